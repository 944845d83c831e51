// skipper.h -- argument block of the SkipPer kernel (ryser_skipper.cu).
#pragma once
#include <cstdint>

#include "perman_common.cuh"

namespace perm {

// Packed sparse operand, one 16-byte-aligned device block staged to shared
// memory whole:  [x0: n doubles][cvals: nnz doubles][rptrs: n+1 ints]
//                [cptrs: n+1 ints][cols: nnz ints][rows: nnz ints]
// with every section starting on a 16-byte boundary.
struct SkipArgs {
  const unsigned char* pack;
  uint32_t pack_bytes;  // multiple of 16
  uint32_t off_cvals, off_rptrs, off_cptrs, off_cols, off_rows;
  int n;
  uint64_t total;    // 2^(n-1) Gray indices
  uint64_t chunk;    // Gray indices per queue entry
  uint64_t nchunks;  // ceil(total / chunk)
  unsigned long long* next_chunk;  // queue head (zeroed before launch)
  unsigned long long* visited;     // evaluated Gray indices (zeroed before launch)
  dd* partials;
  unsigned* ticket;
  double* out;
  int* err;
};

__global__ void skipper_kernel(SkipArgs a);

inline size_t skipper_smem_bytes(uint32_t pack_bytes, int n, int block) {
  return pack_bytes + sizeof(double) * (size_t)n * block + 32 * sizeof(dd) + 16;
}

}  // namespace perm
