// mc_sparse.h -- argument block of the Monte-Carlo kernel for orders above 64
// (mc_sparse.cu).
#pragma once
#include <cstdint>

#include "perman_common.cuh"

namespace perm {

constexpr int kMcSparseMaxOrder = 2047;  // row index packs into 11 bits
constexpr int kMcSparseBlock = 128;      // 4 warps, one trial each at a time

// Packed operand staged whole to shared memory:
//   [rptrs: ptr_ints][cptrs: ptr_ints][cols: idx_ints][rows: idx_ints]
// (int sections padded to multiples of 4 ints).
struct McSparseArgs {
  const unsigned char* pack;
  uint32_t pack_bytes;
  int ptr_ints, idx_ints;
  int n;
  int scaling;  // 0 Rasmussen, 1 scaling
  int y, z;
  uint64_t trials, trial0, seed;
  double* trial_out;
  double* partials;
  unsigned* ticket;
  double* out;
  int* err;
};

__global__ void mc_sparse_kernel(McSparseArgs a);

// per-warp shared bytes: two bitsets, d_r/d_c for scaling, the row counts
__host__ __device__ inline size_t mc_sparse_warp_bytes(int n, int scaling) {
  const size_t W = (size_t)(n + 63) / 64;
  size_t b = 2 * W * sizeof(uint64_t) + (scaling ? 2 * (size_t)n * sizeof(double) : 0) + (size_t)n * sizeof(int);
  return (b + 15) & ~(size_t)15;
}

inline size_t mc_sparse_smem_bytes(uint32_t pack_bytes, int n, int scaling) {
  return pack_bytes + (kMcSparseBlock / 32) * mc_sparse_warp_bytes(n, scaling) +
         (kMcSparseBlock / 32) * 3 * sizeof(double) + 16;
}

}  // namespace perm
