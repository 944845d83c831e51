// batch.h -- argument blocks of the batched persistent kernel (batch.cu).
#pragma once
#include <cstdint>

#include "perman_common.cuh"

namespace perm {

constexpr int kBatchMaxOrder = 40;
// per-warp shared slot: columns [n][np] + x0[np] for the largest order (np = n
// rounded up to even: n (n + 1) doubles hold it for every n)

// One matrix of a batch, in queue order (largest work first).
struct BatchMatrix {
  uint64_t offset;      // first double of its column-major image in `operands`
  uint64_t first_tile;  // tiles [first_tile, first_tile + ntiles) belong to it
  uint32_t ntiles;
  int n;                // order
  int m;                // lane range = 2^m Gray indices (unused below order 9)
  int index;            // position in the caller's batch
  int g;                // 0: FP64 X (column-major doubles, stride np); 5 or 6: int32 X
                        // with product groups of g rows (doubled int columns, stride
                        // np4 = n rounded up to 4, then y0) -- orders >= 9 only
  int r;                // 0: dense walk; > 0: sparse layout, columns 0..2 nonzero in
                        // rows 0..r-1 only (FP64: r in {8, 16, 20, 24}; int32, g = 6: r in
                        // {6, 12, 18, 24}), orders 12..32
};

struct BatchArgs {
  const double* operands;
  const BatchMatrix* mats;
  int count;
  uint64_t total_tiles;
  unsigned long long* next_tile;  // queue head, zero before launch
  dd* tile_partials;              // one per tile
  double* tile_abs;               // sum of |term| per tile
  unsigned* mat_done;             // per-matrix tickets, zero before launch (re-armed by the kernel)
  double* results;                // (hi, lo, sum |term|) per matrix, caller order
};

// per-warp shared slot of a kernel variant whose largest order is max_n:
// columns and x0, then (shared-memory X) 32 lanes' X vectors
__host__ __device__ constexpr int batch_slot_doubles(int max_n, bool xs) {
  return max_n * max_n + max_n + (xs ? 32 * max_n : 0);
}

// A compiled batch kernel: largest order it walks, threads per block, CTAs
// per SM it was compiled for (launch bounds), whether dense FP64 matrices
// keep X in shared memory, entry point.
struct BatchVariant {
  int max_n, block, min_blocks, xs;
  const void* fn;
};
constexpr int kBatchVariantCount = 6;
extern const BatchVariant kBatchVariants[kBatchVariantCount];

inline size_t batch_smem_bytes(const BatchVariant& v) {
  return sizeof(double) * (size_t)batch_slot_doubles(v.max_n, v.xs != 0) * (v.block / 32);
}

// Lane-range exponent used when the autotuner has not measured an order:
// about 2^12 Gray indices per lane, at least 8, at most a 32-lane tile per matrix.
inline int batch_default_m(int n) {
  if (n < 9) return 0;
  int m = 12;
  if (m > n - 1 - 5) m = n - 1 - 5;
  if (m < 3) m = 3;
  return m;
}

}  // namespace perm
