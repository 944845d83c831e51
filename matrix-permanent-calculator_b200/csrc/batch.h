// batch.h -- argument blocks of the batched persistent kernel (batch.cu).
#pragma once
#include <cstdint>

#include "perman_common.cuh"

namespace perm {

constexpr int kBatchMaxOrder = 40;
constexpr int kBatchBlock = 128;  // 4 warps, one tile each at a time
// per-warp shared slot: columns [n][np] + x0[np] for the largest order
constexpr int kBatchSlotDoubles = kBatchMaxOrder * kBatchMaxOrder + kBatchMaxOrder;

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

__global__ void batch_kernel(BatchArgs a);

inline size_t batch_smem_bytes() { return sizeof(double) * (size_t)kBatchSlotDoubles * (kBatchBlock / 32); }

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
