// mc.h -- argument block of the Monte-Carlo trial kernels (mc.cu).
#pragma once
#include <cstdint>

#include "perman_common.cuh"

namespace perm {

// Packed operand staged whole to shared memory (16-byte sections):
//   [rowmask: np uint64][A: n x np doubles, row-major][AT: n x np doubles]
// or, for 0/1 matrices (scaling_kernel_binary), [rowmask][colmask: np uint64].
// np = n rounded up to even.  The Rasmussen kernel stages the row masks only.
struct McArgs {
  const unsigned char* pack;
  uint32_t mask_bytes;  // np * 8
  uint32_t pack_bytes;  // mask_bytes (+ 2 * n * np * 8 for scaling)
  int n, np;
  int y, z;             // scale interval and scale sweeps (scaling only)
  uint64_t trials;
  uint64_t trial0;      // first trial index (streams are keyed by the global index)
  uint64_t seed;
  double* trial_out;    // optional: value of trial t at trial_out[t - trial0]
  double* partials;     // 3 doubles per block: sum, sum of squares, zero trials
  unsigned* ticket;
  double* out;          // out[0..2] = sum, sum of squares, zero-valued trials
  int* err;
};

__global__ void rasmussen_kernel(McArgs a);
__global__ void scaling_kernel(McArgs a);
// 0/1 matrices: pack = [rowmask: np uint64][colmask: np uint64]
__global__ void scaling_kernel_binary(McArgs a);

constexpr int kMcBlock = 256;  // 8 warps, one trial per warp at a time
// per-warp scaling scratch: d_r, d_c, running sums (64 doubles each), 64 column ids
constexpr int kMcWarpDoubles = 64 * 3 + 32;

inline size_t mc_smem_bytes(uint32_t pack_bytes, bool scaling) {
  // pack + per-warp scaling scratch + 3-double reduction slots + mbarrier
  return pack_bytes + (scaling ? (kMcBlock / 32) * kMcWarpDoubles * sizeof(double) : 0) +
         (kMcBlock / 32) * 3 * sizeof(double) + 16;
}

}  // namespace perm
