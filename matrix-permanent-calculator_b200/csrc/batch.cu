// batch.cu -- many exact permanents of mixed order in one persistent launch.
//
// The reference computes one matrix per call (gpu_exact_dense.cu:641-699); a
// batch of thousands of small matrices would be thousands of launches, each
// too small to fill the GPU.  Here the Gray ranges of all matrices are cut
// into tiles -- one warp-sized piece: 32 lanes x 2^m aligned Gray indices -- and
// a persistent grid of warps drains a global tile queue, largest matrices
// first.  A warp stages its tile's matrix into its own shared-memory slot
// (kept when the next tile is from the same matrix), walks the lanes' ranges
// with the same register-X step as ryser_dense.cuh, reduces the tile to one
// double-double and stores it; the warp that completes a matrix's last tile
// (per-matrix atomic ticket) sums that matrix's tile partials in tile order --
// deterministic -- and writes (hi, lo).  Orders 1..kBatchMaxOrder; per-order
// lane-range lengths 2^m come from the autotuner (or a default).
#include <cuda_runtime.h>

#include "batch.h"
#include "ryser_dense.cuh"
#include "ryser_dense_int.cuh"

namespace perm {

namespace {

// Walk lane range [s, e) (aligned, multiple of 8, e > s) of an order-N matrix
// whose columns are at col (stride np) and x0 at x0s.
template <int N>
__device__ __noinline__ void walk_range(const double* col, int np, const double* x0s, uint64_t s, uint64_t e,
                                           Acc& acc, double& abs_sum) {
  double x[N];
#pragma unroll
  for (int j = 0; j < N; j++) x[j] = x0s[j];
  const uint64_t g = s ^ (s >> 1);
#pragma unroll 1
  for (int k = 0; k < N - 1; k++) {
    if ((g >> k) & 1) {
#pragma unroll
      for (int j = 0; j < N; j++) x[j] += col[k * np + j];
    }
  }
  {
    const double p0 = prod_only<N>(x);
    acc.add(p0);
    abs_sum += fabs(p0);
  }
  const double* c0 = col;
  const double* c1 = col + np;
  const double* c2 = col + 2 * np;
  const uint64_t groups = (e - s) >> 3;
  uint64_t base = s;
#pragma unroll 1
  for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) {
    const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
    const uint64_t i8 = base + 8;
    const int k8 = __ffsll((long long)i8) - 1;
    const double s8 = ((i8 >> (k8 + 1)) & 1) ? -1.0 : 1.0;
    double t1 = step<N, +1>(x, c0, 0.0);
    double t2 = step<N, +1>(x, c1, 0.0);
    double t3 = step<N, -1>(x, c0, 0.0);
    double t4 = step<N, 0>(x, c2, s4);
    double t5 = step<N, +1>(x, c0, 0.0);
    double t6 = step<N, -1>(x, c1, 0.0);
    double t7 = step<N, -1>(x, c0, 0.0);
    double t8 = step<N, 0>(x, col + k8 * np, s8);
    acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) + (t8 - t7)));
    abs_sum += ((fabs(t1) + fabs(t2)) + (fabs(t3) + fabs(t4))) + ((fabs(t5) + fabs(t6)) + (fabs(t7) + fabs(t8)));
  }
  const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
  double t1 = step<N, +1>(x, c0, 0.0);
  double t2 = step<N, +1>(x, c1, 0.0);
  double t3 = step<N, -1>(x, c0, 0.0);
  double t4 = step<N, 0>(x, c2, s4);
  double t5 = step<N, +1>(x, c0, 0.0);
  double t6 = step<N, -1>(x, c1, 0.0);
  double t7 = step<N, -1>(x, c0, 0.0);
  acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) - t7));
  abs_sum += ((fabs(t1) + fabs(t2)) + (fabs(t3) + fabs(t4))) + ((fabs(t5) + fabs(t6)) + fabs(t7));
}

// The same walk with y = 2x in int32 (ryser_dense_int.cuh): for integer
// matrices whose product groups of G rows provably fit in int32.  Terms are
// y-products (2^N times the x-products).
template <int N, int G>
__device__ __noinline__ void walk_range_int(const int* col, int np4, const int* y0s, uint64_t s, uint64_t e,
                                            Acc& acc, double& abs_sum) {
  int y[N];
#pragma unroll
  for (int j = 0; j < N; j++) y[j] = y0s[j];
  const uint64_t g = s ^ (s >> 1);
#pragma unroll 1
  for (int k = 0; k < N - 1; k++) {
    if ((g >> k) & 1) {
#pragma unroll
      for (int j = 0; j < N; j++) y[j] += col[k * np4 + j];
    }
  }
  {
    const double p0 = group_product<N, G>(y);
    acc.add(p0);
    abs_sum += fabs(p0);
  }
  const int* c0 = col;
  const int* c1 = col + np4;
  const int* c2 = col + 2 * np4;
  const uint64_t groups = (e - s) >> 3;
  uint64_t base = s;
#pragma unroll 1
  for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) {
    const int s4 = ((base >> 3) & 1) ? -1 : 1;
    const uint64_t i8 = base + 8;
    const int k8 = __ffsll((long long)i8) - 1;
    const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
    double t1 = istep<N, G, +1>(y, c0, 0);
    double t2 = istep<N, G, +1>(y, c1, 0);
    double t3 = istep<N, G, -1>(y, c0, 0);
    double t4 = istep<N, G, 0>(y, c2, s4);
    double t5 = istep<N, G, +1>(y, c0, 0);
    double t6 = istep<N, G, -1>(y, c1, 0);
    double t7 = istep<N, G, -1>(y, c0, 0);
    double t8 = istep<N, G, 0>(y, col + k8 * np4, s8);
    acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) + (t8 - t7)));
    abs_sum += ((fabs(t1) + fabs(t2)) + (fabs(t3) + fabs(t4))) + ((fabs(t5) + fabs(t6)) + (fabs(t7) + fabs(t8)));
  }
  const int s4 = ((base >> 3) & 1) ? -1 : 1;
  double t1 = istep<N, G, +1>(y, c0, 0);
  double t2 = istep<N, G, +1>(y, c1, 0);
  double t3 = istep<N, G, -1>(y, c0, 0);
  double t4 = istep<N, G, 0>(y, c2, s4);
  double t5 = istep<N, G, +1>(y, c0, 0);
  double t6 = istep<N, G, -1>(y, c1, 0);
  double t7 = istep<N, G, -1>(y, c0, 0);
  acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) - t7));
  abs_sum += ((fabs(t1) + fabs(t2)) + (fabs(t3) + fabs(t4))) + ((fabs(t5) + fabs(t6)) + fabs(t7));
}

// Orders below 9 have fewer than 256 Gray indices: lane 0 walks them all.
__device__ void walk_small(const double* col, int np, const double* x0s, int n, Acc& acc, double& abs_sum) {
  double x[8];
  for (int j = 0; j < n; j++) x[j] = x0s[j];
  const uint64_t total = 1ull << (n - 1);
  for (uint64_t i = 0; i < total; i++) {
    if (i) {
      const int k = __ffsll((long long)i) - 1;
      const double s = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
      for (int j = 0; j < n; j++) x[j] = fma(s, col[k * np + j], x[j]);
    }
    double p = x[0];
    for (int j = 1; j < n; j++) p *= x[j];
    acc.add((i & 1) ? -p : p);
    abs_sum += fabs(p);
  }
}

__device__ __forceinline__ void walk_dispatch(int n, const double* col, int np, const double* x0s, uint64_t s,
                                              uint64_t e, Acc& acc, double& abs_sum) {
  switch (n) {
#define PERM_BATCH_CASE(N) \
  case N: walk_range<N>(col, np, x0s, s, e, acc, abs_sum); break;
    PERM_BATCH_CASE(9) PERM_BATCH_CASE(10) PERM_BATCH_CASE(11) PERM_BATCH_CASE(12) PERM_BATCH_CASE(13)
    PERM_BATCH_CASE(14) PERM_BATCH_CASE(15) PERM_BATCH_CASE(16) PERM_BATCH_CASE(17) PERM_BATCH_CASE(18)
    PERM_BATCH_CASE(19) PERM_BATCH_CASE(20) PERM_BATCH_CASE(21) PERM_BATCH_CASE(22) PERM_BATCH_CASE(23)
    PERM_BATCH_CASE(24) PERM_BATCH_CASE(25) PERM_BATCH_CASE(26) PERM_BATCH_CASE(27) PERM_BATCH_CASE(28)
    PERM_BATCH_CASE(29) PERM_BATCH_CASE(30) PERM_BATCH_CASE(31) PERM_BATCH_CASE(32) PERM_BATCH_CASE(33)
    PERM_BATCH_CASE(34) PERM_BATCH_CASE(35) PERM_BATCH_CASE(36) PERM_BATCH_CASE(37) PERM_BATCH_CASE(38)
    PERM_BATCH_CASE(39) PERM_BATCH_CASE(40)
#undef PERM_BATCH_CASE
    default: break;
  }
}

__device__ __forceinline__ void walk_dispatch_int(int n, int g, const int* col, int np4, const int* y0s, uint64_t s,
                                                  uint64_t e, Acc& acc, double& abs_sum) {
  switch (n * 8 + g) {
#define PERM_BATCH_ICASE(N) \
  case N * 8 + 5: walk_range_int<N, 5>(col, np4, y0s, s, e, acc, abs_sum); break; \
  case N * 8 + 6: walk_range_int<N, 6>(col, np4, y0s, s, e, acc, abs_sum); break;
    PERM_BATCH_ICASE(9) PERM_BATCH_ICASE(10) PERM_BATCH_ICASE(11) PERM_BATCH_ICASE(12) PERM_BATCH_ICASE(13)
    PERM_BATCH_ICASE(14) PERM_BATCH_ICASE(15) PERM_BATCH_ICASE(16) PERM_BATCH_ICASE(17) PERM_BATCH_ICASE(18)
    PERM_BATCH_ICASE(19) PERM_BATCH_ICASE(20) PERM_BATCH_ICASE(21) PERM_BATCH_ICASE(22) PERM_BATCH_ICASE(23)
    PERM_BATCH_ICASE(24) PERM_BATCH_ICASE(25) PERM_BATCH_ICASE(26) PERM_BATCH_ICASE(27) PERM_BATCH_ICASE(28)
    PERM_BATCH_ICASE(29) PERM_BATCH_ICASE(30) PERM_BATCH_ICASE(31) PERM_BATCH_ICASE(32) PERM_BATCH_ICASE(33)
    PERM_BATCH_ICASE(34) PERM_BATCH_ICASE(35) PERM_BATCH_ICASE(36) PERM_BATCH_ICASE(37) PERM_BATCH_ICASE(38)
    PERM_BATCH_ICASE(39) PERM_BATCH_ICASE(40)
#undef PERM_BATCH_ICASE
    default: break;
  }
}

__device__ __forceinline__ int find_matrix(const BatchMatrix* mats, int count, uint64_t tile) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {  // last matrix with first_tile <= tile
    const int mid = (lo + hi + 1) >> 1;
    if (mats[mid].first_tile <= tile)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

}  // namespace

__global__ void __launch_bounds__(kBatchBlock) batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* slot = reinterpret_cast<double*>(smem) + (size_t)wib * kBatchSlotDoubles;  // [n][np] + x0[np]
  int cached = -1;
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(a.next_tile, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= a.total_tiles) break;
    const int mi = find_matrix(a.mats, a.count, t);
    const BatchMatrix M = a.mats[mi];
    const int n = M.n, np = (n + 1) & ~1;
    const int np4 = (n + 3) & ~3;
    if (mi != cached) {
      __syncwarp();
      if (M.g) {
        // int32 image: doubled columns then y0, (n + 1) np4 words
        const int* src = reinterpret_cast<const int*>(a.operands + M.offset);
        int* dst = reinterpret_cast<int*>(slot);
        for (int idx = lane; idx < (n + 1) * np4; idx += 32) dst[idx] = src[idx];
      } else {
        const double* src = a.operands + M.offset;
        for (int idx = lane; idx < n * np; idx += 32) slot[idx] = src[idx];
        __syncwarp();
        double* x0 = slot + n * np;
        for (int j = lane; j < n; j += 32) {
          double rs = 0.0;
          for (int k = 0; k < n; k++) rs += slot[k * np + j];
          x0[j] = slot[(n - 1) * np + j] - rs * 0.5;
        }
      }
      __syncwarp();
      cached = mi;
    }
    const double* x0 = slot + n * np;
    Acc acc;
    double abs_sum = 0.0;
    if (n < 9) {
      if (lane == 0) walk_small(slot, np, x0, n, acc, abs_sum);
    } else {
      const uint64_t q = t - M.first_tile;
      const uint64_t L = 1ull << M.m;
      const uint64_t s = (q * 32 + lane) * L;
      if (M.g) {
        const int* ci = reinterpret_cast<const int*>(slot);
        walk_dispatch_int(n, M.g, ci, np4, ci + n * np4, s, s + L, acc, abs_sum);
      } else {
        walk_dispatch(n, slot, np, x0, s, s + L, acc, abs_sum);
      }
    }
    dd v = acc.value();
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      v = dd_add(v, dd_shfl_down(v, d));
      abs_sum += __shfl_down_sync(0xffffffffu, abs_sum, d);
    }
    bool last = false;
    if (lane == 0) {
      a.tile_partials[t] = v;
      a.tile_abs[t] = abs_sum;
      __threadfence();
      const unsigned prev = atomicAdd(&a.mat_done[mi], 1u);
      last = (prev == M.ntiles - 1);
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
      __threadfence();
      dd s = {0.0, 0.0};
      double sa = 0.0;
      for (uint64_t k = lane; k < M.ntiles; k += 32) {
        dd p;
        p.hi = __ldcg(&a.tile_partials[M.first_tile + k].hi);
        p.lo = __ldcg(&a.tile_partials[M.first_tile + k].lo);
        s = dd_add(s, p);
        sa += __ldcg(&a.tile_abs[M.first_tile + k]);
      }
#pragma unroll
      for (int d = 16; d >= 1; d >>= 1) {
        s = dd_add(s, dd_shfl_down(s, d));
        sa += __shfl_down_sync(0xffffffffu, sa, d);
      }
      if (lane == 0) {
        // y-products carry 2^n (exact power-of-two rescaling)
        const double scale = M.g ? ldexp(1.0, -n) : 1.0;
        const double f = ((n & 1) ? 2.0 : -2.0) * scale;
        a.results[3 * M.index] = s.hi * f;
        a.results[3 * M.index + 1] = s.lo * f;
        a.results[3 * M.index + 2] = sa * 2.0 * scale;
        a.mat_done[mi] = 0u;
      }
    }
  }
}

}  // namespace perm
