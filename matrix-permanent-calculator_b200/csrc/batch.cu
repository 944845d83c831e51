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

// ---------------------------------------------------------------------------
// Sparse layout (the batch's per-matrix dense/sparse choice).  The host
// permutes a sparse matrix so that columns 0, 1, 2 -- flipped at seven of
// every eight Gray steps -- have their nonzeros in rows 0..R-1.  At those
// seven steps rows R..N-1 do not change: their product P_out is reused and
// only rows 0..R-1 are updated and multiplied; the eighth step (a column
// >= 3) updates every row and recomputes P_out.
// ---------------------------------------------------------------------------

// product of x[J0..J1) in four chains
template <int J0, int J1, int N>
__device__ __forceinline__ double xprod(const double (&x)[N]) {
  double p[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll
  for (int j = J0; j < J1; j++) p[(j - J0) & 3] = (j - J0 < 4) ? x[j] : p[(j - J0) & 3] * x[j];
  return (p[0] * p[1]) * (p[2] * p[3]);
}

// rows [J0, J1) of x += sign * column (compile-time sign unless kSign == 0)
template <int J0, int J1, int kSign, int N>
__device__ __forceinline__ void xupd(double (&x)[N], const double* c, double s) {
#pragma unroll
  for (int j = J0; j < J1; j++) {
    if (kSign > 0)
      x[j] += c[j];
    else if (kSign < 0)
      x[j] -= c[j];
    else
      x[j] = fma(s, c[j], x[j]);
  }
}

template <int N, int R>
__device__ __noinline__ void walk_range_sparse(const double* col, int np, const double* x0s, uint64_t s, uint64_t e,
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
  double pout = xprod<R, N, N>(x);
  {
    const double p0 = xprod<0, R, N>(x) * pout;
    acc.add(p0);
    abs_sum += fabs(p0);
  }
  const double *c0 = col, *c1 = col + np, *c2 = col + 2 * np;
  const uint64_t groups = (e - s) >> 3;
  uint64_t base = s;
#pragma unroll 1
  for (uint64_t gi = 0; gi < groups; gi++, base += 8) {
    const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
    xupd<0, R, +1, N>(x, c0, 0.0);
    const double t1 = xprod<0, R, N>(x) * pout;
    xupd<0, R, +1, N>(x, c1, 0.0);
    const double t2 = xprod<0, R, N>(x) * pout;
    xupd<0, R, -1, N>(x, c0, 0.0);
    const double t3 = xprod<0, R, N>(x) * pout;
    xupd<0, R, 0, N>(x, c2, s4);
    const double t4 = xprod<0, R, N>(x) * pout;
    xupd<0, R, +1, N>(x, c0, 0.0);
    const double t5 = xprod<0, R, N>(x) * pout;
    xupd<0, R, -1, N>(x, c1, 0.0);
    const double t6 = xprod<0, R, N>(x) * pout;
    xupd<0, R, -1, N>(x, c0, 0.0);
    const double t7 = xprod<0, R, N>(x) * pout;
    double t8 = 0.0;
    if (gi + 1 < groups) {  // the last group of the range has seven steps
      const uint64_t i8 = base + 8;
      const int k8 = __ffsll((long long)i8) - 1;
      const double s8 = ((i8 >> (k8 + 1)) & 1) ? -1.0 : 1.0;
      xupd<0, N, 0, N>(x, col + k8 * np, s8);
      pout = xprod<R, N, N>(x);
      t8 = xprod<0, R, N>(x) * pout;
    }
    acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) + (t8 - t7)));
    abs_sum += ((fabs(t1) + fabs(t2)) + (fabs(t3) + fabs(t4))) + ((fabs(t5) + fabs(t6)) + (fabs(t7) + fabs(t8)));
  }
}

// int32 X (y = 2x) in the sparse layout with product groups of 6 rows (R is
// a multiple of 6, so the inner and outer groups are the dense kernel's
// groups).  For 0/1 and small-integer matrices many terms vanish: when
// P_out is 0 at the start of a group, its seven inner terms are all 0 and
// only their net effect on rows 0..R-1 is applied (column 0 is added and
// subtracted twice, column 1 once each, column 2 once: y += s4 * c2).
template <int N, int R>
__device__ __noinline__ void walk_range_int_sparse(const int* col, int np4, const int* y0s, uint64_t s, uint64_t e,
                                                   Acc& acc, double& abs_sum) {
  constexpr int G = 6;
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
  auto grp = [&](int j0, int j1) {  // exact product of y[j0..j1) (fits int32: checked on the host)
    uint32_t p = (uint32_t)y[j0];
#pragma unroll
    for (int j = j0 + 1; j < j1; j++) p *= (uint32_t)y[j];
    return __int2double_rn((int)p);
  };
  auto outer = [&]() {
    double p0 = 1.0, p1 = 1.0;
#pragma unroll
    for (int j0 = R; j0 < N; j0 += G) {
      const double v = grp(j0, j0 + G < N ? j0 + G : N);
      if (((j0 - R) / G) & 1)
        p1 *= v;
      else
        p0 *= v;
    }
    return p0 * p1;
  };
  auto inner = [&]() {
    double p = grp(0, G);
#pragma unroll
    for (int j0 = G; j0 < R; j0 += G) p *= grp(j0, j0 + G);
    return p;
  };
  auto iupd = [&](const int* c, int sg) {
#pragma unroll
    for (int j = 0; j < R; j++) y[j] += sg * c[j];
  };
  double pout = outer();
  {
    const double p0 = inner() * pout;
    acc.add(p0);
    abs_sum += fabs(p0);
  }
  const int *c0 = col, *c1 = col + np4, *c2 = col + 2 * np4;
  const uint64_t groups = (e - s) >> 3;
  uint64_t base = s;
#pragma unroll 1
  for (uint64_t gi = 0; gi < groups; gi++, base += 8) {
    const int s4 = ((base >> 3) & 1) ? -1 : 1;
    double sum = 0.0, asum = 0.0;
    if (pout == 0.0) {
      iupd(c2, s4);  // seven vanishing terms: net update only
    } else {
      iupd(c0, 1);
      const double t1 = inner() * pout;
      iupd(c1, 1);
      const double t2 = inner() * pout;
      iupd(c0, -1);
      const double t3 = inner() * pout;
      iupd(c2, s4);
      const double t4 = inner() * pout;
      iupd(c0, 1);
      const double t5 = inner() * pout;
      iupd(c1, -1);
      const double t6 = inner() * pout;
      iupd(c0, -1);
      const double t7 = inner() * pout;
      sum = ((t2 - t1) + (t4 - t3)) + ((t6 - t5) - t7);
      asum = ((fabs(t1) + fabs(t2)) + (fabs(t3) + fabs(t4))) + ((fabs(t5) + fabs(t6)) + fabs(t7));
    }
    if (gi + 1 < groups) {  // the last group of the range has seven steps
      const uint64_t i8 = base + 8;
      const int k8 = __ffsll((long long)i8) - 1;
      const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
      const int* c8 = col + k8 * np4;
#pragma unroll
      for (int j = 0; j < N; j++) y[j] += s8 * c8[j];
      pout = outer();
      const double t8 = inner() * pout;
      sum += t8;
      asum += fabs(t8);
    }
    acc.add(sum);
    abs_sum += asum;
  }
}

// FP64 X in shared memory instead of registers: lane l keeps x_j at
// xs[32 j + l] (consecutive lanes, consecutive words: conflict-free), so a
// walk needs few registers and more warps fit an SM; every step loads and
// stores its n entries.  Rolled step loop, eight signed terms summed before
// the compensated add (as the register walk).
template <int N>
__device__ __noinline__ void walk_range_xs(const double* col, int np, const double* x0s, double* xs, uint64_t s,
                                           uint64_t e, Acc& acc, double& abs_sum) {
  const int lane = threadIdx.x & 31;
  double* xl = xs + lane;
  const uint64_t g0 = s ^ (s >> 1);
  double p[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll 1
  for (int j = 0; j < N; j++) {
    double v = x0s[j];
    for (int k = 0; k < N - 1; k++)
      if ((g0 >> k) & 1) v += col[k * np + j];
    xl[32 * j] = v;
    p[j & 3] *= v;
  }
  {
    const double p0 = (p[0] * p[1]) * (p[2] * p[3]);
    acc.add(p0);
    abs_sum += fabs(p0);
  }
#pragma unroll 1
  for (uint64_t base = s; base < e; base += 8) {
    const uint64_t top = base + 8 < e ? base + 8 : e - 1;  // the last group has seven steps
    double sum = 0.0, asum = 0.0;
#pragma unroll 1
    for (uint64_t i = base + 1; i <= top; i++) {
      const int k = __ffsll((long long)i) - 1;
      const double sg = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
      const double* c = col + k * np;
      double q[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll
      for (int j = 0; j < N; j++) {
        const double v = fma(sg, c[j], xl[32 * j]);
        xl[32 * j] = v;
        q[j & 3] = j < 4 ? v : q[j & 3] * v;
      }
      const double t = (q[0] * q[1]) * (q[2] * q[3]);
      sum += (i & 1) ? -t : t;
      asum += fabs(t);
    }
    acc.add(sum);
    abs_sum += asum;
  }
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

template <int kMaxN>
__device__ __forceinline__ void walk_dispatch(int n, const double* col, int np, const double* x0s, uint64_t s,
                                              uint64_t e, Acc& acc, double& abs_sum) {
  switch (n) {
#define PERM_BATCH_CASE(N) \
  case N: if constexpr (N <= kMaxN) walk_range<N>(col, np, x0s, s, e, acc, abs_sum); break;
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

template <int kMaxN>
__device__ __forceinline__ void walk_dispatch_int(int n, int g, const int* col, int np4, const int* y0s, uint64_t s,
                                                  uint64_t e, Acc& acc, double& abs_sum) {
  switch (n * 8 + g) {
#define PERM_BATCH_ICASE(N) \
  case N * 8 + 5: if constexpr (N <= kMaxN) walk_range_int<N, 5>(col, np4, y0s, s, e, acc, abs_sum); break; \
  case N * 8 + 6: if constexpr (N <= kMaxN) walk_range_int<N, 6>(col, np4, y0s, s, e, acc, abs_sum); break;
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

template <int kMaxN>
__device__ __forceinline__ void walk_dispatch_xs(int n, const double* col, int np, const double* x0s, double* xs,
                                                 uint64_t s, uint64_t e, Acc& acc, double& abs_sum) {
  switch (n) {
#define PERM_BATCH_XCASE(N) \
  case N: if constexpr (N <= kMaxN) walk_range_xs<N>(col, np, x0s, xs, s, e, acc, abs_sum); break;
    PERM_BATCH_XCASE(9) PERM_BATCH_XCASE(10) PERM_BATCH_XCASE(11) PERM_BATCH_XCASE(12) PERM_BATCH_XCASE(13)
    PERM_BATCH_XCASE(14) PERM_BATCH_XCASE(15) PERM_BATCH_XCASE(16) PERM_BATCH_XCASE(17) PERM_BATCH_XCASE(18)
    PERM_BATCH_XCASE(19) PERM_BATCH_XCASE(20) PERM_BATCH_XCASE(21) PERM_BATCH_XCASE(22) PERM_BATCH_XCASE(23)
    PERM_BATCH_XCASE(24) PERM_BATCH_XCASE(25) PERM_BATCH_XCASE(26) PERM_BATCH_XCASE(27) PERM_BATCH_XCASE(28)
#undef PERM_BATCH_XCASE
    default: break;
  }
}

template <int kMaxN>
__device__ __forceinline__ void walk_dispatch_sparse(int n, int r, const double* col, int np, const double* x0s,
                                                     uint64_t s, uint64_t e, Acc& acc, double& abs_sum) {
  switch (n * 64 + r) {
#define PERM_BATCH_SCASE(N, R) \
  case N * 64 + R: if constexpr (N <= kMaxN) walk_range_sparse<N, R>(col, np, x0s, s, e, acc, abs_sum); break;
    PERM_BATCH_SCASE(12, 8) PERM_BATCH_SCASE(13, 8) PERM_BATCH_SCASE(14, 8) PERM_BATCH_SCASE(15, 8)
    PERM_BATCH_SCASE(16, 8) PERM_BATCH_SCASE(17, 8) PERM_BATCH_SCASE(18, 8) PERM_BATCH_SCASE(19, 8)
    PERM_BATCH_SCASE(20, 8) PERM_BATCH_SCASE(21, 8) PERM_BATCH_SCASE(22, 8) PERM_BATCH_SCASE(23, 8)
    PERM_BATCH_SCASE(24, 8) PERM_BATCH_SCASE(25, 8) PERM_BATCH_SCASE(26, 8) PERM_BATCH_SCASE(27, 8)
    PERM_BATCH_SCASE(28, 8) PERM_BATCH_SCASE(29, 8) PERM_BATCH_SCASE(30, 8) PERM_BATCH_SCASE(31, 8)
    PERM_BATCH_SCASE(32, 8)
    PERM_BATCH_SCASE(20, 16) PERM_BATCH_SCASE(21, 16) PERM_BATCH_SCASE(22, 16) PERM_BATCH_SCASE(23, 16)
    PERM_BATCH_SCASE(24, 16) PERM_BATCH_SCASE(25, 16) PERM_BATCH_SCASE(26, 16) PERM_BATCH_SCASE(27, 16)
    PERM_BATCH_SCASE(28, 16) PERM_BATCH_SCASE(29, 16) PERM_BATCH_SCASE(30, 16) PERM_BATCH_SCASE(31, 16)
    PERM_BATCH_SCASE(32, 16)
    PERM_BATCH_SCASE(24, 20) PERM_BATCH_SCASE(25, 20) PERM_BATCH_SCASE(26, 20) PERM_BATCH_SCASE(27, 20)
    PERM_BATCH_SCASE(28, 20) PERM_BATCH_SCASE(29, 20) PERM_BATCH_SCASE(30, 20) PERM_BATCH_SCASE(31, 20)
    PERM_BATCH_SCASE(32, 20)
    PERM_BATCH_SCASE(29, 24) PERM_BATCH_SCASE(30, 24) PERM_BATCH_SCASE(31, 24) PERM_BATCH_SCASE(32, 24)
#undef PERM_BATCH_SCASE
    default: break;
  }
}

template <int kMaxN>
__device__ __forceinline__ void walk_dispatch_int_sparse(int n, int r, const int* col, int np4, const int* y0s,
                                                         uint64_t s, uint64_t e, Acc& acc, double& abs_sum) {
  switch (n * 64 + r) {
#define PERM_BATCH_ISCASE(N, R) \
  case N * 64 + R: if constexpr (N <= kMaxN) walk_range_int_sparse<N, R>(col, np4, y0s, s, e, acc, abs_sum); break;
    PERM_BATCH_ISCASE(12, 6) PERM_BATCH_ISCASE(13, 6) PERM_BATCH_ISCASE(14, 6) PERM_BATCH_ISCASE(15, 6)
    PERM_BATCH_ISCASE(16, 6) PERM_BATCH_ISCASE(17, 6) PERM_BATCH_ISCASE(18, 6) PERM_BATCH_ISCASE(19, 6)
    PERM_BATCH_ISCASE(20, 6) PERM_BATCH_ISCASE(21, 6) PERM_BATCH_ISCASE(22, 6) PERM_BATCH_ISCASE(23, 6)
    PERM_BATCH_ISCASE(24, 6) PERM_BATCH_ISCASE(25, 6) PERM_BATCH_ISCASE(26, 6) PERM_BATCH_ISCASE(27, 6)
    PERM_BATCH_ISCASE(28, 6) PERM_BATCH_ISCASE(29, 6) PERM_BATCH_ISCASE(30, 6) PERM_BATCH_ISCASE(31, 6)
    PERM_BATCH_ISCASE(32, 6)
    PERM_BATCH_ISCASE(16, 12) PERM_BATCH_ISCASE(17, 12) PERM_BATCH_ISCASE(18, 12) PERM_BATCH_ISCASE(19, 12)
    PERM_BATCH_ISCASE(20, 12) PERM_BATCH_ISCASE(21, 12) PERM_BATCH_ISCASE(22, 12) PERM_BATCH_ISCASE(23, 12)
    PERM_BATCH_ISCASE(24, 12) PERM_BATCH_ISCASE(25, 12) PERM_BATCH_ISCASE(26, 12) PERM_BATCH_ISCASE(27, 12)
    PERM_BATCH_ISCASE(28, 12) PERM_BATCH_ISCASE(29, 12) PERM_BATCH_ISCASE(30, 12) PERM_BATCH_ISCASE(31, 12)
    PERM_BATCH_ISCASE(32, 12)
    PERM_BATCH_ISCASE(22, 18) PERM_BATCH_ISCASE(23, 18) PERM_BATCH_ISCASE(24, 18) PERM_BATCH_ISCASE(25, 18)
    PERM_BATCH_ISCASE(26, 18) PERM_BATCH_ISCASE(27, 18) PERM_BATCH_ISCASE(28, 18) PERM_BATCH_ISCASE(29, 18)
    PERM_BATCH_ISCASE(30, 18) PERM_BATCH_ISCASE(31, 18) PERM_BATCH_ISCASE(32, 18)
    PERM_BATCH_ISCASE(29, 24) PERM_BATCH_ISCASE(30, 24) PERM_BATCH_ISCASE(31, 24) PERM_BATCH_ISCASE(32, 24)
#undef PERM_BATCH_ISCASE
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

template <int kMaxN, int kBlock, int kMinBlocks, bool kXs>
__global__ void __launch_bounds__(kBlock, kMinBlocks) batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  // [n][np] columns + x0[np], then (kXs) the lanes' X vectors [n][32]
  double* slot = reinterpret_cast<double*>(smem) + (size_t)wib * batch_slot_doubles(kMaxN, kXs);
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
        if (M.r)
          walk_dispatch_int_sparse<kMaxN>(n, M.r, ci, np4, ci + n * np4, s, s + L, acc, abs_sum);
        else
          walk_dispatch_int<kMaxN>(n, M.g, ci, np4, ci + n * np4, s, s + L, acc, abs_sum);
      } else if (M.r) {
        walk_dispatch_sparse<kMaxN>(n, M.r, slot, np, x0, s, s + L, acc, abs_sum);
      } else if (kXs && n <= 28) {
        walk_dispatch_xs<kMaxN>(n, slot, np, x0, slot + kMaxN * (kMaxN + 1), s, s + L, acc, abs_sum);
      } else {
        walk_dispatch<kMaxN>(n, slot, np, x0, s, s + L, acc, abs_sum);
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

// Kernel variants (largest order, threads per block, CTAs per SM asked of
// the compiler, FP64 X of dense matrices in registers or shared memory): the
// general one, and variants for batches of orders <= 28 -- block shapes,
// a register budget for three CTAs per SM, and shared-memory X (few
// registers, more warps per SM).  perm_batch_autotune measures them.
const BatchVariant kBatchVariants[kBatchVariantCount] = {
    {40, 128, 1, 0, reinterpret_cast<const void*>(&batch_kernel<40, 128, 1, false>)},
    {28, 128, 2, 0, reinterpret_cast<const void*>(&batch_kernel<28, 128, 2, false>)},
    {28, 128, 3, 0, reinterpret_cast<const void*>(&batch_kernel<28, 128, 3, false>)},
    {28, 256, 1, 0, reinterpret_cast<const void*>(&batch_kernel<28, 256, 1, false>)},
    {28, 64, 4, 0, reinterpret_cast<const void*>(&batch_kernel<28, 64, 4, false>)},
    {28, 128, 3, 1, reinterpret_cast<const void*>(&batch_kernel<28, 128, 3, true>)},
};

}  // namespace perm
