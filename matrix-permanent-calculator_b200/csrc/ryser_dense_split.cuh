// ryser_dense_split.cuh -- dense exact permanent with an (almost) exact
// row-sum vector for real matrices: the split-X kernel.
//
// Same walk, ranges and reductions as ryser_dense.cuh (the reference's
// kernel_xshared_coalescing_mshared, gpu_exact_dense.cu:330-399, restated).
// The FP64-X walk's error on real matrices with cancellation is dominated by
// the rounding of the X updates, which is correlated from term to term.  Here
// every entry is split on the host into a coarse part on the grid 2^-q and a
// remainder, a = ah + al, with q chosen so that every partial row sum of
// coarse parts fits in 52 bits: the coarse X, xh = x0h + sum +-ah, is then
// computed EXACTLY in FP64, and the remainder xl = x0l + sum +-al is tiny
// (|al| <= 2^-(q+1)), so its rounding is negligible.  Each term uses
// x = fl(xh + xl) -- one rounding per entry that depends only on the subset --
// and the FP64 product, so the per-term errors are independent roundings
// whose sum grows like the square root of the number of terms.
//
// Per Gray step: 2n adds (coarse and remainder), n adds (combine) and n - 1
// multiplies -- about twice the FP64-X work, in a rolled step loop (the two
// X vectors leave no registers for the 8-step schedule); orders 4..40.  The
// walk also sums |t| and t^2 over its own terms, so the independent-rounding
// error estimate of the result is computed from exact moments instead of a
// sample.  Used by the accuracy policy before falling back to double-double.
#pragma once
#include "ryser_dense.cuh"

namespace perm {

struct DenseSplitArgs {
  const double* img;  // [colH: n x np][colL: n x np][x0h: np][x0l: np]
  int np;
  int m;
  uint64_t block0, nblocks;
  dd* partials;
  unsigned* ticket;
  double* out;
  double* sums;  // [sum |t|, sum t^2] over the walked terms (atomic adds; zeroed by the host)
  int* err;
};

template <int N, int kSign>
__device__ __forceinline__ double split_step(double (&xh)[N], double (&xl)[N], const double* colH,
                                             const double* colL, double s) {
  double p0 = 1.0, p1 = 1.0, p2 = 1.0, p3 = 1.0;
#pragma unroll
  for (int j = 0; j < N; j += 2) {
    double h0, h1 = 0.0, l0, l1 = 0.0;
    if (j + 1 < N) {
      const double2 vh = lds2(colH + j), vl = lds2(colL + j);
      h0 = vh.x;
      h1 = vh.y;
      l0 = vl.x;
      l1 = vl.y;
    } else {
      h0 = lds1(colH + j);
      l0 = lds1(colL + j);
    }
    if (kSign > 0) {
      xh[j] = xh[j] + h0;
      xl[j] = xl[j] + l0;
      if (j + 1 < N) {
        xh[j + 1] = xh[j + 1] + h1;
        xl[j + 1] = xl[j + 1] + l1;
      }
    } else if (kSign < 0) {
      xh[j] = xh[j] - h0;
      xl[j] = xl[j] - l0;
      if (j + 1 < N) {
        xh[j + 1] = xh[j + 1] - h1;
        xl[j + 1] = xl[j + 1] - l1;
      }
    } else {
      xh[j] = __fma_rn(s, h0, xh[j]);
      xl[j] = __fma_rn(s, l0, xl[j]);
      if (j + 1 < N) {
        xh[j + 1] = __fma_rn(s, h1, xh[j + 1]);
        xl[j + 1] = __fma_rn(s, l1, xl[j + 1]);
      }
    }
    const double x0 = __dadd_rn(xh[j], xl[j]);
    const double x1 = (j + 1 < N) ? __dadd_rn(xh[j + 1], xl[j + 1]) : 1.0;
    if ((j & 3) == 0) {
      p0 = (j == 0) ? x0 : p0 * x0;
      if (j + 1 < N) p1 = (j == 0) ? x1 : p1 * x1;
    } else {
      p2 = (j == 2) ? x0 : p2 * x0;
      if (j + 1 < N) p3 = (j == 2) ? x1 : p3 * x1;
    }
  }
  return (p0 * p1) * (p2 * p3);
}

template <int N>
__device__ __forceinline__ double split_prod(const double (&xh)[N], const double (&xl)[N]) {
  double p0 = 1.0, p1 = 1.0, p2 = 1.0, p3 = 1.0;
#pragma unroll
  for (int j = 0; j < N; j++) {
    const double x = __dadd_rn(xh[j], xl[j]);
    if ((j & 3) == 0) p0 = (j == 0) ? x : p0 * x;
    if ((j & 3) == 1) p1 = (j == 1) ? x : p1 * x;
    if ((j & 3) == 2) p2 = (j == 2) ? x : p2 * x;
    if ((j & 3) == 3) p3 = (j == 3) ? x : p3 * x;
  }
  return (p0 * p1) * (p2 * p3);
}

__host__ __device__ inline size_t dense_split_smem_bytes(int n) {
  const int np = (n + 1) & ~1;
  return sizeof(double) * (2 * (size_t)n * np + 2 * np) + 32 * sizeof(dd) + 16;
}

// CTAs per SM by order: the two X vectors fit 128 registers up to order 23
// (4 CTAs) and 168 up to order 34 (3 CTAs; without the hint ptxas picked a
// 166-register schedule at order 34 that ran 25% slower); above, 2 CTAs of
// up to 255 registers.
template <int N>
__global__ void __launch_bounds__(128, (N <= 23 ? 4 : N <= 34 ? 3 : 1)) ryser_dense_split_kernel(DenseSplitArgs args) {
  static_assert(N >= 4, "orders below 4 use the other kernels");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sH = reinterpret_cast<double*>(smem_raw);  // whole image, staged once
  const int np = args.np;
  const double* sL = sH + (size_t)N * np;
  const double* sX0h = sL + (size_t)N * np;
  const double* sX0l = sX0h + np;
  dd* red = reinterpret_cast<dd*>(sH + 2 * (size_t)N * np + 2 * np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged =
      stage_to_smem(sH, args.img, (uint32_t)(sizeof(double) * (2 * (size_t)N * np + 2 * np)), bar, args.err);

  Acc acc;
  double m1 = 0.0, m2 = 0.0;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;

  if (staged && b1 > b0) {
    const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
    double xh[N], xl[N];
#pragma unroll
    for (int j = 0; j < N; j++) {
      xh[j] = sX0h[j];
      xl[j] = sX0l[j];
    }
    const uint64_t g = s0 ^ (s0 >> 1);
#pragma unroll 1
    for (int k = 0; k < N - 1; k++) {
      if ((g >> k) & 1) {
#pragma unroll
        for (int j = 0; j < N; j++) {
          xh[j] += sH[k * np + j];
          xl[j] += sL[k * np + j];
        }
      }
    }
    const double t0 = split_prod<N>(xh, xl);
    acc.add(t0);  // index s0 is even: sign +
    m1 = fabs(t0);
    m2 = t0 * t0;

    // rolled step loop (one step's two X vectors already fill the register
    // file): k = ctz(i) is warp-uniform inside aligned ranges, so the column
    // reads stay shared-memory broadcasts
#pragma unroll 1
    for (uint64_t i = s0 + 1; i < e0; i++) {
      const int k = __ffsll((long long)i) - 1;
      const double sg = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
      const double t = split_step<N, 0>(xh, xl, sH + k * np, sL + k * np, sg);
      acc.add((i & 1) ? -t : t);
      m1 += fabs(t);
      m2 = __fma_rn(t, t, m2);
    }
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) {
    m1 += __shfl_down_sync(0xffffffffu, m1, d);
    m2 += __shfl_down_sync(0xffffffffu, m2, d);
  }
  if ((threadIdx.x & 31) == 0 && m1 > 0.0) {
    atomicAdd(args.sums, m1);
    atomicAdd(args.sums + 1, m2);
  }
  dd mine = acc.value();
  dd bt = block_reduce_dd(mine, red);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, (N & 1) ? 2.0 : -2.0, red);
}

}  // namespace perm
