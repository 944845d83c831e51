// ryser_dense_2l.cuh -- the FP64-X walk (ryser_dense.cuh) in the two-level
// row layout of ryser_dense_int_sparse.cuh, and (ryser_dense_3l_kernel) in
// the three-level layout of ryser_dense_int_3l_kernel.
//
// The host permutes the matrix so that columns 0..2 are three columns whose
// nonzeros lie in the fewest rows and those rows come first (rows 0..R-1);
// rows R..N-1 are zero in columns 0..2.  At the seven of every eight Gray
// steps that flip a column 0..2 the kernel updates and multiplies rows
// 0..R-1 only and multiplies by P_out, the product of the other rows, which
// it recomputes at the eighth step (a column >= 3).  Each term is still a
// product of N values formed by N - 1 multiplies, so the FP64-X error bound
// carries over; the outer rows are updated once per eight steps, so their
// rounding drift is smaller.  X is re-anchored (recomputed from x0) at every
// segment of seg_blocks aligned blocks, as in the one-level walk.
#pragma once
#include "ryser_dense.cuh"

namespace perm {

// prod of x over rows [J0, J1), four chains
template <int J0, int J1, int N>
__device__ __forceinline__ double xrows_prod(const double (&x)[N]) {
  constexpr int C = (J1 - J0) >= 4 ? 4 : (J1 - J0);
  double c[4] = {1.0, 1.0, 1.0, 1.0};
#pragma unroll
  for (int t = 0; t < C; t++) c[t] = x[J0 + t];
#pragma unroll
  for (int j = J0 + C; j < J1; j++) c[(j - J0) & 3] *= x[j];
  if (C == 4) return (c[0] * c[1]) * (c[2] * c[3]);
  if (C == 3) return (c[0] * c[1]) * c[2];
  if (C == 2) return c[0] * c[1];
  return c[0];
}

// rows [0, R) of x += s * column (compile-time sign when kSign != 0)
template <int R, int kSign, int N>
__device__ __forceinline__ void xrows_update(double (&x)[N], const double* col, double s) {
#pragma unroll
  for (int j = 0; j < R; j += 2) {
    double v0, v1 = 0.0;
    if (j + 1 < R) {
      const double2 v = lds2(col + j);
      v0 = v.x;
      v1 = v.y;
    } else {
      v0 = lds1(col + j);
    }
    if (kSign > 0) {
      x[j] = x[j] + v0;
      if (j + 1 < R) x[j + 1] = x[j + 1] + v1;
    } else if (kSign < 0) {
      x[j] = x[j] - v0;
      if (j + 1 < R) x[j + 1] = x[j + 1] - v1;
    } else {
      x[j] = fma(s, v0, x[j]);
      if (j + 1 < R) x[j + 1] = fma(s, v1, x[j + 1]);
    }
  }
}

template <int N, int R>
__global__ void __launch_bounds__(128) ryser_dense_2l_kernel(DenseArgs args) {
  static_assert(R >= 2 && R + 2 <= N && (R & 1) == 0, "inner rows: even, and outer rows must remain");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sA = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  double* sX0 = sA + N * np;
  dd* red = reinterpret_cast<dd*>(sX0 + np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged = stage_to_smem(sA, args.colA, (uint32_t)(sizeof(double) * N * np), bar, args.err, args.inject);
  if (threadIdx.x < N) {
    const int j = threadIdx.x;
    double rs = 0.0;
    for (int k = 0; k < N; k++) rs += sA[k * np + j];
    sX0[j] = sA[(N - 1) * np + j] - rs * 0.5;
  }
  __syncthreads();

  Acc acc;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;

  if (staged && b1 > b0) {
    const uint64_t K = args.seg_blocks ? args.seg_blocks : b1 - b0;
    const double* c0 = sA;
    const double* c1 = sA + np;
    const double* c2 = sA + 2 * np;
#pragma unroll 1
    for (uint64_t blk = b0; blk < b1; blk += K) {
      const uint64_t nb = b1 - blk < K ? b1 - blk : K;
      const uint64_t s0 = (args.block0 + blk) << args.m;
      double x[N];
      anchor_x<N>(x, sX0, sA, np, s0);
      double pout = xrows_prod<R, N, N>(x);
      acc.add(xrows_prod<0, R, N>(x) * pout);  // index s0 is even: sign +
      const uint64_t groups = (nb << args.m) >> 3;
      uint64_t base = s0;
      auto seven = [&](double s4, double (&t)[7]) {
        xrows_update<R, +1>(x, c0, 0.0);
        t[0] = xrows_prod<0, R, N>(x) * pout;
        xrows_update<R, +1>(x, c1, 0.0);
        t[1] = xrows_prod<0, R, N>(x) * pout;
        xrows_update<R, -1>(x, c0, 0.0);
        t[2] = xrows_prod<0, R, N>(x) * pout;
        xrows_update<R, 0>(x, c2, s4);
        t[3] = xrows_prod<0, R, N>(x) * pout;
        xrows_update<R, +1>(x, c0, 0.0);
        t[4] = xrows_prod<0, R, N>(x) * pout;
        xrows_update<R, -1>(x, c1, 0.0);
        t[5] = xrows_prod<0, R, N>(x) * pout;
        xrows_update<R, -1>(x, c0, 0.0);
        t[6] = xrows_prod<0, R, N>(x) * pout;
      };
#pragma unroll 1
      for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) {
        const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
        const uint64_t i8 = base + 8;
        const int k8 = __ffsll((long long)i8) - 1;
        const double s8 = ((i8 >> (k8 + 1)) & 1) ? -1.0 : 1.0;
        double t[7];
        seven(s4, t);
        // the eighth step flips column k8 >= 3: every row may change
        xrows_update<N, 0>(x, sA + k8 * np, s8);
        pout = xrows_prod<R, N, N>(x);
        const double t8 = xrows_prod<0, R, N>(x) * pout;
        acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) + (t8 - t[6])));
      }
      {  // last group of the segment: seven steps (the next index starts the next segment)
        const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
        double t[7];
        seven(s4, t);
        acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) - t[6]));
      }
    }
  }

  dd bt = block_reduce_dd(acc.value(), red);
  const double factor = (N & 1) ? 2.0 : -2.0;
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

// Three-level layout: column 0 is zero outside rows [0, R1), columns 1 and 2
// outside rows [0, R2) (the host permuted the matrix so).  With P1, P2, P3
// the products of rows [0, R1), [R1, R2), [R2, N) and P23 = P2 P3: the four
// column-0 steps of every eight update R1 rows and multiply P1 by the stored
// P23, the three column-1/2 steps update R2 rows and re-form P23 from P2 and
// the stored P3, the eighth step updates every row and re-forms P3.  Each
// term is still a product of N values formed by N - 1 multiplies, so the
// FP64-X error bound carries over.  Per 8 steps 8 R1 + 6 R2 + 2n + 13
// operations against 7 (2R + 1) + 2n in the two-level layout.
template <int N, int R1, int R2>
__global__ void __launch_bounds__(128) ryser_dense_3l_kernel(DenseArgs args) {
  static_assert(R1 >= 4 && R1 + 4 <= R2 && R2 + 2 <= N && (R1 & 1) == 0 && (R2 & 1) == 0,
                "levels: even row counts, four rows or more each, outer rows must remain");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sA = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  double* sX0 = sA + N * np;
  dd* red = reinterpret_cast<dd*>(sX0 + np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged = stage_to_smem(sA, args.colA, (uint32_t)(sizeof(double) * N * np), bar, args.err, args.inject);
  if (threadIdx.x < N) {
    const int j = threadIdx.x;
    double rs = 0.0;
    for (int k = 0; k < N; k++) rs += sA[k * np + j];
    sX0[j] = sA[(N - 1) * np + j] - rs * 0.5;
  }
  __syncthreads();

  Acc acc;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;

  if (staged && b1 > b0) {
    const uint64_t K = args.seg_blocks ? args.seg_blocks : b1 - b0;
    const double* c0 = sA;
    const double* c1 = sA + np;
    const double* c2 = sA + 2 * np;
#pragma unroll 1
    for (uint64_t blk = b0; blk < b1; blk += K) {
      const uint64_t nb = b1 - blk < K ? b1 - blk : K;
      const uint64_t s0 = (args.block0 + blk) << args.m;
      double x[N];
      anchor_x<N>(x, sX0, sA, np, s0);
      double p3 = xrows_prod<R2, N, N>(x);
      double p23 = xrows_prod<R1, R2, N>(x) * p3;
      acc.add(xrows_prod<0, R1, N>(x) * p23);  // index s0 is even: sign +
      const uint64_t groups = (nb << args.m) >> 3;
      uint64_t base = s0;
      auto seven = [&](double s4, double (&t)[7]) {
        xrows_update<R1, +1>(x, c0, 0.0);
        t[0] = xrows_prod<0, R1, N>(x) * p23;
        xrows_update<R2, +1>(x, c1, 0.0);
        p23 = xrows_prod<R1, R2, N>(x) * p3;
        t[1] = xrows_prod<0, R1, N>(x) * p23;
        xrows_update<R1, -1>(x, c0, 0.0);
        t[2] = xrows_prod<0, R1, N>(x) * p23;
        xrows_update<R2, 0>(x, c2, s4);
        p23 = xrows_prod<R1, R2, N>(x) * p3;
        t[3] = xrows_prod<0, R1, N>(x) * p23;
        xrows_update<R1, +1>(x, c0, 0.0);
        t[4] = xrows_prod<0, R1, N>(x) * p23;
        xrows_update<R2, -1>(x, c1, 0.0);
        p23 = xrows_prod<R1, R2, N>(x) * p3;
        t[5] = xrows_prod<0, R1, N>(x) * p23;
        xrows_update<R1, -1>(x, c0, 0.0);
        t[6] = xrows_prod<0, R1, N>(x) * p23;
      };
#pragma unroll 1
      for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) {
        const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
        const uint64_t i8 = base + 8;
        const int k8 = __ffsll((long long)i8) - 1;
        const double s8 = ((i8 >> (k8 + 1)) & 1) ? -1.0 : 1.0;
        double t[7];
        seven(s4, t);
        // the eighth step flips column k8 >= 3: every row may change
        xrows_update<N, 0>(x, sA + k8 * np, s8);
        p3 = xrows_prod<R2, N, N>(x);
        p23 = xrows_prod<R1, R2, N>(x) * p3;
        const double t8 = xrows_prod<0, R1, N>(x) * p23;
        acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) + (t8 - t[6])));
      }
      {  // last group of the segment: seven steps (the next index starts the next segment)
        const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
        double t[7];
        seven(s4, t);
        acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) - t[6]));
      }
    }
  }

  dd bt = block_reduce_dd(acc.value(), red);
  const double factor = (N & 1) ? 2.0 : -2.0;
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

}  // namespace perm
