// ryser_dense_intc.cuh -- dense exact permanent for integer matrices with a
// certified error bound: int32 X, double-double products and sum.
//
// Same walk, ranges and reductions as ryser_dense_int.cuh (the reference's
// kernel_xshared_coalescing_mshared, gpu_exact_dense.cu:330-399, restated
// with y = 2x held in int32).  The int32-X kernel's only roundings are its
// ceil(n/G) - 1 FP64 products of exact group values and the FP64 sums of
// terms; its worst-case error bound, (ceil(n/G) + 16) u sum|t| / |perm|,
// cannot certify 1e-10 once the terms cancel by more than ~4e4 (dense
// integer matrices of order 40).  Here both roundings are made error-free:
//  * each group value v_g (an exact int32 product converted exactly to
//    FP64) enters a double-double product as soon as it is formed: the
//    first two by TwoProd (h = v0 v1, l = fma(v0, v1, -h), exact), every
//    further value by h' = h v, l' = fma(l, v, fma(h, v, -h')) (3
//    operations, relative error a few u^2);
//  * with kPair, consecutive int32 group products are first multiplied
//    into one int64 (a 32 x 32 -> 64-bit multiply) and converted once,
//    which is exact because the host proved every pair's |product| < 2^53:
//    a multiply and a conversion replace a 3-operation double-double step
//    and a conversion (order 40, groups of 4 rows: 2446 ms against 2624 ms
//    for groups of 5 in one chain; pairs multiplied in FP64 after two
//    conversions: 2542 ms);
//  * every signed term is added to the thread's total with TwoSum into a
//    (hi, lo) pair whose low part collects every rounding error (Sum2 of
//    Ogita, Rump and Oishi);
//  * the walk also sums |hi| of its own terms, so the bound uses the exact
//    cancellation scale sum|t| instead of a sampled estimate.
// Per Gray step this adds ~2 ceil(n/G) + 9 FP64 operations to the int32-X
// step (which is issue-bound with the FP64 pipe mostly idle).  One product
// chain and one running (hi, lo) per thread: at order 40 this measured 1.4%
// faster than two chains joined at the end with per-group partial sums
// (2628 against 2664 ms; the int32-X walk: 2007 ms).
// Error: below (8 ceil(n/G) + 256 + K^2) u^2 sum|t| for K terms per thread
// (the low part's own rounding over K terms), plus the final rounding.
#pragma once
#include "ryser_dense_int.cuh"

namespace perm {

struct DenseIntcArgs {
  const int* colI;  // column-major doubled matrix, then y0 (as DenseIntArgs)
  int np4;
  int m;
  uint64_t block0, nblocks;
  dd* partials;
  unsigned* ticket;
  double* out;
  double* sums;  // sums[0] += sum |term| over the walked terms (zeroed by the host)
  int* err;
};

// y += s * col (compile-time sign when kSign != 0)
template <int N, int kSign>
__device__ __forceinline__ void iupdate(int (&y)[N], const int* col, int s) {
#pragma unroll
  for (int j = 0; j < N; j += 4) {
    const int4 v = lds4i(col + j);
    const int c[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
      if (j + t < N) {
        if (kSign > 0)
          y[j + t] += c[t];
        else if (kSign < 0)
          y[j + t] -= c[t];
        else
          y[j + t] += s * c[t];
      }
    }
  }
}

// Exact int32 product of y over the rows of group g (the host proved
// |product| < 2^31; the uint32 product wraps to the right two's complement).
template <int N, int G>
__device__ __forceinline__ int group_int(const int (&y)[N], int g) {
  const int j0 = g * G;
  uint32_t pr = (uint32_t)y[j0];
#pragma unroll
  for (int t = 1; t < G; t++)
    if (j0 + t < N) pr = pr * (uint32_t)y[j0 + t];
  return (int)pr;
}

// Exact value of group g converted to FP64.
template <int N, int G>
__device__ __forceinline__ double group_value(const int (&y)[N], int g) {
  return __int2double_rn(group_int<N, G>(y, g));
}

// Factor i of the double-double product: group value i, or with kPair the
// int64 product of groups 2i and 2i + 1 (the last group alone when the
// number of groups is odd) converted exactly (|product| < 2^53).
template <int N, int G, bool kPair>
__device__ __forceinline__ double term_factor(const int (&y)[N], int i) {
  constexpr int NG = (N + G - 1) / G;
  if (!kPair) return group_value<N, G>(y, i);
  long long v = group_int<N, G>(y, 2 * i);
  if (2 * i + 1 < NG) v *= group_int<N, G>(y, 2 * i + 1);
  return __ll2double_rn(v);
}

// Double-double product of the factors (an unevaluated pair), each
// multiplied in as it is formed.
template <int N, int G, bool kPair>
__device__ __forceinline__ dd term_dd(const int (&y)[N]) {
  constexpr int NG = (N + G - 1) / G;
  constexpr int NF = kPair ? (NG + 1) / 2 : NG;
  dd p = {term_factor<N, G, kPair>(y, 0), 0.0};
  if (NF == 1) return p;
  {
    const double v = term_factor<N, G, kPair>(y, 1);
    const double h = __dmul_rn(p.hi, v);
    p.lo = __fma_rn(p.hi, v, -h);
    p.hi = h;
  }
#pragma unroll
  for (int i = 2; i < NF; i++) {
    const double v = term_factor<N, G, kPair>(y, i);
    const double h = __dmul_rn(p.hi, v);
    const double l = __fma_rn(p.hi, v, -h);
    p.lo = __fma_rn(p.lo, v, l);
    p.hi = h;
  }
  return p;
}

// CTAs per SM: 3 up to order 36 (at most 168 registers without a cap), 2
// above: at order 40 a 168-register (3-CTA) schedule fits without spills
// but measured 2% slower than the 203-register one (2680 against 2628 ms;
// paired groups of 4: 2560 against 2534 ms).
template <int N, int G, bool kPair = false, int kMinBlocks = (N <= 36 ? 3 : 2)>
__global__ void __launch_bounds__(128, kMinBlocks) ryser_dense_intc_kernel(DenseIntcArgs args) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np4 = args.np4;
  int* sC = reinterpret_cast<int*>(smem_raw);  // [N][np4] columns, then y0
  dd* red = reinterpret_cast<dd*>(sC + (size_t)(N + 1) * np4);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged = stage_to_smem(sC, args.colI, (uint32_t)(sizeof(int) * (N + 1) * np4), bar, args.err);
  const int* sY0 = sC + (size_t)N * np4;

  double H = 0.0, L = 0.0, m1 = 0.0;  // thread total (Sum2) and sum |term|
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;

  if (staged && b1 > b0) {
    const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
    int y[N];
#pragma unroll
    for (int j = 0; j < N; j++) y[j] = sY0[j];
    const uint64_t g = s0 ^ (s0 >> 1);
#pragma unroll 1
    for (int k = 0; k < N - 1; k++) {
      if ((g >> k) & 1) {
#pragma unroll
        for (int j = 0; j < N; j++) y[j] += sC[k * np4 + j];
      }
    }
    {
      const dd t0 = term_dd<N, G, kPair>(y);  // index s0 is even: sign +
      H = t0.hi;
      L = t0.lo;
      m1 = fabs(t0.hi);
    }

    const int* c0 = sC;
    const int* c1 = sC + np4;
    const int* c2 = sC + 2 * np4;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
    // one group of eight Gray steps, base + 1 .. base + 8 (signs - + - + - + - +);
    // the eighth flips column k8 >= 3 (kLast: only seven steps)
    auto group8 = [&](bool kLast) {
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      iupdate<N, +1>(y, c0, 0);
      dd t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      iupdate<N, +1>(y, c1, 0);
      t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
      iupdate<N, -1>(y, c0, 0);
      t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      iupdate<N, 0>(y, c2, s4);
      t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
      iupdate<N, +1>(y, c0, 0);
      t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      iupdate<N, -1>(y, c1, 0);
      t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
      iupdate<N, -1>(y, c0, 0);
      t = term_dd<N, G, kPair>(y);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      if (!kLast) {
        const uint64_t i8 = base + 8;
        const int k8 = __ffsll((long long)i8) - 1;
        const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
        iupdate<N, 0>(y, sC + k8 * np4, s8);
        t = term_dd<N, G, kPair>(y);
        sum2_add(H, L, t.hi, t.lo);
        m1 += fabs(t.hi);
      }
    };
#pragma unroll 1
    for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) group8(false);
    group8(true);  // last group of the range: index e0 belongs to the next range
  }

#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) m1 += __shfl_down_sync(0xffffffffu, m1, d);
  if ((threadIdx.x & 31) == 0 && m1 > 0.0) atomicAdd(args.sums, m1);
  const dd mine = two_sum(H, L);
  const dd bt = block_reduce_dd(mine, red);
  const double factor = ((N & 1) ? 2.0 : -2.0) * ldexp(1.0, -N);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

}  // namespace perm
