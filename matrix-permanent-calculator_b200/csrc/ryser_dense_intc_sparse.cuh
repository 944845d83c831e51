// ryser_dense_intc_sparse.cuh -- the certified int32-X walk
// (ryser_dense_intc.cuh: double-double products and sum) in the two-level
// row layout of ryser_dense_int_sparse.cuh.
//
// The host permutes the matrix so that columns 0..2 are three columns whose
// nonzeros lie in the fewest rows and those rows come first; the last
// NGO * G rows (NGO whole product groups) are zero in columns 0..2.  At the
// seven of every eight Gray steps that flip a column 0..2 only the inner
// rows change: the kernel updates them and multiplies their factors into
// P_out, the double-double product of the outer groups (an unevaluated
// pair, recomputed at the eighth step).  Factors are group values or, with
// kPair, int64 products of two consecutive groups of the same level (exact:
// the host proved every such pair's |product| < 2^53), as in the one-level
// kernel.  Every term is the same double-double product chain of
// ceil(N / G) group values (or fewer pair values) as there, so the error
// bound (8 ceil(n/G) + 256 + K^2) u^2 sum|t| carries over unchanged.
#pragma once
#include "ryser_dense_int_sparse.cuh"
#include "ryser_dense_intc.cuh"

namespace perm {

// int32 product of rows [j0, j1) (a group, possibly the short last inner one)
template <int N>
__device__ __forceinline__ int rows_int(const int (&y)[N], int j0, int j1) {
  return (int)rows_product<N>(y, j0, j1 - j0);
}

// factor i of one level: rows [J0, J1) in groups of G; with kPair, groups
// 2i and 2i + 1 multiplied in int64 and converted once
template <int N, int G, bool kPair, int J0, int J1>
__device__ __forceinline__ double level_factor(const int (&y)[N], int i) {
  constexpr int NG = (J1 - J0 + G - 1) / G;
  auto grp = [&](int g) {
    const int a = J0 + g * G;
    const int b = a + G < J1 ? a + G : J1;
    return rows_int<N>(y, a, b);
  };
  if (!kPair) return __int2double_rn(grp(i));
  long long v = grp(2 * i);
  if (2 * i + 1 < NG) v *= grp(2 * i + 1);
  return __ll2double_rn(v);
}

template <int G, bool kPair, int J0, int J1>
struct LevelFactors {
  static constexpr int NG = (J1 - J0 + G - 1) / G;
  static constexpr int value = kPair ? (NG + 1) / 2 : NG;
};

// p *= factor (double-double times an exact double, 3 operations)
__device__ __forceinline__ void dd_mul_exact(dd& p, double v) {
  const double h = __dmul_rn(p.hi, v);
  const double l = __fma_rn(p.hi, v, -h);
  p.lo = __fma_rn(p.lo, v, l);
  p.hi = h;
}

// P_out: double-double product of the outer level's factors
template <int N, int G, bool kPair, int NGO>
__device__ __forceinline__ dd outer_dd(const int (&y)[N]) {
  constexpr int RI = N - G * NGO;
  constexpr int F = LevelFactors<G, kPair, RI, N>::value;
  dd p = {level_factor<N, G, kPair, RI, N>(y, 0), 0.0};
  if (F > 1) {
    const double v = level_factor<N, G, kPair, RI, N>(y, 1);
    const double h = __dmul_rn(p.hi, v);
    p.lo = __fma_rn(p.hi, v, -h);
    p.hi = h;
  }
#pragma unroll
  for (int i = 2; i < F; i++) dd_mul_exact(p, level_factor<N, G, kPair, RI, N>(y, i));
  return p;
}

// term: P_out times the inner level's factors
template <int N, int G, bool kPair, int NGO>
__device__ __forceinline__ dd inner_dd(const int (&y)[N], dd pout) {
  constexpr int RI = N - G * NGO;
  constexpr int F = LevelFactors<G, kPair, 0, RI>::value;
#pragma unroll
  for (int i = 0; i < F; i++) dd_mul_exact(pout, level_factor<N, G, kPair, 0, RI>(y, i));
  return pout;
}

template <int N, int G, bool kPair, int NGO, int kMinBlocks = (N <= 36 ? 3 : 2)>
__global__ void __launch_bounds__(128, kMinBlocks) ryser_dense_intc_sparse_kernel(DenseIntcArgs args) {
  static_assert(NGO >= 1 && G * NGO + 3 <= N, "outer groups must leave inner rows");
  constexpr int RI = N - G * NGO;
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
    dd pout = outer_dd<N, G, kPair, NGO>(y);
    {
      const dd t0 = inner_dd<N, G, kPair, NGO>(y, pout);  // index s0 is even: sign +
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
      iupdate_rows<N, RI, +1>(y, c0, 0);
      dd t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      iupdate_rows<N, RI, +1>(y, c1, 0);
      t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
      iupdate_rows<N, RI, -1>(y, c0, 0);
      t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      iupdate_rows<N, RI, 0>(y, c2, s4);
      t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
      iupdate_rows<N, RI, +1>(y, c0, 0);
      t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      iupdate_rows<N, RI, -1>(y, c1, 0);
      t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
      iupdate_rows<N, RI, -1>(y, c0, 0);
      t = inner_dd<N, G, kPair, NGO>(y, pout);
      sum2_add(H, L, -t.hi, -t.lo);
      m1 += fabs(t.hi);
      if (!kLast) {
        const uint64_t i8 = base + 8;
        const int k8 = __ffsll((long long)i8) - 1;
        const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
        iupdate_rows<N, N, 0>(y, sC + k8 * np4, s8);
        pout = outer_dd<N, G, kPair, NGO>(y);
        t = inner_dd<N, G, kPair, NGO>(y, pout);
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

// Three-level row layout (as ryser_dense_int_3l_kernel): column 0 touches
// rows [0, R1) only, columns 1 and 2 rows [0, R2) only, R1 = NG1 G and
// R2 = R1 + NG2 G.  P23 is the double-double product of P_out and the
// second level's factors; a column-0 step multiplies the first level's
// factors into P23, a column-1/2 step recomputes P23 first, the eighth step
// P_out too.  The chain of a term has the same <= ceil(N/G) factors, so the
// bound carries over.
template <int N, int G, bool kPair, int J0, int J1>
__device__ __forceinline__ dd chain_from(const int (&y)[N], dd p) {
  constexpr int F = LevelFactors<G, kPair, J0, J1>::value;
#pragma unroll
  for (int i = 0; i < F; i++) dd_mul_exact(p, level_factor<N, G, kPair, J0, J1>(y, i));
  return p;
}

template <int N, int G, bool kPair, int NG1, int NG2, int kMinBlocks = (N <= 36 ? 3 : 2)>
__global__ void __launch_bounds__(128, kMinBlocks) ryser_dense_intc_3l_kernel(DenseIntcArgs args) {
  constexpr int R1 = NG1 * G, R2 = R1 + NG2 * G;
  static_assert(NG1 >= 1 && NG2 >= 1 && R2 + 2 <= N, "levels must leave outer rows");
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
    auto outer = [&]() {
      constexpr int F = LevelFactors<G, kPair, R2, N>::value;
      dd p = {level_factor<N, G, kPair, R2, N>(y, 0), 0.0};
      if (F > 1) {
        const double v = level_factor<N, G, kPair, R2, N>(y, 1);
        const double h = __dmul_rn(p.hi, v);
        p.lo = __fma_rn(p.hi, v, -h);
        p.hi = h;
      }
#pragma unroll
      for (int i = 2; i < F; i++) dd_mul_exact(p, level_factor<N, G, kPair, R2, N>(y, i));
      return p;
    };
    dd pout = outer();
    dd p23 = chain_from<N, G, kPair, R1, R2>(y, pout);
    {
      const dd t0 = chain_from<N, G, kPair, 0, R1>(y, p23);  // index s0 is even: sign +
      H = t0.hi;
      L = t0.lo;
      m1 = fabs(t0.hi);
    }
    const int* c0 = sC;
    const int* c1 = sC + np4;
    const int* c2 = sC + 2 * np4;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
    auto add = [&](const dd& t, bool neg) {
      if (neg)
        sum2_add(H, L, -t.hi, -t.lo);
      else
        sum2_add(H, L, t.hi, t.lo);
      m1 += fabs(t.hi);
    };
    auto step0 = [&](int sg, bool neg) {
      if (sg > 0)
        iupdate_rows<N, R1, +1>(y, c0, 0);
      else
        iupdate_rows<N, R1, -1>(y, c0, 0);
      add(chain_from<N, G, kPair, 0, R1>(y, p23), neg);
    };
    auto step12 = [&](const int* c, int sg, int ks, bool neg) {
      if (ks > 0)
        iupdate_rows<N, R2, +1>(y, c, 0);
      else if (ks < 0)
        iupdate_rows<N, R2, -1>(y, c, 0);
      else
        iupdate_rows<N, R2, 0>(y, c, sg);
      p23 = chain_from<N, G, kPair, R1, R2>(y, pout);
      add(chain_from<N, G, kPair, 0, R1>(y, p23), neg);
    };
    // one group of eight Gray steps, base + 1 .. base + 8 (signs - + - + - + - +)
    auto group8 = [&](bool kLast) {
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      step0(+1, true);
      step12(c1, 1, +1, false);
      step0(-1, true);
      step12(c2, s4, 0, false);
      step0(+1, true);
      step12(c1, -1, -1, false);
      step0(-1, true);
      if (!kLast) {
        const uint64_t i8 = base + 8;
        const int k8 = __ffsll((long long)i8) - 1;
        const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
        iupdate_rows<N, N, 0>(y, sC + k8 * np4, s8);
        pout = outer();
        p23 = chain_from<N, G, kPair, R1, R2>(y, pout);
        add(chain_from<N, G, kPair, 0, R1>(y, p23), false);
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
