// ryser_dense_int_sparse.cuh -- the int32-X walk (ryser_dense_int.cuh) in a
// two-level row layout.
//
// Seven of every eight Gray steps flip column 0, 1 or 2.  The host permutes
// the matrix (the permanent is invariant under row and column permutations)
// so that columns 0..2 are three columns whose nonzeros lie in the fewest
// rows and those rows come first; the last NGO * G rows ("outer" rows, NGO
// whole product groups) are then zero in columns 0..2.  At the seven steps
// that flip a column 0..2 the kernel updates only the inner rows
// [0, N - NGO G) and multiplies their groups by P_out, the FP64 product of
// the outer groups, which changes only at the eighth step (a column >= 3),
// where every row is updated and P_out is recomputed.  Even a dense matrix
// has such rows: at density 1/2 about n/8 rows are zero in any three
// columns, and the best of the C(n-1, 3) triples does better (the order-40
// bench matrix: 15 of 40 rows, three groups of 5).
//
// Roundings per term are those of the dense int32-X walk: the inner groups
// (ceil((N - NGO G) / G) of them) and the NGO outer groups give ceil(N / G)
// FP64 factors, combined by ceil(N / G) - 1 multiplies.  The host proves
// every group's |product| < 2^31 for this layout's grouping (inner groups
// from row 0, outer groups from row N - NGO G).
#pragma once
#include "ryser_dense_int.cuh"

namespace perm {

// exact int32 product of y over rows [J0, J1) converted to FP64
template <int N, int J0, int J1>
__device__ __forceinline__ double rows_value(const int (&y)[N]) {
  uint32_t pr = (uint32_t)y[J0];
#pragma unroll
  for (int j = J0 + 1; j < J1; j++) pr = pr * (uint32_t)y[j];
  return __int2double_rn((int)pr);
}

// value of inner group g (rows [gG, min(gG + G, RI)))
template <int N, int G, int RI>
__device__ __forceinline__ double inner_group(const int (&y)[N], int g) {
  const int j0 = g * G;
  uint32_t pr = (uint32_t)y[j0];
#pragma unroll
  for (int t = 1; t < G; t++)
    if (j0 + t < RI) pr = pr * (uint32_t)y[j0 + t];
  return __int2double_rn((int)pr);
}

// P_out: product of the NGO outer groups (rows [RI, N))
template <int N, int G, int NGO>
__device__ __forceinline__ double outer_product(const int (&y)[N]) {
  constexpr int RI = N - G * NGO;
  double p = 1.0;
#pragma unroll
  for (int g = 0; g < NGO; g++) {
    const int j0 = RI + g * G;
    uint32_t pr = (uint32_t)y[j0];
#pragma unroll
    for (int t = 1; t < G; t++) pr = pr * (uint32_t)y[j0 + t];
    const double d = __int2double_rn((int)pr);
    p = g == 0 ? d : p * d;
  }
  return p;
}

// term = P_out * prod of the inner groups, four multiply chains (P_out is
// the first factor of chain 0)
template <int N, int G, int NGO>
__device__ __forceinline__ double inner_term(const int (&y)[N], double pout) {
  constexpr int RI = N - G * NGO;
  constexpr int NGI = (RI + G - 1) / G;
  constexpr int F = NGI + 1;  // factors: P_out, then the inner groups
  double c0 = pout, c1 = 1.0, c2 = 1.0, c3 = 1.0;
#pragma unroll
  for (int g = 0; g < NGI; g++) {
    const double d = inner_group<N, G, RI>(y, g);
    const int f = g + 1;
    if ((f & 3) == 0) c0 = c0 * d;
    if ((f & 3) == 1) c1 = f < 4 ? d : c1 * d;
    if ((f & 3) == 2) c2 = f < 4 ? d : c2 * d;
    if ((f & 3) == 3) c3 = f < 4 ? d : c3 * d;
  }
  if (F >= 4) return (c0 * c1) * (c2 * c3);
  if (F == 3) return (c0 * c1) * c2;
  return c0 * c1;
}

// rows [0, R) of y += s * column (compile-time sign when kSign != 0)
template <int N, int R, int kSign>
__device__ __forceinline__ void iupdate_rows(int (&y)[N], const int* col, int s) {
#pragma unroll
  for (int j = 0; j < R; j += 4) {
    const int4 v = lds4i(col + j);
    const int c[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
      if (j + t < R) {
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

template <int N, int G, int NGO>
__global__ void __launch_bounds__(128) ryser_dense_int_sparse_kernel(DenseIntArgs args) {
  static_assert(NGO >= 1 && G * NGO + 3 <= N, "outer groups must leave inner rows");
  constexpr int RI = N - G * NGO;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np4 = args.np4;
  int* sC = reinterpret_cast<int*>(smem_raw);  // [N][np4] columns, then y0
  dd* red = reinterpret_cast<dd*>(sC + (size_t)(N + 1) * np4);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged = stage_to_smem(sC, args.colI, (uint32_t)(sizeof(int) * (N + 1) * np4), bar, args.err);
  const int* sY0 = sC + (size_t)N * np4;

  Acc acc;
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
    double pout = outer_product<N, G, NGO>(y);
    acc.add(inner_term<N, G, NGO>(y, pout));

    const int* c0 = sC;
    const int* c1 = sC + np4;
    const int* c2 = sC + 2 * np4;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
    // one group of eight Gray steps, base + 1 .. base + 8 (signs - + - + - + - +)
    auto seven = [&](int s4, double (&t)[7]) {
      iupdate_rows<N, RI, +1>(y, c0, 0);
      t[0] = inner_term<N, G, NGO>(y, pout);
      iupdate_rows<N, RI, +1>(y, c1, 0);
      t[1] = inner_term<N, G, NGO>(y, pout);
      iupdate_rows<N, RI, -1>(y, c0, 0);
      t[2] = inner_term<N, G, NGO>(y, pout);
      iupdate_rows<N, RI, 0>(y, c2, s4);
      t[3] = inner_term<N, G, NGO>(y, pout);
      iupdate_rows<N, RI, +1>(y, c0, 0);
      t[4] = inner_term<N, G, NGO>(y, pout);
      iupdate_rows<N, RI, -1>(y, c1, 0);
      t[5] = inner_term<N, G, NGO>(y, pout);
      iupdate_rows<N, RI, -1>(y, c0, 0);
      t[6] = inner_term<N, G, NGO>(y, pout);
    };
#pragma unroll 1
    for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) {
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      const uint64_t i8 = base + 8;
      const int k8 = __ffsll((long long)i8) - 1;
      const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
      double t[7];
      seven(s4, t);
      // the eighth step flips column k8 >= 3: every row may change
      iupdate_rows<N, N, 0>(y, sC + k8 * np4, s8);
      pout = outer_product<N, G, NGO>(y);
      const double t8 = inner_term<N, G, NGO>(y, pout);
      acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) + (t8 - t[6])));
    }
    {
      // last group of the range: index e0 belongs to the next range
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      double t[7];
      seven(s4, t);
      acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) - t[6]));
    }
  }

  dd bt = block_reduce_dd(acc.value(), red);
  const double factor = ((N & 1) ? 2.0 : -2.0) * ldexp(1.0, -N);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

// Three-level row layout: column 0 (flipped at every other Gray step)
// touches rows [0, R1) only, columns 1 and 2 (three steps in eight) rows
// [0, R2) only, R1 = NG1 G and R2 = R1 + NG2 G; the host permutes the matrix
// accordingly (rows of a later level may sit in an earlier one: their zero
// entries make the extra updates no-ops).  Column-0 steps update R1 rows and
// multiply their NG1 groups by P23 = P2 P_out; column-1/2 steps update R2
// rows and recompute P1, P2 and P23; the other step of each eight updates
// every row and recomputes P_out too.  Terms keep ceil(N/G) FP64 factors
// combined by ceil(N/G) - 1 multiplies.
template <int N, int J0, int J1, int G>
__device__ __forceinline__ double level_product(const int (&y)[N]) {
  constexpr int NG = (J1 - J0 + G - 1) / G;
  double p = 1.0;
#pragma unroll
  for (int g = 0; g < NG; g++) {
    const int a = J0 + g * G;
    const uint32_t pr = rows_product<N>(y, a, a + G <= J1 ? G : J1 - a);
    const double d = __int2double_rn((int)pr);
    p = g == 0 ? d : p * d;
  }
  return p;
}

template <int N, int G, int NG1, int NG2>
__global__ void __launch_bounds__(128) ryser_dense_int_3l_kernel(DenseIntArgs args) {
  constexpr int R1 = NG1 * G, R2 = R1 + NG2 * G;
  static_assert(NG1 >= 1 && NG2 >= 1 && R2 + 2 <= N, "levels must leave outer rows");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np4 = args.np4;
  int* sC = reinterpret_cast<int*>(smem_raw);  // [N][np4] columns, then y0
  dd* red = reinterpret_cast<dd*>(sC + (size_t)(N + 1) * np4);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged = stage_to_smem(sC, args.colI, (uint32_t)(sizeof(int) * (N + 1) * np4), bar, args.err);
  const int* sY0 = sC + (size_t)N * np4;

  Acc acc;
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
    double pout = level_product<N, R2, N, G>(y);
    double p23 = level_product<N, R1, R2, G>(y) * pout;
    acc.add(level_product<N, 0, R1, G>(y) * p23);

    const int* c0 = sC;
    const int* c1 = sC + np4;
    const int* c2 = sC + 2 * np4;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
    // column-0 step: level 1 only; column-1/2 step: levels 1 and 2
    auto step0 = [&](int sg) {
      if (sg > 0)
        iupdate_rows<N, R1, +1>(y, c0, 0);
      else
        iupdate_rows<N, R1, -1>(y, c0, 0);
      return level_product<N, 0, R1, G>(y) * p23;
    };
    auto step12 = [&](const int* c, int sg, bool known, int ks) {
      if (known && ks > 0)
        iupdate_rows<N, R2, +1>(y, c, 0);
      else if (known)
        iupdate_rows<N, R2, -1>(y, c, 0);
      else
        iupdate_rows<N, R2, 0>(y, c, sg);
      p23 = level_product<N, R1, R2, G>(y) * pout;
      return level_product<N, 0, R1, G>(y) * p23;
    };
    auto seven = [&](int s4, double (&t)[7]) {
      t[0] = step0(+1);
      t[1] = step12(c1, 1, true, +1);
      t[2] = step0(-1);
      t[3] = step12(c2, s4, false, 0);
      t[4] = step0(+1);
      t[5] = step12(c1, -1, true, -1);
      t[6] = step0(-1);
    };
#pragma unroll 1
    for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) {
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      const uint64_t i8 = base + 8;
      const int k8 = __ffsll((long long)i8) - 1;
      const int s8 = ((i8 >> (k8 + 1)) & 1) ? -1 : 1;
      double t[7];
      seven(s4, t);
      iupdate_rows<N, N, 0>(y, sC + k8 * np4, s8);
      pout = level_product<N, R2, N, G>(y);
      p23 = level_product<N, R1, R2, G>(y) * pout;
      const double t8 = level_product<N, 0, R1, G>(y) * p23;
      acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) + (t8 - t[6])));
    }
    {
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      double t[7];
      seven(s4, t);
      acc.add(((t[1] - t[0]) + (t[3] - t[2])) + ((t[5] - t[4]) - t[6]));
    }
  }

  dd bt = block_reduce_dd(acc.value(), red);
  const double factor = ((N & 1) ? 2.0 : -2.0) * ldexp(1.0, -N);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

}  // namespace perm
