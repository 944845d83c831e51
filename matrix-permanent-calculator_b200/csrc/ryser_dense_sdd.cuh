// ryser_dense_sdd.cuh -- exact permanent of real matrices with a certified
// error bound: split X, double-double products and sum ("split-dd").
//
// Same Nijenhuis-Wilf Gray walk, aligned thread ranges and reductions as
// ryser_dense.cuh (the reference's kernel_xshared_coalescing_mshared,
// gpu_exact_dense.cu:330-399, restated).  The operand is the split-X image
// (ryser_dense_split.cuh): every entry a = ah + al with ah on its row's grid
// 2^-q_j, so the coarse row sums xh are EXACT in FP64 and the remainders xl
// are tiny (|al| <= 2^-(q_j+1)).  The pair (xh_j, xl_j) is therefore an
// accurate double-double value of x_j for two FP64 additions per update
// (the double-double kernel's TwoSum update takes seven), and:
//  * the n-way product is formed in double-double on these pairs: exact high
//    product and its error from one FMA, both cross terms by FMAs (4
//    operations per factor, four independent chains);
//  * terms are summed with TwoSum into a (hi, lo) pair per Gray group of
//    eight (Sum2 of Ogita, Rump and Oishi) and the groups into the thread
//    total the same way;
//  * the walk sums |hi| of its own terms: the error bound uses the exact
//    cancellation scale sum|t|.
// About 6n + 10 FP64 operations per Gray step against 11n + 8 for the
// double-double kernel, with a relative error of order n u^2 sum|t| / |perm|.
//
// Three layouts:
//  * ryser_dense_sdd_kernel<N>: every step updates and multiplies all n
//    rows (rolled step loop: the two X vectors fill the register file);
//  * ryser_sparse_sdd_kernel<N, R>: for sparse matrices.  Seven of every
//    eight Gray steps flip column 0, 1 or 2; the host permutes columns so
//    these are three columns whose nonzeros lie in few rows, and rows so that
//    those rows come first (rows 0..R-1).  At those seven steps only rows
//    0..R-1 change: the kernel updates and multiplies them alone and reuses
//    the product of rows R..n-1, which it recomputes at the eighth step (the
//    one that flips a column >= 3).  About (7 (6R + 9) + 6n + 5) / 8
//    operations per step: 78 instead of 221 for n = 36, R = 8;
//  * ryser_sdd_3l_kernel<N, R1, R2>: three levels of rows, for column 0's
//    rows (updated at every other step), the further rows of columns 1 and
//    2 (three steps in eight) and the rest (the eighth step).
#pragma once
#include "ryser_dense.cuh"

namespace perm {

struct DenseSddArgs {
  const double* img;  // [colH: n x np][colL: n x np][x0h: np][x0l: np] (split-X image)
  int np;
  int m;
  uint64_t block0, nblocks;
  dd* partials;
  unsigned* ticket;
  double* out;
  double* sums;  // sums[0] += sum |term| over the walked terms (zeroed by the host)
  int* err;
};

// p *= (xh + xl), both unevaluated pairs: exact high product and its error
// from one FMA, both cross terms by FMAs (the xl x p.lo term is below u^2).
__device__ __forceinline__ void pair_mul(dd& p, double xh, double xl) {
  const double h = __dmul_rn(p.hi, xh);
  double l = __fma_rn(p.hi, xh, -h);
  l = __fma_rn(p.hi, xl, l);
  l = __fma_rn(p.lo, xh, l);
  p.hi = h;
  p.lo = l;
}

// Double-double product of rows [J0, J1) in up to four chains.
template <int J0, int J1, int N>
__device__ __forceinline__ dd rows_product(const double (&xh)[N], const double (&xl)[N]) {
  constexpr int C = (J1 - J0) >= 4 ? 4 : (J1 - J0);
  dd c[4];
#pragma unroll
  for (int t = 0; t < C; t++) c[t] = {xh[J0 + t], xl[J0 + t]};
#pragma unroll
  for (int j = J0 + C; j < J1; j++) pair_mul(c[(j - J0) % C], xh[j], xl[j]);
  if (C == 4) {
    pair_mul(c[0], c[1].hi, c[1].lo);
    pair_mul(c[2], c[3].hi, c[3].lo);
    pair_mul(c[0], c[2].hi, c[2].lo);
  } else {
#pragma unroll
    for (int t = 1; t < C; t++) pair_mul(c[0], c[t].hi, c[t].lo);
  }
  return c[0];
}

// rows [J0, J1) of X += s * column (s = +-1; compile-time when kSign != 0)
template <int J0, int J1, int kSign, int N>
__device__ __forceinline__ void pair_update(double (&xh)[N], double (&xl)[N], const double* colH,
                                            const double* colL, double s) {
#pragma unroll
  for (int j = J0; j < J1; j += 2) {
    double h0, h1 = 0.0, l0, l1 = 0.0;
    if (j + 1 < J1) {
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
      xh[j] = __dadd_rn(xh[j], h0);
      xl[j] = __dadd_rn(xl[j], l0);
      if (j + 1 < J1) {
        xh[j + 1] = __dadd_rn(xh[j + 1], h1);
        xl[j + 1] = __dadd_rn(xl[j + 1], l1);
      }
    } else if (kSign < 0) {
      xh[j] = __dsub_rn(xh[j], h0);
      xl[j] = __dsub_rn(xl[j], l0);
      if (j + 1 < J1) {
        xh[j + 1] = __dsub_rn(xh[j + 1], h1);
        xl[j + 1] = __dsub_rn(xl[j + 1], l1);
      }
    } else {
      xh[j] = __fma_rn(s, h0, xh[j]);
      xl[j] = __fma_rn(s, l0, xl[j]);
      if (j + 1 < J1) {
        xh[j + 1] = __fma_rn(s, h1, xh[j + 1]);
        xl[j + 1] = __fma_rn(s, l1, xl[j + 1]);
      }
    }
  }
}

// Thread start state: X at Gray index s0 directly from gray(s0).
template <int N>
__device__ __forceinline__ void sdd_start(double (&xh)[N], double (&xl)[N], const double* sH, const double* sL,
                                          const double* sX0h, const double* sX0l, int np, uint64_t s0) {
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
        xh[j] = __dadd_rn(xh[j], sH[k * np + j]);
        xl[j] = __dadd_rn(xl[j], sL[k * np + j]);
      }
    }
  }
}

__host__ __device__ inline size_t dense_sdd_smem_bytes(int n) {
  const int np = (n + 1) & ~1;
  return sizeof(double) * (2 * (size_t)n * np + 2 * np) + 32 * sizeof(dd) + 16;
}

// Shared tail: sum |term| to the host accumulator, double-double block and
// grid reduction of the thread totals.
__device__ __forceinline__ void sdd_finish(double H, double L, double m1, const DenseSddArgs& args, dd* red,
                                           double factor) {
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) m1 += __shfl_down_sync(0xffffffffu, m1, d);
  if ((threadIdx.x & 31) == 0 && m1 > 0.0) atomicAdd(args.sums, m1);
  const dd bt = block_reduce_dd(two_sum(H, L), red);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

// CTAs per SM by order: the two X vectors plus the product chains fit 3 CTAs
// (168 registers) up to order 28, 2 above.
template <int N>
__global__ void __launch_bounds__(128, (N <= 28 ? 3 : 2)) ryser_dense_sdd_kernel(DenseSddArgs args) {
  static_assert(N >= 4, "orders below 4 use the other kernels");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sH = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  const double* sL = sH + (size_t)N * np;
  const double* sX0h = sL + (size_t)N * np;
  const double* sX0l = sX0h + np;
  dd* red = reinterpret_cast<dd*>(sH + 2 * (size_t)N * np + 2 * np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged =
      stage_to_smem(sH, args.img, (uint32_t)(sizeof(double) * (2 * (size_t)N * np + 2 * np)), bar, args.err);

  double H = 0.0, L = 0.0, m1 = 0.0;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;

  if (staged && b1 > b0) {
    const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
    double xh[N], xl[N];
    sdd_start<N>(xh, xl, sH, sL, sX0h, sX0l, np, s0);
    const dd t0 = rows_product<0, N, N>(xh, xl);  // index s0 is even: sign +
    H = t0.hi;
    L = t0.lo;
    m1 = fabs(t0.hi);
    // groups of eight steps (s0 and e0 are multiples of 8); the last group
    // of the range has seven (index e0 belongs to the next range)
#pragma unroll 1
    for (uint64_t base = s0; base < e0; base += 8) {
      const uint64_t top = base + 8 < e0 ? base + 8 : e0 - 1;
      double gs = 0.0, gc = 0.0, ma = 0.0;
#pragma unroll 1
      for (uint64_t i = base + 1; i <= top; i++) {
        const int k = __ffsll((long long)i) - 1;
        const double sg = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
        pair_update<0, N, 0, N>(xh, xl, sH + k * np, sL + k * np, sg);
        const dd t = rows_product<0, N, N>(xh, xl);
        if (i & 1)
          sum2_add(gs, gc, -t.hi, -t.lo);
        else
          sum2_add(gs, gc, t.hi, t.lo);
        ma += fabs(t.hi);
      }
      sum2_add(H, L, gs, gc);
      m1 += ma;
    }
  }
  sdd_finish(H, L, m1, args, red, (N & 1) ? 2.0 : -2.0);
}

// The sparse layout.  Columns 0, 1, 2 are zero outside rows 0..R-1 (the host
// checked it); P_out is the product of rows R..N-1, constant between two
// flips of a column >= 3.  Rows 0..R-1 of X live in registers; rows R..N-1
// are touched only at the eighth step of a group, so they live in shared
// memory as (xh, xl) pairs in a [row][thread] layout (consecutive lanes,
// consecutive 16-byte words: conflict-free), which keeps the register file
// for the unrolled inner steps.
__host__ __device__ inline size_t sparse_sdd_smem_bytes(int n, int r, int threads) {
  return dense_sdd_smem_bytes(n) + 16 * (size_t)(n - r) * threads;
}

// Start state of a layout with rows [0, R) in registers and rows [R, N) in
// shared memory ([row][thread] (xh, xl) pairs): X at Gray index s0.
template <int N, int R>
__device__ __forceinline__ void sdd_split_start(double (&xh)[R], double (&xl)[R], double2* sOut, const double* sH,
                                                const double* sL, const double* sX0h, const double* sX0l, int np,
                                                uint64_t s0, int T, int me) {
  const uint64_t g0 = s0 ^ (s0 >> 1);
#pragma unroll
  for (int j = 0; j < R; j++) {
    xh[j] = sX0h[j];
    xl[j] = sX0l[j];
  }
#pragma unroll 1
  for (int k = 0; k < N - 1; k++) {
    if ((g0 >> k) & 1) {
#pragma unroll
      for (int j = 0; j < R; j++) {
        xh[j] = __dadd_rn(xh[j], sH[k * np + j]);
        xl[j] = __dadd_rn(xl[j], sL[k * np + j]);
      }
    }
  }
#pragma unroll 1
  for (int j = R; j < N; j++) {
    double vh = sX0h[j], vl = sX0l[j];
    for (int k = 0; k < N - 1; k++) {
      if ((g0 >> k) & 1) {
        vh = __dadd_rn(vh, sH[k * np + j]);
        vl = __dadd_rn(vl, sL[k * np + j]);
      }
    }
    sOut[(j - R) * T + me] = make_double2(vh, vl);
  }
}

// Product of the shared-memory rows [R, N) (four chains), after adding
// s * column k to them when `upd`.  kRuns: rolled over runs of four rows
// (the three-level kernel: fully unrolled, the compiler hoists the rows'
// loads ahead of the products and spills at some orders); fully unrolled
// otherwise (the sparse layout's unrolled walk, where the eighth step is a
// third of the work, runs 1.3x slower with the rolled runs at n = 36, R = 6).
template <int N, int R, bool kRuns = false>
__device__ __forceinline__ dd sdd_outer(double2* sOut, const double* sH, const double* sL, int np, int T, int me,
                                        bool upd, int k, double s) {
  dd c[4];
  constexpr int C = (N - R) >= 4 ? 4 : (N - R);
  if constexpr (!kRuns) {
#pragma unroll
    for (int j = R; j < N; j++) {
      double2 v = sOut[(j - R) * T + me];
      if (upd) {
        v.x = __fma_rn(s, sH[k * np + j], v.x);
        v.y = __fma_rn(s, sL[k * np + j], v.y);
        sOut[(j - R) * T + me] = v;
      }
      const int t = (j - R) & 3;
      if (j - R < 4)
        c[t] = {v.x, v.y};
      else
        pair_mul(c[t], v.x, v.y);
    }
#pragma unroll
    for (int t = 1; t < C; t++) pair_mul(c[0], c[t].hi, c[t].lo);
    return c[0];
  }
#pragma unroll
  for (int t = 0; t < C; t++) {
    double2 v = sOut[t * T + me];
    if (upd) {
      v.x = __fma_rn(s, sH[k * np + R + t], v.x);
      v.y = __fma_rn(s, sL[k * np + R + t], v.y);
      sOut[t * T + me] = v;
    }
    c[t] = {v.x, v.y};
  }
#pragma unroll 1
  for (int j0 = R + 4; j0 < N; j0 += 4) {
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int j = j0 + t;
      if (j < N) {
        double2 v = sOut[(j - R) * T + me];
        if (upd) {
          v.x = __fma_rn(s, sH[k * np + j], v.x);
          v.y = __fma_rn(s, sL[k * np + j], v.y);
          sOut[(j - R) * T + me] = v;
        }
        pair_mul(c[t], v.x, v.y);
      }
    }
  }
#pragma unroll
  for (int t = 1; t < C; t++) pair_mul(c[0], c[t].hi, c[t].lo);
  return c[0];
}

// kRolled: the step loop is rolled (a runtime column at every step, the
// outer rows updated and P_out recomputed when it is >= 3), which keeps the
// register file to the inner rows for inner-row counts of 20 and more,
// where the unrolled eight-step group spills.
template <int N, int R, int kMinBlocks = 2, bool kRolled = false>
__global__ void __launch_bounds__(128, kMinBlocks) ryser_sparse_sdd_kernel(DenseSddArgs args) {
  static_assert(R >= 2 && R + 2 <= N && (R & 1) == 0, "inner rows: even, and outer rows must remain");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sH = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  const double* sL = sH + (size_t)N * np;
  const double* sX0h = sL + (size_t)N * np;
  const double* sX0l = sX0h + np;
  dd* red = reinterpret_cast<dd*>(sH + 2 * (size_t)N * np + 2 * np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  double2* sOut = reinterpret_cast<double2*>(bar + 2);  // [N - R][blockDim.x]
  const bool staged =
      stage_to_smem(sH, args.img, (uint32_t)(sizeof(double) * (2 * (size_t)N * np + 2 * np)), bar, args.err);

  double H = 0.0, L = 0.0, m1 = 0.0;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;
  const int T = blockDim.x, me = threadIdx.x;

  if (staged && b1 > b0) {
    const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
    // start state: inner rows in registers, outer rows in shared memory
    double xh[R], xl[R];
    sdd_split_start<N, R>(xh, xl, sOut, sH, sL, sX0h, sX0l, np, s0, T, me);
    // product of the outer rows, optionally after adding s * column k to them
    auto outer = [&](bool upd, int k, double s) { return sdd_outer<N, R>(sOut, sH, sL, np, T, me, upd, k, s); };
    dd pout = outer(false, 0, 0.0);
    auto inner_term = [&]() {
      dd t = rows_product<0, R, R>(xh, xl);
      pair_mul(t, pout.hi, pout.lo);
      return t;
    };
    {
      const dd t0 = inner_term();  // index s0 is even: sign +
      H = t0.hi;
      L = t0.lo;
      m1 = fabs(t0.hi);
    }
    if constexpr (kRolled) {
#pragma unroll 1
      for (uint64_t base = s0; base < e0; base += 8) {
        const uint64_t top = base + 8 < e0 ? base + 8 : e0 - 1;
        double gs = 0.0, gc = 0.0, ma = 0.0;
#pragma unroll 1
        for (uint64_t i = base + 1; i <= top; i++) {
          const int k = __ffsll((long long)i) - 1;
          const double sg = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
          pair_update<0, R, 0, R>(xh, xl, sH + k * np, sL + k * np, sg);
          if (k >= 3) pout = outer(true, k, sg);  // the eighth step of a group: every row may change
          const dd t = inner_term();
          if (i & 1)
            sum2_add(gs, gc, -t.hi, -t.lo);
          else
            sum2_add(gs, gc, t.hi, t.lo);
          ma += fabs(t.hi);
        }
        sum2_add(H, L, gs, gc);
        m1 += ma;
      }
    } else {
    const double *h0 = sH, *h1 = sH + np, *h2 = sH + 2 * np;
    const double *l0 = sL, *l1 = sL + np, *l2 = sL + 2 * np;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
    auto group8 = [&](bool kLast) {
      const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
      pair_update<0, R, +1, R>(xh, xl, h0, l0, 0.0);
      dd t = inner_term();
      double gs = -t.hi, gc = -t.lo, ma = fabs(t.hi);
      pair_update<0, R, +1, R>(xh, xl, h1, l1, 0.0);
      t = inner_term();
      sum2_add(gs, gc, t.hi, t.lo);
      ma += fabs(t.hi);
      pair_update<0, R, -1, R>(xh, xl, h0, l0, 0.0);
      t = inner_term();
      sum2_add(gs, gc, -t.hi, -t.lo);
      ma += fabs(t.hi);
      pair_update<0, R, 0, R>(xh, xl, h2, l2, s4);
      t = inner_term();
      sum2_add(gs, gc, t.hi, t.lo);
      ma += fabs(t.hi);
      pair_update<0, R, +1, R>(xh, xl, h0, l0, 0.0);
      t = inner_term();
      sum2_add(gs, gc, -t.hi, -t.lo);
      ma += fabs(t.hi);
      pair_update<0, R, -1, R>(xh, xl, h1, l1, 0.0);
      t = inner_term();
      sum2_add(gs, gc, t.hi, t.lo);
      ma += fabs(t.hi);
      pair_update<0, R, -1, R>(xh, xl, h0, l0, 0.0);
      t = inner_term();
      sum2_add(gs, gc, -t.hi, -t.lo);
      ma += fabs(t.hi);
      if (!kLast) {
        // the eighth step flips column k8 >= 3: every row may change
        const uint64_t i8 = base + 8;
        const int k8 = __ffsll((long long)i8) - 1;
        const double s8 = ((i8 >> (k8 + 1)) & 1) ? -1.0 : 1.0;
        pair_update<0, R, 0, R>(xh, xl, sH + k8 * np, sL + k8 * np, s8);
        pout = outer(true, k8, s8);
        t = inner_term();
        sum2_add(gs, gc, t.hi, t.lo);
        ma += fabs(t.hi);
      }
      sum2_add(H, L, gs, gc);
      m1 += ma;
    };
#pragma unroll 1
    for (uint64_t gi = 0; gi + 1 < groups; gi++, base += 8) group8(false);
    group8(true);
    }
  }
  sdd_finish(H, L, m1, args, red, (N & 1) ? 2.0 : -2.0);
}

// Three-level layout (rolled step loop).  Column 0 is zero outside rows
// [0, R1) and columns 1, 2 outside rows [0, R2) (the host permuted the
// matrix so); rows [0, R2) live in registers, rows [R2, N) in shared memory
// as in the sparse layout.  With P1, P2, P3 the double-double products of
// rows [0, R1), [R1, R2), [R2, N) and P23 = P2 P3: a column-0 step (half of
// all steps) updates rows [0, R1) and multiplies P1 into P23; a column-1/2
// step (three in eight) updates rows [0, R2) and re-forms P2 and P23; the
// eighth step of a group updates every row and re-forms P3 too.  About
// (24 R1 + 18 R2 + 6n + 116) / 8 FP64 operations per step against
// 6n + 10 for the dense layout.  Every term is still the pair_mul chain over
// the N row pairs, so the dense layout's error bound carries over.
__host__ __device__ inline size_t sdd_3l_smem_bytes(int n, int r2, int threads) {
  return sparse_sdd_smem_bytes(n, r2, threads);
}

template <int N, int R1, int R2, int kMinBlocks = 2>
__global__ void __launch_bounds__(128, kMinBlocks) ryser_sdd_3l_kernel(DenseSddArgs args) {
  static_assert(R1 >= 4 && R1 + 4 <= R2 && R2 + 2 <= N && (R1 & 1) == 0 && (R2 & 1) == 0,
                "levels: even row counts, four rows or more each, outer rows must remain");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sH = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  const double* sL = sH + (size_t)N * np;
  const double* sX0h = sL + (size_t)N * np;
  const double* sX0l = sX0h + np;
  dd* red = reinterpret_cast<dd*>(sH + 2 * (size_t)N * np + 2 * np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  double2* sOut = reinterpret_cast<double2*>(bar + 2);  // [N - R2][blockDim.x]
  const bool staged =
      stage_to_smem(sH, args.img, (uint32_t)(sizeof(double) * (2 * (size_t)N * np + 2 * np)), bar, args.err);

  double H = 0.0, L = 0.0, m1 = 0.0;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
  const uint64_t b0 = q * tid + (r * tid) / TT;
  const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;
  const int T = blockDim.x, me = threadIdx.x;

  if (staged && b1 > b0) {
    const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
    double xh[R2], xl[R2];
    sdd_split_start<N, R2>(xh, xl, sOut, sH, sL, sX0h, sX0l, np, s0, T, me);
    dd p3 = sdd_outer<N, R2, true>(sOut, sH, sL, np, T, me, false, 0, 0.0);
    dd p23 = rows_product<R1, R2, R2>(xh, xl);
    pair_mul(p23, p3.hi, p3.lo);
    auto term = [&]() {
      dd t = rows_product<0, R1, R2>(xh, xl);
      pair_mul(t, p23.hi, p23.lo);
      return t;
    };
    {
      const dd t0 = term();  // index s0 is even: sign +
      H = t0.hi;
      L = t0.lo;
      m1 = fabs(t0.hi);
    }
#pragma unroll 1
    for (uint64_t base = s0; base < e0; base += 8) {
      const uint64_t top = base + 8 < e0 ? base + 8 : e0 - 1;
      double gs = 0.0, gc = 0.0, ma = 0.0;
#pragma unroll 1
      for (uint64_t i = base + 1; i <= top; i++) {
        const int k = __ffsll((long long)i) - 1;
        const double sg = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
        if (k == 0) {
          pair_update<0, R1, 0, R2>(xh, xl, sH, sL, sg);
        } else {
          pair_update<0, R2, 0, R2>(xh, xl, sH + k * np, sL + k * np, sg);
          if (k >= 3) p3 = sdd_outer<N, R2, true>(sOut, sH, sL, np, T, me, true, k, sg);
          p23 = rows_product<R1, R2, R2>(xh, xl);
          pair_mul(p23, p3.hi, p3.lo);
        }
        const dd t = term();
        if (i & 1)
          sum2_add(gs, gc, -t.hi, -t.lo);
        else
          sum2_add(gs, gc, t.hi, t.lo);
        ma += fabs(t.hi);
      }
      sum2_add(H, L, gs, gc);
      m1 += ma;
    }
  }
  sdd_finish(H, L, m1, args, red, (N & 1) ? 2.0 : -2.0);
}

}  // namespace perm
