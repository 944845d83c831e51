// ryser_dense_dd.cuh -- dense exact permanent with X, the n-way product and
// the accumulation carried in double-double (about 106-bit significands).
//
// Same walk, aligned thread ranges (warp-uniform columns) and reductions as
// ryser_dense.cuh.  Representation, chosen for the fewest FP64 operations
// that keep double-double accuracy:
//  * x_j is an unevaluated pair (hi, lo): an update adds the column value to
//    hi with TwoSum and the exact rounding error to lo (7 operations);
//  * the product is an unevaluated pair as well: multiplying (ph, pl) by
//    (xh, xl) takes the exact high product and its error from one FMA and
//    adds both cross terms with FMAs (4 operations per factor);
//  * terms are added with TwoSum into the running high part and a plain sum
//    of all low parts.
// About 11n + 8 FP64 operations per Gray step against 2n for the FP64-X
// kernel; the step loop is not unrolled (one step's pairs already fill the
// register file at n = 40).  Used when the FP64 result's estimated relative
// error exceeds the caller's target (heavy cancellation) and as the
// high-precision cross-check of the FP64 kernels at orders the CPU oracle
// cannot reach.
#pragma once
#include "ryser_dense.cuh"

namespace perm {

struct DDX {
  double hi, lo;
};

__device__ __forceinline__ void ddx_add(DDX& x, double a) {
  const double s = __dadd_rn(x.hi, a);
  const double bb = __dsub_rn(s, x.hi);
  const double e = __dadd_rn(__dsub_rn(x.hi, __dsub_rn(s, bb)), __dsub_rn(a, bb));
  x.hi = s;
  x.lo = __dadd_rn(x.lo, e);
}

__device__ __forceinline__ void ddx_mul(DDX& p, const DDX& x) {
  const double h = __dmul_rn(p.hi, x.hi);
  double l = __fma_rn(p.hi, x.hi, -h);
  l = __fma_rn(p.hi, x.lo, l);
  l = __fma_rn(p.lo, x.hi, l);
  p.hi = h;
  p.lo = l;
}

// x += sign * col, then the double-double product of x (unnormalised pair)
template <int N, int kSign>
__device__ __forceinline__ DDX ddstep(DDX (&x)[N], const double* col, double s) {
#pragma unroll
  for (int j = 0; j < N; j += 2) {
    double v0, v1 = 0.0;
    if (j + 1 < N) {
      const double2 v = lds2(col + j);
      v0 = v.x;
      v1 = v.y;
    } else {
      v0 = lds1(col + j);
    }
    if (kSign < 0) {
      v0 = -v0;
      v1 = -v1;
    } else if (kSign == 0) {
      v0 *= s;
      v1 *= s;
    }
    ddx_add(x[j], v0);
    if (j + 1 < N) ddx_add(x[j + 1], v1);
  }
  DDX p = x[0];
#pragma unroll
  for (int j = 1; j < N; j++) ddx_mul(p, x[j]);
  return p;
}

template <int N>
__device__ __forceinline__ DDX ddprod(const DDX (&x)[N]) {
  DDX p = x[0];
#pragma unroll
  for (int j = 1; j < N; j++) ddx_mul(p, x[j]);
  return p;
}

// running sum: TwoSum into hi, every low part into lo
struct DDAcc {
  double hi = 0.0, lo = 0.0;
  __device__ __forceinline__ void add(const DDX& t, bool neg) {
    const double th = neg ? -t.hi : t.hi, tl = neg ? -t.lo : t.lo;
    const dd s = two_sum(hi, th);
    hi = s.hi;
    lo = __dadd_rn(lo, __dadd_rn(s.lo, tl));
  }
};

template <int N>
__global__ void __launch_bounds__(128) ryser_dense_dd_kernel(DenseArgs args) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sA = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  double* sX0 = sA + N * np;  // [N] hi, then [N] lo
  dd* red = reinterpret_cast<dd*>(sX0 + 2 * np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  const bool staged = stage_to_smem(sA, args.colA, (uint32_t)(sizeof(double) * N * np), bar, args.err);
  if (threadIdx.x < N) {
    const int j = threadIdx.x;
    dd rs = {0.0, 0.0};
    for (int k = 0; k < N; k++) rs = dd_add_d(rs, sA[k * np + j]);
    const dd x = dd_add_d({-0.5 * rs.hi, -0.5 * rs.lo}, sA[(N - 1) * np + j]);
    sX0[j] = x.hi;
    sX0[np + j] = x.lo;
  }
  __syncthreads();

  DDAcc acc;
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!staged) {
    // staging failed (error flag set); contribute nothing
  } else if (N < 4) {
    if (tid == 0 && args.block0 == 0) {
      DDX x[N];
#pragma unroll
      for (int j = 0; j < N; j++) x[j] = {sX0[j], sX0[np + j]};
      acc.add(ddprod<N>(x), false);
      for (uint64_t i = 1; i < (1ull << (N - 1)); i++) {
        const int k = __ffsll((long long)i) - 1;
        const bool plus = !((i >> (k + 1)) & 1);
#pragma unroll
        for (int j = 0; j < N; j++) ddx_add(x[j], plus ? sA[k * np + j] : -sA[k * np + j]);
        acc.add(ddprod<N>(x), i & 1);
      }
    }
  } else {
    const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
    const uint64_t b0 = q * tid + (r * tid) / TT;
    const uint64_t b1 = q * (tid + 1) + (r * (tid + 1)) / TT;
    if (b1 > b0) {
      const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
      DDX x[N];
#pragma unroll
      for (int j = 0; j < N; j++) x[j] = {sX0[j], sX0[np + j]};
      const uint64_t g = s0 ^ (s0 >> 1);
#pragma unroll 1
      for (int k = 0; k < N - 1; k++)
        if ((g >> k) & 1)
#pragma unroll
          for (int j = 0; j < N; j++) ddx_add(x[j], sA[k * np + j]);
      acc.add(ddprod<N>(x), false);  // index s0 is even
      // rolled step loop: k = ctz(i) is warp-uniform inside aligned ranges,
      // so the column read stays a shared-memory broadcast
#pragma unroll 1
      for (uint64_t i = s0 + 1; i < e0; i++) {
        const int k = __ffsll((long long)i) - 1;
        const double sg = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
        acc.add(ddstep<N, 0>(x, sA + k * np, sg), i & 1);
      }
    }
  }
  const dd mine = two_sum(acc.hi, acc.lo);
  dd bt = block_reduce_dd(mine, red);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, (N & 1) ? 2.0 : -2.0, red);
}

__host__ __device__ inline size_t dense_dd_smem_bytes(int n) {
  int np = (n + 1) & ~1;
  return sizeof(double) * ((size_t)n * np + 2 * np) + 32 * sizeof(dd) + 16;
}

}  // namespace perm
