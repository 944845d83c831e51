// ryser_dense.cuh -- dense exact permanent: Nijenhuis-Wilf Ryser walked in
// Gray-code order, one contiguous Gray range per thread, X in registers.
//
// Replaces kernel_xshared_coalescing_mshared (gpu_exact_dense.cu:330-399) and
// its host sum (gpu_exact_dense.cu:691-698).  Same mathematics:
//   x_j(0) = a[j][n-1] - rowsum_j / 2                  (gpu_exact_dense.cu:647-654)
//   term(i) = (-1)^i * prod_j x_j(i),  i in [0, 2^(n-1))
//   x(i) = x(i-1) + s * A[:, k],  k = ctz(i),  s = +1 iff bit k of gray(i) is set
//   perm = (4(n&1)-2) * sum_i term(i)                  (gpu_exact_dense.cu:698)
//
// B200 layout:
//  * Each thread owns Gray indices [s, e) with s, e multiples of 2^m (m >= 3).
//    Inside an aligned range the column sequence k = ctz(i) is the same for
//    every lane of a warp, so the column read is a shared-memory broadcast, and
//    seven of every eight steps touch columns 0, 1, 2 with compile-time signs.
//  * The thread computes its starting X directly from gray(s) -- no carry-in.
//  * X (n doubles) stays in registers (n is a template parameter); the n-way
//    product uses four independent multiply chains.
//  * Every 8 signed terms are summed in FP64 and folded into a TwoSum
//    compensated (hi, lo) accumulator; threads are reduced in double-double
//    (warp shuffles, then block, then an ordered last-block grid sum).
#pragma once
#include "perman_common.cuh"

namespace perm {

struct DenseArgs {
  const double* colA;  // column-major a: colA[k * np + j] = a[j][k]
  int np;              // column stride (n rounded up to even: 16-byte columns)
  int m;               // log2 of the range alignment
  uint64_t block0;     // first aligned block of this launch (shards start > 0)
  uint64_t nblocks;    // aligned blocks of 2^m Gray indices, shared out over threads
  dd* partials;        // gridDim.x scratch entries
  unsigned* ticket;    // zero-initialised completion counter
  double* out;         // out[0], out[1] = permanent as (hi, lo)
  int* err;            // set to 1 if the shared-memory staging timed out
  uint64_t seg_blocks; // orders <= kAnchorMaxN: X is recomputed from x0 every seg_blocks
                       // aligned blocks (0: once per thread range)
  uint32_t inject;     // failure injection (tests): staging expects this many extra bytes
};

// Orders up to which the FP64-X walk re-anchors X (recomputes it from x0) at
// every segment: the rounding errors of the X updates then accumulate over at
// most one segment (>= 2^11 steps) instead of a whole thread range (up to
// 2^25 steps), which is what dominates the FP64-X error on real matrices.
// Above this order the extra code makes the compiler spill inside the walk.
constexpr int kAnchorMaxN = 35;

__device__ __forceinline__ double2 lds2(const double* p) {
  double2 v;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ double lds1(const double* p) {
  double v;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}

// x += sgn * col (sgn = +1/-1 known at compile time when kSign != 0; taken
// from `s` otherwise), then return prod_j x_j.
template <int N, int kSign>
__device__ __forceinline__ double step(double (&x)[N], const double* col, double s) {
  double p0 = 1.0, p1 = 1.0, p2 = 1.0, p3 = 1.0;
#pragma unroll
  for (int j = 0; j < N; j += 2) {
    double v0, v1 = 0.0;
    if (j + 1 < N) {
      double2 v = lds2(col + j);
      v0 = v.x;
      v1 = v.y;
    } else {
      v0 = lds1(col + j);
    }
    if (kSign > 0) {
      x[j] = x[j] + v0;
      if (j + 1 < N) x[j + 1] = x[j + 1] + v1;
    } else if (kSign < 0) {
      x[j] = x[j] - v0;
      if (j + 1 < N) x[j + 1] = x[j + 1] - v1;
    } else {
      x[j] = fma(s, v0, x[j]);
      if (j + 1 < N) x[j + 1] = fma(s, v1, x[j + 1]);
    }
    // four chains: j%4 == 0,1,2,3; first touch initialises the chain
    if ((j & 3) == 0) {
      p0 = (j == 0) ? x[j] : p0 * x[j];
      if (j + 1 < N) p1 = (j == 0) ? x[j + 1] : p1 * x[j + 1];
    } else {
      p2 = (j == 2) ? x[j] : p2 * x[j];
      if (j + 1 < N) p3 = (j == 2) ? x[j + 1] : p3 * x[j + 1];
    }
  }
  if (N == 1) return p0;
  if (N == 2) return p0 * p1;
  if (N == 3) return (p0 * p1) * p2;
  return (p0 * p1) * (p2 * p3);
}

// X for Gray index i recomputed from x0 (volatile shared loads: nothing is
// hoisted into registers across the walk)
template <int N>
__device__ __forceinline__ void anchor_x(double (&x)[N], const double* x0, const double* sA, int np, uint64_t i) {
  const uint64_t g = i ^ (i >> 1);
#pragma unroll
  for (int j = 0; j < N; j += 2) {
    if (j + 1 < N) {
      const double2 v = lds2(x0 + j);
      x[j] = v.x;
      x[j + 1] = v.y;
    } else {
      x[j] = lds1(x0 + j);
    }
  }
#pragma unroll 1
  for (int k = 0; k < N - 1; k++) {
    if ((g >> k) & 1) {
      const double* c = sA + k * np;
#pragma unroll
      for (int j = 0; j < N; j += 2) {
        if (j + 1 < N) {
          const double2 v = lds2(c + j);
          x[j] += v.x;
          x[j + 1] += v.y;
        } else {
          x[j] += lds1(c + j);
        }
      }
    }
  }
}

template <int N>
__device__ __forceinline__ double prod_only(const double (&x)[N]) {
  double p0 = x[0], p1 = 1.0, p2 = 1.0, p3 = 1.0;
  if (N > 1) p1 = x[1];
  if (N > 2) p2 = x[2];
  if (N > 3) p3 = x[3];
#pragma unroll
  for (int j = 4; j < N; j++) {
    if ((j & 3) == 0) p0 *= x[j];
    if ((j & 3) == 1) p1 *= x[j];
    if ((j & 3) == 2) p2 *= x[j];
    if ((j & 3) == 3) p3 *= x[j];
  }
  return (p0 * p1) * (p2 * p3);
}

// Shared-memory bytes for an order-N launch.
__host__ __device__ inline size_t dense_smem_bytes(int n) {
  int np = (n + 1) & ~1;
  return sizeof(double) * ((size_t)n * np + np) + 32 * sizeof(dd) + 16;
}

template <int N>
__global__ void __launch_bounds__(128) ryser_dense_kernel(DenseArgs args) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sA = reinterpret_cast<double*>(smem_raw);
  const int np = args.np;
  double* sX0 = sA + N * np;
  dd* red = reinterpret_cast<dd*>(sX0 + np);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);

  // Stage the matrix (at most 32 KB) once per block with a bulk copy; every
  // warp then reads columns as shared-memory broadcasts.
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

  if (!staged) {
    // staging failed (error flag set); contribute nothing
  } else if (N < 4) {
    // Orders 1..3: at most four Gray indices; thread 0 walks them all.
    if (tid == 0 && args.block0 == 0) {
      double x[N];
#pragma unroll
      for (int j = 0; j < N; j++) x[j] = sX0[j];
      uint64_t total = 1ull << (N - 1);
      acc.add(prod_only<N>(x));
      for (uint64_t i = 1; i < total; i++) {
        int k = __ffsll((long long)i) - 1;
        double s = ((i >> (k + 1)) & 1) ? -1.0 : 1.0;
#pragma unroll
        for (int j = 0; j < N; j++) x[j] = fma(s, sA[k * np + j], x[j]);
        double p = prod_only<N>(x);
        acc.add((i & 1) ? -p : p);
      }
    }
  } else if (N <= kAnchorMaxN && b1 > b0) {
    // segments of seg_blocks aligned blocks, each from a freshly computed X
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
      acc.add(prod_only<N>(x));  // index s0 is even: sign +
      const uint64_t groups = (nb << args.m) >> 3;
      uint64_t base = s0;
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
        double t8 = step<N, 0>(x, sA + k8 * np, s8);
        acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) + (t8 - t7)));
      }
      {  // last group of the segment: seven steps (the next index starts the next segment)
        const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
        double t1 = step<N, +1>(x, c0, 0.0);
        double t2 = step<N, +1>(x, c1, 0.0);
        double t3 = step<N, -1>(x, c0, 0.0);
        double t4 = step<N, 0>(x, c2, s4);
        double t5 = step<N, +1>(x, c0, 0.0);
        double t6 = step<N, -1>(x, c1, 0.0);
        double t7 = step<N, -1>(x, c0, 0.0);
        acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) - t7));
      }
    }
  } else if (b1 > b0) {
    const uint64_t s0 = (args.block0 + b0) << args.m, e0 = (args.block0 + b1) << args.m;
    double x[N];
#pragma unroll
    for (int j = 0; j < N; j++) x[j] = sX0[j];
    // Starting X from gray(s0) directly.
    const uint64_t g = s0 ^ (s0 >> 1);
#pragma unroll 1
    for (int k = 0; k < N - 1; k++) {
      if ((g >> k) & 1) {
#pragma unroll
        for (int j = 0; j < N; j++) x[j] += sA[k * np + j];
      }
    }
    acc.add(prod_only<N>(x));  // index s0 is even: sign +

    const double* c0 = sA;
    const double* c1 = sA + np;
    const double* c2 = sA + 2 * np;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
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
      double t8 = step<N, 0>(x, sA + k8 * np, s8);
      acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) + (t8 - t7)));
    }
    {  // last group of the range: seven steps (index e0 belongs to the next range)
      const double s4 = ((base >> 3) & 1) ? -1.0 : 1.0;
      double t1 = step<N, +1>(x, c0, 0.0);
      double t2 = step<N, +1>(x, c1, 0.0);
      double t3 = step<N, -1>(x, c0, 0.0);
      double t4 = step<N, 0>(x, c2, s4);
      double t5 = step<N, +1>(x, c0, 0.0);
      double t6 = step<N, -1>(x, c1, 0.0);
      double t7 = step<N, -1>(x, c0, 0.0);
      acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) - t7));
    }
  }

  dd mine = acc.value();
  dd bt = block_reduce_dd(mine, red);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, (N & 1) ? 2.0 : -2.0, red);
}

}  // namespace perm
