// ryser_dense_dd.cuh -- dense exact permanent with X, the n-way product and
// the accumulation all in double-double (about 106-bit significands).
//
// Same walk, thread ranges and reductions as ryser_dense.cuh; every x_j is a
// (hi, lo) pair updated with TwoSum, products use FMA-based dd multiplication
// and terms are added in dd.  About nine times the FP64-X kernel's work per
// Gray step; used when the FP64 result's estimated relative error exceeds the
// caller's target (heavy cancellation) and as the high-precision cross-check
// of the FP64 kernels at orders the CPU oracle cannot reach.
#pragma once
#include "ryser_dense.cuh"

namespace perm {

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

  dd acc = {0.0, 0.0};
  const uint64_t TT = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t s0, e0;
  if (N < 4) {
    s0 = 0;
    e0 = (tid == 0 && args.block0 == 0) ? (1ull << (N - 1)) : 0;
  } else {
    const uint64_t q = args.nblocks / TT, r = args.nblocks % TT;
    s0 = (args.block0 + q * tid + (r * tid) / TT) << args.m;
    e0 = (args.block0 + q * (tid + 1) + (r * (tid + 1)) / TT) << args.m;
  }
  if (staged && e0 > s0) {
    dd x[N];
#pragma unroll
    for (int j = 0; j < N; j++) x[j] = {sX0[j], sX0[np + j]};
    const uint64_t g = s0 ^ (s0 >> 1);
#pragma unroll 1
    for (int k = 0; k < N - 1; k++)
      if ((g >> k) & 1)
#pragma unroll
        for (int j = 0; j < N; j++) x[j] = dd_add_d(x[j], sA[k * np + j]);
#pragma unroll 1
    for (uint64_t i = s0; i < e0; i++) {
      if (i != s0) {
        const int k = __ffsll((long long)i) - 1;
        const bool plus = !((i >> (k + 1)) & 1);
        const double* col = sA + k * np;
#pragma unroll
        for (int j = 0; j < N; j++) x[j] = dd_add_d(x[j], plus ? col[j] : -col[j]);
      }
      dd p = x[0];
#pragma unroll
      for (int j = 1; j < N; j++) p = dd_mul(p, x[j]);
      if (i & 1) p = {-p.hi, -p.lo};
      acc = dd_add(acc, p);
    }
  }
  dd bt = block_reduce_dd(acc, red);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, (N & 1) ? 2.0 : -2.0, red);
}

__host__ __device__ inline size_t dense_dd_smem_bytes(int n) {
  int np = (n + 1) & ~1;
  return sizeof(double) * ((size_t)n * np + 2 * np) + 32 * sizeof(dd) + 16;
}

}  // namespace perm
