// ryser_dense_int.cuh -- dense exact permanent for integer matrices with
// X held in int32.
//
// Same walk, ranges and reductions as ryser_dense.cuh (kernel_xshared_
// coalescing_mshared, gpu_exact_dense.cu:330-399, restated), but the row-sum
// vector is kept as y = 2x, which is an exact int32 for integer inputs:
//   y_j(0) = 2 a[j][n-1] - rowsum_j,   y += 2 s A[:, k]   (integer adds)
// and the n-way product is split into groups of G consecutive rows whose
// product is formed exactly with 32-bit integer multiplies (the host proves
// prod_{j in group} sum_k |a_jk| < 2^31 before choosing this kernel) and
// converted to FP64 with one (exact) int32 -> double conversion, one
// instruction per group (measured 8% faster at n = 40 than forming 2^52 + u
// from the bits and subtracting).  The group values are multiplied in FP64
// (four chains); terms are accumulated exactly as in the FP64-X kernel and
// the final sum is scaled by (4(n&1)-2) / 2^n (exact).
//
// Per Gray step this moves the X update and (G-1)/G of the product off the
// FP64 pipe onto the integer pipes: ~n integer adds + n integer multiplies +
// ceil(n/G) DADD + ceil(n/G) DMUL instead of n DADD + n DMUL.
#pragma once
#include "ryser_dense.cuh"

namespace perm {

struct DenseIntArgs {
  const int* colI;   // column-major doubled matrix: colI[k * np4 + j] = 2 a[j][k]
  const int* y0;     // y_j(0) = 2 a[j][n-1] - rowsum_j, np4 entries
  int np4;           // column stride, multiple of 4 (16-byte columns)
  int m;             // log2 of the range alignment
  uint64_t block0, nblocks;
  dd* partials;
  unsigned* ticket;
  double* out;
  int* err;
};

__device__ __forceinline__ int4 lds4i(const int* p) {
  int4 v;
  unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v4.s32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}

// Exact int32 product of y[a .. a + len), len <= 8 (uint32 arithmetic wraps
// to the right two's complement value: the host proved |product| < 2^31),
// multiplied as a balanced tree -- ((y0 y1)(y2 y3)) y4 for five rows -- so
// its dependent chain is ceil(log2 len) multiplies deep instead of len - 1.
// Integer multiplication is associative, so the value is the chain's.
template <int N>
__device__ __forceinline__ uint32_t rows_product(const int (&y)[N], int a, int len) {
  uint32_t p[8];
#pragma unroll
  for (int t = 0; t < 8; t++) p[t] = t < len ? (uint32_t)y[a + t] : 1u;
#pragma unroll
  for (int w = 1; w < 8; w *= 2)
#pragma unroll
    for (int t = 0; t + w < 8; t += 2 * w)
      if (t + w < len) p[t] = p[t] * p[t + w];
  return p[0];
}

template <int N, int G>
__device__ __forceinline__ double group_product(const int (&y)[N]) {
  constexpr int NG = (N + G - 1) / G;
  double p0 = 1.0, p1 = 1.0, p2 = 1.0, p3 = 1.0;
#pragma unroll
  for (int g = 0; g < NG; g++) {
    const int j0 = g * G;
    uint32_t pr = (uint32_t)y[j0];
#pragma unroll
    for (int t = 1; t < G; t++)
      if (j0 + t < N) pr = pr * (uint32_t)y[j0 + t];
    const double d = __int2double_rn((int)pr);
    if ((g & 3) == 0) p0 = g < 4 ? d : p0 * d;
    if ((g & 3) == 1) p1 = g < 4 ? d : p1 * d;
    if ((g & 3) == 2) p2 = g < 4 ? d : p2 * d;
    if ((g & 3) == 3) p3 = g < 4 ? d : p3 * d;
  }
  return (p0 * p1) * (p2 * p3);
}

template <int N, int G, int kSign>
__device__ __forceinline__ double istep(int (&y)[N], const int* col, int s) {
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
  return group_product<N, G>(y);
}

__host__ __device__ inline size_t dense_int_smem_bytes(int n) {
  int np4 = (n + 3) & ~3;
  return sizeof(int) * ((size_t)n * np4 + np4) + 32 * sizeof(dd) + 16;
}

template <int N, int G>
__global__ void __launch_bounds__(128) ryser_dense_int_kernel(DenseIntArgs args) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np4 = args.np4;
  int* sC = reinterpret_cast<int*>(smem_raw);  // [N][np4] columns, then y0
  dd* red = reinterpret_cast<dd*>(sC + (size_t)(N + 1) * np4);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);
  // columns and y0 are contiguous in the operand block: one bulk copy
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
    acc.add(group_product<N, G>(y));

    const int* c0 = sC;
    const int* c1 = sC + np4;
    const int* c2 = sC + 2 * np4;
    const uint64_t groups = (e0 - s0) >> 3;
    uint64_t base = s0;
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
      double t8 = istep<N, G, 0>(y, sC + k8 * np4, s8);
      acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) + (t8 - t7)));
    }
    {
      const int s4 = ((base >> 3) & 1) ? -1 : 1;
      double t1 = istep<N, G, +1>(y, c0, 0);
      double t2 = istep<N, G, +1>(y, c1, 0);
      double t3 = istep<N, G, -1>(y, c0, 0);
      double t4 = istep<N, G, 0>(y, c2, s4);
      double t5 = istep<N, G, +1>(y, c0, 0);
      double t6 = istep<N, G, -1>(y, c1, 0);
      double t7 = istep<N, G, -1>(y, c0, 0);
      acc.add(((t2 - t1) + (t4 - t3)) + ((t6 - t5) - t7));
    }
  }

  dd bt = block_reduce_dd(acc.value(), red);
  const double factor = ((N & 1) ? 2.0 : -2.0) * ldexp(1.0, -N);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

}  // namespace perm
