// ryser_skipper.cu -- sparse exact permanent: SkipPer (skip-ahead Ryser) on
// CRS + CCS.
//
// Replaces kernel_xshared_coalescing_mshared_skipper (gpu_exact_sparse.cu:556-670)
// and its wrapper's host sum (gpu_exact_sparse.cu:1124-1190).  Per Gray index i
// the walk
//   * applies gray(i) ^ gray(previous) column by column through the CCS
//     (gpu_exact_sparse.cu:611-633),
//   * multiplies x from row n-1 downwards and stops at the first zero entry
//     (gpu_exact_sparse.cu:634-642),
//   * on a zero product jumps to the next Gray index at which some column of
//     that row flips (gpu_exact_sparse.cu:648-666).
// Differences, all B200-first: X is FP64 (the reference keeps FP32, which is
// inexact for real-valued inputs); it lives in shared memory as x[j][thread],
// so every access of a warp is bank-conflict-free; the packed CRS/CCS/value
// block is staged once per CTA with a bulk (TMA) copy; threads take Gray
// chunks from a global queue (atomic ticket) instead of one static slice, which
// balances the data-dependent skip lengths; products are accumulated with
// TwoSum and reduced in double-double; an FP64 underflow to zero without a
// zero entry is counted as a zero term instead of indexing row -1.
#include "perman_common.cuh"
#include "skipper.h"

namespace perm {

__global__ void __launch_bounds__(128) skipper_kernel(SkipArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n;
  const int BD = blockDim.x;
  const int tid = threadIdx.x;
  double* X = reinterpret_cast<double*>(smem + a.pack_bytes);  // [n][BD]
  dd* red = reinterpret_cast<dd*>(X + (size_t)n * BD);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);

  const bool staged = stage_to_smem(smem, a.pack, a.pack_bytes, bar, a.err);
  const double* x0 = reinterpret_cast<const double*>(smem);
  const double* cvals = reinterpret_cast<const double*>(smem + a.off_cvals);
  const int* rptrs = reinterpret_cast<const int*>(smem + a.off_rptrs);
  const int* cptrs = reinterpret_cast<const int*>(smem + a.off_cptrs);
  const int* cols = reinterpret_cast<const int*>(smem + a.off_cols);
  const int* rows = reinterpret_cast<const int*>(smem + a.off_rows);

  Acc acc;
  unsigned long long visited = 0;
  if (staged) {
    for (;;) {
      unsigned long long c = atomicAdd(a.next_chunk, 1ull);
      if (c >= a.nchunks) break;
      uint64_t i = c * a.chunk;
      uint64_t end = i + a.chunk;
      if (end > a.total) end = a.total;
      for (int j = 0; j < n; j++) X[j * BD + tid] = x0[j];
      uint64_t prev = 0;
      while (i < end) {
        const uint64_t g = i ^ (i >> 1);
        uint64_t diff = prev ^ g;
        while (diff) {
          const int k = __ffsll((long long)diff) - 1;
          diff &= diff - 1;
          const int p0 = cptrs[k], p1 = cptrs[k + 1];
          if ((g >> k) & 1) {
            for (int p = p0; p < p1; p++) X[rows[p] * BD + tid] += cvals[p];
          } else {
            for (int p = p0; p < p1; p++) X[rows[p] * BD + tid] -= cvals[p];
          }
        }
        prev = g;
        double prod = 1.0;
        int last_zero = -1;
        for (int j = n - 1; j >= 0; j--) {
          const double v = X[j * BD + tid];
          prod *= v;
          if (v == 0.0) {
            last_zero = j;
            break;
          }
        }
        visited++;
        if (prod != 0.0 || last_zero < 0) {
          acc.add((i & 1) ? -prod : prod);
          i++;
        } else {
          uint64_t change = ~0ull;
          for (int p = rptrs[last_zero]; p < rptrs[last_zero + 1]; p++) {
            const int col = cols[p];
            const uint64_t first = 1ull << col;  // first index whose ctz is col
            uint64_t ci = first;
            if (i >= first) ci = first + (((i - first) >> (col + 1)) + 1) * (first << 1);
            if (ci < change) change = ci;
          }
          i++;
          if (change > i) i = change;
        }
      }
    }
    atomicAdd(a.visited, visited);
  }
  dd bt = block_reduce_dd(acc.value(), red);
  grid_finish_dd(bt, a.partials, a.ticket, a.out, (n & 1) ? 2.0 : -2.0, red);
}

}  // namespace perm
