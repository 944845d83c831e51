// mc.cu -- Monte-Carlo permanent estimators, one trial per warp.
//
// Rasmussen (replaces kernel_rasmussen, gpu_approximation_dense.cu:156-229, and
// kernel_rasmussen_sparse, gpu_approximation_sparse.cu:198-290): per step take
// the unextracted row with the fewest available nonzeros (lowest index on
// ties), multiply the weight by that count and extract a uniformly chosen
// available column.  An empty row ends the trial with weight 0.
//
// Scaling (replaces kernel_approximation, gpu_approximation_dense.cu:232-369, and
// kernel_approximation_sparse, gpu_approximation_sparse.cu:292-452): same row
// rule; every y steps run z Sinkhorn sweeps (columns then rows) over the
// remaining submatrix in FP64; sample an available column with probability
// proportional to d_r[row] * d_c[col]; weight *= 1 / p.  A zero column or row
// sum ends the trial with weight 0.
//
// Both estimate the permanent of the 0/1 pattern of the matrix (the
// reference's algorithms are documented for binary matrices only).
//
// B200 mapping: a warp runs one trial; lane l owns rows and columns l and
// l + 32, so the minimum-degree row is one popc per lane plus a single
// redux.sync minimum over (count << 8 | row), and each Sinkhorn sweep is a
// column pass (lane = column, walking rows) and a row pass (lane = row, over
// the transposed copy) with no bank conflicts.  Random numbers come from
// Philox4x32-10 keyed by (seed) at counter (trial, step, tag), so trial t is
// reproducible regardless of launch shape.  All FP64 operations use
// explicitly rounded intrinsics in the same order as the CPU restatement, so
// per-trial weights are bit-identical to it.  The trial weight is an FP32
// significand with a separate exponent; trial values are accumulated in FP64.
#include "mc.h"

namespace perm {

namespace {

__device__ __forceinline__ int nth_set_bit(uint64_t m, int idx) {
  for (int i = 0; i < idx; i++) m &= m - 1;
  return __ffsll((long long)m) - 1;
}

// Row rule shared by both estimators: (count << 8 | row) minimum over the
// unextracted rows; returns 0xffffffff if none is left.
__device__ __forceinline__ unsigned min_row_key(const uint64_t* rowmask, int n, uint64_t colext,
                                                uint64_t rowext, int lane) {
  unsigned key = 0xffffffffu;
  int r = lane;
  if (r < n && !((rowext >> r) & 1))
    key = ((unsigned)__popcll(rowmask[r] & ~colext) << 8) | (unsigned)r;
  r = lane + 32;
  if (r < n && !((rowext >> r) & 1)) {
    unsigned k2 = ((unsigned)__popcll(rowmask[r] & ~colext) << 8) | (unsigned)r;
    key = k2 < key ? k2 : key;
  }
  return __reduce_min_sync(0xffffffffu, key);
}

// Block + grid completion of the (sum, sum of squares, zeros) triple.
__device__ __forceinline__ void finish3(double s, double s2, double z, double* slots, const McArgs& a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    slots[warp * 3 + 0] = s;
    slots[warp * 3 + 1] = s2;
    slots[warp * 3 + 2] = z;
  }
  __syncthreads();
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    double t0 = 0, t1 = 0, t2 = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      t0 += slots[w * 3 + 0];
      t1 += slots[w * 3 + 1];
      t2 += slots[w * 3 + 2];
    }
    a.partials[blockIdx.x * 3 + 0] = t0;
    a.partials[blockIdx.x * 3 + 1] = t1;
    a.partials[blockIdx.x * 3 + 2] = t2;
    __threadfence();
    unsigned prev = atomicAdd(a.ticket, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last || threadIdx.x != 0) return;
  __threadfence();
  double t0 = 0, t1 = 0, t2 = 0;
  for (unsigned b = 0; b < gridDim.x; b++) {
    t0 += __ldcg(&a.partials[b * 3 + 0]);
    t1 += __ldcg(&a.partials[b * 3 + 1]);
    t2 += __ldcg(&a.partials[b * 3 + 2]);
  }
  a.out[0] = t0;
  a.out[1] = t1;
  a.out[2] = t2;
  *a.ticket = 0u;
  __threadfence();
}

}  // namespace

__global__ void __launch_bounds__(kMcBlock) rasmussen_kernel(McArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint64_t* rowmask = reinterpret_cast<const uint64_t*>(smem);
  double* slots = reinterpret_cast<double*>(smem + a.pack_bytes);
  uint64_t* bar = reinterpret_cast<uint64_t*>(slots + (kMcBlock / 32) * 3);
  const bool staged = stage_to_smem(smem, a.pack, a.mask_bytes, bar, a.err);

  const int lane = threadIdx.x & 31;
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int n = a.n;
  double s = 0, s2 = 0, zeros = 0;
  if (staged) {
    for (uint64_t q = warp; q < a.trials; q += nwarps) {
      const uint64_t t = a.trial0 + q;
      uint64_t colext = 0, rowext = 0;
      WExp w;
      bool ok = true;
      for (int step = 0; step < n; step++) {
        const unsigned key = min_row_key(rowmask, n, colext, rowext, lane);
        const int best = (int)(key >> 8), row = (int)(key & 0xffu);
        if (best == 0) {
          ok = false;
          break;
        }
        w.mul((float)best);
        const u32x4 rnd = philox_step(a.seed, t, (uint32_t)step, kTagRasmussen);
        const int idx = (int)(((uint64_t)rnd.x * (uint64_t)best) >> 32);
        const int col = nth_set_bit(rowmask[row] & ~colext, idx);
        colext |= 1ull << col;
        rowext |= 1ull << row;
      }
      const double v = ok ? w.value() : 0.0;
      if (lane == 0) {
        s += v;
        s2 += v * v;
        zeros += ok ? 0.0 : 1.0;
        if (a.trial_out) a.trial_out[q] = v;
      }
    }
  }
  finish3(s, s2, zeros, slots, a);
}

// kBinary: every nonzero of the matrix is 1 and the pack holds the row masks
// then the column masks.  A Sinkhorn sum over a 0/1 matrix adds exactly the
// scaling factors of its 1 entries (a * d = d for a = 1; a zero entry adds
// +0.0 to a non-negative sum), so walking the set bits of the masks in
// ascending order gives the same FP64 value as the general sum over the
// rows/columns still in the submatrix.
template <bool kBinary>
__device__ __forceinline__ void scaling_trials(const McArgs& a, unsigned char* smem) {
  const int n = a.n, np = a.np;
  const uint64_t* rowmask = reinterpret_cast<const uint64_t*>(smem);
  const uint64_t* colmask = rowmask + np;                                      // binary pack
  const double* A = reinterpret_cast<const double*>(smem + a.mask_bytes);   // A[i * np + j] (general pack)
  const double* AT = A + (size_t)n * np;                                       // AT[j * np + i]
  double* dwarp = reinterpret_cast<double*>(smem + a.pack_bytes);
  double* slots = dwarp + (kMcBlock / 32) * kMcWarpDoubles;
  uint64_t* bar = reinterpret_cast<uint64_t*>(slots + (kMcBlock / 32) * 3);
  const bool staged = stage_to_smem(smem, a.pack, a.pack_bytes, bar, a.err);

  const int lane = threadIdx.x & 31;
  double* dr = dwarp + (threadIdx.x >> 5) * kMcWarpDoubles;
  double* dc = dr + 64;
  double* prefix = dc + 64;                               // running sums of the column choice
  int* pcol = reinterpret_cast<int*>(prefix + 64);        // their columns
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  double s = 0, s2 = 0, zeros = 0;
  if (staged) {
    for (uint64_t q = warp; q < a.trials; q += nwarps) {
      const uint64_t t = a.trial0 + q;
      dr[lane] = 1.0;
      dr[lane + 32] = 1.0;
      dc[lane] = 1.0;
      dc[lane + 32] = 1.0;
      __syncwarp();
      uint64_t colext = 0, rowext = 0;
      WExp w;
      bool ok = true;
      for (int it = 0; it < n && ok; it++) {
        const unsigned key = min_row_key(rowmask, n, colext, rowext, lane);
        const int row = (int)(key & 0xffu);
        if (it % a.y == 0) {
          const uint64_t full = n == 64 ? ~0ull : ((1ull << n) - 1);
          const uint64_t rows_left = ~rowext & full, cols_left = ~colext & full;
          const int j0 = lane, j1 = lane + 32;
          const bool c0 = (cols_left >> j0) & 1, c1 = j1 < 64 && ((cols_left >> j1) & 1);
          const bool r0 = (rows_left >> j0) & 1, r1 = j1 < 64 && ((rows_left >> j1) & 1);
          for (int k = 0; k < a.z; k++) {
            // column pass: lane owns columns lane, lane + 32
            double cs0 = 0.0, cs1 = 0.0;
            if (kBinary) {
              const uint64_t m0 = c0 ? (colmask[j0] & rows_left) : 0ull;
              const uint64_t m1 = c1 ? (colmask[j1] & rows_left) : 0ull;
              for (int i0 = 0; i0 < n; i0 += 8) {
                const uint32_t b0 = (uint32_t)(m0 >> i0) & 0xFFu, b1 = (uint32_t)(m1 >> i0) & 0xFFu;
#pragma unroll
                for (int u = 0; u < 8; u += 2) {
                  const double2 d = *reinterpret_cast<const double2*>(dr + i0 + u);
                  if (b0 & (1u << u)) cs0 = __dadd_rn(cs0, d.x);
                  if (b1 & (1u << u)) cs1 = __dadd_rn(cs1, d.x);
                  if (b0 & (2u << u)) cs0 = __dadd_rn(cs0, d.y);
                  if (b1 & (2u << u)) cs1 = __dadd_rn(cs1, d.y);
                }
              }
            } else {
              for (uint64_t m = rows_left; m; m &= m - 1) {
                const int i = __ffsll((long long)m) - 1;
                const double d = dr[i];
                const double* Ai = A + i * np;
                if (c0) cs0 = __dadd_rn(cs0, __dmul_rn(d, Ai[j0]));
                if (c1) cs1 = __dadd_rn(cs1, __dmul_rn(d, Ai[j1]));
              }
            }
            bool fail = (c0 && cs0 == 0.0) || (c1 && cs1 == 0.0);
            if (__any_sync(0xffffffffu, fail)) {
              ok = false;
              break;
            }
            if (c0) dc[j0] = __drcp_rn(cs0);
            if (c1) dc[j1] = __drcp_rn(cs1);
            __syncwarp();
            // row pass: lane owns rows lane, lane + 32
            double rs0 = 0.0, rs1 = 0.0;
            if (kBinary) {
              const uint64_t m0 = r0 ? (rowmask[j0] & cols_left) : 0ull;
              const uint64_t m1 = r1 ? (rowmask[j1] & cols_left) : 0ull;
              for (int i0 = 0; i0 < n; i0 += 8) {
                const uint32_t b0 = (uint32_t)(m0 >> i0) & 0xFFu, b1 = (uint32_t)(m1 >> i0) & 0xFFu;
#pragma unroll
                for (int u = 0; u < 8; u += 2) {
                  const double2 d = *reinterpret_cast<const double2*>(dc + i0 + u);
                  if (b0 & (1u << u)) rs0 = __dadd_rn(rs0, d.x);
                  if (b1 & (1u << u)) rs1 = __dadd_rn(rs1, d.x);
                  if (b0 & (2u << u)) rs0 = __dadd_rn(rs0, d.y);
                  if (b1 & (2u << u)) rs1 = __dadd_rn(rs1, d.y);
                }
              }
            } else {
              for (uint64_t m = cols_left; m; m &= m - 1) {
                const int j = __ffsll((long long)m) - 1;
                const double d = dc[j];
                const double* ATj = AT + j * np;
                if (r0) rs0 = __dadd_rn(rs0, __dmul_rn(ATj[j0], d));
                if (r1) rs1 = __dadd_rn(rs1, __dmul_rn(ATj[j1], d));
              }
            }
            fail = (r0 && rs0 == 0.0) || (r1 && rs1 == 0.0);
            if (__any_sync(0xffffffffu, fail)) {
              ok = false;
              break;
            }
            if (r0) dr[j0] = __drcp_rn(rs0);
            if (r1) dr[j1] = __drcp_rn(rs1);
            __syncwarp();
          }
          if (!ok) break;
        }
        // column choice: running sums in ascending column order (recorded),
        // the first one above u * sum (one ballot), the last column if none
        const uint64_t avail = rowmask[row] & ~colext;
        const double drow = dr[row];
        double sum = 0.0;
        int cnt = 0;
        for (uint64_t m = avail; m; m &= m - 1, cnt++) {
          const int j = __ffsll((long long)m) - 1;
          sum = __dadd_rn(sum, __dmul_rn(drow, dc[j]));
          if (lane == 0) {
            prefix[cnt] = sum;
            pcol[cnt] = j;
          }
        }
        if (sum == 0.0) {
          ok = false;
          break;
        }
        __syncwarp();
        const u32x4 rnd = philox_step(a.seed, t, (uint32_t)it, kTagScaling);
        const double u = __dmul_rn(__dadd_rn(__dmul_rn((double)(rnd.x >> 5), 67108864.0), (double)(rnd.y >> 6)),
                                   1.0 / 9007199254740992.0);
        const double target = __dmul_rn(u, sum);
        const unsigned lo = __ballot_sync(0xffffffffu, lane < cnt && target < prefix[lane]);
        const unsigned hi = __ballot_sync(0xffffffffu, lane + 32 < cnt && target < prefix[lane + 32]);
        const int pick = lo ? __ffs(lo) - 1 : (hi ? 32 + __ffs(hi) - 1 : cnt - 1);
        const int col = pcol[pick];
        const double sp = __dmul_rn(drow, dc[col]);
        w.mul(__double2float_rn(__ddiv_rn(sum, sp)));
        colext |= 1ull << col;
        rowext |= 1ull << row;
        __syncwarp();
      }
      const double v = ok ? w.value() : 0.0;
      if (lane == 0) {
        s += v;
        s2 += v * v;
        zeros += ok ? 0.0 : 1.0;
        if (a.trial_out) a.trial_out[q] = v;
      }
      __syncwarp();
    }
  }
  finish3(s, s2, zeros, slots, a);
}

__global__ void __launch_bounds__(kMcBlock) scaling_kernel(McArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  scaling_trials<false>(a, smem);
}

__global__ void __launch_bounds__(kMcBlock) scaling_kernel_binary(McArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  scaling_trials<true>(a, smem);
}

}  // namespace perm
