// mc_sparse.cu -- Monte-Carlo estimators on CRS + CCS for orders above 64.
//
// Same estimators, streams and FP64 operation order as mc.cu (which covers
// orders <= 64 with one 64-bit mask per row); here the extracted-row/column
// sets are bitsets of ceil(n/64) words and the available-neighbour count of
// every row is kept incrementally, as the reference's sparse kernels do with
// their int[21] masks (gpu_approximation_sparse.cu:198-452, orders <= 672).
// One trial per warp:
//  * row rule: lanes scan rows l, l+32, ... for the smallest (count, row) and
//    one redux.sync picks it;
//  * extracting column c decrements the counts of the rows in CCS(c), one
//    row per lane;
//  * Rasmussen picks the idx-th available column of the row in CRS order;
//  * scaling sweeps: lane l owns columns (then rows) l, l+32, ...; each sum
//    walks CCS(j) (CRS(i)) in ascending order over the remaining rows
//    (columns), exactly the CPU restatement's order, so trials are
//    bit-identical to it.
// The pattern's CRS/CCS is staged once per CTA with a bulk copy.
#include "mc.h"
#include "mc_sparse.h"

namespace perm {

namespace {

__device__ __forceinline__ bool bit_get(const uint64_t* b, int i) { return (b[i >> 6] >> (i & 63)) & 1; }

// smallest (count << 11 | row) over unextracted rows
__device__ __forceinline__ unsigned sparse_min_row(const int* cnt, const uint64_t* rowext, int n, int lane) {
  unsigned key = 0xffffffffu;
  for (int r = lane; r < n; r += 32)
    if (!bit_get(rowext, r)) {
      const unsigned k = ((unsigned)cnt[r] << 11) | (unsigned)r;
      key = k < key ? k : key;
    }
  return __reduce_min_sync(0xffffffffu, key);
}

__device__ __forceinline__ void finish3_sparse(double s, double s2, double z, double* slots,
                                               const McSparseArgs& a) {
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

__global__ void __launch_bounds__(kMcSparseBlock) mc_sparse_kernel(McSparseArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n;
  const int W = (n + 63) >> 6;
  const int* rptrs = reinterpret_cast<const int*>(smem);
  const int* cptrs = rptrs + a.ptr_ints;
  const int* cols = cptrs + a.ptr_ints;
  const int* rows = cols + a.idx_ints;
  unsigned char* per_warp = smem + a.pack_bytes;
  const size_t warp_bytes = mc_sparse_warp_bytes(n, a.scaling);
  unsigned char* mine = per_warp + (threadIdx.x >> 5) * warp_bytes;
  uint64_t* colext = reinterpret_cast<uint64_t*>(mine);
  uint64_t* rowext = colext + W;
  double* dr = reinterpret_cast<double*>(rowext + W);   // scaling only
  double* dc = dr + (a.scaling ? n : 0);
  int* cnt = reinterpret_cast<int*>(dc + (a.scaling ? n : 0));
  double* slots = reinterpret_cast<double*>(per_warp + (kMcSparseBlock / 32) * warp_bytes);
  uint64_t* bar = reinterpret_cast<uint64_t*>(slots + (kMcSparseBlock / 32) * 3);
  const bool staged = stage_to_smem(smem, a.pack, a.pack_bytes, bar, a.err);

  const int lane = threadIdx.x & 31;
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  double s = 0, s2 = 0, zeros = 0;
  if (staged) {
    for (uint64_t q = warp; q < a.trials; q += nwarps) {
      const uint64_t t = a.trial0 + q;
      for (int w = lane; w < W; w += 32) colext[w] = rowext[w] = 0ull;
      for (int r = lane; r < n; r += 32) {
        cnt[r] = rptrs[r + 1] - rptrs[r];
        if (a.scaling) dr[r] = dc[r] = 1.0;
      }
      __syncwarp();
      WExp w;
      bool ok = true;
      for (int it = 0; it < n && ok; it++) {
        const unsigned key = sparse_min_row(cnt, rowext, n, lane);
        const int best = (int)(key >> 11), row = (int)(key & 0x7ffu);
        int col = -1;
        if (!a.scaling) {
          if (best == 0) {
            ok = false;
            break;
          }
          w.mul((float)best);
          const u32x4 rnd = philox_step(a.seed, t, (uint32_t)it, kTagRasmussen);
          int idx = (int)(((uint64_t)rnd.x * (uint64_t)best) >> 32);
          for (int p = rptrs[row]; p < rptrs[row + 1]; p++) {
            const int c = cols[p];
            if (bit_get(colext, c)) continue;
            if (idx == 0) {
              col = c;
              break;
            }
            idx--;
          }
        } else {
          if (it % a.y == 0) {
            for (int k = 0; k < a.z && ok; k++) {
              bool fail = false;
              for (int j = lane; j < n; j += 32) {
                if (bit_get(colext, j)) continue;
                double cs = 0.0;
                for (int p = cptrs[j]; p < cptrs[j + 1]; p++)
                  if (!bit_get(rowext, rows[p])) cs = __dadd_rn(cs, dr[rows[p]]);
                if (cs == 0.0)
                  fail = true;
                else
                  dc[j] = __drcp_rn(cs);
              }
              if (__any_sync(0xffffffffu, fail)) {
                ok = false;
                break;
              }
              __syncwarp();
              for (int i = lane; i < n; i += 32) {
                if (bit_get(rowext, i)) continue;
                double rs = 0.0;
                for (int p = rptrs[i]; p < rptrs[i + 1]; p++)
                  if (!bit_get(colext, cols[p])) rs = __dadd_rn(rs, dc[cols[p]]);
                if (rs == 0.0)
                  fail = true;
                else
                  dr[i] = __drcp_rn(rs);
              }
              if (__any_sync(0xffffffffu, fail)) {
                ok = false;
                break;
              }
              __syncwarp();
            }
            if (!ok) break;
          }
          const double drow = dr[row];
          double sum = 0.0;
          for (int p = rptrs[row]; p < rptrs[row + 1]; p++)
            if (!bit_get(colext, cols[p])) sum = __dadd_rn(sum, __dmul_rn(drow, dc[cols[p]]));
          if (sum == 0.0) {
            ok = false;
            break;
          }
          const u32x4 rnd = philox_step(a.seed, t, (uint32_t)it, kTagScaling);
          const double u = __dmul_rn(__dadd_rn(__dmul_rn((double)(rnd.x >> 5), 67108864.0), (double)(rnd.y >> 6)),
                                     1.0 / 9007199254740992.0);
          const double target = __dmul_rn(u, sum);
          double run = 0.0, sp = 0.0;
          for (int p = rptrs[row]; p < rptrs[row + 1]; p++) {
            const int c = cols[p];
            if (bit_get(colext, c)) continue;
            sp = __dmul_rn(drow, dc[c]);
            run = __dadd_rn(run, sp);
            col = c;
            if (target < run) break;
          }
          w.mul(__double2float_rn(__ddiv_rn(sum, sp)));
        }
        __syncwarp();
        if (lane == 0) {
          colext[col >> 6] |= 1ull << (col & 63);
          rowext[row >> 6] |= 1ull << (row & 63);
        }
        for (int p = cptrs[col] + lane; p < cptrs[col + 1]; p += 32) cnt[rows[p]]--;
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
  finish3_sparse(s, s2, zeros, slots, a);
}

}  // namespace perm
