// perman_common.cuh -- shared device helpers for the sm_100a permanent kernels:
// error-free FP64 transformations and double-double (dd) arithmetic, the
// deterministic warp/block/grid dd reductions, and the Philox4x32-10
// counter-based generator used by the Monte-Carlo trial kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace perm {

// ---------------------------------------------------------------------------
// double-double arithmetic.  All FP64 operations here are written with the
// explicitly rounded intrinsics so that nvcc cannot contract them into FMAs
// (which would break the error-free transformations).
// ---------------------------------------------------------------------------
struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
  double s = __dadd_rn(a, b);
  double bb = __dsub_rn(s, a);
  double e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return {s, e};
}
__device__ __forceinline__ dd fast_two_sum(double a, double b) {
  double s = __dadd_rn(a, b);
  double e = __dsub_rn(b, __dsub_rn(s, a));
  return {s, e};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo = __dadd_rn(s.lo, t.hi);
  s = fast_two_sum(s.hi, s.lo);
  s.lo = __dadd_rn(s.lo, t.lo);
  return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd dd_add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  s.lo = __dadd_rn(s.lo, a.lo);
  return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  double p = __dmul_rn(a.hi, b.hi);
  double e = __fma_rn(a.hi, b.hi, -p);
  e = __fma_rn(a.hi, b.lo, e);
  e = __fma_rn(a.lo, b.hi, e);
  return fast_two_sum(p, e);
}
__device__ __forceinline__ dd dd_shfl_down(dd v, int delta) {
  v.hi = __shfl_down_sync(0xffffffffu, v.hi, delta);
  v.lo = __shfl_down_sync(0xffffffffu, v.lo, delta);
  return v;
}

// Sum2 step (Ogita, Rump, Oishi: "Accurate sum and dot product", 2005):
// (s, c) += (th, tl) with the rounding error of the high sum kept in c.
__device__ __forceinline__ void sum2_add(double& s, double& c, double th, double tl) {
  const dd r = two_sum(s, th);
  s = r.hi;
  c = __dadd_rn(c, __dadd_rn(r.lo, tl));
}

// Compensated accumulator: running (hi, lo) with TwoSum on every add.
struct Acc {
  double hi = 0.0, lo = 0.0;
  __device__ __forceinline__ void add(double v) {
    dd s = two_sum(hi, v);
    hi = s.hi;
    lo = __dadd_rn(lo, s.lo);
  }
  __device__ __forceinline__ dd value() const { return fast_two_sum_safe(); }
  __device__ __forceinline__ dd fast_two_sum_safe() const { return two_sum(hi, lo); }
};

// Deterministic dd reduction of one value per thread to thread 0 of the
// block.  `red` must hold blockDim.x / 32 dd entries.  Returns the block
// total in thread 0 (other threads get an unspecified value).
__device__ __forceinline__ dd block_reduce_dd(dd v, dd* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) v = dd_add(v, dd_shfl_down(v, d));
  if (lane == 0) red[warp] = v;
  __syncthreads();
  dd t = {0.0, 0.0};
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    t = lane < nw ? red[lane] : dd{0.0, 0.0};
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) t = dd_add(t, dd_shfl_down(t, d));
  }
  return t;
}

// Grid-level completion: every block stores its dd partial, the block that
// finishes last (atomic ticket) sums all partials in block order -- the
// result is therefore independent of block scheduling -- writes it to *out
// multiplied by `factor` (a power of two, exact), and re-arms the ticket.
// `partials` holds gridDim.x entries, `ticket` starts (and ends) at 0.
__device__ __forceinline__ void grid_finish_dd(dd block_total, dd* partials, unsigned* ticket,
                                               double* out, double factor, dd* red) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = block_total;
    __threadfence();
    unsigned prev = atomicAdd(ticket, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // Ordered sum by warp 0: each lane sums a strided slice in index order,
  // then the 32 lane sums are combined in a fixed tree.
  dd s = {0.0, 0.0};
  if (threadIdx.x < 32) {
    for (unsigned b = threadIdx.x; b < gridDim.x; b += 32) {
      dd p;
      p.hi = __ldcg(&partials[b].hi);
      p.lo = __ldcg(&partials[b].lo);
      s = dd_add(s, p);
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) s = dd_add(s, dd_shfl_down(s, d));
    if (threadIdx.x == 0) {
      out[0] = s.hi * factor;
      out[1] = s.lo * factor;
      *ticket = 0u;
      __threadfence();
    }
  }
  (void)red;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).  Counter = (trial lo, trial hi, step, stream tag),
// key = (seed lo, seed hi).
// ---------------------------------------------------------------------------
struct u32x4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = {hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}

constexpr uint32_t kTagRasmussen = 0x52415330u;  // "RAS0"
constexpr uint32_t kTagScaling = 0x5343414cu;    // "SCAL"

__device__ __forceinline__ u32x4 philox_step(uint64_t seed, uint64_t trial, uint32_t step,
                                             uint32_t tag) {
  return philox4x32_10({(uint32_t)trial, (uint32_t)(trial >> 32), step, tag}, (uint32_t)seed,
                       (uint32_t)(seed >> 32));
}

// Trial weight: FP32 significand in [0.5, 1) with a separate integer binary
// exponent (the integer part of log2 of the weight, kept exactly), so a
// product of up to n factors never leaves FP32 range.  Renormalised by bit
// manipulation after each factor; identical on host and device.
struct WExp {
  float m = 0.5f;
  int e = 1;
  __device__ __forceinline__ void mul(float f) {
    float p = __fmul_rn(m, f);
    uint32_t b = __float_as_uint(p);
    int ex = (int)((b >> 23) & 0xffu) - 126;
    b = (b & 0x807fffffu) | (126u << 23);
    m = __uint_as_float(b);
    e += ex;
  }
  __device__ __forceinline__ double value() const { return ldexp((double)m, e); }
};

}  // namespace perm



namespace perm {

// ---------------------------------------------------------------------------
// Shared-memory staging with the Blackwell bulk-copy (TMA) engine:
// cp.async.bulk global -> shared, completion tracked by an mbarrier
// transaction count.  Source and destination must be 16-byte aligned and the
// size a multiple of 16 (callers pad their packed buffers).  Each CTA copies
// from this GPU's global memory into its own shared memory only.  The wait is
// bounded: after kMbarSpinLimit polls the kernel
// records an error in *err and carries on without the data (callers then
// skip their compute), so a lost completion can never hang the GPU.
// ---------------------------------------------------------------------------
constexpr uint32_t kMbarSpinLimit = 1u << 20;  // x 64 ns backoff: ~0.1 s
constexpr uint32_t kBulkPiece = 32768;

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* sdst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
      "l"(gsrc), "r"(bytes), "r"(b)
      : "memory");
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t it = 0; it < kMbarSpinLimit; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    __nanosleep(64);
  }
  return false;
}

// Stage `bytes` (multiple of 16) from global to shared with bulk copies.
// Every thread of the block must call it; returns false (and sets *err) if
// the completion did not arrive within the spin limit.  `inject_extra` > 0
// is the failure-injection hook: the barrier then expects that many bytes
// more than are copied, so its phase never completes although every copy
// does (nothing stays in flight), and both bounded waits give up.
__device__ __forceinline__ bool stage_to_smem(void* sdst, const void* gsrc, uint32_t bytes,
                                              uint64_t* bar, int* err, uint32_t inject_extra = 0) {
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar, bytes + inject_extra);
    for (uint32_t off = 0; off < bytes; off += kBulkPiece) {
      uint32_t piece = bytes - off < kBulkPiece ? bytes - off : kBulkPiece;
      bulk_g2s((char*)sdst + off, (const char*)gsrc + off, piece, bar);
    }
  }
  bool ok = mbar_wait_bounded(bar, 0);
  if (!ok) {
    atomicExch(err, 1);
    mbar_wait_bounded(bar, 0);  // second bounded wait for the copy in flight
  }
  ok = __syncthreads_and(ok);
  return ok;
}

}  // namespace perm
