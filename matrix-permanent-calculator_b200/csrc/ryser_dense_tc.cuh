// ryser_dense_tc.cuh -- dense exact permanent for small-integer matrices with
// the row-sum vectors generated by the 5th-generation tensor cores (tcgen05,
// kind::i8, accumulators in tensor memory).
//
// Same sum as the int32-X kernel (ryser_dense_int.cuh; the reference's
// kernel_xshared_coalescing_mshared, gpu_exact_dense.cu:330-399, restated):
//   perm(A) = (4(n&1)-2) / 2^n * sum_{S subset of columns 0..n-2} (-1)^|S| prod_j y_j(S),
//   y_j(S) = 2 a[j][n-1] - rowsum_j + sum_{k in S} 2 a[j][k]     (exact integers)
// but the subsets are not walked one column update at a time.  They are split
// into rounds x 4 blocks x 128 lanes (512 subsets per round):
//   * lane l in [0, 128) chooses columns 0..6 (bit k of l <-> column k);
//   * block p in [0, 4) chooses columns 7 and 8;
//   * round r chooses the remaining RB = n - 10 columns 9..n-2 by the Gray
//     code of r, so consecutive rounds differ in one column.
// A round's 128 x 4 x n values y are int32 tensor-memory accumulators of
// one MMA with N = 4 NP columns (NP = n rounded up to 16; block p at column
// p NP):
//   * the first two rounds of a CTA are formed from scratch: D = A0 B^T with
//     K bytes [1, 64, 64 | bits of l] in A0 and [b0, b1, b2 | 2a[j][0..6]] in
//     B, where b0 + 64 b1 + 64 b2 = y_base(r)_j + block p's columns;
//   * every later round advances its buffer (two buffers, rounds alternate)
//     by two Gray steps in place, D += (+-1) 1 c0^T + (+-1) 1 c^T, in ONE
//     accumulate MMA: of two consecutive Gray steps one always toggles round
//     column 0.  B holds every round column's doubled values in its K bytes;
//     the A operand selects two K bytes with their signs and is stored as 8
//     rows only (stride byte offset 0 repeats them for all 128 lanes).
// So the tensor core does the n integer adds of every Gray step, and no
// shared memory is written after start-up.  Consumer threads only form the
// products (grouped int32 multiplies, FP64 across groups, as in the int32-X
// kernel) of the values they read with tcgen05.ld.
//
// CTA (one per SM; it allocates all 512 TMEM columns as two 256-column
// buffers): warps 0-15 are four consumer warpgroups, warpgroup p reading
// block p (thread t of the warpgroup reads TMEM lane t, subset l = t); warp
// 16 issues the MMAs.  A buffer alternates between "full" (an mbarrier that
// tcgen05.commit completes) and "empty" (an mbarrier that the 16 consumer
// warps arrive on once their tcgen05.ld of it has completed, before they form
// the products).  Every wait is bounded and also ends when another thread has
// flagged an abort; after an abort the producer waits (bounded) for its MMAs
// in flight before the tensor memory is freed.
//
// Requirements (checked on the host): integer entries with |2a| <= 127, the
// int32 product grouping of the int32-X kernel, 16 <= n <= 64.
#pragma once
#include "ryser_dense_int.cuh"

namespace perm {

constexpr int kTcLow = 7;                   // subset bits chosen by the MMA's 128 rows
constexpr int kTcBlocks = 4;                // blocks per round = consumer warpgroups
constexpr int kTcThreads = kTcBlocks * 128 + 32;  // plus one MMA-issuing warp
constexpr int kTcBufCols = 256;             // TMEM columns per buffer
constexpr int kTcPairOps = 31 * 4;          // column-pair selectors: K byte 1..31 x 4 signs
constexpr uint32_t kTcMinSmem = 116 * 1024; // keeps residency at one CTA per SM

struct DenseTcArgs {
  const int* colI;   // colI[k * np4 + j] = 2 a[j][k], then y0 (np4 entries)
  int np4;
  uint64_t round0, nrounds;  // rounds of this launch
  dd* partials;
  unsigned* ticket;
  double* out;
  int* err;
  int inject;  // failure injection (tests): the "empty" barriers expect one arrival more than is made
};

__host__ __device__ constexpr int tc_np(int n) { return (n + 15) & ~15; }
__host__ __device__ constexpr int tc_round_bits(int n) { return n - 1 - kTcLow - 2; }

// shared-memory layout (bytes), in order: A0 (4096), the pair selectors
// (kTcPairOps x 256), B of the first two rounds (2 x 4 NP x 32), the round
// columns (2 x 4 NP x 32: columns 0..31, then column 0 and 32..), the staged
// doubled columns and y0, the reduction scratch, 5 mbarriers, the TMEM
// address and the abort flag.
__host__ __device__ inline size_t dense_tc_smem_bytes(int n) {
  const int np = tc_np(n), np4 = (n + 3) & ~3;
  const size_t need = 4096 + (size_t)kTcPairOps * 256 + 4 * (size_t)(4 * np * 32) +
                      sizeof(int) * (size_t)(n + 1) * np4 + 32 * sizeof(dd) + 5 * sizeof(uint64_t) + 16;
  return need < kTcMinSmem ? kTcMinSmem : need;
}

// ---- tcgen05 / TMEM primitives (inline PTX) -------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major without swizzle: core matrices of
// 8 rows x 16 bytes stored contiguously (128 bytes); the second 16-byte K
// chunk of a row group follows at +128 bytes (leading byte offset), the next
// group of 8 rows at +sbo bytes (stride byte offset); bits 46-47 = 1 (sm_100).
// A stride byte offset of 0 makes every group of 8 rows read the same 8
// stored rows (used for operands whose 128 rows are all alike).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t sbo = 256u) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128u >> 4) << 16;
  d |= (uint64_t)(sbo >> 4) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// Instruction descriptor of kind::i8: D s32, A and B signed int8, both
// K-major, N = n_cols, M = 128.
__host__ __device__ constexpr uint32_t i8_idesc(int n_cols) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n_cols >> 3) << 17) | ((128u >> 4) << 24);
}

// D (TMEM) = A B^T, or D += A B^T when `accumulate` is non-zero
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

#define PERM_R(i) "=r"(v[(i)])
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : PERM_R(0), PERM_R(1), PERM_R(2), PERM_R(3), PERM_R(4), PERM_R(5), PERM_R(6), PERM_R(7), PERM_R(8),
        PERM_R(9), PERM_R(10), PERM_R(11), PERM_R(12), PERM_R(13), PERM_R(14), PERM_R(15)
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : PERM_R(0), PERM_R(1), PERM_R(2), PERM_R(3), PERM_R(4), PERM_R(5), PERM_R(6), PERM_R(7)
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : PERM_R(0), PERM_R(1), PERM_R(2), PERM_R(3)
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : PERM_R(0), PERM_R(1) : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld1(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : PERM_R(0) : "r"(taddr));
}
#undef PERM_R

// N consecutive columns of this thread's TMEM lane (taddr carries the warp's
// lane base); the values are valid after tmem_wait<N>.
template <int N>
__device__ __forceinline__ void tmem_load_row(uint32_t taddr, int (&v)[N]) {
  int c = 0;
#pragma unroll
  for (; c + 16 <= N; c += 16) tmem_ld16(taddr + c, v + c);
  if (N - c >= 8) {
    tmem_ld8(taddr + c, v + c);
    c += 8;
  }
  if (N - c >= 4) {
    tmem_ld4(taddr + c, v + c);
    c += 4;
  }
  if (N - c >= 2) {
    tmem_ld2(taddr + c, v + c);
    c += 2;
  }
  if (N - c >= 1) tmem_ld1(taddr + c, v + c);
}
// Wait for this thread's TMEM loads, then tie every loaded register to the
// wait so that no use is scheduled before it.
template <int N>
__device__ __forceinline__ void tmem_wait(int (&v)[N]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < N; j++) asm volatile("" : "+r"(v[j]));
}

// Bounded wait on an mbarrier phase with mbarrier.try_wait (the thread is
// suspended in hardware until the phase completes or a time hint of ~1 us
// runs out, so it wakes as soon as the phase completes): false after
// kMbarSpinLimit tries (about a second) or, when `abort` is not null, as soon
// as *abort is set by another thread of the CTA.
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity, const volatile int* abort) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < kMbarSpinLimit; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(1000u)
        : "memory");
    if (ok) return true;
    if (abort && *abort) return false;
  }
  return false;
}

// int8 digits of a base value: v = b0 + 64 b1 + 64 b2 with b0 in [-32, 31],
// |b1|, |b2| <= 127 (|v| <= 16000 is guaranteed by the host), packed with
// byte 3 of the K row (the value of column 0) into one word.
__device__ __forceinline__ uint32_t base_digits(int v, uint32_t byte3) {
  const int b0 = ((v + 32) & 63) - 32;
  const int rest = (v - b0) >> 6;
  const int b1 = rest > 127 ? 127 : (rest < -127 ? -127 : rest);
  const int b2 = rest - b1;
  return ((uint32_t)b0 & 0xFFu) | (((uint32_t)b1 & 0xFFu) << 8) | (((uint32_t)b2 & 0xFFu) << 16) | (byte3 << 24);
}

// byte offset of (row, k byte) in a K-major no-swizzle 32-byte-K operand
__host__ __device__ constexpr int kmajor_offset(int row, int kb) {
  return (row >> 3) * 256 + (kb >> 4) * 128 + (row & 7) * 16 + (kb & 15);
}

template <int N, int G>
__global__ void __launch_bounds__(kTcThreads, 1) ryser_dense_tc_kernel(DenseTcArgs args) {
  constexpr int NP = tc_np(N), RB = tc_round_bits(N), NALL = kTcBlocks * NP;
  constexpr uint32_t IDESC = i8_idesc(NALL);
  constexpr int BSZ = NALL * 32;  // bytes of one B operand
  static_assert(NALL <= kTcBufCols && RB >= 1 && RB <= 63, "order outside 16..64");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* sA0 = smem_raw;                                 // first-round A
  unsigned char* sSel = sA0 + 4096;                              // pair selectors, 256 B each
  unsigned char* sBI = sSel + kTcPairOps * 256;                  // first-round B [2]
  unsigned char* sBR = sBI + 2 * BSZ;                            // round-column B [2]
  int* sC = reinterpret_cast<int*>(sBR + 2 * BSZ);               // doubled columns, then y0
  const int np4 = args.np4;
  dd* red = reinterpret_cast<dd*>(sC + (size_t)(N + 1) * np4);
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 32);         // [0] staging
  uint64_t* full = bar + 1;                                      // [b]
  uint64_t* empty = bar + 3;                                     // [b]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 5);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int g = warp >> 2;            // block of a consumer warp (kTcBlocks for the producer warp)
  const int l = t & 127;              // TMEM lane = subset of columns 0..6
  constexpr int kProducer = 4 * kTcBlocks;

  const bool staged = stage_to_smem(sC, args.colI, (uint32_t)(sizeof(int) * (N + 1) * np4), bar, args.err);
  const int* sY0 = sC + (size_t)N * np4;
  auto colv = [&](int k, int j) -> int { return sC[k * np4 + j]; };  // 2 a[j][k]

  // this CTA's rounds
  const uint64_t per = args.nrounds / gridDim.x, extra = args.nrounds % gridDim.x;
  const uint64_t r_begin = args.round0 + per * blockIdx.x + (blockIdx.x < extra ? blockIdx.x : extra);
  const uint64_t nr = per + (blockIdx.x < extra ? 1 : 0);

  Acc acc;
  if (staged && nr > 0) {
    // ---- constant operands ----
    if (t < 128) {
      uint32_t w[4] = {1u | (64u << 8) | (64u << 16) | ((uint32_t)(t & 1) << 24), 0u, 0u, 0u};
#pragma unroll
      for (int k = 1; k < kTcLow; k++) w[(3 + k) >> 2] |= (uint32_t)((t >> k) & 1) << (8 * ((3 + k) & 3));
      *reinterpret_cast<uint4*>(sA0 + kmajor_offset(t, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4*>(sA0 + kmajor_offset(t, 16)) = make_uint4(0u, 0u, 0u, 0u);
    }
    // selector (pos, s0, sc): 8 rows [s0 at K byte 0, sc at K byte pos]
    for (int idx = t; idx < kTcPairOps * 8; idx += kTcThreads) {
      const int op = idx >> 3, row = idx & 7, pos = 1 + (op >> 2);
      const uint32_t s0 = (op & 2) ? 0xFFu : 1u, sc = (op & 1) ? 0xFFu : 1u;
      uint32_t w[8] = {s0, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
      w[pos >> 2] |= sc << (8 * (pos & 3));
      unsigned char* m = sSel + op * 256;
      *reinterpret_cast<uint4*>(m + kmajor_offset(row, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4*>(m + kmajor_offset(row, 16)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
    // round-column operands: row p NP + j, K byte kb = 2 a[j][9 + c]
    // (matrix 0: c = kb for kb < 32; matrix 1: c = 0 at kb 0, c = 31 + kb after)
    for (int idx = t; idx < 2 * NALL; idx += kTcThreads) {
      const int m = idx / NALL, row = idx % NALL, j = row % NP;
      uint32_t w[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
      if (j < N) {
#pragma unroll 1
        for (int kb = 0; kb < 32; kb++) {
          const int c = m == 0 ? kb : (kb == 0 ? 0 : 31 + kb);
          if (c < RB) w[kb >> 2] |= ((uint32_t)colv(9 + c, j) & 0xFFu) << (8 * (kb & 3));
        }
      }
      unsigned char* dst = sBR + m * BSZ;
      *reinterpret_cast<uint4*>(dst + kmajor_offset(row, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4*>(dst + kmajor_offset(row, 16)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
    // first two rounds: row p NP + j = [digits of y_base(r)_j + block p's columns | 2a[j][0..6]]
    for (int row = t; row < NALL; row += kTcThreads) {
      const int p = row / NP, j = row % NP;
      uint32_t w[4] = {0u, 0u, 0u, 0u};
      int yb = 0;
      if (j < N) {
#pragma unroll
        for (int k = 0; k < kTcLow; k++) w[(3 + k) >> 2] |= ((uint32_t)colv(k, j) & 0xFFu) << (8 * ((3 + k) & 3));
        yb = sY0[j] + ((p & 1) ? colv(7, j) : 0) + ((p & 2) ? colv(8, j) : 0);
        const uint64_t gr = r_begin ^ (r_begin >> 1);
#pragma unroll 1
        for (int k = 0; k < RB; k++)
          if ((gr >> k) & 1) yb += colv(9 + k, j);
      }
      const uint32_t byte3 = w[0] >> 24;
#pragma unroll
      for (int b = 0; b < 2; b++) {
        if (b == 1 && j < N) {
          const uint64_t r1 = r_begin + 1;  // Gray step to the second round
          const int k = __ffsll((long long)r1) - 1;
          if (k < RB) yb += (((r1 ^ (r1 >> 1)) >> k) & 1) ? colv(9 + k, j) : -colv(9 + k, j);
        }
        const uint32_t w0 = j < N ? base_digits(yb, byte3) : 0u;
        unsigned char* dst = sBI + b * BSZ;
        *reinterpret_cast<uint4*>(dst + kmajor_offset(row, 0)) = make_uint4(w0, w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(dst + kmajor_offset(row, 16)) = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    if (warp == kProducer) {
      tmem_alloc(tslot, 512);
      tmem_relinquish();
    }
    if (t == 0) {
      mbar_init(&full[0], 1);
      mbar_init(&full[1], 1);
      // (with args.inject, one arrival more than the consumers make: the
      // producer's bounded wait for a free buffer gives up at the third
      // round, after which only committed MMAs remain and are drained)
      mbar_init(&empty[0], 4 * kTcBlocks + (args.inject ? 1 : 0));
      mbar_init(&empty[1], 4 * kTcBlocks + (args.inject ? 1 : 0));
      *abort_flag = 0;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    int last_bar = -1;        // producer: barrier and parity of its last commit
    uint32_t last_parity = 0;
    if (warp == kProducer) {
      // ---- producer: lane 0 issues every MMA ----
      if (lane == 0) {
#pragma unroll 1
        for (uint64_t q = 0; q < nr; q++) {
          const int b = (int)(q & 1);
          const uint32_t dcol = tmem + (uint32_t)(b * kTcBufCols);
          if (q < 2) {
            mma_i8(dcol, kmajor_desc(smem_addr(sA0)), kmajor_desc(smem_addr(sBI + b * BSZ)), IDESC, 0u);
          } else {
            // the buffer holds round r - 2 once its consumers are done with it
            if (!tc_wait(&empty[b], (uint32_t)(((q - 2) >> 1) & 1), abort_flag)) {
              atomicExch(args.err, 3);
              *abort_flag = 1;
              break;
            }
            tc_fence_after();
            // Gray steps r-2 -> r-1 and r-1 -> r toggle bits ctz(r-1) and ctz(r):
            // one of them is round column 0
            const uint64_t r = r_begin + q;
            const int k1 = __ffsll((long long)(r - 1)) - 1, k2 = __ffsll((long long)r) - 1;
            const uint64_t g1 = (r - 1) ^ ((r - 1) >> 1), g2 = r ^ (r >> 1);
            const bool add1 = (g1 >> k1) & 1, add2 = (g2 >> k2) & 1;
            const int c = k1 ? k1 : k2;              // the other column
            const bool add0 = k1 ? add2 : add1, addc = k1 ? add1 : add2;
            const int m = c < 32 ? 0 : 1, pos = c < 32 ? c : c - 31;
            const int op = (pos - 1) * 4 + (add0 ? 0 : 2) + (addc ? 0 : 1);
            mma_i8(dcol, kmajor_desc(smem_addr(sSel + op * 256), 0u), kmajor_desc(smem_addr(sBR + m * BSZ)),
                   IDESC, 1u);
          }
          mma_commit(&full[b]);
          last_bar = b;
          last_parity = (uint32_t)((q >> 1) & 1);
          if (*abort_flag) break;
        }
      }
    } else {
      // ---- consumers: warpgroup g reads block g ----
      const uint32_t tl = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(g * NP);
#pragma unroll 1
      for (uint64_t q = 0; q < nr; q++) {
        const int b = (int)(q & 1);
        if (!__all_sync(0xffffffffu, tc_wait(&full[b], (uint32_t)((q >> 1) & 1), abort_flag))) {
          if (lane == 0) {
            atomicExch(args.err, 3);
            *abort_flag = 1;
          }
          break;
        }
        tc_fence_after();
        int y[N];
        tmem_load_row<N>(tl + (uint32_t)(b * kTcBufCols), y);
        tmem_wait<N>(y);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[b]);
        const double s = group_product<N, G>(y);
        acc.add(((r_begin + q) & 1) ? -s : s);  // round sign (-1)^popc(gray(r)) = (-1)^r
      }
    }
    tc_fence_before();
    __syncthreads();
    if (*abort_flag && warp == kProducer && lane == 0 && last_bar >= 0) {
      // MMAs complete in issue order: once the last commit has arrived, none
      // is in flight; wait for it (bounded) before the tensor memory is freed
      if (!tc_wait(&full[last_bar], last_parity, nullptr)) atomicExch(args.err, 3);
    }
    __syncthreads();
    tc_fence_after();
    if (warp == kProducer) tmem_dealloc(tmem, 512);
  }
  dd mine = acc.value();
  if ((__popc(l) + __popc(g & 3)) & 1) mine = {-mine.hi, -mine.lo};  // lane and block signs
  dd bt = block_reduce_dd(mine, red);
  const double factor = ((N & 1) ? 2.0 : -2.0) * ldexp(1.0, -N);
  grid_finish_dd(bt, args.partials, args.ticket, args.out, factor, red);
}

}  // namespace perm
