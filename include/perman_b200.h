/* perman_b200.h -- C ABI of the B200 matrix-permanent engine (libperman_b200.so).
 *
 * The library computes matrix permanents on an NVIDIA B200 (sm_100a) with
 * hand-written CUDA kernels.  Every entry point is plain C: caller-owned host
 * buffers, sizes as ints, an opaque context, int status codes.  There is no
 * CPU fallback: without a usable B200 every compute call fails with
 * PERM_ECUDA and a message.
 *
 * Reference interfaces replaced (berkyaglioglu/matrix-permanent-calculator):
 *   gpu_perman64_xshared_coalescing_mshared<T>          gpu_exact_dense.cu:641
 *   gpu_perman64_xshared_coalescing_mshared_multigpu<T> gpu_exact_dense.cu:702
 *   gpu_perman64_xshared_coalescing_mshared_skipper<T>  gpu_exact_sparse.cu:1124
 *   gpu_perman64_rasmussen<T>                           gpu_approximation_dense.cu:374
 *   gpu_perman64_approximation<T>                       gpu_approximation_dense.cu:528
 *   gpu_perman64_rasmussen_sparse                       gpu_approximation_sparse.cu:455
 *   gpu_perman64_approximation_sparse                   gpu_approximation_sparse.cu:608
 *   ReadMatrix / matrix2compressed[_sortOrder|_skipOrder] util.h:344, 523, 554, 622
 * The reference's templates are C++ functions returning a bare double; the
 * `gpu_perman64_*_{int,float,double}` entry points below keep those exact
 * argument lists for callers that bind them directly, and the perm_* entry
 * points are the status-returning form that new callers should use.
 */
#ifndef PERMAN_B200_H
#define PERMAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define PERM_OK 0
#define PERM_EINVAL (-1)       /* bad argument (size, pointer, option)          */
#define PERM_ECUDA (-2)        /* CUDA runtime error or no usable device        */
#define PERM_ENOMEM (-3)       /* device or pinned host allocation failed       */
#define PERM_EUNSUPPORTED (-4) /* valid request outside this build's limits     */
#define PERM_ETIMEOUT (-5)     /* a bounded device wait gave up (error flag)    */
#define PERM_EIO (-6)          /* matrix file could not be read or parsed       */

/* ---- element types of caller matrices ------------------------------------ */
#define PERM_F64 0
#define PERM_F32 1
#define PERM_I32 2

/* ---- kernels (perm_result.kernel) ---------------------------------------- */
#define PERM_KERNEL_DENSE 1   /* register-X Gray-code Ryser                 */
#define PERM_KERNEL_SKIPPER 2 /* SkipPer on CRS/CCS                          */
#define PERM_KERNEL_DENSE_INT 3 /* int32-X Gray-code Ryser (integer matrices) */
#define PERM_KERNEL_DENSE_DD 4  /* double-double Gray-code Ryser (orders <= 40) */
#define PERM_KERNEL_DENSE_TC 5  /* tensor-core row sums (kind::i8) + int32 products:
                                   integer matrices, |a| <= 63, orders 16..64 */
#define PERM_KERNEL_DENSE_SPLIT 6 /* split-X Gray-code Ryser: exact coarse row sums
                                     plus a small remainder, orders 4..40 */
#define PERM_KERNEL_DENSE_INT_DD 7 /* int32-X Gray-code Ryser with double-double
                                      products and sum: certified error bound for
                                      integer matrices, orders 8..64 */
#define PERM_KERNEL_DENSE_SDD 8 /* split X with double-double products and sum
                                   ("split-dd"): certified error bound for real
                                   matrices, orders 4..40; sparse matrices whose
                                   three sparsest columns touch <= 16 rows walk
                                   only those rows at 7 of 8 steps (orders 12..40) */

/* Limits of this build. */
#define PERM_MAX_EXACT_N 64  /* Gray indices are 64-bit                 */
#define PERM_MAX_MC_N 64     /* dense estimators: trial masks are 64-bit */
#define PERM_MAX_MC_SPARSE_N 2047 /* sparse estimators: bitsets            */

typedef struct perm_ctx perm_ctx;       /* one device, one stream, scratch */
typedef struct perm_matrix perm_matrix; /* device-resident dense matrix    */

typedef struct {
  double value;       /* permanent, hi + lo rounded to double               */
  double hi, lo;      /* double-double result                               */
  double steps;       /* Gray indices whose product was evaluated           */
  double total_steps; /* 2^(n-1), the dense Gray range                      */
  double kernel_ms;   /* device time of the compute kernel (CUDA events)    */
  int kernel;         /* PERM_KERNEL_*                                      */
  int n;
  double abs_term_sum;       /* estimate of sum_i |term(i)| (cancellation scale) */
  double rel_error_estimate; /* estimated relative error of (hi, lo) (0: not estimated);
                                value, their sum rounded once, adds at most 2^-53 */
} perm_result;

typedef struct {
  double mean;        /* estimate of the permanent of the 0/1 pattern       */
  double std_error;   /* sample standard deviation / sqrt(trials)           */
  double trials;
  double zero_trials; /* trials that ended on an empty row / zero sum       */
  double sum, sum_sq; /* raw accumulators                                   */
  double kernel_ms;
} perm_estimate;

/* ---- context --------------------------------------------------------------- */
int perm_version(void);                       /* 10000 * major + 100 * minor  */
int perm_device_count(void);                  /* visible CUDA devices, or <0  */
int perm_ctx_create(int device, perm_ctx** out);
void perm_ctx_destroy(perm_ctx* ctx);
const char* perm_ctx_last_error(const perm_ctx* ctx);
const char* perm_status_string(int status);

/* ---- exact permanents ------------------------------------------------------ */
/* Dense Ryser of a row-major n x n matrix (dtype PERM_F64/F32/I32), 1 <= n <= 64.
 * Replaces gpu_perman64_xshared_coalescing_mshared (gpu_exact_dense.cu:641). */
int perm_exact_dense(perm_ctx* ctx, const void* mat, int n, int dtype, perm_result* out);

/* Share `shard` of `nshards` of the same Gray walk; the permanent is the
 * double-double sum of all shards' (hi, lo).  Ranks of a multi-GPU job call
 * this with their rank and world size (replaces the per-device ranges of
 * gpu_exact_dense.cu:729-752). */
int perm_exact_dense_shard(perm_ctx* ctx, const void* mat, int n, int dtype, int shard, int nshards,
                           perm_result* out);
/* The Gray-index range [*first, *last) that shard `shard` of `nshards`
 * covers for order n.  Host only (no device): depends on (n, shard, nshards)
 * alone, so ranks on different devices always partition [0, 2^(n-1)). */
int perm_shard_range(int n, int shard, int nshards, uint64_t* first, uint64_t* last);
/* One permanent sharded over devices of this process: shard s of `nshards`
 * (1..64) runs perm_exact_dense_ex(variant) on device devices[s] (NULL:
 * device s; a device may appear more than once) in its own host thread and
 * context, and the shards' (hi, lo) are added in shard order in
 * double-double, so the value does not depend on which device finishes
 * first.  Each shard is evaluated once (no accuracy policy, no error
 * estimate: rel_error_estimate and abs_term_sum are 0; a caller wanting the
 * policy on the sum passes `out` to perm_exact_dense_refine); kernel_ms is
 * the slowest shard's.  On failure the failing shard's status is returned
 * and its message printed on stderr.  Replaces
 * gpu_perman64_xshared_coalescing_mshared_multigpu (gpu_exact_dense.cu:702). */
int perm_exact_dense_multi(const void* mat, int n, int dtype, int variant, int nshards, const int* devices,
                           perm_result* out);
/* The whole-walk value (io->hi, io->lo, io->kernel_ms) assembled from all
 * shards of perm_exact_dense_shard, given the error estimate and the
 * context's accuracy policy of perm_exact_dense (see perm_ctx_set_rel_target):
 * io is updated in place, its kernel_ms grows by any cross-check or
 * double-double launch.  No counterpart in the reference (which checks no
 * accuracy). */
int perm_exact_dense_refine(perm_ctx* ctx, const void* mat, int n, int dtype, perm_result* io);

/* SkipPer on CRS (rptrs, cols, rvals) + CCS (cptrs, rows, cvals) of an n x n
 * matrix, 1 <= n <= 64; only the stored entries are used (x0 from the CRS row
 * sums and CCS column n-1, algo.h:751-760).  Replaces
 * gpu_perman64_xshared_coalescing_mshared_skipper (gpu_exact_sparse.cu:1124). */
int perm_exact_sparse(perm_ctx* ctx, int n, const int* rptrs, const int* cols, const double* rvals,
                      const int* cptrs, const int* rows, const double* cvals, perm_result* out);
/* As perm_exact_sparse with an explicit kernel.  variant 0 (what
 * perm_exact_sparse uses) estimates the share of vanishing Gray terms from a
 * fixed sample of 2048 indices and runs SkipPer when at least 75% vanish, the
 * register kernels on the same (CRS) matrix otherwise (through
 * perm_exact_dense_ex's variant 0 and its accuracy policy); PERM_KERNEL_SKIPPER,
 * PERM_KERNEL_DENSE, PERM_KERNEL_DENSE_INT, PERM_KERNEL_DENSE_TC,
 * PERM_KERNEL_DENSE_INT_DD and PERM_KERNEL_DENSE_SDD force a kernel.
 * perm_result.kernel reports which ran. */
int perm_exact_sparse_ex(perm_ctx* ctx, int n, const int* rptrs, const int* cols, const double* rvals,
                         const int* cptrs, const int* rows, const double* cvals, int variant, perm_result* out);

/* Dense Ryser with an explicit kernel: variant 0 picks automatically (the
 * int32-X kernel for integer matrices whose grouped row products provably fit
 * in int32, the FP64-X kernel otherwise; perm_dense_autotune can switch
 * integer inputs to the FP64-X or the tensor-core kernel), PERM_KERNEL_DENSE
 * forces FP64 X, PERM_KERNEL_DENSE_INT forces int32 X, PERM_KERNEL_DENSE_TC
 * the tensor-core kernel (PERM_EUNSUPPORTED where not exact),
 * PERM_KERNEL_DENSE_INT_DD and PERM_KERNEL_DENSE_SDD the certified kernels
 * (integer / real matrices; PERM_EUNSUPPORTED outside their orders).  The
 * tensor-core kernel runs whole walks only: with nshards > 1 its matrices use
 * the int32-X kernel. */
int perm_exact_dense_ex(perm_ctx* ctx, const void* mat, int n, int dtype, int variant, int shard, int nshards,
                        perm_result* out);
/* Whole-walk dense results carry rel_error_estimate, a worst-case bound
 * formed from sum |term|, estimated by a sample of Ryser terms stratified by
 * subset size (exact for the split-X and the certified kernels, whose walks
 * sum their own terms).  The certified kernels' bound is of order
 * n u^2 sum|term| / |perm| (u = 2^-53): it meets 1e-10 unless the terms
 * cancel by more than ~1e18.
 * With variant 0 and a context target (default 1e-10; <= 0 disables the
 * policy; < 0 also skips the estimate):
 *  - a zero pattern without a perfect matching returns exactly 0;
 *  - whole walks of integer matrices whose group products fit in int32 run
 *    PERM_KERNEL_DENSE_INT_DD at once (about 1.4 int32-X walks), and real
 *    matrices of order 12..40 whose three sparsest columns touch so few rows
 *    R that the sparse layout's (7 (6R + 9) + 6n + 5) / 8 FP64 operations
 *    per Gray step are at most FP64 X's 2n run PERM_KERNEL_DENSE_SDD in
 *    that layout: their bound is the estimate, no other step runs;
 *  - for other nonnegative real matrices of order 28..40 the FP64-X walk's
 *    bound is predicted on the device before any walk (stratified sample of
 *    sum |term| and a weighted-Rasmussen estimate of perm, 4096 trials); when
 *    it is above 1.5x the target PERM_KERNEL_DENSE_SDD (about 4.2 FP64-X
 *    walks in the dense layout, less in the sparse one) runs at once and
 *    alone;
 *  - a result whose bound exceeds the target is cross-checked against
 *    B = A^T with its first row times 3 (perm(B) = 3 perm(A), independent
 *    roundings) and kept when max(4-sigma independent-rounding estimate from
 *    sum term^2, 16 |perm(A) - perm(B)/3| / |perm(A)|) meets the target, which
 *    then is the reported estimate; after an FP64-X first pass whose bound is
 *    above 4x the target this check is skipped where split-dd applies
 *    (orders 4..40), since it rarely passes there;
 *  - otherwise it is recomputed by a certified kernel: PERM_KERNEL_DENSE_INT_DD
 *    (integer, orders 8..64, directly after an int32-X first pass),
 *    PERM_KERNEL_DENSE_SDD (orders 4..40, about 4.2 FP64-X walks) or the
 *    double-double kernel (orders <= 40, where neither applies).
 * kernel_ms covers every launch.  PERM_KERNEL_DENSE_DD forces that kernel. */
int perm_ctx_set_rel_target(perm_ctx* ctx, double rel_target);

/* The kernel the accuracy policy starts a whole-walk perm_exact_dense call
 * with for this matrix: PERM_KERNEL_DENSE_INT_DD or PERM_KERNEL_DENSE_SDD
 * when a certified walk goes first and is the whole evaluation, 0 when the
 * FP64-X / int32-X walk goes first or the policy is off.  For nonnegative
 * real matrices of order 28..40 this runs the device prediction above (tens
 * of microseconds) and *fp64_bound (may be NULL) receives the predicted
 * FP64-X bound; otherwise 0.  The request loop uses it to run such requests
 * unsliced.  No counterpart in the reference. */
int perm_exact_dense_plan(perm_ctx* ctx, const void* mat, int n, int dtype, int* kernel, double* fp64_bound);

/* Failure-injection hook for tests of the bounded device waits.  The next
 * `launches` launches of the FP64-X dense kernel (PERM_KERNEL_DENSE) or of
 * the tensor-core kernel (PERM_KERNEL_DENSE_TC) on this context wait on a
 * barrier that never completes: the FP64-X kernel's operand staging expects
 * 16 bytes more than it copies (every copy still lands), the tensor-core
 * kernel's buffer-free barriers expect one arrival more than its consumers
 * make (its issued MMAs still complete and are drained).  Each bounded wait
 * gives up after its limit (a fraction of a second), the call returns
 * PERM_ETIMEOUT with a message naming the wait, nothing is left running on
 * the device, and the context stays usable.  0 switches it off.  No
 * counterpart in the reference (which has no device waits to bound). */
int perm_ctx_inject_wait_timeout(perm_ctx* ctx, int launches);

/* Host only (no device): the layout PERM_KERNEL_DENSE_SDD uses for the
 * row-major n x n matrix `mat`: the number of inner rows R of the sparse
 * layout (6, 8, 12, 16, or 20, 24, 28 with a rolled step loop for dense
 * matrices whose three sparsest columns still miss a quarter or more of the
 * rows: columns 0..2 after its permutation touch rows 0..R-1 only, so 7 of
 * 8 Gray steps walk R rows) or of the three-level layout's second level
 * (16..28, perm_sdd_levels), 0 for the dense layout,
 * PERM_EUNSUPPORTED where the kernel does not apply (orders outside 4..40,
 * row absolute sums at or above 2^1020), PERM_EINVAL for bad arguments.
 * No counterpart in the reference. */
int perm_sdd_layout(const double* mat, int n);

/* Host only: both levels of that layout.  levels[1] = the perm_sdd_layout
 * value; levels[0] = the first level R1 of the three-level layout (orders
 * 24..40: column 0 touches rows 0..R1-1 only, columns 1 and 2 rows
 * 0..levels[1]-1, so half of the Gray steps walk R1 rows and three in eight
 * levels[1]; R1 in 8..20), 0 for the other layouts.  PERM_OK, or the
 * statuses of perm_sdd_layout.  No counterpart in the reference. */
int perm_sdd_levels(const double* mat, int n, int* levels);

/* Host only (no device): the number of inner rows R (16, 20, 24 or 28) of
 * the two-level row layout that PERM_KERNEL_DENSE (the FP64-X walk) uses for
 * the row-major n x n matrix `mat` (orders 20..48: the three columns whose
 * nonzeros lie in the fewest rows go first, their rows to the top, and at
 * seven of every eight Gray steps only those R rows are updated and
 * multiplied), or the second level R2 (20..36) of its three-level layout
 * (perm_fp64_levels), 0 for the one-level walk; PERM_EINVAL for bad
 * arguments.  No counterpart in the reference. */
int perm_fp64_layout(const double* mat, int n);

/* Host only: both levels of that layout.  levels[1] = the perm_fp64_layout
 * value; levels[0] = the first level R1 (8..20) of the three-level layout
 * (orders 28..48: column 0 touches rows 0..R1-1 only, columns 1 and 2 rows
 * 0..levels[1]-1, so half of the Gray steps update R1 rows and three in
 * eight levels[1]), 0 for the other layouts.  PERM_OK or PERM_EINVAL.  No
 * counterpart in the reference. */
int perm_fp64_levels(const double* mat, int n, int* levels);

/* Host only (no device): the layout PERM_KERNEL_DENSE_INT (the int32-X walk)
 * uses for the row-major n x n matrix `mat`: returns the product-group size
 * G (3..6, every group's product fits int32) and fills levels[3]:
 *  - levels[0] > 0: the two-level row layout (orders 20..48): the three
 *    columns whose nonzeros lie in the fewest rows go first, and levels[0]
 *    groups of the rows they never touch keep their product for seven of
 *    every eight Gray steps;
 *  - levels[1], levels[2] > 0: the three-level layout (orders 28..48): the
 *    rows of column 0 (flipped at every other step) form levels[1] groups,
 *    the further rows of columns 1 and 2 levels[2] groups, and each level's
 *    product is recomputed only when a column that touches it flips;
 *  - all 0: the one-level walk.
 * The cheapest layout is taken.  PERM_EUNSUPPORTED where int32 X does not
 * apply, PERM_EINVAL for bad arguments.  No counterpart in the reference. */
int perm_int_layout(const double* mat, int n, int* levels);

/* Host only (no device): the layout PERM_KERNEL_DENSE_INT_DD uses for the
 * row-major n x n matrix `mat`: returns the product-group size G (3..6:
 * every run of G rows has prod(sum_k |a_jk|) < 2^31, so group values are
 * exact int32 products) and sets *pair to 1 when consecutive group values
 * are multiplied in int64 first (every run of 2G rows below 2^53, so those
 * products are exact; orders >= 16), 0 otherwise; the layout with the
 * fewest instructions per Gray step is taken.  levels[0] receives the
 * number of outer groups of the two-level row layout (orders 20..48, as
 * perm_int_layout: groups of 4 or 6 in pairs, or 5 alone), levels[1] and
 * levels[2] the first- and second-level groups of the three-level layout
 * (orders 28..48); all three 0 for one level.  PERM_EUNSUPPORTED for
 * non-integer matrices, |a| >= 2^24, orders below 8 or no fitting G;
 * PERM_EINVAL for bad arguments.  No counterpart in the reference. */
int perm_intc_layout(const double* mat, int n, int* pair, int* levels);

/* Measures, for orders n_lo..n_hi (within 8..40), which of the int32-X, the
 * FP64-X and (n >= 16) the tensor-core kernel is fastest on this device for
 * integer inputs and makes variant 0 follow the measurement in this context.
 * choice_out receives n_hi - n_lo + 1 kernel ids. */
int perm_dense_autotune(perm_ctx* ctx, int n_lo, int n_hi, int* choice_out);

/* Device-resident dense matrices: upload once, run many times (no host copy
 * inside perm_exact_dense_resident). */
int perm_matrix_create_dense(perm_ctx* ctx, const void* mat, int n, int dtype, perm_matrix** out);
int perm_matrix_create_dense_ex(perm_ctx* ctx, const void* mat, int n, int dtype, int variant, perm_matrix** out);
void perm_matrix_destroy(perm_ctx* ctx, perm_matrix* m);
int perm_exact_dense_resident(perm_ctx* ctx, const perm_matrix* m, perm_result* out);
/* Shard `shard` of `nshards` of a resident matrix's walk (the ranges of
 * perm_exact_dense_shard / perm_shard_range); the tensor-core kernel runs
 * whole walks only (PERM_EINVAL for nshards > 1).  Replaces the per-device
 * ranges of gpu_exact_dense.cu:729-752 without a host copy per call. */
int perm_exact_dense_resident_shard(perm_ctx* ctx, const perm_matrix* m, int shard, int nshards,
                                    perm_result* out);

/* The tensor-core kernel over rounds [round0, round0 + nrounds) only: the
 * subsets whose columns 9 .. n-2 follow the Gray code of the round index,
 * every choice of columns 0 .. 8 (512 subsets per round), scaled like the
 * whole sum; round indices go up to 2^(n - 10).  No counterpart in the
 * reference: for verification of the kernel at orders whose full walk is
 * long, and for callers that partition the subsets themselves. */
int perm_exact_dense_tc_rounds(perm_ctx* ctx, const void* mat, int n, int dtype, uint64_t round0,
                               uint64_t nrounds, perm_result* out);

/* ---- allocation-free dense exact permanent ------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory themselves or have it allocated behind their back: code running
 * inside another framework's memory pool, plugins in a host process that owns
 * every device allocation, work issued while allocation is forbidden.  The
 * caller passes a device-resident row-major n x n matrix `d_mat` and a device
 * buffer `d_out` of two doubles that receives (hi, lo); everything else lives
 * in one static device array (~96 KB per GPU that loads this library, held
 * until the process exits).  No cudaMalloc or cudaFree is called.
 *  - the computation is the one-level FP64-X walk with the launch
 *    decomposition and X re-anchoring of perm_exact_dense_ex(PERM_KERNEL_DENSE)'s
 *    one-level walks, so its value equals that call's to the last bit on the
 *    same device wherever that call also walks one level (orders below 20,
 *    and matrices without a sparse enough column triple); where that call
 *    walks a two- or three-level row layout the two agree to rounding.
 *    Unlike perm_exact_dense it returns no error estimate and applies no
 *    accuracy policy (no int32-X, split-dd or double-double pass), so on
 *    matrices with heavy cancellation its error is that of one FP64-X walk;
 *  - orders 1..64; larger orders return PERM_EUNSUPPORTED (the array holds one
 *    64 x 64 operand and partials for 4096 CTAs), null pointers PERM_EINVAL;
 *  - runs asynchronously on `stream` (a cudaStream_t, NULL = default stream);
 *    a staging timeout turns d_out into NaN;
 *  - the first call on a device does that device's one-time set-up (the
 *    array's device address and the kernel's occupancy): make it before any
 *    stream capture;
 *  - all calls on a device share the array and it keeps the last call's
 *    contents: calls that overlap on the GPU race, so order them on one stream
 *    or synchronise between them. */
int perm_exact_dense_noalloc(const double* d_mat, int n, double* d_out, void* stream);

/* ---- batches: many exact permanents in one persistent launch -------------------- */
/* A batch holds `count` row-major matrices concatenated in `values` (matrix i
 * has order orders[i], 1 <= order <= 40, and occupies orders[i]^2 doubles).
 * perm_batch_create uploads them and captures the run (queue reset, one
 * persistent kernel, result readback) as a CUDA graph; perm_batch_run replays
 * it and writes (hi, lo) per matrix into results[2 * count] in caller order
 * (the plain FP64-X values: no error estimate, no accuracy policy).
 * No counterpart in the reference, which computes one matrix per call
 * (gpu_exact_dense.cu:641); each result equals perm_exact_dense's to rounding. */
typedef struct perm_batch perm_batch;
int perm_batch_create(perm_ctx* ctx, int count, const int* orders, const double* values, perm_batch** out);
int perm_batch_run(perm_ctx* ctx, perm_batch* b, double* results, double* kernel_ms);
/* As perm_batch_run, and: the batch kernel also sums |term| per matrix, from
 * which each result's worst-case relative-error bound is formed (rel_err[count],
 * may be NULL); matrices above the context's target (perm_ctx_set_rel_target)
 * go through perm_exact_dense_ex's policy with the batch value as the first
 * evaluation (exact zero, cross-check or double-double), their count in
 * *reruns; kernel_ms includes those launches. */
int perm_batch_run_ex(perm_ctx* ctx, perm_batch* b, double* results, double* rel_err, int* reruns,
                      double* kernel_ms);
void perm_batch_destroy(perm_ctx* ctx, perm_batch* b);
int perm_batch_exact(perm_ctx* ctx, int count, const int* orders, const double* values, double* results,
                     double* kernel_ms);
/* Measures, for each order in [n_lo, n_hi], the batch kernel with every
 * candidate lane-range length and keeps the fastest in the context (used by
 * later perm_batch_create calls); then measures every compiled batch kernel
 * variant that covers order n_hi -- threads per block (64, 128, 256), the
 * register budget it was compiled for (CTAs per SM), and FP64 X of dense
 * matrices in registers or in shared memory -- on a mixed batch of these
 * orders and keeps the fastest for later batches whose orders it covers.
 * m_out receives n_hi - n_lo + 1 exponents.  Per matrix, perm_batch_create
 * also picks the dense or the sparse layout (orders 12..32: three columns
 * whose nonzeros lie in at most 8 / 16 rows for FP64 X, 6 / 12 rows for
 * int32 X; those rows are walked alone at seven of eight Gray steps, and in
 * int32 X a group whose other rows' product is 0 skips its seven vanishing
 * terms). */
int perm_batch_autotune(perm_ctx* ctx, int n_lo, int n_hi, int* m_out);
/* The batch kernel variant later perm_batch_create calls use (0 = the
 * general one, orders up to 40): its largest order, threads per block, CTAs
 * per SM it was compiled for, and whether dense FP64 matrices keep X in
 * shared memory. */
int perm_batch_variant(perm_ctx* ctx, int* variant, int* max_n, int* block, int* min_blocks, int* shared_x);
/* Makes later perm_batch_create calls use batch kernel variant `variant`
 * (0 .. 5; a batch with an order above the variant's largest falls back to
 * variant 0). */
int perm_batch_use_variant(perm_ctx* ctx, int variant);

/* ---- request loop: continuous batching on one GPU ------------------------------
 * No counterpart in the reference.  `slots` worker contexts run requests
 * concurrently (each with its own stream and resident scratch); a request is
 * admitted when a slot is idle and its device-memory need fits the budget
 * (0 = half the free device memory).  Exact requests longer than
 * `slice_steps` Gray indices (0 = 2^31) run as several shard launches so small
 * requests interleave.  The request's matrix is copied at submit.  A request
 * that does not fit the remaining budget may be passed by later, smaller ones
 * at most 8 times; then admission waits for it. */
#define PERM_REQ_EXACT_DENSE 0
#define PERM_REQ_EXACT_SPARSE 1
#define PERM_REQ_RASMUSSEN 2
#define PERM_REQ_SCALING 3
typedef struct {
  int kind;            /* PERM_REQ_*                                      */
  int n;
  const double* mat;   /* row-major n x n                                */
  int64_t trials;      /* Monte-Carlo kinds                              */
  int scale_intervals; /* PERM_REQ_SCALING                               */
  int scale_times;
  uint64_t seed;
} perm_request;
typedef struct {
  int status;          /* PERM_OK or the failing call's status           */
  int kernel;          /* PERM_KERNEL_* for exact kinds                  */
  double value, hi, lo, std_error;
  double t_submit_ms, t_admit_ms, t_done_ms; /* since server creation      */
  double device_ms;    /* sum of the request's kernel times              */
  char message[160];
} perm_response;
typedef struct perm_server perm_server;
int perm_server_create(int device, int slots, size_t memory_budget, uint64_t slice_steps, perm_server** out);
int perm_server_submit(perm_server* s, const perm_request* req, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: forever) and hands the response over once. */
int perm_server_wait(perm_server* s, uint64_t ticket, int timeout_ms, perm_response* out);
/* out5 = submitted, completed, in flight, queued, device bytes in use. */
int perm_server_stats(perm_server* s, double* out5);
/* Finishes the requests already running, ends every queued one with status
 * PERM_EINVAL ("server destroyed before the request ran"), lets threads
 * blocked in perm_server_wait return with their response, then frees the
 * server.  No other call on `s` may start once destroy has begun. */
void perm_server_destroy(perm_server* s);

/* ---- Monte-Carlo estimates of the permanent of the 0/1 pattern -------------- */
/* trials >= 1 run exactly (the reference rounds up to a multiple of 1024);
 * trial t uses Philox stream (seed, t) so results do not depend on the launch
 * shape.  trial_values, if not NULL, receives the `trials` per-trial weights. */
int perm_approx_rasmussen(perm_ctx* ctx, const void* mat, int n, int dtype, int64_t trials,
                          uint64_t seed, double* trial_values, perm_estimate* out);
int perm_approx_scaling(perm_ctx* ctx, const void* mat, int n, int dtype, int64_t trials,
                        int scale_intervals, int scale_times, uint64_t seed, double* trial_values,
                        perm_estimate* out);
/* Trials [trial0, trial0 + trials) of the same estimate (same streams): the
 * multi-GPU split by trial id.  Ranges run on different devices give exactly
 * the per-trial weights of the whole run; their (sum, sum_sq, zero_trials)
 * add up to the whole run's.  Replaces the trial chunks that the
 * reference's multi-GPU estimators hand to each device
 * (gpu_perman64_rasmussen_multigpucpu_chunks, gpu_approximation_dense.cu:412;
 * gpu_perman64_approximation_multigpucpu_chunks, :574). */
int perm_approx_rasmussen_range(perm_ctx* ctx, const void* mat, int n, int dtype, int64_t trial0,
                                int64_t trials, uint64_t seed, double* trial_values, perm_estimate* out);
int perm_approx_scaling_range(perm_ctx* ctx, const void* mat, int n, int dtype, int64_t trial0,
                              int64_t trials, int scale_intervals, int scale_times, uint64_t seed,
                              double* trial_values, perm_estimate* out);
/* Sparse forms take the CRS of the pattern (columns ascending within a row),
 * orders 1..2047 (the reference's sparse kernels stop at 672); above 64 they
 * run a bitset kernel with the same streams and arithmetic, and the CCS
 * arguments of the scaling form are rebuilt from the CRS. */
int perm_approx_rasmussen_sparse(perm_ctx* ctx, int n, const int* rptrs, const int* cols,
                                 int64_t trials, uint64_t seed, double* trial_values,
                                 perm_estimate* out);
int perm_approx_scaling_sparse(perm_ctx* ctx, int n, const int* rptrs, const int* cols,
                               const int* cptrs, const int* rows, int64_t trials,
                               int scale_intervals, int scale_times, uint64_t seed,
                               double* trial_values, perm_estimate* out);
/* Trial ranges of the sparse forms (as perm_approx_*_range; the scaling
 * form rebuilds its CCS from the CRS). */
int perm_approx_rasmussen_sparse_range(perm_ctx* ctx, int n, const int* rptrs, const int* cols,
                                       int64_t trial0, int64_t trials, uint64_t seed, double* trial_values,
                                       perm_estimate* out);
int perm_approx_scaling_sparse_range(perm_ctx* ctx, int n, const int* rptrs, const int* cols,
                                     int64_t trial0, int64_t trials, int scale_intervals, int scale_times,
                                     uint64_t seed, double* trial_values, perm_estimate* out);

/* ---- matrix input (host only; no device needed) ------------------------------ */
/* The reference's grid-graph input mode (util.h:403-520): the dense 0/1
 * adjacency between the two colour classes of an m x n board (order
 * m*n/2, written row-major to out with room for cap_n^2 doubles); its
 * permanent counts the board's domino tilings. */
int perm_grid_graph(int m, int n, int cap_n, double* out, int* nov_out);
/* Reads the reference text format ("n nnz type" then "i j value" lines,
 * util.h:344).  binary != 0 stores 1 for every entry (the -b flag).  `out`
 * must hold cap_n * cap_n doubles; the matrix is written row-major with
 * stride n.  type_out (>= 8 bytes) receives "int", "float" or "double". */
int perm_read_matrix(const char* path, int binary, int cap_n, double* out, int* n_out,
                     int* header_nnz, char* type_out);
/* CRS/CCS of the positive entries; mode 0 plain (util.h:523), 1 sortOrder
 * (util.h:554), 2 skipOrder (util.h:622; permutes mat in place).  Buffers:
 * ptrs n+1, index/value arrays n*n.  Returns the stored count or <0. */
int perm_compress(int mode, double* mat, int n, int* cptrs, int* rows, double* cvals, int* rptrs,
                  int* cols, double* rvals);

/* ---- measurement ------------------------------------------------------------- */
/* FP64 pipe peak of this device: independent DFMA chains, lane-operations
 * per second (DADD, DMUL and DFMA each count as one operation). */
int perm_fp64_peak(perm_ctx* ctx, double* ops_per_second, double* kernel_ms);

/* ---- reference-signature entry points ------------------------------------------
 * Same arguments as the reference's templates; grid_dim/block_dim are accepted
 * and ignored (launch shapes are chosen per device).  They run on the process
 * default context (device from $PERM_DEVICE, else 0) and return NaN on error
 * (message on stderr). */
double gpu_perman64_xshared_coalescing_mshared_int(int* mat, int nov, int grid_dim, int block_dim);
double gpu_perman64_xshared_coalescing_mshared_float(float* mat, int nov, int grid_dim, int block_dim);
double gpu_perman64_xshared_coalescing_mshared_double(double* mat, int nov, int grid_dim,
                                                      int block_dim);
/* gpu_exact_dense.cu:702: devices 0 .. gpu_num - 1 (clamped to the visible
 * devices) through perm_exact_dense_multi; grid_dim and block_dim ignored. */
double gpu_perman64_xshared_coalescing_mshared_multigpu_int(int* mat, int nov, int gpu_num, int grid_dim,
                                                            int block_dim);
double gpu_perman64_xshared_coalescing_mshared_multigpu_float(float* mat, int nov, int gpu_num, int grid_dim,
                                                              int block_dim);
double gpu_perman64_xshared_coalescing_mshared_multigpu_double(double* mat, int nov, int gpu_num, int grid_dim,
                                                               int block_dim);
double gpu_perman64_xshared_coalescing_mshared_skipper_int(int* mat, int* rptrs, int* cols, int* cptrs,
                                                           int* rows, int* cvals, int nov,
                                                           int grid_dim, int block_dim);
double gpu_perman64_xshared_coalescing_mshared_skipper_float(float* mat, int* rptrs, int* cols,
                                                             int* cptrs, int* rows, float* cvals,
                                                             int nov, int grid_dim, int block_dim);
double gpu_perman64_xshared_coalescing_mshared_skipper_double(double* mat, int* rptrs, int* cols,
                                                              int* cptrs, int* rows, double* cvals,
                                                              int nov, int grid_dim, int block_dim);
double gpu_perman64_rasmussen_int(int* mat, int nov, int number_of_times);
double gpu_perman64_rasmussen_float(float* mat, int nov, int number_of_times);
double gpu_perman64_rasmussen_double(double* mat, int nov, int number_of_times);
double gpu_perman64_approximation_int(int* mat, int nov, int number_of_times, int scale_intervals,
                                      int scale_times);
double gpu_perman64_approximation_float(float* mat, int nov, int number_of_times, int scale_intervals,
                                        int scale_times);
double gpu_perman64_approximation_double(double* mat, int nov, int number_of_times,
                                         int scale_intervals, int scale_times);
double gpu_perman64_rasmussen_sparse(int* rptrs, int* cols, int nov, int nnz, int number_of_times,
                                     int grid_graph);
double gpu_perman64_approximation_sparse(int* cptrs, int* rows, int* rptrs, int* cols, int nov,
                                         int nnz, int number_of_times, int scale_intervals,
                                         int scale_times, int grid_graph);

#ifdef __cplusplus
}
#endif
#endif /* PERMAN_B200_H */
