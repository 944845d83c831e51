/* oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's matrix-permanent algorithms
 * (berkyaglioglu/matrix-permanent-calculator), used as the checker for the
 * sm_100a kernels.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load liboracle.so; the product
 * library never links it.
 *
 * Parity pin: the reference ships no golden vectors or known-answer tests.
 * These functions are pinned against (a) closed forms (J_n -> n!, identity ->
 * 1, zero row -> 0, block-diagonal products), (b) three mutually independent
 * algorithms here (Gray-code Ryser in double-double and in __float128, the
 * subset dynamic programme, exact multi-modular integer Ryser) and (c) the
 * reference's own functions compiled from its sources into
 * oracle/_ref/libperman_ref.so (tests/test_oracle_pin.py).
 *
 * All matrices are row-major n x n doubles unless stated otherwise.
 */
#ifndef PERMAN_ORACLE_H
#define PERMAN_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Nijenhuis-Wilf Ryser in double-double over Gray indices [i0, i1) of
 * [0, 2^(n-1)); out = (hi, lo) of the raw signed sum (no final factor).
 * Follows algo.h:1032-1088 (perman64) and the start-state construction of
 * gpu_exact_dense.cu:354-371. */
void orc_ryser_dd_range(const double* a, int n, int64_t i0, int64_t i1, int threads, double out[2]);
/* Full permanent (4(n&1)-2) * sum, double-double. */
void orc_perm_dd(const double* a, int n, int threads, double out[2]);
/* Same walk in __float128 (n <= 30 practical). */
void orc_perm_q(const double* a, int n, int threads, double out[2]);
/* Subset dynamic programme perm = sum over row-expansions (independent of
 * Ryser), __float128 accumulation, n <= 24. */
void orc_perm_dp(const double* a, int n, double out[2]);
/* Exact permanent of an integer matrix by Gray-code Ryser modulo several
 * 31-bit primes and Chinese remaindering.  Writes the decimal string to dec
 * (cap bytes) and the nearest double to *approx.  Returns 0 on success. */
int orc_perm_exact_int(const int64_t* a, int n, int threads, char* dec, int cap, double* approx);

/* SkipPer in double, restating parallel_skip_perman64_w_balanced
 * (algo.h:886-1023) on CRS+CCS with `chunks` dynamic chunks.  Also reports the
 * number of Gray indices whose product was evaluated. */
double orc_skipper(const int* rptrs, const int* cols, const double* rvals, const int* cptrs,
                   const int* rows, const double* cvals, int n, int chunks, int threads,
                   double* visited);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Monte-Carlo estimators, one trial per index, with the same counter-based
 * streams as the device kernels: counter = (trial lo, trial hi, step, tag),
 * key = (seed lo, seed hi).  Values of trials [t0, t0+count) are written to
 * out; the pattern used is a[i*n+j] != 0.  n <= 64.
 *   Rasmussen: gpu_approximation_dense.cu:156-229 / algo.h:270-364.
 *   Scaling:   gpu_approximation_dense.cu:232-369 / algo.h:472-566. */
void orc_rasmussen_trials(const double* a, int n, uint64_t seed, int64_t t0, int64_t count,
                          double* out);
void orc_scaling_trials(const double* a, int n, int y, int z, uint64_t seed, int64_t t0,
                        int64_t count, double* out);

/* Sparse estimators for any order on CRS + CCS of the 0/1 pattern. */
void orc_rasmussen_sparse_trials(const int* rptrs, const int* cols, const int* cptrs, const int* rows, int n,
                                 uint64_t seed, int64_t t0, int64_t count, double* out);
void orc_scaling_sparse_trials(const int* rptrs, const int* cols, const int* cptrs, const int* rows, int n, int y,
                               int z, uint64_t seed, int64_t t0, int64_t count, double* out);
/* Dense 0/1 grid-graph matrix of an m x n board (util.h:403-520). */
int orc_grid_graph(int m, int n, double* mat, int cap);

#ifdef __cplusplus
}
#endif
#endif
