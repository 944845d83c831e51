/* oracle.c -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * CPU restatement of the reference's permanent algorithms, written to be
 * slow and obviously right.  Compiled with -ffp-contract=off so that the
 * FP64 operation sequence of the Monte-Carlo restatements is exactly the one
 * the device kernels perform (they use explicitly rounded intrinsics).
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <omp.h>
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* double-double arithmetic (Dekker / Knuth error-free transformations)      */
/* ------------------------------------------------------------------------ */
typedef struct {
  double hi, lo;
} dd;

static inline dd two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  dd r = {s, e};
  return r;
}
static inline dd fast_two_sum(double a, double b) {
  double s = a + b;
  double e = b - (s - a);
  dd r = {s, e};
  return r;
}
static inline dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
static inline dd dd_add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  s.lo += a.lo;
  return fast_two_sum(s.hi, s.lo);
}
static inline dd dd_mul(dd a, dd b) {
  double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return fast_two_sum(p, e);
}
static inline dd dd_neg(dd a) {
  dd r = {-a.hi, -a.lo};
  return r;
}

static inline int ctz64(uint64_t v) { return __builtin_ctzll(v); }

/* ------------------------------------------------------------------------ */
/* Ryser / Nijenhuis-Wilf in double-double                                   */
/* x_j = a[j][n-1] - rowsum_j / 2 (algo.h:1048-1053); Gray index i runs over */
/* [0, 2^(n-1)); term i = (-1)^i prod_j x_j(i), x(i) = x0 + sum of columns k */
/* whose bit is set in gray(i) = i ^ (i >> 1) (gpu_exact_dense.cu:363-371);  */
/* result = (4(n&1)-2) * sum (algo.h:1087).                                  */
/* ------------------------------------------------------------------------ */
static void x0_dd(const double* a, int n, dd* x) {
  for (int j = 0; j < n; j++) {
    dd rs = {0.0, 0.0};
    for (int k = 0; k < n; k++) rs = dd_add_d(rs, a[j * n + k]);
    dd half = {rs.hi * 0.5, rs.lo * 0.5};
    x[j] = dd_add_d(dd_neg(half), a[j * n + (n - 1)]);
  }
}

void orc_ryser_dd_range(const double* a, int n, int64_t i0, int64_t i1, int threads, double out[2]) {
  dd x0[64];
  x0_dd(a, n, x0);
  int64_t total = i1 - i0;
  if (threads < 1) threads = 1;
  if (total < threads) threads = 1;
  dd* part = (dd*)calloc((size_t)threads, sizeof(dd));
#pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    int64_t s = i0 + total * t / threads;
    int64_t e = i0 + total * (t + 1) / threads;
    dd x[64];
    memcpy(x, x0, sizeof(dd) * n);
    uint64_t gray = (uint64_t)s ^ ((uint64_t)s >> 1);
    for (int k = 0; k < n - 1; k++)
      if ((gray >> k) & 1)
        for (int j = 0; j < n; j++) x[j] = dd_add_d(x[j], a[j * n + k]);
    dd acc = {0.0, 0.0};
    for (int64_t i = s; i < e; i++) {
      if (i != s) {
        int k = ctz64((uint64_t)i);
        gray ^= 1ULL << k;
        int plus = (gray >> k) & 1;
        for (int j = 0; j < n; j++) x[j] = dd_add_d(x[j], plus ? a[j * n + k] : -a[j * n + k]);
      }
      dd prod = x[0];
      for (int j = 1; j < n; j++) prod = dd_mul(prod, x[j]);
      acc = dd_add(acc, (i & 1) ? dd_neg(prod) : prod);
    }
    part[t] = acc;
  }
  dd sum = {0.0, 0.0};
  for (int t = 0; t < threads; t++) sum = dd_add(sum, part[t]);
  free(part);
  out[0] = sum.hi;
  out[1] = sum.lo;
}

void orc_perm_dd(const double* a, int n, int threads, double out[2]) {
  if (n <= 0) {
    out[0] = 1.0;
    out[1] = 0.0;
    return;
  }
  if (n == 1) {
    out[0] = a[0];
    out[1] = 0.0;
    return;
  }
  double s[2];
  orc_ryser_dd_range(a, n, 0, (int64_t)1 << (n - 1), threads, s);
  double f = (n & 1) ? 2.0 : -2.0;
  out[0] = s[0] * f;
  out[1] = s[1] * f;
}

/* ------------------------------------------------------------------------ */
/* The same walk in __float128                                                */
/* ------------------------------------------------------------------------ */
static void q_to_dd(__float128 q, double out[2]) {
  double hi = (double)q;
  double lo = (double)(q - (__float128)hi);
  out[0] = hi;
  out[1] = lo;
}

void orc_perm_q(const double* a, int n, int threads, double out[2]) {
  if (n <= 0) {
    out[0] = 1.0;
    out[1] = 0.0;
    return;
  }
  if (n == 1) {
    out[0] = a[0];
    out[1] = 0.0;
    return;
  }
  __float128 x0[64];
  for (int j = 0; j < n; j++) {
    __float128 rs = 0;
    for (int k = 0; k < n; k++) rs += (__float128)a[j * n + k];
    x0[j] = (__float128)a[j * n + n - 1] - rs / 2;
  }
  int64_t total = (int64_t)1 << (n - 1);
  if (threads < 1) threads = 1;
  if (total < threads) threads = 1;
  __float128* part = (__float128*)calloc((size_t)threads, sizeof(__float128));
#pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    int64_t s = total * t / threads;
    int64_t e = total * (t + 1) / threads;
    __float128 x[64];
    memcpy(x, x0, sizeof(__float128) * n);
    uint64_t gray = (uint64_t)s ^ ((uint64_t)s >> 1);
    for (int k = 0; k < n - 1; k++)
      if ((gray >> k) & 1)
        for (int j = 0; j < n; j++) x[j] += a[j * n + k];
    __float128 acc = 0;
    for (int64_t i = s; i < e; i++) {
      if (i != s) {
        int k = ctz64((uint64_t)i);
        gray ^= 1ULL << k;
        int plus = (gray >> k) & 1;
        for (int j = 0; j < n; j++) x[j] += plus ? (__float128)a[j * n + k] : -(__float128)a[j * n + k];
      }
      __float128 prod = x[0];
      for (int j = 1; j < n; j++) prod *= x[j];
      acc += (i & 1) ? -prod : prod;
    }
    part[t] = acc;
  }
  __float128 sum = 0;
  for (int t = 0; t < threads; t++) sum += part[t];
  free(part);
  sum *= (n & 1) ? 2 : -2;
  q_to_dd(sum, out);
}

/* ------------------------------------------------------------------------ */
/* Subset dynamic programme: P[S] = sum_{j in S} a[|S|-1][j] P[S \ {j}],     */
/* perm = P[all].  Independent of Ryser; no cancellation for a >= 0.         */
/* ------------------------------------------------------------------------ */
void orc_perm_dp(const double* a, int n, double out[2]) {
  if (n <= 0) {
    out[0] = 1.0;
    out[1] = 0.0;
    return;
  }
  size_t full = (size_t)1 << n;
  __float128* P = (__float128*)malloc(full * sizeof(__float128));
  P[0] = 1;
  for (size_t S = 1; S < full; S++) {
    int r = __builtin_popcountll(S) - 1;
    __float128 acc = 0;
    for (size_t rest = S; rest; rest &= rest - 1) {
      int j = ctz64(rest);
      double v = a[r * n + j];
      if (v != 0.0) acc += (__float128)v * P[S & ~((size_t)1 << j)];
    }
    P[S] = acc;
  }
  q_to_dd(P[full - 1], out);
  free(P);
}

/* ------------------------------------------------------------------------ */
/* Exact integer permanent: Gray-code Ryser modulo 31-bit primes + CRT       */
/* With y_j = 2 x_j (integers), sum_i (-1)^i prod_j y_j(i) = 2^n * S where   */
/* perm = (4(n&1)-2) * S, i.e. perm = (n odd ? +1 : -1) * T / 2^(n-1).       */
/* ------------------------------------------------------------------------ */
static int is_prime_u32(uint32_t p) {
  if (p < 2) return 0;
  for (uint32_t d = 2; (uint64_t)d * d <= p; d++)
    if (p % d == 0) return 0;
  return 1;
}

typedef struct {
  uint32_t p, pinv_neg, r2; /* r2 = 2^64 mod p */
} mont_t;

static mont_t mont_make(uint32_t p) {
  mont_t m;
  m.p = p;
  uint32_t inv = 1; /* inverse of p mod 2^32 by Newton */
  for (int i = 0; i < 5; i++) inv *= 2 - p * inv;
  m.pinv_neg = (uint32_t)(0u - inv);
  uint64_t r = ((uint64_t)1 << 32) % p;
  m.r2 = (uint32_t)((r * r) % p);
  return m;
}
static inline uint32_t mont_mul(const mont_t* m, uint32_t a, uint32_t b) {
  uint64_t t = (uint64_t)a * b;
  uint32_t q = (uint32_t)t * m->pinv_neg;
  uint64_t u = (t + (uint64_t)q * m->p) >> 32;
  return (uint32_t)(u >= m->p ? u - m->p : u);
}
static inline uint32_t mod_from_i64(int64_t v, uint32_t p) {
  int64_t r = v % (int64_t)p;
  if (r < 0) r += p;
  return (uint32_t)r;
}
static inline uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
  uint32_t s = a + b;
  return s >= p ? s - p : s;
}
static inline uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) { return a >= b ? a - b : a + p - b; }

/* signed residue walk; returns T mod p */
static uint32_t ryser_mod_p(const int64_t* a, int n, uint32_t p, int threads) {
  mont_t m = mont_make(p);
  /* Montgomery images of y0 and of the 2*a columns */
  uint32_t y0[64], col[64][64];
  for (int j = 0; j < n; j++) {
    int64_t rs = 0;
    for (int k = 0; k < n; k++) rs += a[j * n + k];
    y0[j] = mont_mul(&m, mod_from_i64(2 * a[j * n + n - 1] - rs, p), m.r2);
    for (int k = 0; k < n; k++) col[k][j] = mont_mul(&m, mod_from_i64(2 * a[j * n + k], p), m.r2);
  }
  int64_t total = (int64_t)1 << (n - 1);
  if (threads < 1) threads = 1;
  if (total < threads) threads = 1;
  uint64_t* part = (uint64_t*)calloc((size_t)threads, sizeof(uint64_t));
#pragma omp parallel num_threads(threads)
  {
    int t = omp_get_thread_num();
    int64_t s = total * t / threads;
    int64_t e = total * (t + 1) / threads;
    uint32_t y[64];
    memcpy(y, y0, sizeof(uint32_t) * n);
    uint64_t gray = (uint64_t)s ^ ((uint64_t)s >> 1);
    for (int k = 0; k < n - 1; k++)
      if ((gray >> k) & 1)
        for (int j = 0; j < n; j++) y[j] = add_mod(y[j], col[k][j], p);
    uint32_t acc = 0;
    for (int64_t i = s; i < e; i++) {
      if (i != s) {
        int k = ctz64((uint64_t)i);
        gray ^= 1ULL << k;
        if ((gray >> k) & 1)
          for (int j = 0; j < n; j++) y[j] = add_mod(y[j], col[k][j], p);
        else
          for (int j = 0; j < n; j++) y[j] = sub_mod(y[j], col[k][j], p);
      }
      uint32_t prod = y[0];
      for (int j = 1; j < n; j++) prod = mont_mul(&m, prod, y[j]);
      acc = (i & 1) ? sub_mod(acc, prod, p) : add_mod(acc, prod, p);
    }
    part[t] = acc;
  }
  uint32_t acc = 0;
  for (int t = 0; t < threads; t++) acc = add_mod(acc, (uint32_t)part[t], p);
  free(part);
  /* acc is the Montgomery image T*2^32; leave the domain: multiply by 1 */
  return mont_mul(&m, acc, 1);
}

/* little-endian base-2^32 unsigned big integers */
#define BIG_LIMBS 80
typedef struct {
  uint32_t d[BIG_LIMBS];
} big_t;

static void big_mul_small(big_t* a, uint32_t m) {
  uint64_t carry = 0;
  for (int i = 0; i < BIG_LIMBS; i++) {
    uint64_t v = (uint64_t)a->d[i] * m + carry;
    a->d[i] = (uint32_t)v;
    carry = v >> 32;
  }
}
static void big_add_small(big_t* a, uint32_t v) {
  uint64_t carry = v;
  for (int i = 0; i < BIG_LIMBS && carry; i++) {
    uint64_t s = (uint64_t)a->d[i] + carry;
    a->d[i] = (uint32_t)s;
    carry = s >> 32;
  }
}
static int big_cmp(const big_t* a, const big_t* b) {
  for (int i = BIG_LIMBS - 1; i >= 0; i--) {
    if (a->d[i] != b->d[i]) return a->d[i] < b->d[i] ? -1 : 1;
  }
  return 0;
}
static void big_sub(big_t* a, const big_t* b) { /* a -= b, a >= b */
  int64_t borrow = 0;
  for (int i = 0; i < BIG_LIMBS; i++) {
    int64_t v = (int64_t)a->d[i] - b->d[i] - borrow;
    borrow = v < 0;
    a->d[i] = (uint32_t)(v + (borrow ? ((int64_t)1 << 32) : 0));
  }
}
static uint32_t big_div_small(big_t* a, uint32_t m) { /* returns remainder */
  uint64_t rem = 0;
  for (int i = BIG_LIMBS - 1; i >= 0; i--) {
    uint64_t cur = (rem << 32) | a->d[i];
    a->d[i] = (uint32_t)(cur / m);
    rem = cur % m;
  }
  return (uint32_t)rem;
}
static int big_is_zero(const big_t* a) {
  for (int i = 0; i < BIG_LIMBS; i++)
    if (a->d[i]) return 0;
  return 1;
}
static double big_to_double(const big_t* a) {
  double r = 0;
  for (int i = BIG_LIMBS - 1; i >= 0; i--) r = r * 4294967296.0 + a->d[i];
  return r;
}

static uint32_t pow_mod(uint64_t b, uint64_t e, uint32_t p) {
  uint64_t r = 1;
  b %= p;
  while (e) {
    if (e & 1) r = r * b % p;
    b = b * b % p;
    e >>= 1;
  }
  return (uint32_t)r;
}

int orc_perm_exact_int(const int64_t* a, int n, int threads, char* dec, int cap, double* approx) {
  if (n == 1) {
    snprintf(dec, cap, "%lld", (long long)a[0]);
    *approx = (double)a[0];
    return 0;
  }
  if (n < 2 || n > 63) return -1;
  /* |T| <= 2^(n-1) * prod_j sum_k |2 a_jk| ; log2 bound */
  double bits = (double)(n - 1);
  for (int j = 0; j < n; j++) {
    double rs = 0;
    for (int k = 0; k < n; k++) rs += fabs(2.0 * (double)a[j * n + k]);
    if (rs == 0) {
      snprintf(dec, cap, "0");
      *approx = 0.0;
      return 0;
    }
    bits += log2(rs);
  }
  bits += 2; /* sign and slack */
  int np = (int)ceil(bits / 30.0) + 1;
  if (np > 64 || (np + 2) * 32 > BIG_LIMBS * 32) return -2;
  uint32_t primes[64], res[64];
  uint32_t cand = 2147483647u;
  for (int i = 0; i < np; i++) {
    while (!is_prime_u32(cand)) cand -= 2;
    primes[i] = cand;
    cand -= 2;
  }
  for (int i = 0; i < np; i++) res[i] = ryser_mod_p(a, n, primes[i], threads);
  /* Garner mixed-radix digits */
  uint32_t v[64];
  for (int i = 0; i < np; i++) {
    uint64_t t = res[i];
    for (int j = 0; j < i; j++) {
      uint64_t inv = pow_mod(primes[j], primes[i] - 2, primes[i]);
      t = (t + primes[i] - v[j] % primes[i]) % primes[i];
      t = t * inv % primes[i];
    }
    v[i] = (uint32_t)t;
  }
  big_t X, M;
  memset(&X, 0, sizeof X);
  memset(&M, 0, sizeof M);
  M.d[0] = 1;
  for (int i = np - 1; i >= 0; i--) {
    big_mul_small(&X, primes[i]);
    big_add_small(&X, v[i]);
  }
  for (int i = 0; i < np; i++) big_mul_small(&M, primes[i]);
  /* signed: X > M/2 -> negative */
  big_t half = M;
  big_div_small(&half, 2);
  int neg = 0;
  if (big_cmp(&X, &half) > 0) {
    big_t t = M;
    big_sub(&t, &X);
    X = t;
    neg = 1;
  }
  /* divide by 2^(n-1) exactly */
  for (int i = 0; i < n - 1; i++) {
    if (X.d[0] & 1) return -3; /* not divisible: bound or arithmetic error */
    big_div_small(&X, 2);
  }
  if (!(n & 1)) neg = !neg;
  if (big_is_zero(&X)) neg = 0;
  *approx = (neg ? -1.0 : 1.0) * big_to_double(&X);
  char buf[1024];
  int len = 0;
  big_t t = X;
  if (big_is_zero(&t)) buf[len++] = '0';
  while (!big_is_zero(&t) && len < 1000) buf[len++] = (char)('0' + big_div_small(&t, 10));
  if (neg) buf[len++] = '-';
  if (len + 1 > cap) return -4;
  for (int i = 0; i < len; i++) dec[i] = buf[len - 1 - i];
  dec[len] = 0;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* SkipPer in double (algo.h:886-1023)                                       */
/* ------------------------------------------------------------------------ */
double orc_skipper(const int* rptrs, const int* cols, const double* rvals, const int* cptrs,
                   const int* rows, const double* cvals, int n, int chunks, int threads,
                   double* visited_out) {
  double x[64];
  for (int j = 0; j < n; j++) {
    double rs = 0;
    for (int p = rptrs[j]; p < rptrs[j + 1]; p++) rs += rvals[p];
    x[j] = -rs / 2.0;
  }
  for (int p = cptrs[n - 1]; p < cptrs[n]; p++) x[rows[p]] += cvals[p];
  double prod = 1;
  for (int j = 0; j < n; j++) prod *= x[j];
  double total = prod;
  uint64_t start = 1;
  for (int j = 0; j < n; j++) {
    if (x[j] == 0) {
      uint64_t change = ~0ULL;
      for (int p = rptrs[j]; p < rptrs[j + 1]; p++) {
        uint64_t ci = 1ULL << cols[p];
        if (ci < change) change = ci;
      }
      if (change > start) start = change;
    }
  }
  uint64_t end = 1ULL << (n - 1);
  uint64_t chunk = (end - start + 1) / (uint64_t)chunks + 1;
  double vis = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(+ : total, vis)
  for (int cid = 0; cid < chunks; cid++) {
    uint64_t my_start = start + cid * chunk;
    uint64_t my_end = start + (cid + 1) * chunk;
    if (my_end > end) my_end = end;
    double my_x[64];
    memcpy(my_x, x, sizeof(double) * n);
    uint64_t prev = 0;
    double my_p = 0;
    uint64_t i = my_start;
    while (i < my_end) {
      uint64_t g = i ^ (i >> 1);
      uint64_t diff = prev ^ g;
      for (int k = 0; diff; k++) {
        uint64_t bit = 1ULL << k;
        if (diff & bit) {
          diff ^= bit;
          if (g & bit)
            for (int p = cptrs[k]; p < cptrs[k + 1]; p++) my_x[rows[p]] += cvals[p];
          else
            for (int p = cptrs[k]; p < cptrs[k + 1]; p++) my_x[rows[p]] -= cvals[p];
        }
      }
      prev = g;
      int last_zero = -1;
      double pr = 1;
      for (int j = n - 1; j >= 0; j--) {
        pr *= my_x[j];
        if (my_x[j] == 0) {
          last_zero = j;
          break;
        }
      }
      vis += 1;
      if (pr != 0) {
        my_p += ((i & 1) ? -1.0 : 1.0) * pr;
        i++;
      } else {
        uint64_t change = ~0ULL;
        for (int p = rptrs[last_zero]; p < rptrs[last_zero + 1]; p++) {
          uint64_t step_start = 1ULL << cols[p];
          uint64_t period = step_start << 1;
          uint64_t ci = step_start;
          if (i >= step_start) ci = step_start + ((i - step_start) / period + 1) * period;
          if (ci < change) change = ci;
        }
        i++;
        if (change > i) i = change;
      }
    }
    total += my_p;
  }
  if (visited_out) *visited_out = vis;
  return ((n & 1) ? 2.0 : -2.0) * total;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                             */
/* ------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Stream tags: the fourth counter word separates the estimators. */
#define TAG_RASMUSSEN 0x52415330u /* "RAS0" */
#define TAG_SCALING 0x5343414cu   /* "SCAL" */

static void philox_step(uint64_t seed, int64_t trial, int step, uint32_t tag, uint32_t out[4]) {
  uint32_t ctr[4] = {(uint32_t)trial, (uint32_t)((uint64_t)trial >> 32), (uint32_t)step, tag};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  orc_philox4x32_10(ctr, key, out);
}

/* Trial weight: FP32 significand with a separate binary exponent (the
 * integer part of log2 kept exactly), renormalised after every factor. */
typedef struct {
  float m;
  int e;
} wexp_t;
static inline void w_mul(wexp_t* w, float f) {
  float m = w->m * f;
  uint32_t b;
  memcpy(&b, &m, 4);
  int ex = (int)((b >> 23) & 0xff) - 126;
  b = (b & 0x807fffffu) | (126u << 23);
  memcpy(&m, &b, 4);
  w->m = m;
  w->e += ex;
}
static inline double w_value(wexp_t w) { return ldexp((double)w.m, w.e); }

static int nth_set_bit(uint64_t v, int idx) {
  for (int i = 0; i < idx; i++) v &= v - 1;
  return ctz64(v);
}

void orc_rasmussen_trials(const double* a, int n, uint64_t seed, int64_t t0, int64_t count,
                          double* out) {
  uint64_t rowmask[64];
  for (int r = 0; r < n; r++) {
    rowmask[r] = 0;
    for (int c = 0; c < n; c++)
      if (a[r * n + c] != 0.0) rowmask[r] |= 1ULL << c;
  }
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < count; q++) {
    int64_t t = t0 + q;
    uint64_t colext = 0, rowext = 0;
    wexp_t w = {0.5f, 1};
    double value = 0;
    int ok = 1;
    for (int step = 0; step < n; step++) {
      int best = n + 1, row = -1;
      for (int r = 0; r < n; r++) {
        if ((rowext >> r) & 1) continue;
        int c = __builtin_popcountll(rowmask[r] & ~colext);
        if (c < best) {
          best = c;
          row = r;
        }
      }
      if (best == 0) {
        ok = 0;
        break;
      }
      w_mul(&w, (float)best);
      uint32_t rnd[4];
      philox_step(seed, t, step, TAG_RASMUSSEN, rnd);
      int idx = (int)(((uint64_t)rnd[0] * (uint64_t)best) >> 32);
      int col = nth_set_bit(rowmask[row] & ~colext, idx);
      colext |= 1ULL << col;
      rowext |= 1ULL << row;
    }
    if (ok) value = w_value(w);
    out[q] = value;
  }
}

void orc_scaling_trials(const double* a, int n, int y, int z, uint64_t seed, int64_t t0,
                        int64_t count, double* out) {
  uint64_t rowmask[64];
  for (int r = 0; r < n; r++) {
    rowmask[r] = 0;
    for (int c = 0; c < n; c++)
      if (a[r * n + c] != 0.0) rowmask[r] |= 1ULL << c;
  }
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < count; q++) {
    int64_t t = t0 + q;
    uint64_t colext = 0, rowext = 0;
    double dr[64], dc[64];
    for (int i = 0; i < n; i++) dr[i] = dc[i] = 1.0;
    wexp_t w = {0.5f, 1};
    int ok = 1;
    for (int it = 0; it < n && ok; it++) {
      int best = n + 1, row = -1;
      for (int r = 0; r < n; r++) {
        if ((rowext >> r) & 1) continue;
        int c = __builtin_popcountll(rowmask[r] & ~colext);
        if (c < best) {
          best = c;
          row = r;
        }
      }
      if (it % y == 0) {
        for (int k = 0; k < z && ok; k++) {
          for (int j = 0; j < n && ok; j++) {
            if ((colext >> j) & 1) continue;
            double cs = 0;
            for (int i = 0; i < n; i++)
              if (!((rowext >> i) & 1)) cs = cs + dr[i] * a[i * n + j];
            if (cs == 0) ok = 0;
            else dc[j] = 1.0 / cs;
          }
          for (int i = 0; i < n && ok; i++) {
            if ((rowext >> i) & 1) continue;
            double rs = 0;
            for (int j = 0; j < n; j++)
              if (!((colext >> j) & 1)) rs = rs + a[i * n + j] * dc[j];
            if (rs == 0) ok = 0;
            else dr[i] = 1.0 / rs;
          }
        }
        if (!ok) break;
      }
      uint64_t avail = rowmask[row] & ~colext;
      double sum = 0;
      for (uint64_t m = avail; m; m &= m - 1) sum = sum + dr[row] * dc[ctz64(m)];
      if (sum == 0) {
        ok = 0;
        break;
      }
      uint32_t rnd[4];
      philox_step(seed, t, it, TAG_SCALING, rnd);
      double u = ((double)(rnd[0] >> 5) * 67108864.0 + (double)(rnd[1] >> 6)) * (1.0 / 9007199254740992.0);
      double target = u * sum;
      double run = 0, s = 0;
      int col = -1;
      for (uint64_t m = avail; m; m &= m - 1) {
        int j = ctz64(m);
        s = dr[row] * dc[j];
        run = run + s;
        col = j;
        if (target < run) break;
      }
      w_mul(&w, (float)(sum / s));
      colext |= 1ULL << col;
      rowext |= 1ULL << row;
    }
    out[q] = ok ? w_value(w) : 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* Sparse estimators for any order (CRS + CCS of the 0/1 pattern), restating */
/* rasmussen_sparse (algo.h:172-268) and approximation_perman64_sparse       */
/* (algo.h:366-470) / the GPU sparse kernels (gpu_approximation_sparse.cu:    */
/* 198-452) with the device kernels' streams and FP64 order.  For n <= 64    */
/* they equal orc_rasmussen_trials / orc_scaling_trials on the pattern.      */
/* ------------------------------------------------------------------------ */
static int bit_get(const uint64_t* b, int i) { return (int)((b[i >> 6] >> (i & 63)) & 1); }
static void bit_set(uint64_t* b, int i) { b[i >> 6] |= 1ULL << (i & 63); }

void orc_rasmussen_sparse_trials(const int* rptrs, const int* cols, const int* cptrs, const int* rows, int n,
                                 uint64_t seed, int64_t t0, int64_t count, double* out) {
#pragma omp parallel
  {
    int* cnt = (int*)malloc(sizeof(int) * (size_t)n);
    uint64_t* colext = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)((n + 63) / 64));
    uint64_t* rowext = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)((n + 63) / 64));
#pragma omp for schedule(static)
    for (int64_t q = 0; q < count; q++) {
      const int64_t t = t0 + q;
      memset(colext, 0, sizeof(uint64_t) * (size_t)((n + 63) / 64));
      memset(rowext, 0, sizeof(uint64_t) * (size_t)((n + 63) / 64));
      for (int r = 0; r < n; r++) cnt[r] = rptrs[r + 1] - rptrs[r];
      wexp_t w = {0.5f, 1};
      int ok = 1;
      for (int step = 0; step < n; step++) {
        int best = n + 1, row = -1;
        for (int r = 0; r < n; r++)
          if (!bit_get(rowext, r) && cnt[r] < best) {
            best = cnt[r];
            row = r;
          }
        if (best == 0) {
          ok = 0;
          break;
        }
        w_mul(&w, (float)best);
        uint32_t rnd[4];
        philox_step(seed, t, step, TAG_RASMUSSEN, rnd);
        int idx = (int)(((uint64_t)rnd[0] * (uint64_t)best) >> 32);
        int col = -1;
        for (int p = rptrs[row]; p < rptrs[row + 1]; p++) {
          int c = cols[p];
          if (bit_get(colext, c)) continue;
          if (idx == 0) {
            col = c;
            break;
          }
          idx--;
        }
        bit_set(colext, col);
        bit_set(rowext, row);
        for (int p = cptrs[col]; p < cptrs[col + 1]; p++) cnt[rows[p]]--;
      }
      out[q] = ok ? w_value(w) : 0.0;
    }
    free(cnt);
    free(colext);
    free(rowext);
  }
}

void orc_scaling_sparse_trials(const int* rptrs, const int* cols, const int* cptrs, const int* rows, int n, int y,
                               int z, uint64_t seed, int64_t t0, int64_t count, double* out) {
#pragma omp parallel
  {
    int* cnt = (int*)malloc(sizeof(int) * (size_t)n);
    double* dr = (double*)malloc(sizeof(double) * (size_t)n);
    double* dc = (double*)malloc(sizeof(double) * (size_t)n);
    const int W = (n + 63) / 64;
    uint64_t* colext = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)W);
    uint64_t* rowext = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)W);
#pragma omp for schedule(static)
    for (int64_t q = 0; q < count; q++) {
      const int64_t t = t0 + q;
      memset(colext, 0, sizeof(uint64_t) * (size_t)W);
      memset(rowext, 0, sizeof(uint64_t) * (size_t)W);
      for (int r = 0; r < n; r++) {
        cnt[r] = rptrs[r + 1] - rptrs[r];
        dr[r] = dc[r] = 1.0;
      }
      wexp_t w = {0.5f, 1};
      int ok = 1;
      for (int it = 0; it < n && ok; it++) {
        int best = n + 1, row = -1;
        for (int r = 0; r < n; r++)
          if (!bit_get(rowext, r) && cnt[r] < best) {
            best = cnt[r];
            row = r;
          }
        if (it % y == 0) {
          for (int k = 0; k < z && ok; k++) {
            for (int j = 0; j < n && ok; j++) {
              if (bit_get(colext, j)) continue;
              double cs = 0;
              for (int p = cptrs[j]; p < cptrs[j + 1]; p++)
                if (!bit_get(rowext, rows[p])) cs = cs + dr[rows[p]];
              if (cs == 0) ok = 0;
              else dc[j] = 1.0 / cs;
            }
            for (int i = 0; i < n && ok; i++) {
              if (bit_get(rowext, i)) continue;
              double rs = 0;
              for (int p = rptrs[i]; p < rptrs[i + 1]; p++)
                if (!bit_get(colext, cols[p])) rs = rs + dc[cols[p]];
              if (rs == 0) ok = 0;
              else dr[i] = 1.0 / rs;
            }
          }
          if (!ok) break;
        }
        double sum = 0;
        for (int p = rptrs[row]; p < rptrs[row + 1]; p++)
          if (!bit_get(colext, cols[p])) sum = sum + dr[row] * dc[cols[p]];
        if (sum == 0) {
          ok = 0;
          break;
        }
        uint32_t rnd[4];
        philox_step(seed, t, it, TAG_SCALING, rnd);
        double u = ((double)(rnd[0] >> 5) * 67108864.0 + (double)(rnd[1] >> 6)) * (1.0 / 9007199254740992.0);
        double target = u * sum, run = 0, sp = 0;
        int col = -1;
        for (int p = rptrs[row]; p < rptrs[row + 1]; p++) {
          int c = cols[p];
          if (bit_get(colext, c)) continue;
          sp = dr[row] * dc[c];
          run = run + sp;
          col = c;
          if (target < run) break;
        }
        w_mul(&w, (float)(sum / sp));
        bit_set(colext, col);
        bit_set(rowext, row);
        for (int p = cptrs[col]; p < cptrs[col + 1]; p++) cnt[rows[p]]--;
      }
      out[q] = ok ? w_value(w) : 0.0;
    }
    free(cnt);
    free(dr);
    free(dc);
    free(colext);
    free(rowext);
  }
}

/* Grid graph of an m x n board (util.h:403-520 restated): the bipartite
 * adjacency of its two colour classes, whose permanent counts the board's
 * domino tilings.  Writes the dense nov x nov 0/1 matrix (nov = m*n/2);
 * returns nov, or -1 when both sides are odd. */
int orc_grid_graph(int m, int n, double* mat, int cap) {
  if ((m & 1) && (n & 1)) return -1;
  int row, col;
  if (m % 2 == 0) {
    row = n;
    col = m;
  } else {
    row = m;
    col = n;
  }
  const int nov = m * n / 2;
  if (nov > cap) return -2;
  memset(mat, 0, sizeof(double) * (size_t)nov * nov);
  for (int i = 0; i < row; i++)
    for (int j = 0; j < col; j++) {
      const int x = i * (col / 2) + j / 2;
      const int black = ((i + j) & 1) == 0;
      /* neighbours of cell (i, j) in the other colour class, indexed the same way */
      int nb[4], k = 0;
      if (x - col / 2 >= 0) nb[k++] = x - col / 2;
      if (x + col / 2 < nov) nb[k++] = x + col / 2;
      if (j % 2 == 0) {
        if (j != 0) nb[k++] = x - 1;
        nb[k++] = x;
      } else {
        nb[k++] = x;
        if (j != col - 1) nb[k++] = x + 1;
      }
      for (int t = 0; t < k; t++) {
        if (black)
          mat[(size_t)x * nov + nb[t]] = 1.0;
        else
          mat[(size_t)nb[t] * nov + x] = 1.0;
      }
    }
  return nov;
}
