/* Helpers shared by the oracle's restatements (opir_oracle.c for
 * CONFIG_N2048_K1_COMP, opir_oracle_c4.c for CONFIG_N4096_K2_MP). TEST
 * INFRASTRUCTURE ONLY, like the rest of oracle/. Exact modular arithmetic on
 * u64/u128, and libstdc++ 13's mt19937_64, uniform_int_distribution<int> and
 * normal_distribution<double> restated so seeded clients reproduce the
 * reference client's draws bit for bit.
 */
#ifndef OPIR_ORACLE_COMMON_H
#define OPIR_ORACLE_COMMON_H

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ======================================================================
 * modular helpers
 * ====================================================================== */
typedef unsigned __int128 u128;
typedef __int128 i128;

/* ======================================================================
 * modular helpers
 * ====================================================================== */
typedef struct { uint64_t q, mu_lo, mu_hi; } barrett_t;

static inline barrett_t barrett_make(uint64_t q) {
  barrett_t b;
  u128 mu = (~(u128)0) / q;
  b.q = q; b.mu_lo = (uint64_t)mu; b.mu_hi = (uint64_t)(mu >> 64);
  return b;
}
static inline uint64_t barrett_reduce(const barrett_t *b, u128 x) {
  uint64_t x_lo = (uint64_t)x, x_hi = (uint64_t)(x >> 64);
  u128 t = (u128)x_lo * b->mu_lo;
  u128 m1 = (u128)x_lo * b->mu_hi + (t >> 64);
  u128 m2 = (u128)x_hi * b->mu_lo + (uint64_t)m1;
  uint64_t qhat = (uint64_t)((u128)x_hi * b->mu_hi + (m1 >> 64) + (m2 >> 64));
  uint64_t r = x_lo - qhat * b->q;
  while (r >= b->q) r -= b->q;
  return r;
}
static inline uint64_t mulmod(const barrett_t *b, uint64_t x, uint64_t y) {
  return barrett_reduce(b, (u128)x * y);
}
static inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) {
  uint64_t s = a + b; return s >= q ? s - q : s;
}
static inline uint64_t submod(uint64_t a, uint64_t b, uint64_t q) {
  return a >= b ? a - b : a + q - b;
}
static inline uint64_t powmod(uint64_t b, uint64_t e, uint64_t q) {
  u128 r = 1 % q, x = b % q;
  while (e) { if (e & 1) r = r * x % q; x = x * x % q; e >>= 1; }
  return (uint64_t)r;
}
/* utils.cpp:155-163: extended Euclid; returns 0 if not invertible. */
static inline int invmod(uint64_t v, uint64_t m, uint64_t *res) {
  if (v == 0) return 0;
  int64_t s0 = 1, s1 = 0, r0 = (int64_t)v, r1 = (int64_t)m;
  while (r1 != 0) {
    int64_t qq = r0 / r1, tmp;
    tmp = r1; r1 = r0 - qq * r1; r0 = tmp;
    tmp = s1; s1 = s0 - qq * s1; s0 = tmp;
  }
  if (r0 != 1) return 0;
  *res = s0 < 0 ? (uint64_t)(s0 + (int64_t)m) : (uint64_t)s0;
  return 1;
}
static inline uint64_t bitrev(uint64_t x, uint32_t bits) {
  uint64_t y = 0;
  for (uint32_t i = 0; i < bits; ++i) { y = (y << 1) | (x & 1); x >>= 1; }
  return y;
}
static inline uint32_t log2u(uint64_t n) { uint32_t l = 0; while ((1ULL << l) < n) ++l; return l; }

/* ======================================================================
 * libstdc++ 13 random engines/distributions (restated)
 * ====================================================================== */
typedef struct { uint64_t mt[312]; int idx; } mt64;

static inline void mt_seed(mt64 *g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i)
    g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->idx = 312;
}
static inline uint64_t mt_next(mt64 *g) {
  if (g->idx >= 312) {
    const uint64_t UP = 0xFFFFFFFF80000000ULL, LO = 0x7FFFFFFFULL, A = 0xB5026F5AA96619E9ULL;
    for (int i = 0; i < 312; ++i) {
      uint64_t x = (g->mt[i] & UP) | (g->mt[(i + 1) % 312] & LO);
      uint64_t xa = x >> 1;
      if (x & 1) xa ^= A;
      g->mt[i] = g->mt[(i + 156) % 312] ^ xa;
    }
    g->idx = 0;
  }
  uint64_t y = g->mt[g->idx++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= y >> 43;
  return y;
}
/* uniform_int_distribution<int>(0, 2) with a 64-bit engine: Lemire's
 * nearly-divisionless method on u128 (uniform_int_dist.h _S_nd). */
static inline int uniform_0_2(mt64 *g) {
  const uint64_t range = 3;
  u128 prod = (u128)mt_next(g) * range;
  uint64_t low = (uint64_t)prod;
  if (low < range) {
    uint64_t threshold = (0 - range) % range;
    while (low < threshold) { prod = (u128)mt_next(g) * range; low = (uint64_t)prod; }
  }
  return (int)(prod >> 64);
}
/* generate_canonical<double, 53>(mt19937_64) */
static inline double canonical(mt64 *g) {
  double sum = (double)mt_next(g);
  double ret = sum / 18446744073709551616.0;
  if (ret >= 1.0) ret = nextafter(1.0, 0.0);
  return ret;
}
typedef struct { double saved; int have; double sigma; } normal_t;
/* normal_distribution<double>::operator() (random.tcc, polar method) */
static inline double normal_next(normal_t *n, mt64 *g) {
  double ret;
  if (n->have) { n->have = 0; ret = n->saved; }
  else {
    double x, y, r2;
    do {
      x = 2.0 * canonical(g) - 1.0;
      y = 2.0 * canonical(g) - 1.0;
      r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0.0);
    double mult = sqrt(-2 * log(r2) / r2);
    n->saved = x * mult; n->have = 1;
    ret = y * mult;
  }
  return ret * n->sigma + 0.0;
}
/* utils.cpp:421-430 */
static inline void sample_uniform(uint64_t *out, uint32_t N, uint64_t q, mt64 *g) {
  const uint64_t limit = (~0ULL) - ((~0ULL) % q);
  for (uint32_t i = 0; i < N; ++i) { uint64_t r; do { r = mt_next(g); } while (r >= limit); out[i] = r % q; }
}

static inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

#endif
