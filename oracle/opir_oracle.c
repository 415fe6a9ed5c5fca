/* CPU oracle for the OnionPIRv2 server hot path. TEST INFRASTRUCTURE ONLY:
 * the checker for tests/, smoke() and bench.py's cpu_baseline leg; never the
 * product. Each function names the reference file:line it restates (paths
 * relative to the reference's src/). Arithmetic is exact integer arithmetic;
 * the only floating point is the client's Gaussian sampler, restated from
 * libstdc++ 13 (normal_distribution polar method over generate_canonical) so
 * seeded clients reproduce the reference client's draws bit for bit. Build
 * with -ffp-contract=off and no FMA target (see oracle/Makefile).
 */
#include "opir_oracle.h"
#include "oracle_common.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ======================================================================
 * primes and roots (utils.cpp:126-287, pir.cpp:14-63)
 * ====================================================================== */
static int mr_witness(uint64_t n, uint64_t d, int r, uint64_t a) {
  uint64_t x = powmod(a, d, n);
  if (x == 1 || x == n - 1) return 0;
  for (int i = 0; i < r - 1; ++i) {
    x = (uint64_t)((u128)x * x % n);
    if (x == n - 1) return 0;
  }
  return 1;
}
int oracle_is_prime(uint64_t n) {
  static const uint64_t sp[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return 0;
  for (int i = 0; i < 12; ++i) { if (n == sp[i]) return 1; if (n % sp[i] == 0) return 0; }
  uint64_t d = n - 1; int r = 0;
  while ((d & 1) == 0) { d >>= 1; ++r; }
  for (int i = 0; i < 12; ++i) if (mr_witness(n, d, r, sp[i])) return 0;
  return 1;
}
/* utils.cpp:240-251: smallest prime >= 2^(bw-1)+1, odd candidates. */
uint64_t oracle_generate_prime(uint32_t bw) {
  uint64_t c = 1ULL << (bw - 1);
  do { c++; c |= 1; } while (!oracle_is_prime(c));
  return c;
}
/* utils.cpp:253-287: largest p < 2^bw, p = 1 mod 2N; repeated widths continue
 * downward. */
int oracle_ntt_primes(const uint32_t *bws, uint32_t count, uint32_t N, uint64_t *out) {
  const uint64_t step = 2ULL * N;
  uint64_t next[64]; int have[64];
  memset(have, 0, sizeof have);
  for (uint32_t i = 0; i < count; ++i) {
    uint32_t bw = bws[i];
    if (bw < 2 || bw > 63) return -1;
    uint64_t c;
    if (!have[bw]) { c = (1ULL << bw) - 1; c -= (c - 1) % step; }
    else c = next[bw];
    for (;;) { if (c < 2) return -1; if (oracle_is_prime(c)) break; c -= step; }
    out[i] = c;
    next[bw] = c >= step ? c - step : 0; have[bw] = 1;
  }
  return 0;
}
/* HEXL MinimalPrimitiveRoot(degree, q) for prime q: minimum over the odd
 * powers of any generator of the degree-th roots of unity. */
uint64_t oracle_min_primitive_root(uint64_t degree, uint64_t q) {
  uint64_t g = 0;
  for (uint64_t x = 2; x < q; ++x) {
    uint64_t c = powmod(x, (q - 1) / degree, q);
    if (powmod(c, degree / 2, q) == q - 1) { g = c; break; }
  }
  if (!g) return 0;
  barrett_t b = barrett_make(q);
  uint64_t g2 = mulmod(&b, g, g), cur = g, best = g;
  for (uint64_t i = 0; i < degree / 2; ++i) { if (cur < best) best = cur; cur = mulmod(&b, cur, g2); }
  return best;
}
/* utils.cpp:229-238 */
static uint64_t crt_combine(uint64_t w1, uint64_t q1, uint64_t w2, uint64_t q2) {
  uint64_t inv = 0;
  invmod(q1 % q2, q2, &inv);
  uint64_t diff = (w2 + q2 - (w1 % q2)) % q2;
  uint64_t k = (uint64_t)((u128)diff * inv % q2);
  return (uint64_t)((u128)q1 * k + w1);
}
/* utils.cpp:376-401 */
int oracle_calc_db_shape(uint64_t target, uint64_t l, uint32_t h, int pow2,
                         uint64_t *fst, uint64_t *dims) {
  if (target == 0 || l == 0 || h >= 64) return -1;
  const uint64_t capacity = 1ULL << h;
  const uint64_t max_dims = 1 + (capacity - 1) / l;
  for (uint64_t nd = 1; nd <= max_dims + 1; nd++) {
    uint64_t reserved = l * (nd - 1);
    if (reserved >= capacity) break;
    uint64_t slack = capacity - reserved;
    uint64_t f = slack;
    if (pow2) { f = 1; while ((f << 1) <= slack) f <<= 1; }
    if (nd - 1 < 64 && f * (1ULL << (nd - 1)) >= target) { *fst = f; *dims = nd; return 0; }
  }
  return -1;
}
/* pir.cpp:14-98,100-128 with CONFIG_N2048_K1_COMP constants. */
int oracle_params_init(uint64_t target, uint32_t h, int pow2, opir_oracle_params *p) {
  memset(p, 0, sizeof *p);
  p->N = 2048;
  if (target == 0 || h > log2u(p->N)) return -1;
  const uint32_t bits[2] = {29, 29};
  uint64_t pr[2];
  if (oracle_ntt_primes(bits, 2, p->N, pr)) return -1;
  p->q1 = pr[0]; p->q2 = pr[1]; p->q = pr[0] * pr[1];
  p->w1 = oracle_min_primitive_root(2ULL * p->N, p->q1);
  p->w2 = oracle_min_primitive_root(2ULL * p->N, p->q2);
  p->w_crt = crt_combine(p->w1, p->q1, p->w2, p->q2);
  if (!invmod(p->q1 % p->q2, p->q2, &p->q1_inv_mod_q2)) return -1;
  p->t = oracle_generate_prime(13);
  const uint32_t sbits = 22;
  if (oracle_ntt_primes(&sbits, 1, p->N, &p->small_q)) return -1;
  p->small_q_width = (uint32_t)ceil(log2((double)p->small_q));
  p->ct_mod_width = 58;
  p->l_ep = 6; p->l_key = 10; p->l_ks = 8;
  p->base_ep = (p->ct_mod_width + p->l_ep - 1) / p->l_ep;     /* pir.cpp:82 */
  p->base_key = (p->ct_mod_width + p->l_key - 1) / p->l_key;  /* pir.cpp:83 */
  p->base_ks = p->ct_mod_width / p->l_ks + 1;                 /* bv_keyswitch.cpp:73-76 */
  uint64_t fst, dims;
  if (oracle_calc_db_shape(target, p->l_ep, h, pow2, &fst, &dims)) return -1;
  p->target_num_pt = target; p->expansion_height = h; p->fst_dim_pow2 = pow2 ? 1 : 0;
  p->fst_dim_sz = fst; p->num_dims = (uint32_t)dims;
  p->other_dim_sz = (target + fst - 1) / fst;
  p->num_pt = fst * p->other_dim_sz;
  return 0;
}

/* pir.cpp:14-98 with CONFIG_N2048_K1 (database_constants.h:61-76): one real
 * NTT prime q of 60 bits (RnsMods {60}, no composite split: q1 = q2 = 0
 * marks the single-prime set below), w_crt = its minimal 2N-th root,
 * PlainMod 14, SmallQWidth 22, L_EP 5, L_KEY 8, L_KS 8; ct_mod_width 60. */
int oracle_k1p_params_init(uint64_t target, uint32_t h, int pow2, opir_oracle_params *p) {
  memset(p, 0, sizeof *p);
  p->N = 2048;
  if (target == 0 || h > log2u(p->N)) return -1;
  const uint32_t bits = 60;
  uint64_t q = 0;
  if (oracle_ntt_primes(&bits, 1, p->N, &q)) return -1;
  p->q = q;
  p->q1 = p->q2 = 0;
  p->w_crt = oracle_min_primitive_root(2ULL * p->N, q);
  p->t = oracle_generate_prime(14);
  const uint32_t sbits = 22;
  if (oracle_ntt_primes(&sbits, 1, p->N, &p->small_q)) return -1;
  p->small_q_width = (uint32_t)ceil(log2((double)p->small_q));
  p->ct_mod_width = 60;
  p->l_ep = 5; p->l_key = 8; p->l_ks = 8;
  p->base_ep = (p->ct_mod_width + p->l_ep - 1) / p->l_ep;
  p->base_key = (p->ct_mod_width + p->l_key - 1) / p->l_key;
  p->base_ks = p->ct_mod_width / p->l_ks + 1;
  uint64_t fst, dims;
  if (oracle_calc_db_shape(target, p->l_ep, h, pow2, &fst, &dims)) return -1;
  p->target_num_pt = target; p->expansion_height = h; p->fst_dim_pow2 = pow2 ? 1 : 0;
  p->fst_dim_sz = fst; p->num_dims = (uint32_t)dims;
  p->other_dim_sz = (target + fst - 1) / fst;
  p->num_pt = fst * p->other_dim_sz;
  return 0;
}

/* ======================================================================
 * negacyclic NTT (HEXL NTT semantics as restated in oracle/hexl_standin)
 * ====================================================================== */
typedef struct {
  uint32_t N; uint64_t q, root;
  uint64_t *fw, *iw; uint64_t ninv;
} ntt_tab;

#define NTT_CACHE 8
static ntt_tab g_ntt[NTT_CACHE];
static int g_ntt_n = 0;

static const ntt_tab *ntt_get(uint32_t N, uint64_t q, uint64_t root) {
  const int n = __atomic_load_n(&g_ntt_n, __ATOMIC_ACQUIRE);
  for (int i = 0; i < n; ++i)
    if (__atomic_load_n(&g_ntt[i].N, __ATOMIC_ACQUIRE) == N && g_ntt[i].q == q &&
        g_ntt[i].root == root)
      return &g_ntt[i];
  ntt_tab *t;
#pragma omp critical(opir_ntt_cache)
  {
    int found = -1;
    for (int i = 0; i < g_ntt_n; ++i)
      if (g_ntt[i].N == N && g_ntt[i].q == q && g_ntt[i].root == root) found = i;
    if (found >= 0) {
      t = &g_ntt[found];
    } else {
      int slot = g_ntt_n < NTT_CACHE ? g_ntt_n : NTT_CACHE - 1;
      t = &g_ntt[slot];
      barrett_t b = barrett_make(q);
      uint32_t lg = log2u(N);
      uint64_t rinv = 0; invmod(root % q, q, &rinv);
      uint64_t *pw = malloc(N * sizeof *pw), *ipw = malloc(N * sizeof *ipw);
      pw[0] = 1; ipw[0] = 1;
      for (uint32_t i = 1; i < N; ++i) { pw[i] = mulmod(&b, pw[i - 1], root); ipw[i] = mulmod(&b, ipw[i - 1], rinv); }
      uint64_t *fw = malloc(N * sizeof *fw), *iw = malloc(N * sizeof *iw);
      for (uint32_t k = 0; k < N; ++k) { uint64_t e = bitrev(k, lg); fw[k] = pw[e]; iw[k] = ipw[e]; }
      free(pw); free(ipw);
      uint64_t ninv = 0; invmod(N % q, q, &ninv);
      t->fw = fw; t->iw = iw; t->ninv = ninv; t->q = q; t->root = root;
      __atomic_store_n(&t->N, N, __ATOMIC_RELEASE);
      if (slot == g_ntt_n) __atomic_store_n(&g_ntt_n, g_ntt_n + 1, __ATOMIC_RELEASE);
    }
  }
  return t;
}

/* Forward: merged Cooley-Tukey, output in bit-reversed order. */
void oracle_ntt_fwd(uint64_t *a, uint32_t N, uint64_t q, uint64_t root) {
  const ntt_tab *T = ntt_get(N, q, root);
  barrett_t b = barrett_make(q);
  uint32_t t = N;
  for (uint32_t m = 1; m < N; m <<= 1) {
    t >>= 1;
    for (uint32_t i = 0; i < m; ++i) {
      uint64_t w = T->fw[m + i];
      uint64_t *x = a + 2 * i * t, *y = x + t;
      for (uint32_t j = 0; j < t; ++j) {
        uint64_t u = x[j], v = mulmod(&b, y[j], w);
        x[j] = addmod(u, v, q); y[j] = submod(u, v, q);
      }
    }
  }
}
/* Inverse: Gentleman-Sande from bit-reversed input, scaled by N^-1. */
void oracle_ntt_inv(uint64_t *a, uint32_t N, uint64_t q, uint64_t root) {
  const ntt_tab *T = ntt_get(N, q, root);
  barrett_t b = barrett_make(q);
  uint32_t t = 1;
  for (uint32_t m = N >> 1; m >= 1; m >>= 1) {
    for (uint32_t i = 0; i < m; ++i) {
      uint64_t w = T->iw[m + i];
      uint64_t *x = a + 2 * i * t, *y = x + t;
      for (uint32_t j = 0; j < t; ++j) {
        uint64_t u = x[j], v = y[j];
        x[j] = addmod(u, v, q); y[j] = mulmod(&b, submod(u, v, q), w);
      }
    }
    t <<= 1;
  }
  for (uint32_t i = 0; i < N; ++i) a[i] = mulmod(&b, a[i], T->ninv);
}

/* The logical-modulus NTT used everywhere on the server: N, q, w_crt
 * (utils.cpp:26-56 registers w_crt for the composite q). */
static void ntt_q(const opir_oracle_params *p, uint64_t *a) { oracle_ntt_fwd(a, p->N, p->q, p->w_crt); }
static void intt_q(const opir_oracle_params *p, uint64_t *a) { oracle_ntt_inv(a, p->N, p->q, p->w_crt); }
static uint64_t small_root(const opir_oracle_params *p) { return oracle_min_primitive_root(2ULL * p->N, p->small_q); }

/* utils.cpp:58-72 */
void oracle_automorphism(const uint64_t *in, uint32_t N, uint32_t k, uint64_t q, uint64_t *out) {
  const uint64_t two_n = 2ULL * N;
  for (uint64_t i = 0; i < N; ++i) {
    uint64_t dest = (i * k) % two_n;
    if (dest < N) out[dest] = in[i];
    else out[dest - N] = in[i] == 0 ? 0 : q - in[i];
  }
}
/* utils.cpp:166-186 */
void oracle_negacyclic_shift(const uint64_t *in, uint32_t N, uint64_t shift, uint64_t q, uint64_t *out) {
  if (shift == 0) { memcpy(out, in, N * sizeof *in); return; }
  uint64_t idx = shift;
  const uint64_t mask = (uint64_t)N - 1;
  for (uint32_t i = 0; i < N; ++i, ++idx) {
    uint64_t pos = idx & mask;
    if (!(idx & (uint64_t)N) || !in[i]) out[pos] = in[i];
    else out[pos] = q - in[i];
  }
}
/* utils.cpp:445-462 (C truncating division matches C++ __int128) */
uint64_t oracle_rescale(uint64_t a, uint64_t inp_mod, uint64_t out_mod) {
  const int64_t inp_i = (int64_t)inp_mod;
  const i128 out_i = (i128)out_mod;
  int64_t v = (int64_t)(a % inp_mod);
  if (v >= inp_i / 2) v -= inp_i;
  const int64_t sign = v >= 0 ? 1 : -1;
  i128 val = (i128)v * (i128)out_mod;
  i128 r = (val + (i128)(sign * (inp_i / 2))) / (i128)inp_mod;
  r = (r + (i128)((inp_mod / out_mod) * out_mod) + 2 * out_i) % out_i;
  return (uint64_t)((r + out_i) % out_i);
}
/* bv_keyswitch.cpp:20-40 */
void oracle_signed_decompose(uint64_t val, uint32_t base_log2, uint64_t q, uint64_t *out, uint32_t nd) {
  const uint64_t half_q = q >> 1;
  const int sh = 64 - (int)base_log2;
  int64_t d = val > half_q ? (int64_t)val - (int64_t)q : (int64_t)val;
  for (uint32_t i = 0; i < nd; ++i) {
    int64_t r = (int64_t)((uint64_t)d << sh) >> sh;
    d -= r;
    d >>= base_log2;
    out[i] = r >= 0 ? (uint64_t)r : (uint64_t)(r + (int64_t)q);
  }
}

uint64_t oracle_mt_test(uint64_t seed, uint64_t skip) {
  mt64 g; mt_seed(&g, seed);
  uint64_t v = 0;
  for (uint64_t i = 0; i <= skip; ++i) v = mt_next(&g);
  return v;
}

/* rlwe.cpp:196-215 (K = 1): fresh distribution per call */
static void sample_gaussian(uint64_t *out, uint32_t N, uint64_t q, double sigma, mt64 *g) {
  normal_t nd = {0.0, 0, sigma};
  for (uint32_t i = 0; i < N; ++i) {
    int64_t v = llround(normal_next(&nd, g));
    if (v >= 0) out[i] = (uint64_t)v % q;
    else { uint64_t a = (uint64_t)(-v) % q; out[i] = a == 0 ? 0 : q - a; }
  }
}
/* rlwe.cpp:177-193 (K = 1) */
static void sample_ternary(uint64_t *out, uint32_t N, uint64_t q, mt64 *g) {
  for (uint32_t i = 0; i < N; ++i) {
    int v = uniform_0_2(g);
    out[i] = v == 0 ? 0 : (v == 1 ? 1 : q - 1);
  }
}

/* ======================================================================
 * client (rlwe.cpp, bv_keyswitch.cpp, gsw.cpp, client.cpp)
 * ====================================================================== */
#define SIGMA 2.55
static const uint64_t kBvSalt = 0x5BD1E9955BD1E995ULL;
static const uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

uint64_t oracle_db_coeff(uint64_t seed, uint64_t pt, uint64_t c, uint64_t N, uint64_t t) {
  return mix64(seed + (pt * N + c + 1) * kGolden) % t;
}
void oracle_db_plaintext(uint64_t seed, uint64_t pt, const opir_oracle_params *p, uint16_t *out) {
  for (uint32_t c = 0; c < p->N; ++c) out[c] = (uint16_t)oracle_db_coeff(seed, pt, c, p->N, p->t);
}

struct oracle_client {
  opir_oracle_params p;
  uint64_t *sk;   /* NTT form mod q */
  uint64_t *bv;   /* h * l_ks * 2N */
  uint64_t *gsw;  /* 2 l_key * 2N */
  mt64 rng;
};

/* rlwe.cpp:230-276 (K = 1), coefficient-form output */
/* given_a: the uniform polynomial (c1) supplied by the caller (a seed-
 * compressed query) instead of drawn from the generator; NULL draws it. */
static void encrypt_zero_a(const opir_oracle_params *p, const uint64_t *sk, mt64 *g,
                           const uint64_t *given_a, uint64_t *ct, int64_t *e_out) {
  const uint32_t N = p->N; const uint64_t q = p->q;
  uint64_t *c0 = ct, *c1 = ct + N;
  barrett_t b = barrett_make(q);
  if (given_a) memcpy(c1, given_a, N * sizeof *c1);
  else sample_uniform(c1, N, q, g);
  uint64_t *e = malloc(N * sizeof *e), *a = malloc(N * sizeof *a);
  sample_gaussian(e, N, q, SIGMA, g);
  if (e_out)
    for (uint32_t i = 0; i < N; ++i) e_out[i] = e[i] > q / 2 ? -(int64_t)(q - e[i]) : (int64_t)e[i];
  memcpy(a, c1, N * sizeof *a);
  ntt_q(p, a);
  for (uint32_t i = 0; i < N; ++i) c0[i] = mulmod(&b, a[i], sk[i]);
  intt_q(p, c0);
  for (uint32_t i = 0; i < N; ++i) c0[i] = submod(0, addmod(c0[i], e[i], q), q);
  free(e); free(a);
}

/* bv_keyswitch.cpp:191-259 */
/* cap_a / cap_e (may be NULL): each row's uniform a (coefficient form, N)
 * and signed Gaussian e (N), in generation order. */
static void gen_bv_key(const opir_oracle_params *p, const uint64_t *sk, uint32_t galois_k,
                       mt64 *g, uint64_t *rows, uint64_t *cap_a, int64_t *cap_e) {
  const uint32_t N = p->N; const uint64_t q = p->q;
  barrett_t b = barrett_make(q);
  uint64_t *sig = malloc(N * sizeof *sig), *tmp = malloc(N * sizeof *tmp);
  uint64_t *msg = malloc(N * sizeof *msg), *e = malloc(N * sizeof *e);
  memcpy(tmp, sk, N * sizeof *tmp);
  intt_q(p, tmp);
  oracle_automorphism(tmp, N, galois_k, q, sig);
  ntt_q(p, sig);
  for (uint32_t i = 0; i < p->l_ks; ++i) {
    uint64_t Bi = 1 % q;
    for (uint32_t bb = 0; bb < i * p->base_ks; ++bb) Bi = (uint64_t)(((u128)Bi << 1) % q);
    for (uint32_t j = 0; j < N; ++j) msg[j] = mulmod(&b, sig[j], Bi);
    uint64_t *rb = rows + (size_t)i * 2 * N, *ra = rb + N;
    sample_uniform(ra, N, q, g);
    sample_gaussian(e, N, q, SIGMA, g);
    if (cap_a) memcpy(cap_a + (size_t)i * N, ra, N * sizeof *ra);
    if (cap_e)
      for (uint32_t j = 0; j < N; ++j)
        cap_e[(size_t)i * N + j] = e[j] > q / 2 ? -(int64_t)(q - e[j]) : (int64_t)e[j];
    ntt_q(p, ra);
    ntt_q(p, e);
    for (uint32_t j = 0; j < N; ++j)
      rb[j] = addmod(submod(msg[j], mulmod(&b, ra[j], sk[j]), q), e[j], q);
  }
  free(sig); free(tmp); free(msg); free(e);
}

/* utils.cpp:206-222: gadget[j] = B^(l-1-j) mod q */
static void gadget(uint32_t l, uint32_t base, uint64_t q, uint64_t *out) {
  uint64_t pw = 1;
  for (int j = (int)l - 1; j >= 0; --j) { out[j] = pw; pw = (uint64_t)(((u128)pw << base) % q); }
}

/* gsw.cpp:359-422 (K = 1) */
static void plain_to_gsw(const opir_oracle_params *p, const uint64_t *pt, const uint64_t *sk,
                         uint32_t l, uint32_t base, mt64 *g, uint64_t *out, uint64_t *cap_a,
                         int64_t *cap_e) {
  const uint32_t N = p->N; const uint64_t q = p->q;
  uint64_t gd[64];
  gadget(l, base, q, gd);
  for (uint32_t half = 0; half < 2; ++half)
    for (uint32_t r = 0; r < l; ++r) {
      uint64_t *row = out + (size_t)(half * l + r) * 2 * N;
      const size_t at = (size_t)(half * l + r) * N;
      encrypt_zero_a(p, sk, g, NULL, row, cap_e ? cap_e + at : NULL);
      if (cap_a) memcpy(cap_a + at, row + N, N * sizeof *row);
      uint64_t *tgt = row + (size_t)half * N;
      for (uint32_t c = 0; c < N; ++c) {
        uint64_t val = (uint64_t)((u128)(pt[c] % q) * gd[r] % q);
        tgt[c] = (tgt[c] + val) % q;
      }
      ntt_q(p, row);
      ntt_q(p, row + N);
    }
}

static oracle_client *client_new(const opir_oracle_params *p, uint64_t seed, uint64_t *bv_a,
                                 int64_t *bv_e, uint64_t *gsw_a, int64_t *gsw_e) {
  const uint32_t N = p->N; const uint64_t q = p->q;
  oracle_client *c = calloc(1, sizeof *c);
  c->p = *p;
  mt_seed(&c->rng, seed);
  c->sk = malloc(N * sizeof *c->sk);
  sample_ternary(c->sk, N, q, &c->rng);        /* rlwe.cpp:219-228 */
  ntt_q(p, c->sk);
  mt64 gbv; mt_seed(&gbv, seed ^ kBvSalt);
  const uint32_t h = p->expansion_height;
  c->bv = malloc((size_t)(h ? h : 1) * p->l_ks * 2 * N * sizeof *c->bv);
  for (uint32_t i = 0; i < h; ++i)              /* bv_keyswitch.cpp:270-274 */
    gen_bv_key(p, c->sk, (N >> i) + 1, &gbv, c->bv + (size_t)i * p->l_ks * 2 * N,
               bv_a ? bv_a + (size_t)i * p->l_ks * N : NULL,
               bv_e ? bv_e + (size_t)i * p->l_ks * N : NULL);
  uint64_t *skc = malloc(N * sizeof *skc);
  memcpy(skc, c->sk, N * sizeof *skc);
  intt_q(p, skc);                               /* client.cpp:25-38 */
  c->gsw = malloc((size_t)2 * p->l_key * 2 * N * sizeof *c->gsw);
  plain_to_gsw(p, skc, c->sk, p->l_key, p->base_key, &c->rng, c->gsw, gsw_a, gsw_e);
  free(skc);
  return c;
}
oracle_client *oracle_client_new(const opir_oracle_params *p, uint64_t seed) {
  return client_new(p, seed, NULL, NULL, NULL, NULL);
}
oracle_client *oracle_client_new_keygen_parts(const opir_oracle_params *p, uint64_t seed,
                                              uint64_t *bv_a, int64_t *bv_e, uint64_t *gsw_a,
                                              int64_t *gsw_e) {
  return client_new(p, seed, bv_a, bv_e, gsw_a, gsw_e);
}
void oracle_client_free(oracle_client *c) {
  if (!c) return;
  free(c->sk); free(c->bv); free(c->gsw); free(c);
}
void oracle_client_bv_keys(const oracle_client *c, uint64_t *out) {
  memcpy(out, c->bv, (size_t)c->p.expansion_height * c->p.l_ks * 2 * c->p.N * sizeof *out);
}
void oracle_client_gsw_key(const oracle_client *c, uint64_t *out) {
  memcpy(out, c->gsw, (size_t)2 * c->p.l_key * 2 * c->p.N * sizeof *out);
}

/* client.cpp:48-98 */
static uint32_t query_indices(const opir_oracle_params *p, uint64_t idx, uint64_t *out) {
  uint64_t col = idx % p->fst_dim_sz, row = idx / p->fst_dim_sz;
  uint64_t other = p->other_dim_sz, d = p->num_dims;
  uint32_t n = 0;
  out[n++] = col;
  if (d == 1) return n;
  uint64_t h = d - 1;
  uint64_t r = 2 * other - (1ULL << h), sl = other - r, perfect;
  if (row < sl) { out[n++] = 0; perfect = row; }
  else { uint64_t corr = row - sl; out[n++] = corr % 2; perfect = sl + corr / 2; }
  if (h > 1)
    for (uint64_t k = h - 2; k + 1 > 0; k--) { out[n++] = (perfect >> k) & 1ULL; if (k == 0) break; }
  return n;
}
/* client.cpp:107-225 (K = 1) */
static int client_query(oracle_client *c, uint64_t pt_idx, const uint64_t *given_a,
                        uint64_t *out, int64_t *e_out) {
  const opir_oracle_params *p = &c->p;
  if (pt_idx >= p->num_pt) return -1;
  const uint64_t q = p->q;
  uint64_t qi[70];
  uint32_t nq = query_indices(p, pt_idx, qi);
  const uint32_t h = p->expansion_height;
  const uint64_t capacity = 1ULL << h;
  uint64_t inverse = 0;
  invmod(capacity % p->t, p->t, &inverse);
  encrypt_zero_a(p, c->sk, &c->rng, given_a, out, e_out);
  uint64_t rev = bitrev(qi[0], h);
  uint64_t scaled = (uint64_t)((((u128)q * inverse) + (p->t >> 1)) / p->t) % q;
  out[rev] = (out[rev] + scaled) % q;
  if (nq > 1) {
    uint64_t inv = 0, gd[64];
    invmod(capacity, q, &inv);
    gadget(p->l_ep, p->base_ep, q, gd);
    for (uint32_t i = 1; i < nq; ++i) {
      if (qi[i] != 1) continue;
      for (uint32_t k = 0; k < p->l_ep; ++k) {
        uint64_t pos = p->fst_dim_sz + (uint64_t)(i - 1) * p->l_ep + k;
        uint64_t ridx = bitrev(pos, h);
        uint64_t coef = (uint64_t)((u128)gd[k] * inv % q);
        out[ridx] = (out[ridx] + coef) % q;
      }
    }
  }
  return 0;
}
int oracle_client_query(oracle_client *c, uint64_t pt_idx, uint64_t *out) {
  return client_query(c, pt_idx, NULL, out, NULL);
}
int oracle_client_query_with_a(oracle_client *c, uint64_t pt_idx, const uint64_t *a,
                               uint64_t *out) {
  return client_query(c, pt_idx, a, out, NULL);
}
int oracle_client_query_parts(oracle_client *c, uint64_t pt_idx, const uint64_t *a,
                              uint64_t *out, int64_t *e_out) {
  return client_query(c, pt_idx, a, out, e_out);
}
void oracle_client_secret(const oracle_client *c, int8_t *out) {
  const opir_oracle_params *p = &c->p;
  uint64_t *s = malloc(p->N * sizeof *s);
  memcpy(s, c->sk, p->N * sizeof *s);
  intt_q(p, s);
  for (uint32_t i = 0; i < p->N; ++i) out[i] = s[i] == 0 ? 0 : s[i] == 1 ? 1 : -1;
  free(s);
}
/* tree_query.cpp:142-196 (K = 1), make_tree_query: an encryption of zero
 * from the client's generator, the alpha one-hot as the BFV lift of
 * W^-1 mod t at BitRev(alpha, h_q) (add_bfv_query_constant, :70-111), and for
 * every set bit of group g (b beta bits, then r gamma bits) the L_EP data
 * gadget rows scaled by W^-1 mod q at BitRev(N0 + g L_EP + row, h_q)
 * (add_rlwe_star_constant, :113-140). */
static int client_tree_query(oracle_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                             const uint8_t *bits, uint32_t groups, const uint64_t *given_a,
                             uint64_t *out, int64_t *e_out) {
  const opir_oracle_params *p = &c->p;
  const uint64_t q = p->q, t = p->t, W = 1ULL << h_q;
  if (h_q > 11 || alpha >= N0 || N0 + (uint64_t)groups * p->l_ep > W) return -1;
  uint64_t w_inv_t = 0, w_inv_q = 0, gd[64];
  if (!invmod(W % t, t, &w_inv_t) || !invmod(W % q, q, &w_inv_q)) return -1;
  encrypt_zero_a(p, c->sk, &c->rng, given_a, out, e_out);
  const uint64_t rev = bitrev(alpha, h_q);
  const uint64_t scaled = (uint64_t)((((u128)q * w_inv_t) + (t >> 1)) / t) % q;
  out[rev] = (out[rev] + scaled) % q;
  gadget(p->l_ep, p->base_ep, q, gd);
  for (uint32_t g = 0; g < groups; ++g) {
    if (!bits[g]) continue;
    for (uint32_t row = 0; row < p->l_ep; ++row) {
      const uint64_t idx = bitrev(N0 + (uint64_t)g * p->l_ep + row, h_q);
      const uint64_t v = (uint64_t)((u128)gd[row] * w_inv_q % q);
      out[idx] = (out[idx] + v) % q;
    }
  }
  return 0;
}
int oracle_client_tree_query(oracle_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                             const uint8_t *bits, uint32_t groups, uint64_t *out) {
  return client_tree_query(c, N0, h_q, alpha, bits, groups, NULL, out, NULL);
}
int oracle_client_tree_query_parts(oracle_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                                   const uint8_t *bits, uint32_t groups, const uint64_t *a,
                                   uint64_t *out, int64_t *e_out) {
  return client_tree_query(c, N0, h_q, alpha, bits, groups, a, out, e_out);
}
/* decrypt_rns (rlwe.cpp:310-348, K = 1): phase = c0 + c1 s mod q, then the
 * centred rescale q -> t per coefficient; ct coefficient form [c0][c1]. */
void oracle_client_decrypt_q(const oracle_client *c, const uint64_t *ct, uint64_t *pt_out) {
  const opir_oracle_params *p = &c->p;
  const uint32_t N = p->N;
  const uint64_t q = p->q;
  barrett_t b = barrett_make(q);
  uint64_t *c1 = malloc(N * 8);
  memcpy(c1, ct + N, N * 8);
  ntt_q(p, c1);
  for (uint32_t i = 0; i < N; ++i) c1[i] = mulmod(&b, c1[i], c->sk[i]);
  intt_q(p, c1);
  for (uint32_t i = 0; i < N; ++i) pt_out[i] = oracle_rescale(addmod(c1[i], ct[i], q), q, p->t);
  free(c1);
}
/* The noise figure decrypt_mod_q reports (client.cpp:389-407): max over
 * the coefficients of |phase - round(sq m / t)| mod sq, centred. */
static uint64_t noise_of(uint64_t phase, uint64_t m, uint64_t sq, uint64_t t) {
  const uint64_t approx = (uint64_t)((((u128)sq * m) + (t >> 1)) / t) % sq;
  const uint64_t pos = phase >= approx ? phase - approx : sq - approx + phase;
  return pos > sq / 2 ? sq - pos : pos;
}
/* client.cpp:364-430 */
void oracle_client_decrypt_noise(const oracle_client *c, const uint64_t *resp, uint64_t *pt_out,
                                 uint64_t *max_noise) {
  const opir_oracle_params *p = &c->p;
  const uint32_t N = p->N; const uint64_t sq = p->small_q, t = p->t;
  const uint64_t root = small_root(p);
  barrett_t b = barrett_make(sq);
  uint64_t *skc = malloc(N * 8), *sks = malloc(N * 8), *c0 = malloc(N * 8), *c1 = malloc(N * 8), *ph = malloc(N * 8);
  memcpy(skc, c->sk, N * 8);
  intt_q(p, skc);
  for (uint32_t i = 0; i < N; ++i) sks[i] = skc[i] > 1 ? sq - 1 : skc[i];
  oracle_ntt_fwd(sks, N, sq, root);
  for (uint32_t i = 0; i < N; ++i) { c0[i] = resp[i] % sq; c1[i] = resp[N + i] % sq; }
  oracle_ntt_fwd(c1, N, sq, root);
  for (uint32_t i = 0; i < N; ++i) ph[i] = mulmod(&b, c1[i], sks[i]);
  oracle_ntt_inv(ph, N, sq, root);
  uint64_t worst = 0;
  for (uint32_t i = 0; i < N; ++i) {
    uint64_t v = addmod(ph[i], c0[i], sq);
    pt_out[i] = (uint64_t)((((u128)v * t) + (sq >> 1)) / sq) % t;
    const uint64_t nz = noise_of(v, pt_out[i], sq, t);
    if (nz > worst) worst = nz;
  }
  if (max_noise) *max_noise = worst;
  free(skc); free(sks); free(c0); free(c1); free(ph);
}
void oracle_client_decrypt(const oracle_client *c, const uint64_t *resp, uint64_t *pt_out) {
  oracle_client_decrypt_noise(c, resp, pt_out, NULL);
}

/* ======================================================================
 * server
 * ====================================================================== */
struct oracle_server {
  opir_oracle_params p;
  uint32_t *db_lo, *db_hi;  /* [coeff][pt] residues mod q1 / q2 (server.h:117-118) */
  uint64_t *db64;           /* [coeff][pt] mod q, single-prime set (server.h:110-116) */
  uint64_t *bv, *gsw;
  int has_keys;
};

static int single_prime(const opir_oracle_params *p) { return p->q1 == 0; }

oracle_server *oracle_server_new(const opir_oracle_params *p) {
  oracle_server *s = calloc(1, sizeof *s);
  s->p = *p;
  size_t n = (size_t)p->num_pt * p->N;
  if (single_prime(p)) {
    s->db64 = calloc(n, sizeof *s->db64);
    if (!s->db64) { oracle_server_free(s); return NULL; }
    return s;
  }
  s->db_lo = calloc(n, sizeof *s->db_lo);
  s->db_hi = calloc(n, sizeof *s->db_hi);
  if (!s->db_lo || !s->db_hi) { oracle_server_free(s); return NULL; }
  return s;
}
void oracle_server_free(oracle_server *s) {
  if (!s) return;
  free(s->db_lo); free(s->db_hi); free(s->db64); free(s->bv); free(s->gsw); free(s);
}

/* server.cpp:80-171 (composite path) */
static int load_impl(oracle_server *s, uint64_t logical, const uint16_t *coeffs, uint64_t seed, int seeded) {
  const opir_oracle_params *p = &s->p;
  const uint32_t N = p->N;
  if (logical > p->num_pt) return -1;
  if (!seeded)
    for (size_t i = 0; i < (size_t)logical * N; ++i) if (coeffs[i] >= p->t) return -2;
  long long np = (long long)p->num_pt;
#pragma omp parallel
  {
    uint64_t *buf = malloc(N * sizeof *buf);
#pragma omp for schedule(static)
    for (long long pt = 0; pt < np; ++pt) {
      for (uint32_t c = 0; c < N; ++c) {
        if ((uint64_t)pt >= logical) buf[c] = 0;
        else if (seeded) buf[c] = oracle_db_coeff(seed, (uint64_t)pt, c, N, p->t);
        else buf[c] = coeffs[(size_t)pt * N + c];
      }
      ntt_q(p, buf);
      if (single_prime(p)) {
        for (uint32_t c = 0; c < N; ++c) s->db64[(size_t)c * p->num_pt + pt] = buf[c];
        continue;
      }
      for (uint32_t c = 0; c < N; ++c) {
        s->db_lo[(size_t)c * p->num_pt + pt] = (uint32_t)(buf[c] % p->q1);
        s->db_hi[(size_t)c * p->num_pt + pt] = (uint32_t)(buf[c] % p->q2);
      }
    }
    free(buf);
  }
  return 0;
}
int oracle_server_load_seeded(oracle_server *s, uint64_t logical, uint64_t seed) { return load_impl(s, logical, NULL, seed, 1); }
int oracle_server_load(oracle_server *s, uint64_t logical, const uint16_t *coeffs) { return load_impl(s, logical, coeffs, 0, 0); }

int oracle_server_set_keys(oracle_server *s, const uint64_t *bv, const uint64_t *gsw) {
  const opir_oracle_params *p = &s->p;
  size_t nbv = (size_t)p->expansion_height * p->l_ks * 2 * p->N;
  size_t ng = (size_t)2 * p->l_key * 2 * p->N;
  free(s->bv); free(s->gsw);
  s->bv = malloc((nbv ? nbv : 1) * 8); s->gsw = malloc(ng * 8);
  if (nbv) memcpy(s->bv, bv, nbv * 8);
  memcpy(s->gsw, gsw, ng * 8);
  s->has_keys = 1;
  return 0;
}

/* bv_keyswitch.cpp:296-367 (K = 1). key_rows: l_ks x [b | a] NTT form. */
void oracle_bv_apply_galois(const opir_oracle_params *p, uint64_t *ct, uint32_t galois_k, const uint64_t *key) {
  const uint32_t N = p->N, L = p->l_ks; const uint64_t q = p->q;
  barrett_t b = barrett_make(q);
  uint64_t *c0p = malloc(N * 8), *c1p = malloc(N * 8), *db = calloc(N, 8), *da = calloc(N, 8);
  uint64_t *dig = malloc((size_t)L * N * 8);
  oracle_automorphism(ct, N, galois_k, q, c0p);
  oracle_automorphism(ct + N, N, galois_k, q, c1p);
  uint64_t dv[64];
  for (uint32_t k = 0; k < N; ++k) {
    oracle_signed_decompose(c1p[k], p->base_ks, q, dv, L);
    for (uint32_t i = 0; i < L; ++i) dig[(size_t)i * N + k] = dv[i];
  }
  for (uint32_t i = 0; i < L; ++i) {
    uint64_t *d = dig + (size_t)i * N;
    const uint64_t *kb = key + (size_t)i * 2 * N, *ka = kb + N;
    ntt_q(p, d);
    for (uint32_t j = 0; j < N; ++j) {
      db[j] = addmod(db[j], mulmod(&b, d[j], kb[j]), q);
      da[j] = addmod(da[j], mulmod(&b, d[j], ka[j]), q);
    }
  }
  intt_q(p, db);
  intt_q(p, da);
  for (uint32_t j = 0; j < N; ++j) { ct[j] = addmod(c0p[j], db[j], q); ct[N + j] = da[j]; }
  free(c0p); free(c1p); free(db); free(da); free(dig);
}

/* server.cpp:731-816. out: u x 2N leaves, u = N0 + L_EP (d - 1). */
int oracle_server_expand(const oracle_server *s, const uint64_t *query, uint64_t *out) {
  const opir_oracle_params *p = &s->p;
  const uint32_t N = p->N; const uint64_t q = p->q;
  const uint64_t useful = p->fst_dim_sz + (uint64_t)p->l_ep * (p->num_dims - 1);
  const uint32_t h = p->expansion_height;
  const uint64_t cap = 1ULL << h;
  if (!s->has_keys && h > 0) return -1;
  const size_t ct = 2 * (size_t)N;
  uint64_t *heap = malloc(2 * cap * ct * 8);
  uint64_t *cp = malloc(ct * 8);
  memcpy(heap + 1 * ct, query, ct * 8);
  for (uint64_t i = 1; i < cap; ++i) {
    uint32_t lvl = 0; while ((2ULL << lvl) <= i) ++lvl;      /* floor(log2 i) */
    const uint64_t k = 1ULL << lvl;
    const uint64_t left_leaf = i * cap / k - cap;
    if (left_leaf >= useful) continue;
    uint64_t *ci = heap + i * ct;
    memcpy(cp, ci, ct * 8);
    const uint32_t galois_k = (uint32_t)(N / k + 1);
    oracle_bv_apply_galois(p, cp, galois_k, s->bv + (size_t)lvl * p->l_ks * 2 * N);
    uint64_t *l = heap + 2 * i * ct, *r = heap + (2 * i + 1) * ct;
    for (size_t j = 0; j < ct; ++j) { l[j] = addmod(ci[j], cp[j], q); ci[j] = submod(ci[j], cp[j], q); }
    oracle_negacyclic_shift(ci, N, (uint64_t)0 - k, q, r);
    oracle_negacyclic_shift(ci + N, N, (uint64_t)0 - k, q, r + N);
  }
  memcpy(out, heap + cap * ct, useful * ct * 8);
  free(heap); free(cp);
  return 0;
}

/* gsw.cpp:252-295 */
static void decomp_single_mod(const opir_oracle_params *p, const uint64_t *ct, uint32_t l, uint32_t base, uint64_t *rows) {
  const uint32_t N = p->N; const uint64_t q = p->q, half = q >> 1;
  const int sh = 64 - (int)base;
  for (uint32_t poly = 0; poly < 2; ++poly)
    for (uint32_t k = 0; k < N; ++k) {
      uint64_t v = ct[(size_t)poly * N + k];
      int64_t d = v > half ? (int64_t)v - (int64_t)q : (int64_t)v;
      for (uint32_t i = 0; i < l; ++i) {
        int64_t r = (int64_t)((uint64_t)d << sh) >> sh;
        d = (d - r) >> base;
        rows[(size_t)(poly * l + (l - 1 - i)) * N + k] = r >= 0 ? (uint64_t)r : (uint64_t)(r + (int64_t)q);
      }
    }
}
/* gsw.cpp:119-182: output in NTT form. */
void oracle_external_product(const opir_oracle_params *p, const uint64_t *rgsw, uint32_t l, uint32_t base,
                             const uint64_t *ct, uint64_t *out) {
  const uint32_t N = p->N; const uint64_t q = p->q;
  barrett_t b = barrett_make(q);
  uint64_t *rows = malloc((size_t)2 * l * N * 8);
  decomp_single_mod(p, ct, l, base, rows);
  for (uint32_t j = 0; j < 2 * l; ++j) ntt_q(p, rows + (size_t)j * N);
  for (uint32_t k = 0; k < 2; ++k)
    for (uint32_t c = 0; c < N; ++c) {
      uint64_t acc = 0;
      for (uint32_t j = 0; j < 2 * l; ++j)
        acc = addmod(acc, mulmod(&b, rows[(size_t)j * N + c], rgsw[(size_t)j * 2 * N + (size_t)k * N + c]), q);
      out[(size_t)k * N + c] = acc;
    }
  free(rows);
}

/* server.cpp:823-855 + gsw.cpp:317-357. out: (d-1) selectors x 2 L_EP rows x 2N. */
int oracle_server_complete_selectors(const oracle_server *s, const uint64_t *expanded, uint64_t *out) {
  const opir_oracle_params *p = &s->p;
  const uint32_t N = p->N, l = p->l_ep;
  const size_t ct = 2 * (size_t)N;
  const uint32_t nsel = p->num_dims - 1;
  if (nsel && !s->has_keys) return -1;
  for (uint32_t i = 0; i < nsel; ++i) {
    uint64_t *sel = out + (size_t)i * 2 * l * ct;
    for (uint32_t r = 0; r < l; ++r) {
      const uint64_t *row = expanded + (size_t)(p->fst_dim_sz + (uint64_t)i * l + r) * ct;
      uint64_t *top = sel + (size_t)r * ct, *bot = sel + (size_t)(l + r) * ct;
      memcpy(top, row, ct * 8);
      ntt_q(p, top);
      ntt_q(p, top + N);
      oracle_external_product(p, s->gsw, p->l_key, p->base_key, row, bot);
    }
  }
  return 0;
}

/* matrix.cpp:315-350 semantics: out[lvl][i][c] = sum_k A[lvl][i][k] B[lvl][k][c] mod q */
void oracle_level_mat_mat_32(const uint32_t *A, const uint32_t *B, uint64_t *out,
                             uint64_t m, uint64_t n, uint64_t levels, uint64_t q) {
  long long L = (long long)levels;
#pragma omp parallel for schedule(static)
  for (long long lvl = 0; lvl < L; ++lvl) {
    const uint32_t *Ap = A + (size_t)lvl * m * n, *Bp = B + (size_t)lvl * n * 2;
    uint64_t *Cp = out + (size_t)lvl * m * 2;
    for (uint64_t i = 0; i < m; ++i) {
      u128 t0 = 0, t1 = 0;
      const uint32_t *Ar = Ap + i * n;
      for (uint64_t k = 0; k < n; ++k) { t0 += (u128)((uint64_t)Ar[k] * Bp[2 * k]); t1 += (u128)((uint64_t)Ar[k] * Bp[2 * k + 1]); }
      Cp[2 * i] = (uint64_t)(t0 % q); Cp[2 * i + 1] = (uint64_t)(t1 % q);
    }
  }
}

/* matrix.cpp:36-151 (level_mat_mat, u64 x u64 -> u128 chunks): per NTT
 * level, C = A B mod q with A [m x n], B [n x 2], values < q < 2^60; at most
 * 255 products (< 2^120 each) are summed before a reduction. */
static void level_mat_mat_64(const uint64_t *A, const uint64_t *B, uint64_t *out, uint64_t m,
                             uint64_t n, uint64_t levels, uint64_t q) {
  long long L = (long long)levels;
#pragma omp parallel for schedule(static)
  for (long long lvl = 0; lvl < L; ++lvl) {
    const uint64_t *Ap = A + (size_t)lvl * m * n, *Bp = B + (size_t)lvl * n * 2;
    uint64_t *Cp = out + (size_t)lvl * m * 2;
    for (uint64_t i = 0; i < m; ++i) {
      u128 t0 = 0, t1 = 0;
      const uint64_t *Ar = Ap + i * n;
      for (uint64_t k = 0; k < n; ++k) {
        t0 += (u128)Ar[k] * Bp[2 * k];
        t1 += (u128)Ar[k] * Bp[2 * k + 1];
        if ((k & 127) == 127) { t0 %= q; t1 %= q; }
      }
      Cp[2 * i] = (uint64_t)(t0 % q); Cp[2 * i + 1] = (uint64_t)(t1 % q);
    }
  }
}

/* server.cpp:313-405 for the single-prime set: query NTT, level_mat_mat mod
 * q, inter_to_cts (server.cpp:408-527) with an INTT per candidate. */
static int first_dim_single(const oracle_server *s, const uint64_t *fst_query, uint64_t *out) {
  const opir_oracle_params *p = &s->p;
  const uint32_t N = p->N;
  const uint64_t n0 = p->fst_dim_sz, m = p->other_dim_sz;
  const size_t ct = 2 * (size_t)N;
  uint64_t *qm = malloc((size_t)N * n0 * 2 * 8), *tmp = malloc(ct * 8);
  for (uint64_t i = 0; i < n0; ++i) {
    memcpy(tmp, fst_query + i * ct, ct * 8);
    ntt_q(p, tmp); ntt_q(p, tmp + N);
    for (uint32_t lv = 0; lv < N; ++lv)
      for (uint32_t c = 0; c < 2; ++c) qm[(size_t)lv * n0 * 2 + i * 2 + c] = tmp[(size_t)c * N + lv];
  }
  uint64_t *inter = malloc((size_t)N * m * 2 * 8);
  level_mat_mat_64(s->db64, qm, inter, m, n0, N, p->q);
  for (uint64_t j = 0; j < m; ++j) {
    uint64_t *o = out + j * ct;
    for (uint32_t lv = 0; lv < N; ++lv)
      for (uint32_t c = 0; c < 2; ++c) o[(size_t)c * N + lv] = inter[(size_t)lv * m * 2 + j * 2 + c];
    intt_q(p, o); intt_q(p, o + N);
  }
  free(qm); free(tmp); free(inter);
  return 0;
}

/* server.cpp:313-361 + 264-304 + 529-597. fst_query: N0 x 2N coeff form;
 * out: other_dim x 2N coeff form. */
int oracle_server_first_dim(const oracle_server *s, const uint64_t *fst_query, uint64_t *out) {
  const opir_oracle_params *p = &s->p;
  if (single_prime(p)) return first_dim_single(s, fst_query, out);
  const uint32_t N = p->N;
  const uint64_t n0 = p->fst_dim_sz, m = p->other_dim_sz;
  const size_t ct = 2 * (size_t)N;
  uint32_t *qlo = malloc(N * n0 * 2 * 4), *qhi = malloc(N * n0 * 2 * 4);
  uint64_t *tmp = malloc(ct * 8);
  for (uint64_t i = 0; i < n0; ++i) {
    memcpy(tmp, fst_query + i * ct, ct * 8);
    ntt_q(p, tmp); ntt_q(p, tmp + N);
    for (uint32_t lv = 0; lv < N; ++lv)
      for (uint32_t c = 0; c < 2; ++c) {
        uint64_t v = tmp[(size_t)c * N + lv];
        qlo[(size_t)lv * n0 * 2 + i * 2 + c] = (uint32_t)(v % p->q1);
        qhi[(size_t)lv * n0 * 2 + i * 2 + c] = (uint32_t)(v % p->q2);
      }
  }
  uint64_t *ilo = malloc((size_t)N * m * 2 * 8), *ihi = malloc((size_t)N * m * 2 * 8);
  oracle_level_mat_mat_32(s->db_lo, qlo, ilo, m, n0, N, p->q1);
  oracle_level_mat_mat_32(s->db_hi, qhi, ihi, m, n0, N, p->q2);
  for (uint64_t j = 0; j < m; ++j) {
    uint64_t *o = out + j * ct;
    for (uint32_t lv = 0; lv < N; ++lv)
      for (uint32_t c = 0; c < 2; ++c) {
        size_t b = (size_t)lv * m * 2 + j * 2 + c;
        uint64_t lo = ilo[b], hi = ihi[b];
        uint64_t diff = (hi + p->q2 - lo % p->q2) % p->q2;
        uint64_t kk = (diff * p->q1_inv_mod_q2) % p->q2;
        o[(size_t)c * N + lv] = lo + p->q1 * kk;
      }
    intt_q(p, o); intt_q(p, o + N);
  }
  free(qlo); free(qhi); free(tmp); free(ilo); free(ihi);
  return 0;
}

/* server.cpp:652-722. x, y coeff form; y is clobbered; result may alias x. */
static void ext_prod_mux(const opir_oracle_params *p, const uint64_t *x, uint64_t *y, const uint64_t *sel, uint64_t *res) {
  const uint32_t N = p->N; const uint64_t q = p->q;
  const size_t ct = 2 * (size_t)N;
  for (size_t j = 0; j < ct; ++j) y[j] = submod(y[j], x[j], q);
  uint64_t *tmp = malloc(ct * 8);
  oracle_external_product(p, sel, p->l_ep, p->base_ep, y, tmp);
  intt_q(p, tmp); intt_q(p, tmp + N);
  for (size_t j = 0; j < ct; ++j) res[j] = addmod(x[j], tmp[j], q);
  free(tmp);
}

void oracle_ext_prod_mux(const opir_oracle_params *p, const uint64_t *x, uint64_t *y,
                         const uint64_t *sel, uint64_t *res) {
  ext_prod_mux(p, x, y, sel, res);
}

/* server.cpp:599-649. mid: other_dim x 2N (consumed). */
int oracle_server_other_dim(const oracle_server *s, uint64_t *mid, const uint64_t *selectors, uint64_t *out) {
  const opir_oracle_params *p = &s->p;
  const size_t ct = 2 * (size_t)p->N;
  const size_t sel_sz = (size_t)2 * p->l_ep * ct;
  if (p->num_dims == 1) { memcpy(out, mid, ct * 8); return 0; }
  const uint64_t h = p->num_dims - 1, other = p->other_dim_sz;
  const uint64_t perfect = 1ULL << (h - 1);
  if (other < perfect) return -1;
  const uint64_t last = 2 * other - (1ULL << h), offset = other - last;
  for (uint64_t i = 0; i < last; i += 2) {
    uint64_t ci = i + offset;
    ext_prod_mux(p, mid + ci * ct, mid + (ci + 1) * ct, selectors, mid + (i / 2 + offset) * ct);
  }
  for (uint64_t a = 1; a < h; ++a) {
    const uint64_t half = (1ULL << (h - a)) >> 1;
    for (uint64_t i = 0; i < half; ++i)
      ext_prod_mux(p, mid + i * ct, mid + (i + half) * ct, selectors + a * sel_sz, mid + i * ct);
  }
  memcpy(out, mid, ct * 8);
  return 0;
}

/* server.cpp:1025-1043 */
void oracle_mod_switch(const opir_oracle_params *p, uint64_t *ct) {
  for (uint32_t i = 0; i < 2 * p->N; ++i) ct[i] = oracle_rescale(ct[i], p->q, p->small_q);
}
/* server.cpp:950-1009 */
size_t oracle_serialize(const opir_oracle_params *p, const uint64_t *resp, uint8_t *out) {
  const uint32_t w = p->small_q_width;
  uint8_t buf = 0; uint32_t filled = 0; size_t nb = 0;
  for (uint32_t i = 0; i < 2 * p->N; ++i) {
    uint64_t c = resp[i] & ((1ULL << w) - 1);
    uint32_t written = 0;
    while (written < w) {
      uint32_t room = 8 - filled, take = w - written < room ? w - written : room;
      uint8_t chunk = (uint8_t)((c >> written) & ((1ULL << take) - 1));
      buf |= (uint8_t)(chunk << filled);
      filled += take; written += take;
      if (filled == 8) { out[nb++] = buf; buf = 0; filled = 0; }
    }
  }
  if (filled) out[nb++] = buf;
  return nb;
}

/* server.cpp:895-947 */
int oracle_server_make_query(const oracle_server *s, const uint64_t *query, uint64_t *resp) {
  const opir_oracle_params *p = &s->p;
  const size_t ct = 2 * (size_t)p->N;
  const uint64_t useful = p->fst_dim_sz + (uint64_t)p->l_ep * (p->num_dims - 1);
  const uint32_t nsel = p->num_dims - 1;
  uint64_t *exp = malloc(useful * ct * 8);
  uint64_t *sel = malloc((nsel ? nsel : 1) * (size_t)2 * p->l_ep * ct * 8);
  uint64_t *mid = malloc(p->other_dim_sz * ct * 8);
  int rc = oracle_server_expand(s, query, exp);
  if (!rc) rc = oracle_server_complete_selectors(s, exp, sel);
  if (!rc) rc = oracle_server_first_dim(s, exp, mid);
  if (!rc) rc = oracle_server_other_dim(s, mid, sel, resp);
  if (!rc) oracle_mod_switch(p, resp);
  free(exp); free(sel); free(mid);
  return rc;
}
