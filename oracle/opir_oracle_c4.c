/* CPU oracle for CONFIG_N4096_K2_MP (database_constants.h:111-125): N = 4096,
 * two 60-bit RNS limbs q0, q1 (logical Q = q0 q1 ~ 2^120), t =
 * generate_prime(40), small_q = 50-bit NTT prime, L_EP = 5, L_KEY = 8,
 * L_KS = 8. TEST INFRASTRUCTURE ONLY, like the rest of oracle/: the checker
 * for tests/ and bench.py's cpu_baseline leg, never the product. Each
 * function names the reference file:line it restates (paths relative to the
 * reference's src/).
 *
 * Layouts (u64, limb-major: [limb 0 (N)][limb 1 (N)]):
 *   ciphertext : [c0 (2N)][c1 (2N)]                          (rlwe.h:17-31)
 *   BV keys    : [level < h][row < L_KS][b (2N)][a (2N)], NTT form per limb
 *   RGSW       : [row < 2l][c0 (2N)][c1 (2N)], NTT form per limb (gsw.h:8-17)
 */
#include "opir_oracle.h"
#include "oracle_common.h"

#define C4_N 4096u
#define C4_K 2u
#define SIGMA_C4 2.55
static const uint64_t kBvSaltC4 = 0x5BD1E9955BD1E995ULL;

/* ---- parameters: pir.cpp:49-134 with RnsMods = {60, 60}, PlainMod 40,
 *      SmallQWidth 50; ct_mod_width = 120 (pir.cpp:188-194), data/key gadget
 *      bases ceil(120 / l), BV base 120 / L_KS + 1 (bv_keyswitch.cpp:73-76) */
int oracle_c4_params_init(uint64_t target, uint32_t h, int pow2, opir_oracle_c4_params *p) {
  memset(p, 0, sizeof *p);
  p->N = C4_N;
  p->K = C4_K;
  const uint32_t widths[2] = {60, 60};
  if (oracle_ntt_primes(widths, 2, C4_N, p->q) != 0) return -1;
  for (int k = 0; k < 2; ++k) p->w[k] = oracle_min_primitive_root(2ULL * C4_N, p->q[k]);
  if (!invmod(p->q[0] % p->q[1], p->q[1], &p->q0_inv_mod_q1)) return -1;
  for (int k = 0; k < 2; ++k) p->r64_mod_q[k] = (uint64_t)(((u128)1 << 64) % p->q[k]);
  p->t = oracle_generate_prime(40);
  const uint32_t sw = 50;
  if (oracle_ntt_primes(&sw, 1, C4_N, &p->small_q) != 0) return -1;
  p->small_q_width = 50;
  p->ct_mod_width = 120;
  p->l_ep = 5; p->l_key = 8; p->l_ks = 8;
  p->base_ep = (120 + 5 - 1) / 5;
  p->base_key = (120 + 8 - 1) / 8;
  p->base_ks = 120 / 8 + 1;
  if (target == 0 || h > 12) return -1;
  uint64_t fst = 0, nd = 0;
  if (oracle_calc_db_shape(target, p->l_ep, h, pow2, &fst, &nd) != 0) return -1;
  p->target_num_pt = target;
  p->expansion_height = h;
  p->fst_dim_pow2 = pow2 ? 1 : 0;
  p->fst_dim_sz = fst;
  p->num_dims = (uint32_t)nd;
  p->other_dim_sz = (target + fst - 1) / fst;
  p->num_pt = fst * p->other_dim_sz;
  return 0;
}

/* ---- CONFIG_N2048_K2_MP (database_constants.h:96-110): the same K = 2 MP
 *      pipeline at N = 2048 with RnsMods = {29, 29}, PlainMod 10,
 *      SmallQWidth 22; ct_mod_width = 58, data/key gadget bases ceil(58 / l)
 *      (pir.cpp:101-103), BV base 58 / L_KS + 1 (bv_keyswitch.cpp:73-76).
 *      Every routine below is written for any N and limb width below 2^62, so
 *      both two-limb sets share them. */
int oracle_k2mp_params_init(uint64_t target, uint32_t h, int pow2, opir_oracle_c4_params *p) {
  memset(p, 0, sizeof *p);
  p->N = 2048u;
  p->K = C4_K;
  const uint32_t widths[2] = {29, 29};
  if (oracle_ntt_primes(widths, 2, p->N, p->q) != 0) return -1;
  for (int k = 0; k < 2; ++k) p->w[k] = oracle_min_primitive_root(2ULL * p->N, p->q[k]);
  if (!invmod(p->q[0] % p->q[1], p->q[1], &p->q0_inv_mod_q1)) return -1;
  for (int k = 0; k < 2; ++k) p->r64_mod_q[k] = (uint64_t)(((u128)1 << 64) % p->q[k]);
  p->t = oracle_generate_prime(10);
  const uint32_t sw = 22;
  if (oracle_ntt_primes(&sw, 1, p->N, &p->small_q) != 0) return -1;
  p->small_q_width = 22;
  p->ct_mod_width = 58;
  p->l_ep = 5; p->l_key = 8; p->l_ks = 8;
  p->base_ep = (58 + 5 - 1) / 5;
  p->base_key = (58 + 8 - 1) / 8;
  p->base_ks = 58 / 8 + 1;
  if (target == 0 || h > 11) return -1;
  uint64_t fst = 0, nd = 0;
  if (oracle_calc_db_shape(target, p->l_ep, h, pow2, &fst, &nd) != 0) return -1;
  p->target_num_pt = target;
  p->expansion_height = h;
  p->fst_dim_pow2 = pow2 ? 1 : 0;
  p->fst_dim_sz = fst;
  p->num_dims = (uint32_t)nd;
  p->other_dim_sz = (target + fst - 1) / fst;
  p->num_pt = fst * p->other_dim_sz;
  return 0;
}

static void ntt_k(const opir_oracle_c4_params *p, uint32_t k, uint64_t *a) {
  oracle_ntt_fwd(a, p->N, p->q[k], p->w[k]);
}
static void intt_k(const opir_oracle_c4_params *p, uint32_t k, uint64_t *a) {
  oracle_ntt_inv(a, p->N, p->q[k], p->w[k]);
}
/* a signed value reduced into [0, q) */
static uint64_t sreduce(int64_t v, uint64_t q) {
  if (v >= 0) return (uint64_t)v % q;
  const uint64_t a = (uint64_t)(-v) % q;
  return a == 0 ? 0 : q - a;
}

/* ======================================================================
 * client
 * ====================================================================== */
struct oracle_c4_client {
  opir_oracle_c4_params p;
  uint64_t *sk;   /* 2N, NTT form per limb */
  uint64_t *bv;   /* h x L_KS x [b (2N)][a (2N)] */
  uint64_t *gsw;  /* 2 L_KEY x [c0 (2N)][c1 (2N)] */
  mt64 rng;
};

/* rlwe.cpp:230-276: per-limb uniform c1, one shared Gaussian e reduced per
 * limb (rlwe.cpp:196-215), c0_k = -(a_k s_k + e_k); coefficient form. */
/* given_a (2N, limb-major): the uniform c1 supplied by the caller instead of
 * drawn from the generator (NULL draws it); e_out receives the shared error. */
static void encrypt_zero_c4_a(const opir_oracle_c4_params *p, const uint64_t *sk, mt64 *g,
                              const uint64_t *given_a, uint64_t *ct, int64_t *e_out) {
  const uint32_t N = p->N;
  uint64_t *c0 = ct, *c1 = ct + 2 * (size_t)N;
  if (given_a) memcpy(c1, given_a, 2 * (size_t)N * sizeof *c1);
  else for (uint32_t k = 0; k < 2; ++k) sample_uniform(c1 + (size_t)k * N, N, p->q[k], g);
  int64_t *e = malloc(N * sizeof *e);
  normal_t nd = {0.0, 0, SIGMA_C4};
  for (uint32_t i = 0; i < N; ++i) e[i] = llround(normal_next(&nd, g));
  if (e_out) memcpy(e_out, e, N * sizeof *e);
  uint64_t *a = malloc(N * sizeof *a);
  for (uint32_t k = 0; k < 2; ++k) {
    const uint64_t q = p->q[k];
    barrett_t b = barrett_make(q);
    uint64_t *c0k = c0 + (size_t)k * N;
    memcpy(a, c1 + (size_t)k * N, N * sizeof *a);
    ntt_k(p, k, a);
    for (uint32_t i = 0; i < N; ++i) c0k[i] = mulmod(&b, a[i], sk[(size_t)k * N + i]);
    intt_k(p, k, c0k);
    for (uint32_t i = 0; i < N; ++i) c0k[i] = submod(0, addmod(c0k[i], sreduce(e[i], q), q), q);
  }
  free(e); free(a);
}

/* bv_keyswitch.cpp:191-259 (K = 2): sigma_k(s) per limb (utils.cpp:74-82),
 * row i encrypts sigma_k(s) 2^(i base) under both limbs with per-limb
 * uniform a and one shared Gaussian e (bv_keyswitch.cpp:166-186). */
static void gen_bv_key_c4(const opir_oracle_c4_params *p, const uint64_t *sk, uint32_t galois_k,
                          mt64 *g, uint64_t *rows, uint64_t *cap_a, int64_t *cap_e) {
  const uint32_t N = p->N;
  const size_t KN = 2 * (size_t)N;
  uint64_t *sig = malloc(KN * 8), *tmp = malloc(N * 8), *msg = malloc(KN * 8);
  int64_t *e = malloc(N * sizeof *e);
  for (uint32_t k = 0; k < 2; ++k) {
    memcpy(tmp, sk + (size_t)k * N, N * 8);
    intt_k(p, k, tmp);
    oracle_automorphism(tmp, N, galois_k, p->q[k], sig + (size_t)k * N);
    ntt_k(p, k, sig + (size_t)k * N);
  }
  for (uint32_t i = 0; i < p->l_ks; ++i) {
    for (uint32_t k = 0; k < 2; ++k) {
      const uint64_t q = p->q[k];
      barrett_t b = barrett_make(q);
      uint64_t Bi = 1 % q;
      for (uint32_t bb = 0; bb < i * p->base_ks; ++bb) Bi = (uint64_t)(((u128)Bi << 1) % q);
      for (uint32_t j = 0; j < N; ++j) msg[(size_t)k * N + j] = mulmod(&b, sig[(size_t)k * N + j], Bi);
    }
    uint64_t *rb = rows + (size_t)i * 2 * KN, *ra = rb + KN;
    for (uint32_t k = 0; k < 2; ++k) sample_uniform(ra + (size_t)k * N, N, p->q[k], g);
    normal_t nd = {0.0, 0, SIGMA_C4};
    for (uint32_t j = 0; j < N; ++j) e[j] = llround(normal_next(&nd, g));
    if (cap_a) memcpy(cap_a + (size_t)i * KN, ra, KN * sizeof *ra);
    if (cap_e) memcpy(cap_e + (size_t)i * N, e, N * sizeof *e);
    for (uint32_t k = 0; k < 2; ++k) {
      const uint64_t q = p->q[k];
      barrett_t b = barrett_make(q);
      uint64_t *ak = ra + (size_t)k * N, *bk = rb + (size_t)k * N;
      for (uint32_t j = 0; j < N; ++j) tmp[j] = sreduce(e[j], q);
      ntt_k(p, k, ak);
      ntt_k(p, k, tmp);
      for (uint32_t j = 0; j < N; ++j)
        bk[j] = addmod(submod(msg[(size_t)k * N + j], mulmod(&b, ak[j], sk[(size_t)k * N + j]), q), tmp[j], q);
    }
  }
  free(sig); free(tmp); free(msg); free(e);
}

/* utils.cpp:206-222: gadget[k][j] = B^(l-1-j) mod q_k */
static void gadget_c4(uint32_t l, uint32_t base, uint64_t q, uint64_t *out) {
  uint64_t pw = 1;
  for (int j = (int)l - 1; j >= 0; --j) { out[j] = pw; pw = (uint64_t)(((u128)pw << base) % q); }
}

/* gsw.cpp:359-422 (K = 2): the plaintext arrives mod q0 and is
 * re-canonicalised per limb (a value above q0/2 is negative). */
static void plain_to_gsw_c4(const opir_oracle_c4_params *p, const uint64_t *pt, const uint64_t *sk,
                            uint32_t l, uint32_t base, mt64 *g, uint64_t *out, uint64_t *cap_a,
                            int64_t *cap_e) {
  const uint32_t N = p->N;
  const size_t KN = 2 * (size_t)N;
  uint64_t gd[2][64];
  for (uint32_t k = 0; k < 2; ++k) gadget_c4(l, base, p->q[k], gd[k]);
  const uint64_t q0 = p->q[0], half_q0 = q0 >> 1;
  for (uint32_t half = 0; half < 2; ++half)
    for (uint32_t r = 0; r < l; ++r) {
      uint64_t *row = out + (size_t)(half * l + r) * 2 * KN;
      encrypt_zero_c4_a(p, sk, g, NULL, row, cap_e ? cap_e + (size_t)(half * l + r) * N : NULL);
      if (cap_a) memcpy(cap_a + (size_t)(half * l + r) * KN, row + KN, KN * sizeof *row);
      for (uint32_t k = 0; k < 2; ++k) {
        const uint64_t qk = p->q[k];
        uint64_t *tgt = row + (size_t)half * KN + (size_t)k * N;
        for (uint32_t c = 0; c < N; ++c) {
          uint64_t mj;
          if (pt[c] <= half_q0) mj = pt[c] % qk;
          else { const uint64_t abs_v = q0 - pt[c]; mj = abs_v >= qk ? (qk - abs_v % qk) % qk : qk - abs_v; }
          const uint64_t val = (uint64_t)((u128)mj * gd[k][r] % qk);
          tgt[c] = (uint64_t)(((u128)tgt[c] + val) % qk);
        }
      }
      for (uint32_t k = 0; k < 2; ++k) {
        ntt_k(p, k, row + (size_t)k * N);
        ntt_k(p, k, row + KN + (size_t)k * N);
      }
    }
}

/* client.cpp:20-38 with the driver's seeding: rng(seed) for s (rlwe.cpp:
 * 177-228, one ternary draw shared by both limbs), RGSW(s) and queries;
 * rng(seed ^ salt) for the BV keys. */
static oracle_c4_client *c4_client_new(const opir_oracle_c4_params *p, uint64_t seed,
                                       uint64_t *bv_a, int64_t *bv_e, uint64_t *gsw_a,
                                       int64_t *gsw_e) {
  const uint32_t N = p->N;
  oracle_c4_client *c = calloc(1, sizeof *c);
  c->p = *p;
  mt_seed(&c->rng, seed);
  c->sk = malloc(2 * (size_t)N * sizeof *c->sk);
  for (uint32_t i = 0; i < N; ++i) {
    const int v = uniform_0_2(&c->rng);
    for (uint32_t k = 0; k < 2; ++k)
      c->sk[(size_t)k * N + i] = v == 0 ? 0 : (v == 1 ? 1 : p->q[k] - 1);
  }
  for (uint32_t k = 0; k < 2; ++k) ntt_k(p, k, c->sk + (size_t)k * N);
  mt64 gbv; mt_seed(&gbv, seed ^ kBvSaltC4);
  const uint32_t h = p->expansion_height;
  const size_t key_words = (size_t)p->l_ks * 2 * 2 * N;
  c->bv = malloc((h ? h : 1) * key_words * sizeof *c->bv);
  for (uint32_t i = 0; i < h; ++i)
    gen_bv_key_c4(p, c->sk, (N >> i) + 1, &gbv, c->bv + (size_t)i * key_words,
                  bv_a ? bv_a + (size_t)i * p->l_ks * 2 * N : NULL,
                  bv_e ? bv_e + (size_t)i * p->l_ks * N : NULL);
  uint64_t *skc = malloc(N * sizeof *skc);
  memcpy(skc, c->sk, N * sizeof *skc);
  intt_k(p, 0, skc);
  c->gsw = malloc((size_t)2 * p->l_key * 2 * 2 * N * sizeof *c->gsw);
  plain_to_gsw_c4(p, skc, c->sk, p->l_key, p->base_key, &c->rng, c->gsw, gsw_a, gsw_e);
  free(skc);
  return c;
}
oracle_c4_client *oracle_c4_client_new(const opir_oracle_c4_params *p, uint64_t seed) {
  return c4_client_new(p, seed, NULL, NULL, NULL, NULL);
}
oracle_c4_client *oracle_c4_client_new_keygen_parts(const opir_oracle_c4_params *p, uint64_t seed,
                                                    uint64_t *bv_a, int64_t *bv_e,
                                                    uint64_t *gsw_a, int64_t *gsw_e) {
  return c4_client_new(p, seed, bv_a, bv_e, gsw_a, gsw_e);
}
void oracle_c4_client_free(oracle_c4_client *c) {
  if (!c) return;
  free(c->sk); free(c->bv); free(c->gsw); free(c);
}
void oracle_c4_client_bv_keys(const oracle_c4_client *c, uint64_t *out) {
  memcpy(out, c->bv, (size_t)c->p.expansion_height * c->p.l_ks * 2 * 2 * c->p.N * 8);
}
void oracle_c4_client_gsw_key(const oracle_c4_client *c, uint64_t *out) {
  memcpy(out, c->gsw, (size_t)2 * c->p.l_key * 2 * 2 * c->p.N * 8);
}

/* client.cpp:48-98 */
static uint32_t query_indices_c4(const opir_oracle_c4_params *p, uint64_t idx, uint64_t *out) {
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
/* client.cpp:107-225 (K = 2): the message Delta (2^h)^-1 lifted under Q,
 * then reduced per limb; gadget rows written under every limb. */
static int c4_client_query(oracle_c4_client *c, uint64_t pt_idx, const uint64_t *given_a,
                           uint64_t *out, int64_t *e_out) {
  const opir_oracle_c4_params *p = &c->p;
  if (pt_idx >= p->num_pt) return -1;
  const uint32_t N = p->N;
  uint64_t qi[70];
  const uint32_t nq = query_indices_c4(p, pt_idx, qi);
  const uint32_t h = p->expansion_height;
  const uint64_t capacity = 1ULL << h, t = p->t;
  uint64_t inverse = 0;
  invmod(capacity % t, t, &inverse);
  encrypt_zero_c4_a(p, c->sk, &c->rng, given_a, out, e_out);
  const uint64_t rev = bitrev(qi[0], h);
  const u128 Q = (u128)p->q[0] * p->q[1];
  const u128 Delta = Q / t;
  const uint64_t r = (uint64_t)(Q - Delta * t);
  const uint64_t r_inv_round = (uint64_t)(((u128)r * inverse + (t >> 1)) / t);
  const u128 scaled = Delta * inverse + r_inv_round;
  for (uint32_t k = 0; k < 2; ++k) {
    const uint64_t sk = (uint64_t)(scaled % p->q[k]);
    const size_t idx = (size_t)k * N + rev;
    out[idx] = (uint64_t)(((u128)out[idx] + sk) % p->q[k]);
  }
  if (nq > 1) {
    uint64_t inv[2], gd[2][64];
    for (uint32_t k = 0; k < 2; ++k) {
      invmod(capacity % p->q[k], p->q[k], &inv[k]);
      gadget_c4(p->l_ep, p->base_ep, p->q[k], gd[k]);
    }
    for (uint32_t i = 1; i < nq; ++i) {
      if (qi[i] != 1) continue;
      for (uint32_t k = 0; k < p->l_ep; ++k) {
        const uint64_t pos = p->fst_dim_sz + (uint64_t)(i - 1) * p->l_ep + k;
        const uint64_t ridx = bitrev(pos, h);
        for (uint32_t m = 0; m < 2; ++m) {
          const uint64_t coef = (uint64_t)((u128)gd[m][k] * inv[m] % p->q[m]);
          const size_t at = (size_t)m * N + ridx;
          out[at] = (uint64_t)(((u128)out[at] + coef) % p->q[m]);
        }
      }
    }
  }
  return 0;
}
int oracle_c4_client_query(oracle_c4_client *c, uint64_t pt_idx, uint64_t *out) {
  return c4_client_query(c, pt_idx, NULL, out, NULL);
}
int oracle_c4_client_query_parts(oracle_c4_client *c, uint64_t pt_idx, const uint64_t *a,
                                 uint64_t *out, int64_t *e_out) {
  return c4_client_query(c, pt_idx, a, out, e_out);
}
void oracle_c4_client_secret(const oracle_c4_client *c, int8_t *out) {
  const opir_oracle_c4_params *p = &c->p;
  uint64_t *s = malloc(p->N * sizeof *s);
  memcpy(s, c->sk, p->N * sizeof *s);
  intt_k(p, 0, s);
  for (uint32_t i = 0; i < p->N; ++i) out[i] = s[i] == 0 ? 0 : s[i] == 1 ? 1 : -1;
  free(s);
}
/* make_tree_query (tree_query.cpp:142-196) for K = 2: a fresh encryption of
 * zero from the client's generator, the alpha one-hot as the BFV lift of
 * W^-1 mod t computed under Q = q0 q1 and reduced per limb
 * (add_bfv_query_constant, :70-111), and for every set bit of group g
 * (b beta bits, then r gamma bits) the L_EP data gadget rows scaled by
 * W^-1 mod q_k, per limb, at BitRev(N0 + g L_EP + row, h_q)
 * (add_rlwe_star_constant, :113-140). */
static int c4_client_tree_query(oracle_c4_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                                const uint8_t *bits, uint32_t groups, const uint64_t *given_a,
                                uint64_t *out, int64_t *e_out) {
  const opir_oracle_c4_params *p = &c->p;
  const uint32_t N = p->N;
  const uint64_t t = p->t, W = 1ULL << h_q;
  if (h_q > 12 || alpha >= N0 || N0 + (uint64_t)groups * p->l_ep > W) return -1;
  uint64_t w_inv_t = 0;
  if (!invmod(W % t, t, &w_inv_t)) return -1;
  encrypt_zero_c4_a(p, c->sk, &c->rng, given_a, out, e_out);
  const uint64_t rev = bitrev(alpha, h_q);
  const u128 Q = (u128)p->q[0] * p->q[1];
  const u128 Delta = Q / t;
  const uint64_t r = (uint64_t)(Q - Delta * t);
  const uint64_t r_round = (uint64_t)(((u128)r * w_inv_t + (t >> 1)) / t);
  const u128 scaled = Delta * w_inv_t + r_round;
  for (uint32_t k = 0; k < 2; ++k) {
    const size_t idx = (size_t)k * N + rev;
    out[idx] = (uint64_t)(((u128)out[idx] + (uint64_t)(scaled % p->q[k])) % p->q[k]);
  }
  uint64_t inv[2], gd[2][64];
  for (uint32_t k = 0; k < 2; ++k) {
    if (!invmod(W % p->q[k], p->q[k], &inv[k])) return -1;
    gadget_c4(p->l_ep, p->base_ep, p->q[k], gd[k]);
  }
  for (uint32_t g = 0; g < groups; ++g) {
    if (!bits[g]) continue;
    for (uint32_t row = 0; row < p->l_ep; ++row) {
      const uint64_t ridx = bitrev(N0 + (uint64_t)g * p->l_ep + row, h_q);
      for (uint32_t m = 0; m < 2; ++m) {
        const uint64_t coef = (uint64_t)((u128)gd[m][row] * inv[m] % p->q[m]);
        const size_t at = (size_t)m * N + ridx;
        out[at] = (uint64_t)(((u128)out[at] + coef) % p->q[m]);
      }
    }
  }
  return 0;
}
int oracle_c4_client_tree_query(oracle_c4_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                                const uint8_t *bits, uint32_t groups, uint64_t *out) {
  return c4_client_tree_query(c, N0, h_q, alpha, bits, groups, NULL, out, NULL);
}
int oracle_c4_client_tree_query_parts(oracle_c4_client *c, uint64_t N0, uint32_t h_q,
                                      uint64_t alpha, const uint8_t *bits, uint32_t groups,
                                      const uint64_t *a, uint64_t *out, int64_t *e_out) {
  return c4_client_tree_query(c, N0, h_q, alpha, bits, groups, a, out, e_out);
}

/* client.cpp:364-430 under small_q: s from limb 0, ternary re-mapped;
 * max_noise (may be NULL) as in the reference's noise report (:389-407). */
void oracle_c4_client_decrypt_noise(const oracle_c4_client *c, const uint64_t *resp,
                                    uint64_t *pt_out, uint64_t *max_noise) {
  const opir_oracle_c4_params *p = &c->p;
  const uint32_t N = p->N;
  const uint64_t sq = p->small_q, t = p->t;
  const uint64_t root = oracle_min_primitive_root(2ULL * N, sq);
  barrett_t b = barrett_make(sq);
  uint64_t *skc = malloc(N * 8), *sks = malloc(N * 8), *c0 = malloc(N * 8), *c1 = malloc(N * 8), *ph = malloc(N * 8);
  memcpy(skc, c->sk, N * 8);
  intt_k(p, 0, skc);
  for (uint32_t i = 0; i < N; ++i) sks[i] = skc[i] > 1 ? sq - 1 : skc[i];
  oracle_ntt_fwd(sks, N, sq, root);
  for (uint32_t i = 0; i < N; ++i) { c0[i] = resp[i] % sq; c1[i] = resp[N + i] % sq; }
  oracle_ntt_fwd(c1, N, sq, root);
  for (uint32_t i = 0; i < N; ++i) ph[i] = mulmod(&b, c1[i], sks[i]);
  oracle_ntt_inv(ph, N, sq, root);
  uint64_t worst = 0;
  for (uint32_t i = 0; i < N; ++i) {
    const uint64_t v = addmod(ph[i], c0[i], sq);
    const uint64_t m = (uint64_t)((((u128)v * t) + (sq >> 1)) / sq) % t;
    pt_out[i] = m;
    const uint64_t approx = (uint64_t)((((u128)sq * m) + (t >> 1)) / t) % sq;
    const uint64_t pos = v >= approx ? v - approx : sq - approx + v;
    const uint64_t nz = pos > sq / 2 ? sq - pos : pos;
    if (nz > worst) worst = nz;
  }
  if (max_noise) *max_noise = worst;
  free(skc); free(sks); free(c0); free(c1); free(ph);
}
void oracle_c4_client_decrypt(const oracle_c4_client *c, const uint64_t *resp, uint64_t *pt_out) {
  oracle_c4_client_decrypt_noise(c, resp, pt_out, NULL);
}
void oracle_c4_db_plaintext(uint64_t seed, uint64_t pt, const opir_oracle_c4_params *p, uint64_t *out) {
  for (uint32_t c = 0; c < p->N; ++c) out[c] = oracle_db_coeff(seed, pt, c, p->N, p->t);
}

/* ======================================================================
 * server
 * ====================================================================== */
struct oracle_c4_server {
  opir_oracle_c4_params p;
  uint64_t *db;   /* [limb][coeff][pt] (server.cpp:172-194) */
  uint64_t *bv, *gsw;
  int has_keys;
};

oracle_c4_server *oracle_c4_server_new(const opir_oracle_c4_params *p) {
  oracle_c4_server *s = calloc(1, sizeof *s);
  s->p = *p;
  s->db = calloc((size_t)p->num_pt * 2 * p->N, 8);
  if (!s->db) { free(s); return NULL; }
  return s;
}
void oracle_c4_server_free(oracle_c4_server *s) {
  if (!s) return;
  free(s->db); free(s->bv); free(s->gsw); free(s);
}
/* server.cpp:80-203 (standard path): per limb, pt mod q_k, NTT, transpose */
int oracle_c4_server_load_seeded(oracle_c4_server *s, uint64_t logical, uint64_t seed) {
  const opir_oracle_c4_params *p = &s->p;
  const uint32_t N = p->N;
  if (logical > p->num_pt) return -1;
  const long long np = (long long)p->num_pt;
#pragma omp parallel
  {
    uint64_t *buf = malloc(N * 8);
#pragma omp for schedule(static)
    for (long long pt = 0; pt < np; ++pt)
      for (uint32_t k = 0; k < 2; ++k) {
        for (uint32_t c = 0; c < N; ++c)
          buf[c] = (uint64_t)pt < logical ? oracle_db_coeff(seed, (uint64_t)pt, c, N, p->t) % p->q[k] : 0;
        ntt_k(p, k, buf);
        for (uint32_t c = 0; c < N; ++c) s->db[((size_t)k * N + c) * p->num_pt + (size_t)pt] = buf[c];
      }
    free(buf);
  }
  return 0;
}
int oracle_c4_server_set_keys(oracle_c4_server *s, const uint64_t *bv, const uint64_t *gsw) {
  const opir_oracle_c4_params *p = &s->p;
  const size_t nbv = (size_t)p->expansion_height * p->l_ks * 2 * 2 * p->N;
  const size_t ng = (size_t)2 * p->l_key * 2 * 2 * p->N;
  free(s->bv); free(s->gsw);
  s->bv = malloc((nbv ? nbv : 1) * 8);
  s->gsw = malloc(ng * 8);
  if (nbv) memcpy(s->bv, bv, nbv * 8);
  memcpy(s->gsw, gsw, ng * 8);
  s->has_keys = 1;
  return 0;
}

/* Garner compose of a residue pair into [0, q0 q1) (gsw.cpp:22-53) */
static u128 compose_c4(const opir_oracle_c4_params *p, uint64_t r0, uint64_t r1) {
  const uint64_t q0 = p->q[0], q1 = p->q[1];
  const uint64_t diff = (r1 + q1 - r0 % q1) % q1;
  const uint64_t sv = (uint64_t)((u128)diff * p->q0_inv_mod_q1 % q1);
  return (u128)q0 * sv + r0;
}

/* bv_keyswitch.cpp:373-481 (K = 2); key_rows: L_KS x [b (2N)][a (2N)] */
void oracle_c4_bv_apply_galois(const opir_oracle_c4_params *p, uint64_t *ct, uint32_t galois_k,
                               const uint64_t *key) {
  const uint32_t N = p->N, L = p->l_ks, B = p->base_ks;
  const size_t KN = 2 * (size_t)N;
  uint64_t *c0p = malloc(KN * 8), *c1p = malloc(KN * 8);
  for (uint32_t k = 0; k < 2; ++k) {
    oracle_automorphism(ct + (size_t)k * N, N, galois_k, p->q[k], c0p + (size_t)k * N);
    oracle_automorphism(ct + KN + (size_t)k * N, N, galois_k, p->q[k], c1p + (size_t)k * N);
  }
  /* signed_gadget_decompose_mp (bv_keyswitch.cpp:42-62): digits in
   * (-B/2, B/2], LSB first, from the centred composition */
  int64_t *sd = malloc((size_t)L * N * sizeof *sd);
  const u128 Q = (u128)p->q[0] * p->q[1], half_Q = Q >> 1;
  const uint64_t Bv = 1ULL << B, half_B = Bv >> 1, mask = Bv - 1;
  for (uint32_t j = 0; j < N; ++j) {
    const u128 v = compose_c4(p, c1p[j], c1p[N + j]);
    i128 d = v > half_Q ? (i128)v - (i128)Q : (i128)v;
    for (uint32_t i = 0; i < L; ++i) {
      const uint64_t low = (uint64_t)d & mask;
      int64_t r;
      if (low > half_B) { r = (int64_t)low - (int64_t)Bv; d = (d >> B) + 1; }
      else { r = (int64_t)low; d >>= B; }
      sd[(size_t)i * N + j] = r;
    }
  }
  uint64_t *dig = malloc(N * 8), *db = malloc(N * 8), *da = malloc(N * 8);
  for (uint32_t k = 0; k < 2; ++k) {
    const uint64_t q = p->q[k];
    barrett_t b = barrett_make(q);
    memset(db, 0, N * 8); memset(da, 0, N * 8);
    for (uint32_t i = 0; i < L; ++i) {
      for (uint32_t j = 0; j < N; ++j) dig[j] = sreduce(sd[(size_t)i * N + j], q);
      ntt_k(p, k, dig);
      const uint64_t *kb = key + (size_t)i * 2 * KN + (size_t)k * N;
      const uint64_t *ka = key + (size_t)i * 2 * KN + KN + (size_t)k * N;
      for (uint32_t j = 0; j < N; ++j) {
        db[j] = addmod(db[j], mulmod(&b, dig[j], kb[j]), q);
        da[j] = addmod(da[j], mulmod(&b, dig[j], ka[j]), q);
      }
    }
    intt_k(p, k, db);
    intt_k(p, k, da);
    for (uint32_t j = 0; j < N; ++j) {
      ct[(size_t)k * N + j] = addmod(c0p[(size_t)k * N + j], db[j], q);
      ct[KN + (size_t)k * N + j] = da[j];
    }
  }
  free(c0p); free(c1p); free(sd); free(dig); free(db); free(da);
}

/* server.cpp:731-816. out: u x [c0 (2N)][c1 (2N)] leaves. */
int oracle_c4_server_expand(const oracle_c4_server *s, const uint64_t *query, uint64_t *out) {
  const opir_oracle_c4_params *p = &s->p;
  const uint32_t N = p->N;
  const uint64_t useful = p->fst_dim_sz + (uint64_t)p->l_ep * (p->num_dims - 1);
  const uint32_t h = p->expansion_height;
  const uint64_t cap = 1ULL << h;
  if (!s->has_keys && h > 0) return -1;
  const size_t KN = 2 * (size_t)N, ct = 2 * KN;
  uint64_t *heap = malloc(2 * cap * ct * 8);
  uint64_t *cp = malloc(ct * 8);
  memcpy(heap + 1 * ct, query, ct * 8);
  for (uint64_t i = 1; i < cap; ++i) {
    uint32_t lvl = 0; while ((2ULL << lvl) <= i) ++lvl;
    const uint64_t k = 1ULL << lvl;
    const uint64_t left_leaf = i * cap / k - cap;
    if (left_leaf >= useful) continue;
    uint64_t *ci = heap + i * ct;
    memcpy(cp, ci, ct * 8);
    oracle_c4_bv_apply_galois(p, cp, (uint32_t)(N / k + 1),
                              s->bv + (size_t)lvl * p->l_ks * 2 * KN);
    uint64_t *l = heap + 2 * i * ct, *r = heap + (2 * i + 1) * ct;
    for (uint32_t poly = 0; poly < 2; ++poly)
      for (uint32_t m = 0; m < 2; ++m) {
        const uint64_t q = p->q[m];
        const size_t off = (size_t)poly * KN + (size_t)m * N;
        for (uint32_t j = 0; j < N; ++j) {
          l[off + j] = addmod(ci[off + j], cp[off + j], q);
          ci[off + j] = submod(ci[off + j], cp[off + j], q);
        }
        oracle_negacyclic_shift(ci + off, N, (uint64_t)0 - k, q, r + off);
      }
  }
  memcpy(out, heap + cap * ct, useful * ct * 8);
  free(heap); free(cp);
  return 0;
}

/* gsw.cpp:184-250 (decomp_rlwe_mp): compose to Q, unsigned base-2^B digits,
 * rows MSB-first (row poly*l + (l-1-p) holds digit p), then back to RNS. */
static void decomp_mp(const opir_oracle_c4_params *p, const uint64_t *ct, uint32_t l, uint32_t base,
                      uint64_t *rows) {
  const uint32_t N = p->N;
  const size_t KN = 2 * (size_t)N;
  const uint64_t mask = (1ULL << base) - 1;
  for (uint32_t poly = 0; poly < 2; ++poly)
    for (uint32_t j = 0; j < N; ++j) {
      const u128 v = compose_c4(p, ct[(size_t)poly * KN + j], ct[(size_t)poly * KN + N + j]);
      for (uint32_t d = 0; d < l; ++d) {
        const uint64_t dig = (uint64_t)(v >> (d * base)) & mask;
        uint64_t *row = rows + (size_t)(poly * l + (l - 1 - d)) * KN;
        row[j] = dig % p->q[0];
        row[N + j] = dig % p->q[1];
      }
    }
}
/* gsw.cpp:119-182 (K = 2): output in NTT form per limb */
void oracle_c4_external_product(const opir_oracle_c4_params *p, const uint64_t *rgsw, uint32_t l,
                                uint32_t base, const uint64_t *ct, uint64_t *out) {
  const uint32_t N = p->N;
  const size_t KN = 2 * (size_t)N;
  uint64_t *rows = malloc((size_t)2 * l * KN * 8);
  decomp_mp(p, ct, l, base, rows);
  for (uint32_t j = 0; j < 2 * l; ++j)
    for (uint32_t k = 0; k < 2; ++k) ntt_k(p, k, rows + (size_t)j * KN + (size_t)k * N);
  for (uint32_t poly = 0; poly < 2; ++poly)
    for (uint32_t k = 0; k < 2; ++k) {
      const uint64_t q = p->q[k];
      barrett_t b = barrett_make(q);
      for (uint32_t c = 0; c < N; ++c) {
        uint64_t acc = 0;
        for (uint32_t j = 0; j < 2 * l; ++j)
          acc = addmod(acc, mulmod(&b, rows[(size_t)j * KN + (size_t)k * N + c],
                                   rgsw[(size_t)j * 2 * KN + (size_t)poly * KN + (size_t)k * N + c]), q);
        out[(size_t)poly * KN + (size_t)k * N + c] = acc;
      }
    }
  free(rows);
}

/* server.cpp:823-855 + gsw.cpp:317-357 */
int oracle_c4_server_complete_selectors(const oracle_c4_server *s, const uint64_t *expanded, uint64_t *out) {
  const opir_oracle_c4_params *p = &s->p;
  const uint32_t N = p->N, l = p->l_ep;
  const size_t KN = 2 * (size_t)N, ct = 2 * KN;
  const uint32_t nsel = p->num_dims - 1;
  if (nsel && !s->has_keys) return -1;
  for (uint32_t i = 0; i < nsel; ++i) {
    uint64_t *sel = out + (size_t)i * 2 * l * ct;
    for (uint32_t r = 0; r < l; ++r) {
      const uint64_t *row = expanded + (size_t)(p->fst_dim_sz + (uint64_t)i * l + r) * ct;
      uint64_t *top = sel + (size_t)r * ct, *bot = sel + (size_t)(l + r) * ct;
      memcpy(top, row, ct * 8);
      for (uint32_t poly = 0; poly < 2; ++poly)
        for (uint32_t k = 0; k < 2; ++k) ntt_k(p, k, top + (size_t)poly * KN + (size_t)k * N);
      oracle_c4_external_product(p, s->gsw, p->l_key, p->base_key, row, bot);
    }
  }
  return 0;
}

/* server.cpp:313-405 (standard path) + matrix.cpp:36-151 + server.cpp:
 * 405-527: per limb and NTT level C = A B mod q_k, then INTT per limb. */
int oracle_c4_server_first_dim(const oracle_c4_server *s, const uint64_t *fst_query, uint64_t *out) {
  const opir_oracle_c4_params *p = &s->p;
  const uint32_t N = p->N;
  const uint64_t n0 = p->fst_dim_sz, m = p->other_dim_sz;
  const size_t KN = 2 * (size_t)N, ct = 2 * KN;
  uint64_t *qm = malloc(KN * n0 * 2 * 8);   /* [level][k][c] */
  uint64_t *tmp = malloc(ct * 8);
  for (uint64_t i = 0; i < n0; ++i) {
    memcpy(tmp, fst_query + i * ct, ct * 8);
    for (uint32_t poly = 0; poly < 2; ++poly)
      for (uint32_t k = 0; k < 2; ++k) ntt_k(p, k, tmp + (size_t)poly * KN + (size_t)k * N);
    for (size_t lv = 0; lv < KN; ++lv)
      for (uint32_t c = 0; c < 2; ++c) qm[lv * n0 * 2 + i * 2 + c] = tmp[(size_t)c * KN + lv];
  }
  const long long levels = (long long)KN;
  for (uint64_t j = 0; j < m; ++j) memset(out + j * ct, 0, ct * 8);
#pragma omp parallel for schedule(static)
  for (long long lv = 0; lv < levels; ++lv) {
    const uint64_t q = p->q[(size_t)lv / N];
    const uint64_t *A = s->db + (size_t)lv * p->num_pt;
    const uint64_t *Bq = qm + (size_t)lv * n0 * 2;
    for (uint64_t r = 0; r < m; ++r) {
      u128 t0 = 0, t1 = 0;
      for (uint64_t k = 0; k < n0; ++k) {
        const uint64_t a = A[r * n0 + k];
        t0 = (t0 + (u128)a * Bq[2 * k]) % q;
        t1 = (t1 + (u128)a * Bq[2 * k + 1]) % q;
      }
      out[r * ct + (size_t)lv] = (uint64_t)t0;
      out[r * ct + KN + (size_t)lv] = (uint64_t)t1;
    }
  }
  for (uint64_t j = 0; j < m; ++j)
    for (uint32_t poly = 0; poly < 2; ++poly)
      for (uint32_t k = 0; k < 2; ++k) intt_k(p, k, out + j * ct + (size_t)poly * KN + (size_t)k * N);
  free(qm); free(tmp);
  return 0;
}

/* server.cpp:652-722 (K = 2). y is clobbered; result may alias x. */
static void ext_prod_mux_c4(const opir_oracle_c4_params *p, const uint64_t *x, uint64_t *y,
                            const uint64_t *sel, uint64_t *res) {
  const uint32_t N = p->N;
  const size_t KN = 2 * (size_t)N, ct = 2 * KN;
  for (size_t j = 0; j < ct; ++j) { const uint64_t q = p->q[(j % KN) / N]; y[j] = submod(y[j], x[j], q); }
  uint64_t *tmp = malloc(ct * 8);
  oracle_c4_external_product(p, sel, p->l_ep, p->base_ep, y, tmp);
  for (uint32_t poly = 0; poly < 2; ++poly)
    for (uint32_t k = 0; k < 2; ++k) intt_k(p, k, tmp + (size_t)poly * KN + (size_t)k * N);
  for (size_t j = 0; j < ct; ++j) { const uint64_t q = p->q[(j % KN) / N]; res[j] = addmod(x[j], tmp[j], q); }
  free(tmp);
}
void oracle_c4_ext_prod_mux(const opir_oracle_c4_params *p, const uint64_t *x, uint64_t *y,
                            const uint64_t *sel, uint64_t *res) {
  ext_prod_mux_c4(p, x, y, sel, res);
}

/* server.cpp:599-649 */
int oracle_c4_server_other_dim(const oracle_c4_server *s, uint64_t *mid, const uint64_t *selectors,
                               uint64_t *out) {
  const opir_oracle_c4_params *p = &s->p;
  const size_t ct = 4 * (size_t)p->N;
  const size_t sel_sz = (size_t)2 * p->l_ep * ct;
  if (p->num_dims == 1) { memcpy(out, mid, ct * 8); return 0; }
  const uint64_t h = p->num_dims - 1, other = p->other_dim_sz;
  if (other < (1ULL << (h - 1))) return -1;
  const uint64_t last = 2 * other - (1ULL << h), offset = other - last;
  for (uint64_t i = 0; i < last; i += 2) {
    const uint64_t ci = i + offset;
    ext_prod_mux_c4(p, mid + ci * ct, mid + (ci + 1) * ct, selectors, mid + (i / 2 + offset) * ct);
  }
  for (uint64_t a = 1; a < h; ++a) {
    const uint64_t half = (1ULL << (h - a)) >> 1;
    for (uint64_t i = 0; i < half; ++i)
      ext_prod_mux_c4(p, mid + i * ct, mid + (i + half) * ct, selectors + a * sel_sz, mid + i * ct);
  }
  memcpy(out, mid, ct * 8);
  return 0;
}

/* server.cpp:1044-1075: drop q1 with rounding, then the centred rescale
 * q0 -> small_q; in: [c0 (2N)][c1 (2N)], out: [c0 (N)][c1 (N)] */
void oracle_c4_mod_switch(const opir_oracle_c4_params *p, const uint64_t *ct, uint64_t *out) {
  const uint32_t N = p->N;
  const uint64_t q0 = p->q[0], q1 = p->q[1];
  for (uint32_t poly = 0; poly < 2; ++poly)
    for (uint32_t i = 0; i < N; ++i) {
      const uint64_t r0 = ct[(size_t)poly * 2 * N + i], r1 = ct[(size_t)poly * 2 * N + N + i];
      const u128 x = compose_c4(p, r0, r1);
      uint64_t v = (uint64_t)((x + ((u128)q1 >> 1)) / q1);
      if (v >= q0) v -= q0;
      out[(size_t)poly * N + i] = oracle_rescale(v, q0, p->small_q);
    }
}

/* server.cpp:895-947 */
int oracle_c4_server_make_query(const oracle_c4_server *s, const uint64_t *query, uint64_t *resp) {
  const opir_oracle_c4_params *p = &s->p;
  const size_t ct = 4 * (size_t)p->N;
  const uint64_t useful = p->fst_dim_sz + (uint64_t)p->l_ep * (p->num_dims - 1);
  const uint32_t nsel = p->num_dims - 1;
  uint64_t *exp = malloc(useful * ct * 8);
  uint64_t *sel = malloc((nsel ? nsel : 1) * (size_t)2 * p->l_ep * ct * 8);
  uint64_t *mid = malloc(p->other_dim_sz * ct * 8);
  uint64_t *fin = malloc(ct * 8);
  int rc = oracle_c4_server_expand(s, query, exp);
  if (!rc) rc = oracle_c4_server_complete_selectors(s, exp, sel);
  if (!rc) rc = oracle_c4_server_first_dim(s, exp, mid);
  if (!rc) rc = oracle_c4_server_other_dim(s, mid, sel, fin);
  if (!rc) oracle_c4_mod_switch(p, fin, resp);
  free(exp); free(sel); free(mid); free(fin);
  return rc;
}

/* server.cpp:950-1009 with small_q_width = 50: c0 then c1, LSB-first */
size_t oracle_c4_serialize(const opir_oracle_c4_params *p, const uint64_t *resp, uint8_t *out) {
  const uint32_t w = p->small_q_width;
  uint8_t buf = 0;
  uint32_t filled = 0;
  size_t nb = 0;
  for (uint32_t i = 0; i < 2 * p->N; ++i) {
    const uint64_t c = resp[i] & ((1ULL << w) - 1);
    uint32_t written = 0;
    while (written < w) {
      const uint32_t room = 8 - filled, take = w - written < room ? w - written : room;
      const uint8_t chunk = (uint8_t)((c >> written) & ((1ULL << take) - 1));
      buf |= (uint8_t)(chunk << filled);
      filled += take;
      written += take;
      if (filled == 8) { out[nb++] = buf; buf = 0; filled = 0; }
    }
  }
  if (filled) out[nb++] = buf;
  return nb;
}
