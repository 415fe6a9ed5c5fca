/* CPU oracle for the OnionPIRv2 server hot path (PirServer::make_query).
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference's
 * algorithm, used by tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py as the checker. Nothing in the product links or calls it.
 *
 * Parameter set: CONFIG_N2048_K1_COMP (database_constants.h:77-94): N = 2048,
 * logical q = q1*q2 (two 29-bit NTT primes), t = generate_prime(13),
 * small_q = 22-bit NTT prime, L_EP = 6, L_KEY = 10, L_KS = 8.
 *
 * Layouts (all little-endian u64, values canonical in [0, q)):
 *   ciphertext   : [c0 (N)][c1 (N)]                                 (rlwe.h:17-31)
 *   BV keys      : [level i < h][row j < L_KS][b (N)][a (N)], NTT form,
 *                  galois_k(level i) = (N >> i) + 1             (bv_keyswitch.h:48-66)
 *   RGSW (GSWCt) : [row r < 2l][c0 (N)][c1 (N)], NTT form          (gsw.h:8-17)
 */
#ifndef OPIR_ORACLE_H
#define OPIR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint32_t N;
  uint64_t q, q1, q2;           /* logical modulus and its CRT factors   */
  uint64_t w1, w2, w_crt;       /* minimal 2N-th roots mod q1, q2; CRT   */
  uint64_t q1_inv_mod_q2;
  uint64_t t, small_q;
  uint32_t small_q_width;
  uint32_t ct_mod_width;        /* 58: sum of configured limb bit widths */
  uint32_t l_ep, l_key, l_ks;
  uint32_t base_ep, base_key, base_ks;
  uint64_t target_num_pt, num_pt, fst_dim_sz, other_dim_sz;
  uint32_t num_dims, expansion_height, fst_dim_pow2;
} opir_oracle_params;

/* ---- parameters (pir.cpp, utils.cpp) ---- */
int oracle_is_prime(uint64_t n);
uint64_t oracle_generate_prime(uint32_t bit_width);
int oracle_ntt_primes(const uint32_t *bit_widths, uint32_t count, uint32_t N,
                      uint64_t *out);
uint64_t oracle_min_primitive_root(uint64_t degree, uint64_t q);
int oracle_calc_db_shape(uint64_t target, uint64_t l, uint32_t h, int pow2,
                         uint64_t *fst_dim_sz, uint64_t *num_dims);
int oracle_params_init(uint64_t target_num_pt, uint32_t expansion_height,
                       int fst_dim_pow2, opir_oracle_params *out);
/* CONFIG_N2048_K1 (the reference's default): one 60-bit prime q, q1 = q2 = 0 */
int oracle_k1p_params_init(uint64_t target_num_pt, uint32_t expansion_height,
                           int fst_dim_pow2, opir_oracle_params *out);

/* ---- ring primitives ---- */
void oracle_ntt_fwd(uint64_t *a, uint32_t N, uint64_t q, uint64_t root);
void oracle_ntt_inv(uint64_t *a, uint32_t N, uint64_t q, uint64_t root);
void oracle_automorphism(const uint64_t *in, uint32_t N, uint32_t k, uint64_t q,
                         uint64_t *out);
void oracle_negacyclic_shift(const uint64_t *in, uint32_t N, uint64_t shift,
                             uint64_t q, uint64_t *out);
uint64_t oracle_rescale(uint64_t a, uint64_t inp_mod, uint64_t out_mod);
void oracle_signed_decompose(uint64_t val, uint32_t base_log2, uint64_t q,
                             uint64_t *out, uint32_t num_digits);

/* ---- seeded client (the reference client with seeded generators) ---- */
uint64_t oracle_mt_test(uint64_t seed, uint64_t skip);
uint64_t oracle_db_coeff(uint64_t seed, uint64_t pt, uint64_t c, uint64_t N,
                         uint64_t t);
void oracle_db_plaintext(uint64_t seed, uint64_t pt, const opir_oracle_params *p,
                         uint16_t *out);

typedef struct oracle_client oracle_client;
oracle_client *oracle_client_new(const opir_oracle_params *p, uint64_t seed);
/* The same client, also returning the randomness its key generation drew,
 * in generation order: bv_a (h x L_KS x N, coefficient form) and bv_e
 * (h x L_KS x N, signed) for the BV keys, gsw_a / gsw_e (2 L_KEY x N) for
 * the RGSW rows (create_session_keys, client.cpp:40-45). */
oracle_client *oracle_client_new_keygen_parts(const opir_oracle_params *p, uint64_t seed,
                                              uint64_t *bv_a, int64_t *bv_e, uint64_t *gsw_a,
                                              int64_t *gsw_e);
void oracle_client_free(oracle_client *c);
void oracle_client_bv_keys(const oracle_client *c, uint64_t *out);
void oracle_client_gsw_key(const oracle_client *c, uint64_t *out);
int oracle_client_query(oracle_client *c, uint64_t pt_idx, uint64_t *out);
/* The same query with its uniform polynomial c1 = a given by the caller
 * (a seed-compressed query: a = Expand(seed)); the error still comes from
 * the client's generator. */
int oracle_client_query_with_a(oracle_client *c, uint64_t pt_idx, const uint64_t *a,
                               uint64_t *out);
/* The same, also returning the error e (N signed values) it drew. */
int oracle_client_query_parts(oracle_client *c, uint64_t pt_idx, const uint64_t *a,
                              uint64_t *out, int64_t *e_out);
/* The secret key in coefficient form, N values in {-1, 0, 1}. */
void oracle_client_secret(const oracle_client *c, int8_t *out);
/* tree_query.cpp:142-196 (K = 1): packed tree query; bits = b beta bits
 * then r gamma bits (little-endian coordinates), groups = b + r. */
int oracle_client_tree_query(oracle_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                             const uint8_t *bits, uint32_t groups, uint64_t *out);
/* The same with c1 = a given (N), also returning the error drawn (N). */
int oracle_client_tree_query_parts(oracle_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                                   const uint8_t *bits, uint32_t groups, const uint64_t *a,
                                   uint64_t *out, int64_t *e_out);
/* decrypt_rns (rlwe.cpp:310-348, K = 1) of a coefficient-form ciphertext. */
void oracle_client_decrypt_q(const oracle_client *c, const uint64_t *ct, uint64_t *pt_out);
void oracle_client_decrypt(const oracle_client *c, const uint64_t *resp,
                           uint64_t *pt_out);
/* The same, also returning the response's max noise (client.cpp:389-407). */
void oracle_client_decrypt_noise(const oracle_client *c, const uint64_t *resp, uint64_t *pt_out,
                                 uint64_t *max_noise);

/* ---- server (server.cpp, gsw.cpp, bv_keyswitch.cpp, matrix.cpp) ---- */
typedef struct oracle_server oracle_server;
oracle_server *oracle_server_new(const opir_oracle_params *p);
void oracle_server_free(oracle_server *s);
int oracle_server_load_seeded(oracle_server *s, uint64_t logical_num_pt,
                              uint64_t seed);
int oracle_server_load(oracle_server *s, uint64_t logical_num_pt,
                       const uint16_t *coeffs);
int oracle_server_set_keys(oracle_server *s, const uint64_t *bv_keys,
                           const uint64_t *gsw_key);
int oracle_server_expand(const oracle_server *s, const uint64_t *query,
                         uint64_t *out);
int oracle_server_complete_selectors(const oracle_server *s,
                                     const uint64_t *expanded, uint64_t *out);
int oracle_server_first_dim(const oracle_server *s, const uint64_t *fst_query,
                            uint64_t *out);
int oracle_server_other_dim(const oracle_server *s, uint64_t *mid,
                            const uint64_t *selectors, uint64_t *out);
int oracle_server_make_query(const oracle_server *s, const uint64_t *query,
                             uint64_t *resp);
/* PirServer::ext_prod_mux (server.cpp:652-722): res = x + INTT(ExtProd(sel,
 * y - x)); x, y coefficient form (2N u64), y is clobbered, res may alias x;
 * sel = 2 L_EP rows x 2N u64, NTT form. */
void oracle_ext_prod_mux(const opir_oracle_params *p, const uint64_t *x, uint64_t *y,
                         const uint64_t *sel, uint64_t *res);
void oracle_mod_switch(const opir_oracle_params *p, uint64_t *ct);
size_t oracle_serialize(const opir_oracle_params *p, const uint64_t *resp,
                        uint8_t *out);
void oracle_external_product(const opir_oracle_params *p, const uint64_t *rgsw,
                             uint32_t l, uint32_t base_log2,
                             const uint64_t *ct, uint64_t *out);
void oracle_bv_apply_galois(const opir_oracle_params *p, uint64_t *ct,
                            uint32_t galois_k, const uint64_t *key_rows);
void oracle_level_mat_mat_32(const uint32_t *A, const uint32_t *B, uint64_t *out,
                             uint64_t m, uint64_t n, uint64_t levels, uint64_t q);

/* ---- CONFIG_N4096_K2_MP (opir_oracle_c4.c): N = 4096, two 60-bit RNS
 *      limbs, limb-major layouts [limb 0 (N)][limb 1 (N)] per polynomial ---- */
typedef struct {
  uint32_t N, K;
  uint64_t q[2], w[2];          /* limbs and their minimal 2N-th roots   */
  uint64_t q0_inv_mod_q1, r64_mod_q[2];
  uint64_t t, small_q;
  uint32_t small_q_width, ct_mod_width;
  uint32_t l_ep, l_key, l_ks;
  uint32_t base_ep, base_key, base_ks;
  uint64_t target_num_pt, num_pt, fst_dim_sz, other_dim_sz;
  uint32_t num_dims, expansion_height, fst_dim_pow2;
} opir_oracle_c4_params;

int oracle_c4_params_init(uint64_t target_num_pt, uint32_t expansion_height,
                          int fst_dim_pow2, opir_oracle_c4_params *out);
/* CONFIG_N2048_K2_MP: the same two-limb routines at N = 2048, limbs of 29 bits */
int oracle_k2mp_params_init(uint64_t target_num_pt, uint32_t expansion_height,
                            int fst_dim_pow2, opir_oracle_c4_params *out);
void oracle_c4_db_plaintext(uint64_t seed, uint64_t pt,
                            const opir_oracle_c4_params *p, uint64_t *out);

typedef struct oracle_c4_client oracle_c4_client;
oracle_c4_client *oracle_c4_client_new(const opir_oracle_c4_params *p, uint64_t seed);
/* Two-limb form: bv_a h x L_KS x 2N, gsw_a 2 L_KEY x 2N (limb-major), the
 * errors N each (shared by the limbs). */
oracle_c4_client *oracle_c4_client_new_keygen_parts(const opir_oracle_c4_params *p, uint64_t seed,
                                                    uint64_t *bv_a, int64_t *bv_e,
                                                    uint64_t *gsw_a, int64_t *gsw_e);
void oracle_c4_client_free(oracle_c4_client *c);
void oracle_c4_client_bv_keys(const oracle_c4_client *c, uint64_t *out);
void oracle_c4_client_gsw_key(const oracle_c4_client *c, uint64_t *out);
int oracle_c4_client_query(oracle_c4_client *c, uint64_t pt_idx, uint64_t *out);
/* tree_query.cpp:142-196 (K = 2): packed tree query; bits as for
 * oracle_client_tree_query; out: 4N u64 limb-major. */
int oracle_c4_client_tree_query(oracle_c4_client *c, uint64_t N0, uint32_t h_q, uint64_t alpha,
                                const uint8_t *bits, uint32_t groups, uint64_t *out);
int oracle_c4_client_tree_query_parts(oracle_c4_client *c, uint64_t N0, uint32_t h_q,
                                      uint64_t alpha, const uint8_t *bits, uint32_t groups,
                                      const uint64_t *a, uint64_t *out, int64_t *e_out);
/* Query with a given uniform c1 (2N, limb-major), returning the shared
 * error (N signed values); the secret in coefficient form (N in {-1,0,1}). */
int oracle_c4_client_query_parts(oracle_c4_client *c, uint64_t pt_idx, const uint64_t *a,
                                 uint64_t *out, int64_t *e_out);
void oracle_c4_client_secret(const oracle_c4_client *c, int8_t *out);
void oracle_c4_client_decrypt(const oracle_c4_client *c, const uint64_t *resp,
                              uint64_t *pt_out);
void oracle_c4_client_decrypt_noise(const oracle_c4_client *c, const uint64_t *resp,
                                    uint64_t *pt_out, uint64_t *max_noise);

typedef struct oracle_c4_server oracle_c4_server;
oracle_c4_server *oracle_c4_server_new(const opir_oracle_c4_params *p);
void oracle_c4_server_free(oracle_c4_server *s);
int oracle_c4_server_load_seeded(oracle_c4_server *s, uint64_t logical_num_pt,
                                 uint64_t seed);
int oracle_c4_server_set_keys(oracle_c4_server *s, const uint64_t *bv_keys,
                              const uint64_t *gsw_key);
int oracle_c4_server_expand(const oracle_c4_server *s, const uint64_t *query,
                            uint64_t *out);
int oracle_c4_server_complete_selectors(const oracle_c4_server *s,
                                        const uint64_t *expanded, uint64_t *out);
int oracle_c4_server_first_dim(const oracle_c4_server *s,
                               const uint64_t *fst_query, uint64_t *out);
int oracle_c4_server_other_dim(const oracle_c4_server *s, uint64_t *mid,
                               const uint64_t *selectors, uint64_t *out);
int oracle_c4_server_make_query(const oracle_c4_server *s, const uint64_t *query,
                                uint64_t *resp);
/* ext_prod_mux under CONFIG_N4096_K2_MP: 4N u64 ciphertexts (limb-major). */
void oracle_c4_ext_prod_mux(const opir_oracle_c4_params *p, const uint64_t *x, uint64_t *y,
                            const uint64_t *sel, uint64_t *res);
void oracle_c4_mod_switch(const opir_oracle_c4_params *p, const uint64_t *ct,
                          uint64_t *out);
void oracle_c4_external_product(const opir_oracle_c4_params *p,
                                const uint64_t *rgsw, uint32_t l, uint32_t base,
                                const uint64_t *ct, uint64_t *out);
void oracle_c4_bv_apply_galois(const opir_oracle_c4_params *p, uint64_t *ct,
                               uint32_t galois_k, const uint64_t *key_rows);
size_t oracle_c4_serialize(const opir_oracle_c4_params *p, const uint64_t *resp,
                           uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
