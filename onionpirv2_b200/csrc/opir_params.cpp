// Parameter derivation (host). Restates src/pir.cpp:14-134 and the helpers it
// uses in src/utils.cpp (primes :136-287, crt_combine :229-238,
// calculate_db_shape :376-401) for CONFIG_N2048_K1_COMP, plus HEXL's
// MinimalPrimitiveRoot (the smallest primitive 2N-th root of unity mod a
// prime).
#include "opir_params.h"

#include <cmath>
#include <limits>
#include <stdexcept>

namespace opir {

using u128 = unsigned __int128;

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
  u128 r = 1 % m, x = b % m;
  while (e) {
    if (e & 1) r = r * x % m;
    x = x * x % m;
    e >>= 1;
  }
  return static_cast<uint64_t>(r);
}

bool is_prime_u64(uint64_t n) {
  static const uint64_t sp[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return false;
  for (uint64_t p : sp) {
    if (n == p) return true;
    if (n % p == 0) return false;
  }
  uint64_t d = n - 1;
  int r = 0;
  while ((d & 1) == 0) { d >>= 1; ++r; }
  for (uint64_t a : sp) {
    uint64_t x = powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool composite = true;
    for (int i = 0; i < r - 1; ++i) {
      x = static_cast<uint64_t>(static_cast<u128>(x) * x % n);
      if (x == n - 1) { composite = false; break; }
    }
    if (composite) return false;
  }
  return true;
}

uint64_t generate_prime(uint32_t bit_width) {
  if (bit_width < 2) throw std::invalid_argument("Bit width must be at least 2.");
  uint64_t c = 1ull << (bit_width - 1);
  do { ++c; c |= 1; } while (!is_prime_u64(c));
  return c;
}

std::vector<uint64_t> ntt_friendly_primes(const std::vector<uint32_t> &bws, uint32_t n) {
  const uint64_t step = 2ull * n;
  std::vector<uint64_t> out;
  uint64_t next[64] = {0};
  bool have[64] = {false};
  for (uint32_t bw : bws) {
    if (bw < 2 || bw > 63) throw std::invalid_argument("bit width out of range [2, 63]");
    uint64_t c;
    if (!have[bw]) { c = (1ull << bw) - 1; c -= (c - 1) % step; }
    else c = next[bw];
    for (;;) {
      if (c < 2) throw std::runtime_error("No NTT-friendly prime found");
      if (is_prime_u64(c)) break;
      c -= step;
    }
    out.push_back(c);
    next[bw] = c >= step ? c - step : 0;
    have[bw] = true;
  }
  return out;
}

uint64_t min_primitive_root(uint64_t degree, uint64_t q) {
  uint64_t g = 0;
  for (uint64_t x = 2; x < q; ++x) {
    const uint64_t c = powmod(x, (q - 1) / degree, q);
    if (powmod(c, degree / 2, q) == q - 1) { g = c; break; }
  }
  if (!g) throw std::runtime_error("no primitive root");
  const uint64_t g2 = static_cast<uint64_t>(static_cast<u128>(g) * g % q);
  uint64_t cur = g, best = g;
  for (uint64_t i = 0; i < degree / 2; ++i) {
    if (cur < best) best = cur;
    cur = static_cast<uint64_t>(static_cast<u128>(cur) * g2 % q);
  }
  return best;
}

bool invert_mod(uint64_t v, uint64_t m, uint64_t &out) {
  if (v == 0) return false;
  int64_t s0 = 1, s1 = 0, r0 = static_cast<int64_t>(v), r1 = static_cast<int64_t>(m);
  while (r1 != 0) {
    const int64_t qq = r0 / r1;
    int64_t t = r1; r1 = r0 - qq * r1; r0 = t;
    t = s1; s1 = s0 - qq * s1; s0 = t;
  }
  if (r0 != 1) return false;
  out = s0 < 0 ? static_cast<uint64_t>(s0 + static_cast<int64_t>(m)) : static_cast<uint64_t>(s0);
  return true;
}

std::pair<uint64_t, uint64_t> calc_db_shape(uint64_t target, uint64_t l, uint32_t h, bool pow2) {
  if (target == 0) throw std::invalid_argument("calculate_db_shape target must be positive");
  if (l == 0) throw std::invalid_argument("calculate_db_shape gadget length must be positive");
  if (h >= 64) throw std::invalid_argument("calculate_db_shape height is too large");
  const uint64_t capacity = 1ull << h;
  const uint64_t max_dims = 1 + (capacity - 1) / l;
  for (uint64_t nd = 1; nd <= max_dims + 1; ++nd) {
    const uint64_t reserved = l * (nd - 1);
    if (reserved >= capacity) break;
    const uint64_t slack = capacity - reserved;
    uint64_t f = slack;
    if (pow2) { f = 1; while ((f << 1) <= slack) f <<= 1; }
    if (nd - 1 < 63 && f * (1ull << (nd - 1)) >= target) return {f, nd};
  }
  throw std::runtime_error("Failed to calculate database shape");
}

opir_params derive_params(const opir_layout &layout) {
  constexpr uint32_t N = 2048;
  opir_params p{};
  p.poly_degree = N;
  p.num_limbs = 1;
  const auto pr = ntt_friendly_primes({29, 29}, N);
  p.q1 = pr[0];
  p.q2 = pr[1];
  p.q = p.q1 * p.q2;
  p.w1 = min_primitive_root(2ull * N, p.q1);
  p.w2 = min_primitive_root(2ull * N, p.q2);
  uint64_t inv = 0;
  if (!invert_mod(p.q1 % p.q2, p.q2, inv)) throw std::runtime_error("q1, q2 must be coprime");
  p.q1_inv_mod_q2 = inv;
  const uint64_t diff = (p.w2 + p.q2 - p.w1 % p.q2) % p.q2;
  const uint64_t k = static_cast<uint64_t>(static_cast<u128>(diff) * inv % p.q2);
  p.w_crt = static_cast<uint64_t>(static_cast<u128>(p.q1) * k + p.w1);
  p.plain_mod = generate_prime(13);
  p.small_q = ntt_friendly_primes({22}, N)[0];
  p.small_q_width = static_cast<uint32_t>(std::ceil(std::log2(static_cast<double>(p.small_q))));
  p.ct_mod_width = 58;
  p.l_ep = 6;
  p.l_key = 10;
  p.l_ks = 8;
  p.base_log2 = (p.ct_mod_width + p.l_ep - 1) / p.l_ep;
  p.base_log2_key = (p.ct_mod_width + p.l_key - 1) / p.l_key;
  p.base_log2_ks = p.ct_mod_width / p.l_ks + 1;
  // apply_layout (pir.cpp:100-128)
  if (layout.target_num_pt == 0)
    throw std::invalid_argument("PirParams: target_num_pt must be positive");
  if (layout.expansion_height > 11)
    throw std::invalid_argument("PirParams: expansion_height exceeds the ring automorphism capacity");
  const auto shape = calc_db_shape(layout.target_num_pt, p.l_ep, layout.expansion_height,
                                   layout.fst_dim_pow2 != 0);
  const uint64_t other = (layout.target_num_pt + shape.first - 1) / shape.first;
  if (other > std::numeric_limits<uint64_t>::max() / shape.first)
    throw std::overflow_error("PirParams: rounded database shape overflows");
  p.target_num_pt = layout.target_num_pt;
  p.expansion_height = layout.expansion_height;
  p.fst_dim_pow2 = layout.fst_dim_pow2 ? 1 : 0;
  p.fst_dim_sz = shape.first;
  p.num_dims = static_cast<uint32_t>(shape.second);
  p.other_dim_sz = other;
  p.num_pt = shape.first * other;
  return p;
}

opir_params derive_params_k2mp(const opir_layout &layout) {
  // pir.cpp:49-134 with CONFIG_N2048_K2_MP (database_constants.h:96-110):
  // RnsMods {29, 29} as two real RNS limbs, PlainMod 10, SmallQWidth 22,
  // L_EP 5, L_KEY 8, L_KS 8. The limbs are the same primes as the
  // composite split of CONFIG_N2048_K1_COMP, and q = q1 q2 fits 64 bits.
  constexpr uint32_t N = 2048;
  opir_params p{};
  p.poly_degree = N;
  p.num_limbs = 2;
  const auto pr = ntt_friendly_primes({29, 29}, N);
  p.q1 = pr[0];  // the two RNS limbs (q0, q1 in the reference's naming)
  p.q2 = pr[1];
  p.q = p.q1 * p.q2;
  p.w1 = min_primitive_root(2ull * N, p.q1);
  p.w2 = min_primitive_root(2ull * N, p.q2);
  uint64_t inv = 0;
  if (!invert_mod(p.q1 % p.q2, p.q2, inv)) throw std::runtime_error("limbs must be coprime");
  p.q1_inv_mod_q2 = inv;
  p.w_crt = 0;  // each limb runs its own NTT
  p.plain_mod = generate_prime(10);
  p.small_q = ntt_friendly_primes({22}, N)[0];
  p.small_q_width = static_cast<uint32_t>(std::ceil(std::log2(static_cast<double>(p.small_q))));
  p.ct_mod_width = 58;  // pir.cpp:188-194: sum of the configured limb widths
  p.l_ep = 5;
  p.l_key = 8;
  p.l_ks = 8;
  p.base_log2 = (p.ct_mod_width + p.l_ep - 1) / p.l_ep;
  p.base_log2_key = (p.ct_mod_width + p.l_key - 1) / p.l_key;
  p.base_log2_ks = p.ct_mod_width / p.l_ks + 1;
  if (layout.target_num_pt == 0)
    throw std::invalid_argument("PirParams: target_num_pt must be positive");
  if (layout.expansion_height > 11)
    throw std::invalid_argument("PirParams: expansion_height exceeds the ring automorphism capacity");
  const auto shape = calc_db_shape(layout.target_num_pt, p.l_ep, layout.expansion_height,
                                   layout.fst_dim_pow2 != 0);
  const uint64_t other = (layout.target_num_pt + shape.first - 1) / shape.first;
  if (other > std::numeric_limits<uint64_t>::max() / shape.first)
    throw std::overflow_error("PirParams: rounded database shape overflows");
  p.target_num_pt = layout.target_num_pt;
  p.expansion_height = layout.expansion_height;
  p.fst_dim_pow2 = layout.fst_dim_pow2 ? 1 : 0;
  p.fst_dim_sz = shape.first;
  p.num_dims = static_cast<uint32_t>(shape.second);
  p.other_dim_sz = other;
  p.num_pt = shape.first * other;
  return p;
}

opir_params derive_params_k1p(const opir_layout &layout) {
  // pir.cpp:49-134 with CONFIG_N2048_K1 (database_constants.h:61-76), the
  // reference's default ACTIVE_CONFIG: RnsMods {60} (one real NTT prime, no
  // composite split), PlainMod 14, SmallQWidth 22, L_EP 5, L_KEY 8, L_KS 8.
  constexpr uint32_t N = 2048;
  opir_params p{};
  p.poly_degree = N;
  p.num_limbs = 1;
  p.q = ntt_friendly_primes({60}, N)[0];
  p.q1 = p.q2 = 0;  // no composite first-dimension split
  p.w1 = min_primitive_root(2ull * N, p.q);
  p.w2 = 0;
  p.w_crt = p.w1;
  p.q1_inv_mod_q2 = 0;
  p.plain_mod = generate_prime(14);
  p.small_q = ntt_friendly_primes({22}, N)[0];
  p.small_q_width = static_cast<uint32_t>(std::ceil(std::log2(static_cast<double>(p.small_q))));
  p.ct_mod_width = 60;
  p.l_ep = 5;
  p.l_key = 8;
  p.l_ks = 8;
  p.base_log2 = (p.ct_mod_width + p.l_ep - 1) / p.l_ep;
  p.base_log2_key = (p.ct_mod_width + p.l_key - 1) / p.l_key;
  p.base_log2_ks = p.ct_mod_width / p.l_ks + 1;
  if (layout.target_num_pt == 0)
    throw std::invalid_argument("PirParams: target_num_pt must be positive");
  if (layout.expansion_height > 11)
    throw std::invalid_argument("PirParams: expansion_height exceeds the ring automorphism capacity");
  const auto shape = calc_db_shape(layout.target_num_pt, p.l_ep, layout.expansion_height,
                                   layout.fst_dim_pow2 != 0);
  const uint64_t other = (layout.target_num_pt + shape.first - 1) / shape.first;
  if (other > std::numeric_limits<uint64_t>::max() / shape.first)
    throw std::overflow_error("PirParams: rounded database shape overflows");
  p.target_num_pt = layout.target_num_pt;
  p.expansion_height = layout.expansion_height;
  p.fst_dim_pow2 = layout.fst_dim_pow2 ? 1 : 0;
  p.fst_dim_sz = shape.first;
  p.num_dims = static_cast<uint32_t>(shape.second);
  p.other_dim_sz = other;
  p.num_pt = shape.first * other;
  return p;
}

static uint32_t bitrev(uint32_t x, uint32_t bits) {
  uint32_t y = 0;
  for (uint32_t i = 0; i < bits; ++i) { y = (y << 1) | (x & 1); x >>= 1; }
  return y;
}

LimbTables make_limb_tables(uint32_t n, uint32_t q, uint32_t root) {
  LimbTables t;
  t.q = q;
  t.mu = static_cast<uint64_t>((static_cast<u128>(1) << 64) / q);
  uint32_t lg = 0;
  while ((1u << lg) < n) ++lg;
  uint64_t rinv = 0;
  invert_mod(root, q, rinv);
  std::vector<uint32_t> pw(n), ipw(n);
  pw[0] = ipw[0] = 1;
  for (uint32_t i = 1; i < n; ++i) {
    pw[i] = static_cast<uint32_t>(static_cast<uint64_t>(pw[i - 1]) * root % q);
    ipw[i] = static_cast<uint32_t>(static_cast<uint64_t>(ipw[i - 1]) * rinv % q);
  }
  auto shoup = [q](uint32_t w) {
    return static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / q);
  };
  t.fw.resize(n); t.fw_sh.resize(n); t.iw.resize(n); t.iw_sh.resize(n);
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t e = bitrev(k, lg);
    t.fw[k] = pw[e]; t.fw_sh[k] = shoup(pw[e]);
    t.iw[k] = ipw[e]; t.iw_sh[k] = shoup(ipw[e]);
  }
  uint64_t ninv = 0;
  invert_mod(n % q, q, ninv);
  t.n_inv = static_cast<uint32_t>(ninv);
  t.n_inv_sh = shoup(t.n_inv);
  return t;
}

opir_params derive_params_c4(const opir_layout &layout) {
  // pir.cpp:49-134 with CONFIG_N4096_K2_MP (database_constants.h:111-125):
  // RnsMods {60, 60}, PlainMod 40, SmallQWidth 50, L_EP 5, L_KEY 8, L_KS 8.
  constexpr uint32_t N = 4096;
  opir_params p{};
  p.poly_degree = N;
  p.num_limbs = 2;
  const auto pr = ntt_friendly_primes({60, 60}, N);
  p.q1 = pr[0];  // the two RNS limbs (q0, q1 in the reference's naming)
  p.q2 = pr[1];
  p.q = 0;       // the product exceeds 64 bits
  p.w1 = min_primitive_root(2ull * N, p.q1);
  p.w2 = min_primitive_root(2ull * N, p.q2);
  uint64_t inv = 0;
  if (!invert_mod(p.q1 % p.q2, p.q2, inv)) throw std::runtime_error("limbs must be coprime");
  p.q1_inv_mod_q2 = inv;
  p.w_crt = 0;
  p.plain_mod = generate_prime(40);
  p.small_q = ntt_friendly_primes({50}, N)[0];
  p.small_q_width = 50;
  p.ct_mod_width = 120;  // pir.cpp:188-194: sum of the configured limb widths
  p.l_ep = 5;
  p.l_key = 8;
  p.l_ks = 8;
  p.base_log2 = (p.ct_mod_width + p.l_ep - 1) / p.l_ep;
  p.base_log2_key = (p.ct_mod_width + p.l_key - 1) / p.l_key;
  p.base_log2_ks = p.ct_mod_width / p.l_ks + 1;
  if (layout.target_num_pt == 0)
    throw std::invalid_argument("PirParams: target_num_pt must be positive");
  if (layout.expansion_height > 12)
    throw std::invalid_argument("PirParams: expansion_height exceeds the ring automorphism capacity");
  const auto shape = calc_db_shape(layout.target_num_pt, p.l_ep, layout.expansion_height,
                                   layout.fst_dim_pow2 != 0);
  const uint64_t other = (layout.target_num_pt + shape.first - 1) / shape.first;
  if (other > std::numeric_limits<uint64_t>::max() / shape.first)
    throw std::overflow_error("PirParams: rounded database shape overflows");
  p.target_num_pt = layout.target_num_pt;
  p.expansion_height = layout.expansion_height;
  p.fst_dim_pow2 = layout.fst_dim_pow2 ? 1 : 0;
  p.fst_dim_sz = shape.first;
  p.num_dims = static_cast<uint32_t>(shape.second);
  p.other_dim_sz = other;
  p.num_pt = shape.first * other;
  return p;
}

LimbTables64 make_limb_tables64(uint32_t n, uint64_t q, uint64_t root) {
  LimbTables64 t;
  t.q = q;
  uint32_t lg = 0;
  while ((1u << lg) < n) ++lg;
  uint64_t rinv = 0;
  invert_mod(root % q, q, rinv);
  std::vector<uint64_t> pw(n), ipw(n);
  pw[0] = ipw[0] = 1;
  for (uint32_t i = 1; i < n; ++i) {
    pw[i] = static_cast<uint64_t>(static_cast<u128>(pw[i - 1]) * root % q);
    ipw[i] = static_cast<uint64_t>(static_cast<u128>(ipw[i - 1]) * rinv % q);
  }
  auto shoup = [q](uint64_t w) { return static_cast<uint64_t>((static_cast<u128>(w) << 64) / q); };
  t.fw.resize(n); t.fw_sh.resize(n); t.iw.resize(n); t.iw_sh.resize(n);
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t e = bitrev(k, lg);
    t.fw[k] = pw[e]; t.fw_sh[k] = shoup(pw[e]);
    t.iw[k] = ipw[e]; t.iw_sh[k] = shoup(ipw[e]);
  }
  uint64_t ninv = 0;
  invert_mod(n % q, q, ninv);
  t.n_inv = ninv;
  t.n_inv_sh = shoup(ninv);
  t.w1_ninv = static_cast<uint64_t>(static_cast<u128>(t.iw[1]) * ninv % q);
  t.w1_ninv_sh = shoup(t.w1_ninv);
  return t;
}

}  // namespace opir
