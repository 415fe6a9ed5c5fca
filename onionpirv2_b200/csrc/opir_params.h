// Host-side parameter derivation for CONFIG_N2048_K1_COMP (and
// CONFIG_N4096_K2_MP): primes, roots,
// gadget bases, database shape, NTT twiddle tables for the two CRT limbs.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/onionpir_b200.h"

namespace opir {

bool is_prime_u64(uint64_t n);
uint64_t generate_prime(uint32_t bit_width);
std::vector<uint64_t> ntt_friendly_primes(const std::vector<uint32_t> &bit_widths,
                                          uint32_t n);
uint64_t min_primitive_root(uint64_t degree, uint64_t q);
bool invert_mod(uint64_t v, uint64_t m, uint64_t &out);
// {fst_dim_sz, num_dims}; throws std::invalid_argument / std::runtime_error.
std::pair<uint64_t, uint64_t> calc_db_shape(uint64_t target, uint64_t l, uint32_t h,
                                            bool pow2);
// PirParams().with_layout(layout); throws like the reference.
opir_params derive_params(const opir_layout &layout);

// Per-limb NTT tables (u32 values and Shoup companions).
struct LimbTables {
  uint32_t q = 0, n_inv = 0, n_inv_sh = 0;
  uint64_t mu = 0;
  std::vector<uint32_t> fw, fw_sh, iw, iw_sh;
};
LimbTables make_limb_tables(uint32_t n, uint32_t q, uint32_t root);

// CONFIG_N4096_K2_MP: N = 4096, two 60-bit RNS limbs (q1, q2 fields hold the
// limbs, q = 0), t = generate_prime(40), small_q 50-bit, L_EP 5, L_KEY 8, L_KS 8.
opir_params derive_params_c4(const opir_layout &layout);
// PirParams under CONFIG_N2048_K2_MP (two 29-bit RNS limbs at N = 2048).
opir_params derive_params_k2mp(const opir_layout &layout);
// PirParams under CONFIG_N2048_K1 (one 60-bit prime at N = 2048; q1 = q2 = 0).
opir_params derive_params_k1p(const opir_layout &layout);

// 64-bit limb tables: bit-reversed powers with Shoup companions
// floor(w 2^64 / q), N^-1 and iw[1] N^-1 with theirs.
struct LimbTables64 {
  uint64_t q = 0, n_inv = 0, n_inv_sh = 0, w1_ninv = 0, w1_ninv_sh = 0;
  std::vector<uint64_t> fw, fw_sh, iw, iw_sh;
};
LimbTables64 make_limb_tables64(uint32_t n, uint64_t q, uint64_t root);

}  // namespace opir
