// Host-side tree PIR layer (the reference's src/tree_index.cpp,
// src/tree_query.cpp and src/tree_select.cpp index math): tree parameters,
// level plans, the query-shape view, and the arrangement of one level's
// packed plaintexts as the matrix the GPU select contracts.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/onionpir_b200.h"

namespace opir {

// make_tree_pir_params (src/tree_index.cpp:47-92) + validate_tree_params
// (:93-150); throws std::invalid_argument on any violated constraint.
opir_tree_params make_tree_params(uint64_t L, uint64_t a, uint64_t n, uint64_t ell_beta,
                                  uint64_t ell_gamma, uint64_t t,
                                  const std::vector<uint64_t> &rns_moduli);
void validate_tree_params(const opir_tree_params &p, const std::vector<uint64_t> &rns_moduli);

// make_tree_pir_params_for_scheme (src/tree_query.cpp:42-62).
opir_tree_params tree_params_for_scheme(uint64_t L, uint64_t a, const opir_params &scheme);

// RNS moduli of a scheme as the reference reports them (get_rns_mods): the
// logical q for the single-modulus set, the two limbs for the two-limb one.
std::vector<uint64_t> scheme_moduli(const opir_params &scheme);

// build_level_plans (src/tree_index.cpp:177-225).
std::vector<opir_tree_level_plan> level_plans(const opir_tree_params &p);

// PirParams::with_query_shape (src/pir.cpp:136-166).
opir_params with_query_shape(const opir_params &scheme, const opir_query_shape &shape);

// The contraction that select_level (src/tree_select.cpp:203-238) performs
// on one level: candidate row m = sum over the N0 alpha ciphertexts k of
// M[m][k] * alpha_k, then `fold` MSB-first ext_prod_mux steps over the rows.
//   AlphaBeta       : rows 2^d, M[delta][k] = D[k 2^d + delta] (the sec. 6.2
//                     matrix view of evaluate_alpha_dimension, :146-173)
//   CoarsenedAlpha  : one row, M[0][k] = D[k >> c] (pyramid level c sums the
//                     alpha ciphertexts of each block of 2^c, :122-144)
//   Single          : one row, M[0][k] = D[0] (the pyramid apex sums all)
// `plaintexts` is the level in pack_tree_level order (R x n); the result is
// rows x N0 plaintexts (row-major, n coefficients each).
struct LevelMatrix {
  uint64_t rows = 0, cols = 0, fold = 0;
  std::vector<uint64_t> coeffs;
};
LevelMatrix arrange_level(const opir_tree_params &p, const opir_tree_level_plan &plan,
                          const uint64_t *plaintexts);

}  // namespace opir
