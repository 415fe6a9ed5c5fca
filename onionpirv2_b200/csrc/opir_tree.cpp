// Tree PIR index math: restated from the reference's src/tree_index.cpp,
// src/tree_query.cpp and src/pir.cpp (with_query_shape), plus the level
// matrix the GPU select contracts (opir_tree.h).
#include "opir_tree.h"

#include <algorithm>
#include <limits>
#include <stdexcept>
#include <string>

namespace opir {

namespace {

void require(bool ok, const char *msg) {
  if (!ok) throw std::invalid_argument(std::string("TreePirParams: ") + msg);
}

bool is_pow2(uint64_t v) { return v != 0 && (v & (v - 1)) == 0; }

uint64_t log2_exact(uint64_t v, const char *name) {
  if (!is_pow2(v)) throw std::invalid_argument(std::string("TreePirParams: ") + name +
                                               " must be a power of two");
  uint64_t l = 0;
  while ((1ull << l) < v) ++l;
  return l;
}

uint64_t bit_ceil(uint64_t v) {
  uint64_t c = 1;
  while (c < v) c <<= 1;
  return c;
}

uint64_t gcd(uint64_t a, uint64_t b) {
  while (b) { const uint64_t t = a % b; a = b; b = t; }
  return a;
}

// Overflow-checked N0 + ell_beta b + ell_gamma r (src/tree_index.cpp:26-44).
uint64_t packed_width(uint64_t N0, uint64_t ell_beta, uint64_t b, uint64_t ell_gamma, uint64_t r) {
  const uint64_t M = std::numeric_limits<uint64_t>::max();
  auto mul = [&](uint64_t x, uint64_t y) {
    if (x != 0 && y > M / x) throw std::invalid_argument("TreePirParams: packed width overflows");
    return x * y;
  };
  auto add = [&](uint64_t x, uint64_t y) {
    if (y > M - x) throw std::invalid_argument("TreePirParams: packed width overflows");
    return x + y;
  };
  return add(N0, add(mul(ell_beta, b), mul(ell_gamma, r)));
}

}  // namespace

void validate_tree_params(const opir_tree_params &p, const std::vector<uint64_t> &rns_moduli) {
  require(p.L > 0 && p.L < 63, "tree height is out of range");
  require(p.a < 63, "first-dimension width is out of range");
  require(is_pow2(p.N), "N must be a power of two");
  require(is_pow2(p.n), "n must be a power of two");
  require(is_pow2(p.N0), "N0 must be a power of two");
  require(p.N == 1ull << p.L, "N must equal 2^L");
  require(p.N0 == 1ull << p.a, "N0 must equal 2^a");
  require(p.g == 1, "the MVP supports only g = 1");
  require(p.rho == p.n / p.g, "rho must equal n / g");
  require(p.r == log2_exact(p.rho, "rho"), "r must equal log2(rho)");
  require(p.n <= p.N, "rho = n must fit below the leaf count");
  require(p.N0 >= 2, "N0 must be at least 2");
  require(p.N0 <= p.N / p.n, "N0 exceeds N / n");
  require(p.N % (p.n * p.N0) == 0, "N must be divisible by n * N0");
  require(p.L >= p.r + p.a, "L is below r + a");
  require(p.b == p.L - p.r - p.a, "b must be L - r - a");
  require(p.P == p.N / p.rho, "P must equal N / rho");
  require(p.B == 1ull << p.b, "B must equal 2^b");
  require(p.ell_beta > 0 && p.ell_gamma > 0, "gadget lengths must be positive");
  require(p.w == packed_width(p.N0, p.ell_beta, p.b, p.ell_gamma, p.r),
          "w must equal N0 + ell_beta*b + ell_gamma*r");
  require(p.w <= p.n, "packed width exceeds the ring degree");
  require(p.W == bit_ceil(p.w), "W must be the next power of two of w");
  require(p.W == 1ull << p.h_q, "h_q must equal log2(W)");
  require(p.W <= p.n, "W exceeds the ring degree");
  require(gcd(p.W, p.t) == 1, "W must be invertible modulo t");
  for (uint64_t q : rns_moduli) {
    require((q & 1) == 1, "every RNS modulus must be odd");
    require(gcd(p.W, q) == 1, "W must be invertible modulo every RNS modulus");
  }
}

opir_tree_params make_tree_params(uint64_t L, uint64_t a, uint64_t n, uint64_t ell_beta,
                                  uint64_t ell_gamma, uint64_t t,
                                  const std::vector<uint64_t> &rns_moduli) {
  require(L > 0 && L < 63, "tree height is out of range");
  require(a < 63, "first-dimension width is out of range");
  require(n > 0, "ring degree must be positive");
  require(ell_beta > 0 && ell_gamma > 0, "gadget lengths must be positive");
  opir_tree_params p{};
  p.L = L;
  p.N = 1ull << L;
  p.n = n;
  p.g = 1;
  p.rho = n;
  p.r = log2_exact(n, "ring degree");
  p.a = a;
  p.N0 = 1ull << a;
  require(p.L >= p.r + p.a, "tree height is below r + a; no beta bits remain");
  p.b = p.L - p.r - p.a;
  p.P = p.N / p.rho;
  p.B = 1ull << p.b;
  p.ell_beta = ell_beta;
  p.ell_gamma = ell_gamma;
  p.w = packed_width(p.N0, ell_beta, p.b, ell_gamma, p.r);
  require(p.w <= p.n, "packed width exceeds the ring degree");
  p.W = bit_ceil(p.w);
  p.h_q = log2_exact(p.W, "W");
  p.t = t;
  validate_tree_params(p, rns_moduli);
  return p;
}

std::vector<uint64_t> scheme_moduli(const opir_params &scheme) {
  if (scheme.num_limbs == 2) return {scheme.q1, scheme.q2};
  return {scheme.q};
}

opir_tree_params tree_params_for_scheme(uint64_t L, uint64_t a, const opir_params &scheme) {
  const opir_tree_params p = make_tree_params(L, a, scheme.poly_degree, scheme.l_ep, scheme.l_ep,
                                              scheme.plain_mod, scheme_moduli(scheme));
  if (p.h_q > scheme.expansion_height)
    throw std::invalid_argument(
        "tree query expansion height exceeds the scheme's session-key coverage");
  return p;
}

std::vector<opir_tree_level_plan> level_plans(const opir_tree_params &p) {
  std::vector<opir_tree_level_plan> plans;
  for (uint64_t level = 0; level <= p.L; ++level) {
    opir_tree_level_plan pl{};
    pl.level = level;
    pl.R = level >= p.r ? 1ull << (level - p.r) : 1;
    if (pl.R == 1) {
      pl.select_case = OPIR_TREE_SINGLE;
      pl.coarsen_count = p.a;
    } else if (pl.R < p.N0) {
      pl.select_case = OPIR_TREE_COARSENED_ALPHA;
      pl.coarsen_count = p.a - (level - p.r);
    } else {
      pl.select_case = OPIR_TREE_ALPHA_BETA;
      pl.coarsen_count = 0;
    }
    if (pl.select_case == OPIR_TREE_ALPHA_BETA) {
      pl.beta_begin = p.L - level;
      pl.beta_count = level - p.r - p.a;
    } else {
      pl.beta_begin = p.b;
      pl.beta_count = 0;
    }
    if (level >= p.r) {
      pl.gamma_begin = 0;
      pl.gamma_count = p.r;
    } else {
      pl.gamma_begin = p.r - level;
      pl.gamma_count = level;
    }
    pl.projection_depth = level < p.r ? level : p.r;
    plans.push_back(pl);
  }
  return plans;
}

opir_params with_query_shape(const opir_params &scheme, const opir_query_shape &shape) {
  uint32_t max_h = 0;
  while ((1u << (max_h + 1)) <= scheme.poly_degree) ++max_h;
  if (shape.expansion_height > max_h)
    throw std::invalid_argument("PirParams: query shape exceeds the ring automorphism capacity");
  if (shape.fst_dim_sz == 0)
    throw std::invalid_argument("PirParams: query shape needs a positive first dimension");
  const uint64_t capacity = 1ull << shape.expansion_height;
  if (shape.fst_dim_sz > capacity ||
      shape.num_selector_bits > (capacity - shape.fst_dim_sz) / scheme.l_ep)
    throw std::invalid_argument("PirParams: query shape does not fit the expansion capacity");
  opir_params r = scheme;
  r.fst_dim_sz = shape.fst_dim_sz;
  r.num_dims = 1 + shape.num_selector_bits;
  r.expansion_height = shape.expansion_height;
  r.num_pt = shape.fst_dim_sz;
  r.target_num_pt = shape.fst_dim_sz;
  r.other_dim_sz = 1;
  r.view = OPIR_VIEW_QUERY_SHAPE;
  return r;
}

LevelMatrix arrange_level(const opir_tree_params &p, const opir_tree_level_plan &plan,
                          const uint64_t *plaintexts) {
  const uint64_t n = p.n, N0 = p.N0;
  LevelMatrix m;
  m.cols = N0;
  if (plan.select_case == OPIR_TREE_ALPHA_BETA) {
    m.rows = 1ull << plan.beta_count;
    m.fold = plan.beta_count;
    if (plan.R != N0 * m.rows) throw std::invalid_argument("tree_select: AlphaBeta level has R = N0 * 2^d");
  } else {
    m.rows = 1;
    m.fold = 0;
  }
  m.coeffs.resize(m.rows * m.cols * n);
  for (uint64_t row = 0; row < m.rows; ++row)
    for (uint64_t k = 0; k < N0; ++k) {
      uint64_t src;
      if (plan.select_case == OPIR_TREE_ALPHA_BETA) src = k * m.rows + row;
      else if (plan.select_case == OPIR_TREE_COARSENED_ALPHA) src = k >> plan.coarsen_count;
      else src = 0;
      if (src >= plan.R) throw std::invalid_argument("tree_select: level plaintext index out of range");
      const uint64_t *from = plaintexts + src * n;
      std::copy(from, from + n, m.coeffs.begin() + (row * m.cols + k) * n);
    }
  return m;
}

}  // namespace opir
