// C ABI of the wire codec (opir_codec.h): seed-compressed queries and client
// keys in the layouts of include/onionpir_b200.h.
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/onionpir_b200.h"
#include "opir_codec.h"
#include "opir_tree.h"

namespace {

using opir::codec::expand_uniform;
using opir::codec::pack_bits;
using opir::codec::unpack_bits;
using opir::codec::width_of;

const uint8_t kQueryMagic[4] = {'O', 'P', 'Q', '1'};
const uint8_t kKeysMagic[4] = {'O', 'P', 'K', '1'};

template <typename F>
opir_status run(F &&f) {
  try {
    f();
    return OPIR_OK;
  } catch (const std::invalid_argument &) {
    return OPIR_ERR_INVALID_ARGUMENT;
  } catch (const std::out_of_range &) {
    return OPIR_ERR_OUT_OF_RANGE;
  } catch (const std::bad_alloc &) {
    return OPIR_ERR_NO_MEMORY;
  } catch (...) {
    return OPIR_ERR_RUNTIME;
  }
}

struct Shape {
  std::vector<uint64_t> mods;
  uint32_t n = 0;
  size_t poly_bytes = 0;  // one packed K-limb polynomial
  size_t kn() const { return mods.size() * n; }
};

Shape shape_of(const opir_params &p) {
  if (p.poly_degree == 0 || (p.num_limbs != 1 && p.num_limbs != 2))
    throw std::invalid_argument("codec: unsupported parameter set");
  Shape s;
  s.mods = opir::scheme_moduli(p);
  s.n = p.poly_degree;
  for (uint64_t q : s.mods) s.poly_bytes += (static_cast<size_t>(s.n) * width_of(q) + 7) / 8;
  return s;
}

void check_reduced(const Shape &s, const uint64_t *poly, const char *what) {
  for (size_t k = 0; k < s.mods.size(); ++k)
    for (uint32_t j = 0; j < s.n; ++j)
      if (poly[k * s.n + j] >= s.mods[k])
        throw std::invalid_argument(std::string("codec: ") + what + " not reduced mod its limb");
}

uint8_t *pack_poly(const Shape &s, const uint64_t *poly, uint8_t *out) {
  for (size_t k = 0; k < s.mods.size(); ++k)
    out += pack_bits(poly + k * s.n, s.n, width_of(s.mods[k]), out);
  return out;
}

const uint8_t *unpack_poly(const Shape &s, const uint8_t *in, uint64_t *poly) {
  for (size_t k = 0; k < s.mods.size(); ++k) {
    const uint32_t w = width_of(s.mods[k]);
    unpack_bits(in, s.n, w, poly + k * s.n);
    in += (static_cast<size_t>(s.n) * w + 7) / 8;
  }
  check_reduced(s, poly, "decoded coefficient");
  return in;
}

// The uniform polynomial must be Expand(seed, domain, index).
void require_expanded(const Shape &s, const uint8_t *seed, uint32_t domain, uint64_t index,
                      const uint64_t *poly, const char *what) {
  std::vector<uint64_t> e(s.kn());
  expand_uniform(seed, domain, index, s.mods, s.n, e.data());
  if (std::memcmp(e.data(), poly, e.size() * 8) != 0)
    throw std::invalid_argument(std::string("codec: ") + what + " is not Expand(seed)");
}

size_t keys_bytes(const opir_params &p, const Shape &s) {
  const size_t rows = static_cast<size_t>(p.expansion_height) * p.l_ks + 2ull * p.l_key;
  return 4 + OPIR_SEED_BYTES + rows * s.poly_bytes;
}

}  // namespace

extern "C" {

opir_status opir_prf_expand(const opir_params *params, const uint8_t *seed, uint32_t domain,
                            uint64_t index, uint64_t *out) {
  if (!params || !seed || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return run([&] {
    const Shape s = shape_of(*params);
    expand_uniform(seed, domain, index, s.mods, s.n, out);
  });
}

size_t opir_query_wire_bytes(const opir_params *params) {
  if (!params) return 0;
  try {
    return 4 + OPIR_SEED_BYTES + shape_of(*params).poly_bytes;
  } catch (...) {
    return 0;
  }
}

size_t opir_keys_wire_bytes(const opir_params *params) {
  if (!params) return 0;
  try {
    return keys_bytes(*params, shape_of(*params));
  } catch (...) {
    return 0;
  }
}

opir_status opir_query_encode(const opir_params *params, const uint8_t *seed,
                              const uint64_t *query, uint8_t *out, size_t cap) {
  if (!params || !seed || !query || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return run([&] {
    const Shape s = shape_of(*params);
    if (cap < 4 + OPIR_SEED_BYTES + s.poly_bytes) throw std::invalid_argument("codec: buffer too small");
    check_reduced(s, query, "query c0");
    check_reduced(s, query + s.kn(), "query c1");
    require_expanded(s, seed, OPIR_PRF_QUERY, 0, query + s.kn(), "query c1");
    std::memcpy(out, kQueryMagic, 4);
    std::memcpy(out + 4, seed, OPIR_SEED_BYTES);
    pack_poly(s, query, out + 4 + OPIR_SEED_BYTES);
  });
}

opir_status opir_query_decode(const opir_params *params, const uint8_t *in, size_t len,
                              uint64_t *query) {
  if (!params || !in || !query) return OPIR_ERR_INVALID_ARGUMENT;
  return run([&] {
    const Shape s = shape_of(*params);
    if (len != 4 + OPIR_SEED_BYTES + s.poly_bytes || std::memcmp(in, kQueryMagic, 4) != 0)
      throw std::invalid_argument("codec: not a query of this parameter set");
    const uint8_t *seed = in + 4;
    unpack_poly(s, in + 4 + OPIR_SEED_BYTES, query);
    expand_uniform(seed, OPIR_PRF_QUERY, 0, s.mods, s.n, query + s.kn());
  });
}

opir_status opir_keys_encode(const opir_params *params, const uint8_t *seed,
                             const uint64_t *bv_keys, const uint64_t *gsw_key, uint8_t *out,
                             size_t cap) {
  if (!params || !seed || !gsw_key || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return run([&] {
    const opir_params &p = *params;
    const Shape s = shape_of(p);
    if (cap < keys_bytes(p, s)) throw std::invalid_argument("codec: buffer too small");
    const size_t rows_bv = static_cast<size_t>(p.expansion_height) * p.l_ks;
    if (rows_bv && !bv_keys) throw std::invalid_argument("codec: null BV keys");
    std::memcpy(out, kKeysMagic, 4);
    std::memcpy(out + 4, seed, OPIR_SEED_BYTES);
    uint8_t *o = out + 4 + OPIR_SEED_BYTES;
    for (size_t r = 0; r < rows_bv; ++r) {  // BvRlweCt row: [b][a]
      const uint64_t *b = bv_keys + r * 2 * s.kn(), *a = b + s.kn();
      check_reduced(s, b, "BV key b");
      require_expanded(s, seed, OPIR_PRF_BV_KEY, r, a, "BV key a");
      o = pack_poly(s, b, o);
    }
    for (size_t r = 0; r < 2ull * p.l_key; ++r) {  // RGSW row: [c0][c1]
      const uint64_t *c0 = gsw_key + r * 2 * s.kn(), *c1 = c0 + s.kn();
      check_reduced(s, c0, "RGSW c0");
      require_expanded(s, seed, OPIR_PRF_GSW_KEY, r, c1, "RGSW c1");
      o = pack_poly(s, c0, o);
    }
  });
}

opir_status opir_keys_decode(const opir_params *params, const uint8_t *in, size_t len,
                             uint64_t *bv_keys, uint32_t *galois_ks, uint64_t *gsw_key) {
  if (!params || !in || !gsw_key) return OPIR_ERR_INVALID_ARGUMENT;
  return run([&] {
    const opir_params &p = *params;
    const Shape s = shape_of(p);
    if (len != keys_bytes(p, s) || std::memcmp(in, kKeysMagic, 4) != 0)
      throw std::invalid_argument("codec: not a key bundle of this parameter set");
    const size_t rows_bv = static_cast<size_t>(p.expansion_height) * p.l_ks;
    if (rows_bv && (!bv_keys || !galois_ks)) throw std::invalid_argument("codec: null BV keys");
    const uint8_t *seed = in + 4;
    const uint8_t *i = in + 4 + OPIR_SEED_BYTES;
    for (size_t r = 0; r < rows_bv; ++r) {
      uint64_t *b = bv_keys + r * 2 * s.kn();
      i = unpack_poly(s, i, b);
      expand_uniform(seed, OPIR_PRF_BV_KEY, r, s.mods, s.n, b + s.kn());
    }
    for (uint32_t d = 0; d < p.expansion_height; ++d) galois_ks[d] = p.poly_degree / (1u << d) + 1;
    for (size_t r = 0; r < 2ull * p.l_key; ++r) {
      uint64_t *c0 = gsw_key + r * 2 * s.kn();
      i = unpack_poly(s, i, c0);
      expand_uniform(seed, OPIR_PRF_GSW_KEY, r, s.mods, s.n, c0 + s.kn());
    }
  });
}

}  // extern "C"
