// HEXL-API stand-in used ONLY to compile the unmodified OnionPIRv2 reference
// sources into the CPU oracle binary (oracle/_ref). Test infrastructure, not
// product code.
//
// Intel HEXL 1.2.6 (pinned by the reference's CMakeLists.txt:38) is not
// vendored in the reference and is not installed on this machine. The
// reference uses six HEXL entry points (utils.cpp:26-44,84-90, pir.cpp:32-33,
// rlwe.cpp, bv_keyswitch.cpp, gsw.cpp, server.cpp, client.cpp):
//   NTT(N, q) / NTT(N, q, root), NTT::ComputeForward / ComputeInverse,
//   EltwiseAddMod, EltwiseSubMod, EltwiseMultMod, EltwiseFMAMod,
//   MinimalPrimitiveRoot.
// Only the names and signatures follow HEXL. The bodies restate the published
// mathematics:
//   * element-wise modular add / sub / mult / fused-mult-add with canonical
//     outputs in [0, q) (inputs are canonical: every reference call site
//     passes input_mod_factor = 1);
//   * MinimalPrimitiveRoot(2N, q): the smallest primitive 2N-th root of unity
//     mod a prime q (found by taking any generator g of the 2N-th roots and
//     minimising over its odd powers g^(2i+1), i < N);
//   * the negacyclic NTT over Z_q[X]/(X^N+1) in the merged Cooley-Tukey form:
//     forward output in bit-reversed order, out[j] = a(psi^(2*brv(j)+1)),
//     inverse taking bit-reversed input (Gentleman-Sande) and scaling by N^-1.
//     This is the ordering HEXL documents for ComputeForward. Every reference
//     output that leaves the server (the coefficient-form response) is
//     independent of the NTT ordering, because clients sample every
//     polynomial in coefficient form.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <vector>

namespace intel {
namespace hexl {

namespace standin {

using u128 = unsigned __int128;

// floor(2^128 / q) split into two 64-bit words (q odd, q >= 3).
struct Barrett128 {
  uint64_t q, mu_lo, mu_hi;
  explicit Barrett128(uint64_t modulus) : q(modulus) {
    const u128 mu = (~static_cast<u128>(0)) / modulus;
    mu_lo = static_cast<uint64_t>(mu);
    mu_hi = static_cast<uint64_t>(mu >> 64);
  }
  // x mod q for any 128-bit x with the result needing one correction.
  inline uint64_t reduce(u128 x) const {
    const uint64_t x_lo = static_cast<uint64_t>(x);
    const uint64_t x_hi = static_cast<uint64_t>(x >> 64);
    const u128 t = static_cast<u128>(x_lo) * mu_lo;
    const u128 m1 = static_cast<u128>(x_lo) * mu_hi + (t >> 64);
    const u128 m2 = static_cast<u128>(x_hi) * mu_lo + static_cast<uint64_t>(m1);
    const uint64_t qhat = static_cast<uint64_t>(
        static_cast<u128>(x_hi) * mu_hi + (m1 >> 64) + (m2 >> 64));
    uint64_t r = x_lo - qhat * q;
    while (r >= q) r -= q;
    return r;
  }
  inline uint64_t mul(uint64_t a, uint64_t b) const {
    return reduce(static_cast<u128>(a) * b);
  }
};

inline uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t q) {
  u128 r = 1 % q, x = b % q;
  while (e) {
    if (e & 1) r = r * x % q;
    x = x * x % q;
    e >>= 1;
  }
  return static_cast<uint64_t>(r);
}

inline uint64_t inv_mod(uint64_t a, uint64_t q) {
  // extended Euclid over signed 128-bit values
  __int128 t = 0, nt = 1, r = q, nr = a % q;
  while (nr != 0) {
    const __int128 quo = r / nr;
    __int128 tmp = t - quo * nt; t = nt; nt = tmp;
    tmp = r - quo * nr; r = nr; nr = tmp;
  }
  if (r != 1) throw std::invalid_argument("hexl stand-in: value not invertible");
  if (t < 0) t += q;
  return static_cast<uint64_t>(t);
}

inline uint64_t bit_rev(uint64_t x, unsigned bits) {
  uint64_t y = 0;
  for (unsigned i = 0; i < bits; ++i) { y = (y << 1) | (x & 1); x >>= 1; }
  return y;
}

// Shoup companion floor(w * 2^64 / q) of a constant multiplier w < q.
inline uint64_t shoup(uint64_t w, uint64_t q) {
  return static_cast<uint64_t>((static_cast<u128>(w) << 64) / q);
}
// (x * w) mod q for x < 2^64 and w < q < 2^63.
inline uint64_t mul_shoup(uint64_t x, uint64_t w, uint64_t w_sh, uint64_t q) {
  const uint64_t qhat = static_cast<uint64_t>((static_cast<u128>(x) * w_sh) >> 64);
  uint64_t r = x * w - qhat * q;
  if (r >= q) r -= q;
  return r;
}

}  // namespace standin

inline uint64_t MinimalPrimitiveRoot(uint64_t degree, uint64_t modulus) {
  if (degree < 2 || (degree & (degree - 1)) != 0 || (modulus - 1) % degree != 0)
    throw std::invalid_argument("MinimalPrimitiveRoot: bad degree/modulus");
  // A generator of the degree-th roots: x^((q-1)/degree) with
  // g^(degree/2) == -1 (degree is a power of two).
  uint64_t g = 0;
  for (uint64_t x = 2; x < modulus; ++x) {
    const uint64_t c = standin::pow_mod(x, (modulus - 1) / degree, modulus);
    if (standin::pow_mod(c, degree / 2, modulus) == modulus - 1) { g = c; break; }
  }
  if (g == 0) throw std::runtime_error("MinimalPrimitiveRoot: none found");
  const standin::Barrett128 b(modulus);
  const uint64_t g2 = b.mul(g, g);
  uint64_t cur = g, best = g;
  for (uint64_t i = 0; i < degree / 2; ++i) {  // odd powers g^(2i+1)
    if (cur < best) best = cur;
    cur = b.mul(cur, g2);
  }
  return best;
}

inline void EltwiseAddMod(uint64_t *result, const uint64_t *a, const uint64_t *b,
                          uint64_t n, uint64_t q) {
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t s = a[i] + b[i];
    result[i] = s >= q ? s - q : s;
  }
}

inline void EltwiseAddMod(uint64_t *result, const uint64_t *a, uint64_t b,
                          uint64_t n, uint64_t q) {
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t s = a[i] + b;
    result[i] = s >= q ? s - q : s;
  }
}

inline void EltwiseSubMod(uint64_t *result, const uint64_t *a, const uint64_t *b,
                          uint64_t n, uint64_t q) {
  for (uint64_t i = 0; i < n; ++i)
    result[i] = a[i] >= b[i] ? a[i] - b[i] : a[i] + q - b[i];
}

inline void EltwiseMultMod(uint64_t *result, const uint64_t *a, const uint64_t *b,
                           uint64_t n, uint64_t q, uint64_t input_mod_factor) {
  const standin::Barrett128 bar(q);
  if (input_mod_factor == 1) {
    for (uint64_t i = 0; i < n; ++i) result[i] = bar.mul(a[i], b[i]);
  } else {
    for (uint64_t i = 0; i < n; ++i) result[i] = bar.mul(a[i] % q, b[i] % q);
  }
}

// result = (a * scalar + c) mod q; c may be nullptr.
inline void EltwiseFMAMod(uint64_t *result, const uint64_t *a, uint64_t scalar,
                          const uint64_t *c, uint64_t n, uint64_t q,
                          uint64_t input_mod_factor) {
  const standin::Barrett128 bar(q);
  const uint64_t s = scalar % q;
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t ai = input_mod_factor == 1 ? a[i] : a[i] % q;
    uint64_t v = bar.mul(ai, s);
    if (c != nullptr) {
      const uint64_t ci = input_mod_factor == 1 ? c[i] : c[i] % q;
      v += ci;
      if (v >= q) v -= q;
    }
    result[i] = v;
  }
}

class NTT {
 public:
  NTT() = default;
  NTT(uint64_t degree, uint64_t q)
      : NTT(degree, q, MinimalPrimitiveRoot(2 * degree, q)) {}
  NTT(uint64_t degree, uint64_t q, uint64_t root_of_unity)
      : n_(degree), q_(q), root_(root_of_unity) {
    if (degree < 2 || (degree & (degree - 1)) != 0)
      throw std::invalid_argument("NTT: degree must be a power of two");
    if (standin::pow_mod(root_of_unity, degree, q) != q - 1)
      throw std::invalid_argument("NTT: root is not a primitive 2N-th root");
    unsigned lg = 0;
    while ((uint64_t{1} << lg) < degree) ++lg;
    const standin::Barrett128 bar(q);
    const uint64_t root_inv = standin::inv_mod(root_of_unity, q);
    std::vector<uint64_t> pw(degree), ipw(degree);
    pw[0] = 1; ipw[0] = 1;
    for (uint64_t i = 1; i < degree; ++i) {
      pw[i] = bar.mul(pw[i - 1], root_of_unity);
      ipw[i] = bar.mul(ipw[i - 1], root_inv);
    }
    fw_.resize(degree); fw_sh_.resize(degree);
    iw_.resize(degree); iw_sh_.resize(degree);
    for (uint64_t k = 0; k < degree; ++k) {
      const uint64_t e = standin::bit_rev(k, lg);
      fw_[k] = pw[e]; fw_sh_[k] = standin::shoup(fw_[k], q);
      iw_[k] = ipw[e]; iw_sh_[k] = standin::shoup(iw_[k], q);
    }
    n_inv_ = standin::inv_mod(degree % q, q);
    n_inv_sh_ = standin::shoup(n_inv_, q);
  }

  uint64_t GetDegree() const { return n_; }
  uint64_t GetModulus() const { return q_; }
  uint64_t GetMinimalRootOfUnity() const { return root_; }

  void ComputeForward(uint64_t *result, const uint64_t *operand,
                      uint64_t input_mod_factor, uint64_t /*output_mod_factor*/) {
    const uint64_t q = q_;
    if (result != operand)
      for (uint64_t i = 0; i < n_; ++i) result[i] = operand[i];
    if (input_mod_factor != 1)
      for (uint64_t i = 0; i < n_; ++i) result[i] %= q;
    uint64_t t = n_;
    for (uint64_t m = 1; m < n_; m <<= 1) {
      t >>= 1;
      for (uint64_t i = 0; i < m; ++i) {
        const uint64_t w = fw_[m + i], wsh = fw_sh_[m + i];
        uint64_t *x = result + 2 * i * t;
        uint64_t *y = x + t;
        for (uint64_t j = 0; j < t; ++j) {
          const uint64_t u = x[j];
          const uint64_t v = standin::mul_shoup(y[j], w, wsh, q);
          const uint64_t s = u + v;
          x[j] = s >= q ? s - q : s;
          y[j] = u >= v ? u - v : u + q - v;
        }
      }
    }
  }

  void ComputeInverse(uint64_t *result, const uint64_t *operand,
                      uint64_t input_mod_factor, uint64_t /*output_mod_factor*/) {
    const uint64_t q = q_;
    if (result != operand)
      for (uint64_t i = 0; i < n_; ++i) result[i] = operand[i];
    if (input_mod_factor != 1)
      for (uint64_t i = 0; i < n_; ++i) result[i] %= q;
    uint64_t t = 1;
    for (uint64_t m = n_ >> 1; m >= 1; m >>= 1) {
      for (uint64_t i = 0; i < m; ++i) {
        const uint64_t w = iw_[m + i], wsh = iw_sh_[m + i];
        uint64_t *x = result + 2 * i * t;
        uint64_t *y = x + t;
        for (uint64_t j = 0; j < t; ++j) {
          const uint64_t u = x[j], v = y[j];
          const uint64_t s = u + v;
          x[j] = s >= q ? s - q : s;
          y[j] = standin::mul_shoup(u >= v ? u - v : u + q - v, w, wsh, q);
        }
      }
      t <<= 1;
    }
    for (uint64_t i = 0; i < n_; ++i)
      result[i] = standin::mul_shoup(result[i], n_inv_, n_inv_sh_, q);
  }

 private:
  uint64_t n_ = 0, q_ = 0, root_ = 0, n_inv_ = 0, n_inv_sh_ = 0;
  std::vector<uint64_t> fw_, fw_sh_, iw_, iw_sh_;
};

}  // namespace hexl
}  // namespace intel
