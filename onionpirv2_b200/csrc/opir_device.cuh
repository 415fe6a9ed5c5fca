// Device-side arithmetic for the OnionPIRv2 server path on sm_100a.
//
// Representation. The reference computes modulo the logical composite
// q = q1*q2 (~2^58) with a CRT-combined NTT root (src/pir.cpp:14-47,
// src/utils.cpp:26-56). Z_q is isomorphic to Z_q1 x Z_q2, and the composite
// negacyclic NTT with root w_crt is the CRT of the NTTs mod q1 (root w1) and
// mod q2 (root w2). So every polynomial lives on the device as two 29-bit
// residue planes ("residue pair") and all ring arithmetic runs in 32-bit
// integer lanes. Only the operations that need the canonical integer in
// [0, q) -- signed gadget decomposition (src/gsw.cpp:252-295,
// src/bv_keyswitch.cpp:20-40) and the final rescale (src/utils.cpp:445-462)
// -- Garner-compose the pair back into a u64. Results are therefore the
// reference's values exactly.
//
// Ciphertext layout: [poly p in {c0,c1}][residue r in {q1,q2}][N] u32.
#pragma once

#include <cstdint>

namespace opir {

constexpr int kN = 2048;        // CONFIG_N2048_K1_COMP PolyDegree
constexpr int kLogN = 11;
constexpr int kThreads = 256;   // every polynomial kernel: 256 threads
constexpr int kPer = kN / kThreads;  // coefficient positions per thread (8)
constexpr int kCtWords = 4 * kN;     // u32 words per ciphertext residue pair

struct ResidueTables {
  const uint32_t *fw, *fw_sh;   // psi^brv(k), Shoup companions (forward)
  const uint32_t *iw, *iw_sh;   // psi^-brv(k), Shoup companions (inverse)
  uint32_t q;
  uint32_t n_inv, n_inv_sh;
  uint32_t pad;
  uint64_t mu;                  // floor(2^64 / q), for 64-bit Barrett
};

struct DevParams {
  ResidueTables r[2];
  uint64_t q;                   // q1 * q2
  uint64_t half_q;              // q >> 1
  uint32_t q1, q2;
  uint32_t q1_inv, q1_inv_sh;   // q1^-1 mod q2 and its Shoup companion
  uint64_t small_q;
  uint32_t small_q_width;
  uint32_t pad;
};

// ---------------------------------------------------------------- modular ops
__device__ __forceinline__ uint32_t mul_shoup_lazy(uint32_t a, uint32_t w,
                                                   uint32_t w_sh, uint32_t q) {
  // a * w mod q in [0, 2q) for any 32-bit a (Shoup, w_sh = floor(w 2^32 / q)).
  const uint32_t qhat = __umulhi(a, w_sh);
  return a * w - qhat * q;
}
__device__ __forceinline__ uint32_t red2q(uint32_t x, uint32_t q) {
  return x >= q ? x - q : x;
}
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t q) {
  const uint32_t s = a + b;
  return s >= q ? s - q : s;
}
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t q) {
  return a >= b ? a - b : a + q - b;
}
__device__ __forceinline__ uint32_t neg_mod(uint32_t a, uint32_t q) {
  return a ? q - a : 0u;
}
// x mod q for any 64-bit x (Barrett with mu = floor(2^64/q); error < 3q).
__device__ __forceinline__ uint32_t reduce64(uint64_t x, uint32_t q, uint64_t mu) {
  const uint64_t qhat = __umul64hi(x, mu);
  uint64_t r = x - qhat * q;
  if (r >= q) r -= q;
  if (r >= q) r -= q;
  return static_cast<uint32_t>(r);
}

// Garner CRT compose of a residue pair into the canonical value in [0, q)
// (the compose of src/server.cpp:548-553).
__device__ __forceinline__ uint64_t crt_compose(uint32_t r1, uint32_t r2,
                                                const DevParams &P) {
  const uint32_t r1m = r1 >= P.q2 ? r1 - P.q2 : r1;  // q1 < 2 q2
  const uint32_t diff = sub_mod(r2, r1m, P.q2);
  const uint32_t k = red2q(mul_shoup_lazy(diff, P.q1_inv, P.q1_inv_sh, P.q2), P.q2);
  return static_cast<uint64_t>(r1) + static_cast<uint64_t>(P.q1) * k;
}
// Centre [0, q) -> (-q/2, q/2] (src/gsw.cpp:277-281, bv_keyswitch.cpp:25-28).
__device__ __forceinline__ int64_t centre(uint64_t v, const DevParams &P) {
  return v > P.half_q ? static_cast<int64_t>(v) - static_cast<int64_t>(P.q)
                      : static_cast<int64_t>(v);
}
// Next balanced digit in [-B/2, B/2), LSB first (src/gsw.cpp:288-289).
__device__ __forceinline__ int32_t next_digit(int64_t &d, int base_log2) {
  const int sh = 64 - base_log2;
  const int64_t r = static_cast<int64_t>(static_cast<uint64_t>(d) << sh) >> sh;
  d = (d - r) >> base_log2;
  return static_cast<int32_t>(r);
}
__device__ __forceinline__ uint32_t digit_residue(int32_t r, uint32_t q) {
  return r >= 0 ? static_cast<uint32_t>(r) : static_cast<uint32_t>(r + static_cast<int32_t>(q));
}

// ------------------------------------------------------------------- NTT
// Block-cooperative negacyclic NTT over `np` planes of kN u32 in shared
// memory (plane stride kN). Forward: merged Cooley-Tukey, natural-order input,
// bit-reversed output, out[j] = a(psi^(2 brv(j) + 1)). Inverse:
// Gentleman-Sande from bit-reversed input, scaled by N^-1. Harvey lazy
// butterflies keep values in [0, 4q) (q < 2^29 so 4q < 2^31); outputs are
// canonical. Callers synchronise before the call; the call ends synchronised.
__device__ __forceinline__ void ntt_fwd_planes(uint32_t *sm, int np,
                                               const ResidueTables &T) {
  const uint32_t q = T.q, two_q = 2 * q;
  const int total = np * (kN / 2);
#pragma unroll 1
  for (int lt = kLogN - 1, m = 1; lt >= 0; --lt, m <<= 1) {
    const int t = 1 << lt;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int plane = idx >> (kLogN - 1);
      const int b = idx & (kN / 2 - 1);
      const int i = b >> lt;
      const int x = (i << (lt + 1)) + (b & (t - 1));
      uint32_t *P = sm + plane * kN;
      const uint32_t w = __ldg(T.fw + m + i), ws = __ldg(T.fw_sh + m + i);
      uint32_t X = P[x];
      const uint32_t Y = P[x + t];
      X = X >= two_q ? X - two_q : X;
      const uint32_t V = mul_shoup_lazy(Y, w, ws, q);
      P[x] = X + V;
      P[x + t] = X - V + two_q;
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < np * kN; idx += blockDim.x) {
    uint32_t v = sm[idx];
    v = v >= two_q ? v - two_q : v;
    sm[idx] = v >= q ? v - q : v;
  }
  __syncthreads();
}

__device__ __forceinline__ void ntt_inv_planes(uint32_t *sm, int np,
                                               const ResidueTables &T) {
  const uint32_t q = T.q, two_q = 2 * q;
  const int total = np * (kN / 2);
#pragma unroll 1
  for (int lt = 0, m = kN / 2; lt < kLogN; ++lt, m >>= 1) {
    const int t = 1 << lt;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int plane = idx >> (kLogN - 1);
      const int b = idx & (kN / 2 - 1);
      const int i = b >> lt;
      const int x = (i << (lt + 1)) + (b & (t - 1));
      uint32_t *P = sm + plane * kN;
      const uint32_t w = __ldg(T.iw + m + i), ws = __ldg(T.iw_sh + m + i);
      const uint32_t X = P[x], Y = P[x + t];
      uint32_t U = X + Y;
      U = U >= two_q ? U - two_q : U;
      P[x] = U;
      P[x + t] = mul_shoup_lazy(X - Y + two_q, w, ws, q);
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < np * kN; idx += blockDim.x) {
    const uint32_t v = mul_shoup_lazy(sm[idx], T.n_inv, T.n_inv_sh, q);
    sm[idx] = v >= q ? v - q : v;
  }
  __syncthreads();
}

}  // namespace opir
