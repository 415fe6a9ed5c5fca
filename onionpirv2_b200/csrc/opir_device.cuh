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
  const uint2 *fwt, *iwt;       // the same, interleaved (w, w_sh) pairs
  const uint2 *pwt;             // (psi^m, Shoup companion) for m < 2N
  uint32_t q;
  uint32_t n_inv, n_inv_sh;
  uint32_t w1_ninv, w1_ninv_sh; // iw[1] * N^-1 (last inverse stage)
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
  // ciphertext limbs at the boundary: 0 or 1 = one u64 per coefficient mod
  // q1 q2 (CONFIG_N2048_K1_COMP); 2 = two RNS limbs q1, q2, limb-major, one
  // u64 per limb (CONFIG_N2048_K2_MP, the same residue pair on the device)
  uint32_t limbs;
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

// ------------------------------------------------- register-resident NTT
// The radix-8/8/8/4 form used by the query-path kernels. A block of 256
// threads transforms a 2048-coefficient plane with each thread holding eight
// values in registers; the eleven butterfly stages run as four passes
// (3 + 3 + 3 + 2 stages) with three exchanges through a shared-memory plane
// padded by one word per 32 (conflict-free for every pass). Positions held
// by thread t in each pass:
//   A: t + 256 k                       (stages t = 1024, 512, 256)
//   B: (t >> 5) 256 + (t & 31) + 32 k  (128, 64, 32)
//   C: (t & 63) 32 + (t >> 6) + 4 k    (16, 8, 4)
//   D: 4 (t + 256 (k >> 2)) + (k & 3)  (2, 1)
// The forward transform enters in A-order (natural coefficient positions)
// and leaves in D-order; the inverse enters in D-order and leaves in A-order.
// Same convention and twiddle indexing as ntt_fwd_planes / ntt_inv_planes.
constexpr int kPad = kN + kN / 32;  // padded plane stride in words
__device__ __forceinline__ int padi(int p) { return p + (p >> 5); }
__device__ __forceinline__ int posA(int t, int k) { return t + 256 * k; }
__device__ __forceinline__ int posB(int t, int k) { return ((t >> 5) << 8) + (t & 31) + 32 * k; }
__device__ __forceinline__ int posC(int t, int k) { return ((t & 63) << 5) + (t >> 6) + 4 * k; }
__device__ __forceinline__ int posD(int t, int k) { return ((t + ((k >> 2) << 8)) << 2) + (k & 3); }

__device__ __forceinline__ void bf_f(uint32_t &X, uint32_t &Y, uint2 w, uint32_t q, uint32_t q2) {
  const uint32_t x = X >= q2 ? X - q2 : X;
  const uint32_t t = mul_shoup_lazy(Y, w.x, w.y, q);
  X = x + t;
  Y = x - t + q2;
}
__device__ __forceinline__ void bf_i(uint32_t &X, uint32_t &Y, uint2 w, uint32_t q, uint32_t q2) {
  uint32_t u = X + Y;
  u = u >= q2 ? u - q2 : u;
  Y = mul_shoup_lazy(X - Y + q2, w.x, w.y, q);
  X = u;
}
__device__ __forceinline__ uint2 tw(const uint2 *t, int i) { return __ldg(t + i); }

// forward, values in [0, 4q) between passes (inputs canonical)
__device__ __forceinline__ void fwdA(uint32_t (&v)[8], const ResidueTables &T) {
  const uint32_t q = T.q, q2 = 2 * q;
  uint2 w = tw(T.fwt, 1);
  bf_f(v[0], v[4], w, q, q2); bf_f(v[1], v[5], w, q, q2);
  bf_f(v[2], v[6], w, q, q2); bf_f(v[3], v[7], w, q, q2);
  w = tw(T.fwt, 2); bf_f(v[0], v[2], w, q, q2); bf_f(v[1], v[3], w, q, q2);
  w = tw(T.fwt, 3); bf_f(v[4], v[6], w, q, q2); bf_f(v[5], v[7], w, q, q2);
  bf_f(v[0], v[1], tw(T.fwt, 4), q, q2); bf_f(v[2], v[3], tw(T.fwt, 5), q, q2);
  bf_f(v[4], v[5], tw(T.fwt, 6), q, q2); bf_f(v[6], v[7], tw(T.fwt, 7), q, q2);
}
// pass B (base 8) and pass C (base 64) share one shape
__device__ __forceinline__ void fwdBC(uint32_t (&v)[8], const ResidueTables &T, int base, int g) {
  const uint32_t q = T.q, q2 = 2 * q;
  uint2 w = tw(T.fwt, base + g);
  bf_f(v[0], v[4], w, q, q2); bf_f(v[1], v[5], w, q, q2);
  bf_f(v[2], v[6], w, q, q2); bf_f(v[3], v[7], w, q, q2);
  w = tw(T.fwt, 2 * base + 2 * g); bf_f(v[0], v[2], w, q, q2); bf_f(v[1], v[3], w, q, q2);
  w = tw(T.fwt, 2 * base + 2 * g + 1); bf_f(v[4], v[6], w, q, q2); bf_f(v[5], v[7], w, q, q2);
  bf_f(v[0], v[1], tw(T.fwt, 4 * base + 4 * g + 0), q, q2);
  bf_f(v[2], v[3], tw(T.fwt, 4 * base + 4 * g + 1), q, q2);
  bf_f(v[4], v[5], tw(T.fwt, 4 * base + 4 * g + 2), q, q2);
  bf_f(v[6], v[7], tw(T.fwt, 4 * base + 4 * g + 3), q, q2);
}
// pass D, then reduction to canonical [0, q)
__device__ __forceinline__ void fwdD(uint32_t (&v)[8], const ResidueTables &T, int t) {
  const uint32_t q = T.q, q2 = 2 * q;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int b4 = t + 256 * h;
    uint32_t *u = v + 4 * h;
    const uint2 w = tw(T.fwt, 512 + b4);
    bf_f(u[0], u[2], w, q, q2); bf_f(u[1], u[3], w, q, q2);
    bf_f(u[0], u[1], tw(T.fwt, 1024 + 2 * b4), q, q2);
    bf_f(u[2], u[3], tw(T.fwt, 1025 + 2 * b4), q, q2);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    uint32_t x = v[k];
    x = x >= q2 ? x - q2 : x;
    v[k] = x >= q ? x - q : x;
  }
}
// inverse, values in [0, 2q) between passes (inputs canonical)
__device__ __forceinline__ void invD(uint32_t (&v)[8], const ResidueTables &T, int t) {
  const uint32_t q = T.q, q2 = 2 * q;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int b4 = t + 256 * h;
    uint32_t *u = v + 4 * h;
    bf_i(u[0], u[1], tw(T.iwt, 1024 + 2 * b4), q, q2);
    bf_i(u[2], u[3], tw(T.iwt, 1025 + 2 * b4), q, q2);
    const uint2 w = tw(T.iwt, 512 + b4);
    bf_i(u[0], u[2], w, q, q2); bf_i(u[1], u[3], w, q, q2);
  }
}
__device__ __forceinline__ void invBC(uint32_t (&v)[8], const ResidueTables &T, int base, int g) {
  const uint32_t q = T.q, q2 = 2 * q;
  bf_i(v[0], v[1], tw(T.iwt, 4 * base + 4 * g + 0), q, q2);
  bf_i(v[2], v[3], tw(T.iwt, 4 * base + 4 * g + 1), q, q2);
  bf_i(v[4], v[5], tw(T.iwt, 4 * base + 4 * g + 2), q, q2);
  bf_i(v[6], v[7], tw(T.iwt, 4 * base + 4 * g + 3), q, q2);
  uint2 w = tw(T.iwt, 2 * base + 2 * g); bf_i(v[0], v[2], w, q, q2); bf_i(v[1], v[3], w, q, q2);
  w = tw(T.iwt, 2 * base + 2 * g + 1); bf_i(v[4], v[6], w, q, q2); bf_i(v[5], v[7], w, q, q2);
  w = tw(T.iwt, base + g);
  bf_i(v[0], v[4], w, q, q2); bf_i(v[1], v[5], w, q, q2);
  bf_i(v[2], v[6], w, q, q2); bf_i(v[3], v[7], w, q, q2);
}
// last pass: stages t = 256, 512, then t = 1024 with the N^-1 scaling
// folded in; outputs canonical
__device__ __forceinline__ void invA(uint32_t (&v)[8], const ResidueTables &T) {
  const uint32_t q = T.q, q2 = 2 * q;
  bf_i(v[0], v[1], tw(T.iwt, 4), q, q2); bf_i(v[2], v[3], tw(T.iwt, 5), q, q2);
  bf_i(v[4], v[5], tw(T.iwt, 6), q, q2); bf_i(v[6], v[7], tw(T.iwt, 7), q, q2);
  uint2 w = tw(T.iwt, 2); bf_i(v[0], v[2], w, q, q2); bf_i(v[1], v[3], w, q, q2);
  w = tw(T.iwt, 3); bf_i(v[4], v[6], w, q, q2); bf_i(v[5], v[7], w, q, q2);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t X = v[k], Y = v[k + 4];
    uint32_t a = mul_shoup_lazy(X + Y, T.n_inv, T.n_inv_sh, q);
    uint32_t b = mul_shoup_lazy(X - Y + q2, T.w1_ninv, T.w1_ninv_sh, q);
    v[k] = a >= q ? a - q : a;
    v[k + 4] = b >= q ? b - q : b;
  }
}

// Shared-memory plane traffic between passes (padded indexing).
template <int P>
__device__ __forceinline__ void st_plane(uint32_t *pl, const uint32_t (&v)[8], int t) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int p = P == 0 ? posA(t, k) : P == 1 ? posB(t, k) : P == 2 ? posC(t, k) : posD(t, k);
    pl[padi(p)] = v[k];
  }
}
template <int P>
__device__ __forceinline__ void ld_plane(const uint32_t *pl, uint32_t (&v)[8], int t) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int p = P == 0 ? posA(t, k) : P == 1 ? posB(t, k) : P == 2 ? posC(t, k) : posD(t, k);
    v[k] = pl[padi(p)];
  }
}

// Forward NTT of `np` padded planes whose A-pass input has already been
// stored by the caller (after fwdA) in A-order: runs passes B and C in shared
// memory. The caller then loads D-order, runs fwdD and consumes the values.
// Must be entered with the A-pass stores complete up to a __syncthreads.
__device__ __forceinline__ void fwd_mid(uint32_t *sm, int np, const ResidueTables &T) {
  const int t = threadIdx.x;
  for (int i = 0; i < np; ++i) {
    uint32_t v[8];
    ld_plane<1>(sm + i * kPad, v, t);
    fwdBC(v, T, 8, t >> 5);
    st_plane<1>(sm + i * kPad, v, t);
  }
  __syncthreads();
  for (int i = 0; i < np; ++i) {
    uint32_t v[8];
    ld_plane<2>(sm + i * kPad, v, t);
    fwdBC(v, T, 64, t & 63);
    st_plane<2>(sm + i * kPad, v, t);
  }
  __syncthreads();
}
// Inverse counterpart: planes hold D-order values after invD; runs C and B.
__device__ __forceinline__ void inv_mid(uint32_t *sm, int np, const ResidueTables &T) {
  const int t = threadIdx.x;
  for (int i = 0; i < np; ++i) {
    uint32_t v[8];
    ld_plane<2>(sm + i * kPad, v, t);
    invBC(v, T, 64, t & 63);
    st_plane<2>(sm + i * kPad, v, t);
  }
  __syncthreads();
  for (int i = 0; i < np; ++i) {
    uint32_t v[8];
    ld_plane<1>(sm + i * kPad, v, t);
    invBC(v, T, 8, t >> 5);
    st_plane<1>(sm + i * kPad, v, t);
  }
  __syncthreads();
}

}  // namespace opir
