// Device arithmetic and the register-resident NTT-4096 for the
// CONFIG_N4096_K2_MP parameter set (includes/database_constants.h:111-125):
// N = 4096, two RNS limbs q0 = 2^60 - 2^14 + 1 and q1 = 2^60 - 2^16 - 2^15 + 1
// (the reference's generate_ntt_friendly_primes({60, 60}, 4096)), every
// polynomial as [limb 0 (N)][limb 1 (N)] u64. Included by opir_c4_kernels.cu only
// (it defines constant-memory arrays).
//
// NTT: 512 threads hold 8 coefficients each; the 12 butterfly stages run as
// four radix-8 passes (3 stages each) with three exchanges through a shared
// plane padded by one word per 8 (p -> p + p/8). Thread t holds, per pass,
//   A: t + 512 k            B: 512 (t >> 6) + (t & 63) + 64 k
//   C: 64 (t >> 3) + (t & 7) + 8 k                D: 8 t + k
// and a pass with twiddle base b and group g uses w[b + g] (stage 1),
// w[2b + 2g (+1)] (stage 2), w[4b + 4g + 0..3] (stage 3): A (1, 0),
// B (8, t >> 6), C (64, t >> 3), D (512, t). Merged Cooley-Tukey forward with
// bit-reversed output and Gentleman-Sande inverse scaled by N^-1, the HEXL
// convention of the reference (utils.cpp:26-56). Forward butterflies are
// Harvey/Shoup lazy with X corrected only on stages 4, 6, 8, 10, 12 (values
// stay below 8q < 2^63, outputs below 6q); inverse ones keep [0, 2q).
#pragma once

#include <cstdint>

#include "opir_c4_kernels.h"

namespace opir4 {

constexpr int kThreads = 512;
constexpr int kPad = kN + kN / 8;           // u64 words per padded plane

template <int L>
struct Limb {
  static constexpr uint64_t q = L ? kQ1 : kQ0;
};

// (w, floor(w 2^64 / q)) for twiddle indices < 64: [limb][index]
static __constant__ ulonglong2 c4_fwt[2][64];
static __constant__ ulonglong2 c4_iwt[2][64];
// {N^-1, Shoup} and {iw[1] N^-1, Shoup} per limb
static __constant__ ulonglong2 c4_ninv[2], c4_w1ninv[2];

__device__ __forceinline__ int pad(int p) { return p + (p >> 3); }
__device__ __forceinline__ int posA(int t, int k) { return t + 512 * k; }
__device__ __forceinline__ int posB(int t, int k) { return ((t >> 6) << 9) + (t & 63) + 64 * k; }
__device__ __forceinline__ int posC(int t, int k) { return ((t >> 3) << 6) + (t & 7) + 8 * k; }
__device__ __forceinline__ int posD(int t, int k) { return 8 * t + k; }

// a w mod q in [0, 2q) for any 64-bit a (Shoup; ws = floor(w 2^64 / q))
template <uint64_t Q>
__device__ __forceinline__ uint64_t mul_shoup(uint64_t a, uint64_t w, uint64_t ws) {
  return a * w - __umul64hi(a, ws) * Q;
}
template <uint64_t Q>
__device__ __forceinline__ uint64_t canon8(uint64_t x) {  // [0, 8q) -> [0, q)
  x = min(x, x - 4 * Q);
  x = min(x, x - 2 * Q);
  return min(x, x - Q);
}
template <uint64_t Q>
__device__ __forceinline__ uint64_t add_mod(uint64_t a, uint64_t b) {
  const uint64_t s = a + b;
  return min(s, s - Q);
}
template <uint64_t Q>
__device__ __forceinline__ uint64_t sub_mod(uint64_t a, uint64_t b) {
  const uint64_t d = a - b + Q;
  return min(d, d - Q);
}
template <uint64_t Q>
__device__ __forceinline__ uint64_t neg_mod(uint64_t a) {
  return a ? Q - a : 0;
}

// x mod q for x < 2^126: x = h 2^64 + l, h 2^64 mod q by Shoup with
// c = 2^64 mod q, l mod q by a 64-bit Barrett estimate.
template <uint64_t Q>
__device__ __forceinline__ uint64_t red128(unsigned __int128 x) {
  constexpr uint64_t c = static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) % Q);
  constexpr uint64_t cs = static_cast<uint64_t>((static_cast<unsigned __int128>(c) << 64) / Q);
  constexpr uint64_t mu = ~0ull / Q;  // floor(2^64 / q)
  const uint64_t h = static_cast<uint64_t>(x >> 64), l = static_cast<uint64_t>(x);
  const uint64_t r1 = mul_shoup<Q>(h, c, cs);            // [0, 2q)
  const uint64_t r2 = l - __umul64hi(l, mu) * Q;          // [0, 3q)
  uint64_t r = r1 + r2;                                   // [0, 5q) < 2^63
  r = min(r, r - 4 * Q);
  r = min(r, r - 2 * Q);
  return min(r, r - Q);
}

// ----------------------------------------------------------------- NTT
template <uint64_t Q, bool C>
__device__ __forceinline__ void fbf(uint64_t &X, uint64_t &Y, ulonglong2 w) {
  uint64_t x = X;
  if (C) x = min(x, x - 4 * Q);
  const uint64_t t = mul_shoup<Q>(Y, w.x, w.y);
  X = x + t;
  Y = x - t + 2 * Q;
}
template <uint64_t Q, bool C1, bool C2, bool C3>
__device__ __forceinline__ void fpass(uint64_t (&v)[8], const ulonglong2 (&w)[7]) {
  fbf<Q, C1>(v[0], v[4], w[0]); fbf<Q, C1>(v[1], v[5], w[0]);
  fbf<Q, C1>(v[2], v[6], w[0]); fbf<Q, C1>(v[3], v[7], w[0]);
  fbf<Q, C2>(v[0], v[2], w[1]); fbf<Q, C2>(v[1], v[3], w[1]);
  fbf<Q, C2>(v[4], v[6], w[2]); fbf<Q, C2>(v[5], v[7], w[2]);
  fbf<Q, C3>(v[0], v[1], w[3]); fbf<Q, C3>(v[2], v[3], w[4]);
  fbf<Q, C3>(v[4], v[5], w[5]); fbf<Q, C3>(v[6], v[7], w[6]);
}
template <uint64_t Q>
__device__ __forceinline__ void ibf(uint64_t &X, uint64_t &Y, ulonglong2 w) {
  uint64_t u = X + Y;
  u = min(u, u - 2 * Q);
  const uint64_t d = X - Y + 2 * Q;
  Y = mul_shoup<Q>(d, w.x, w.y);
  X = u;
}
template <uint64_t Q>
__device__ __forceinline__ void ipass(uint64_t (&v)[8], const ulonglong2 (&w)[7]) {
  ibf<Q>(v[0], v[1], w[3]); ibf<Q>(v[2], v[3], w[4]);
  ibf<Q>(v[4], v[5], w[5]); ibf<Q>(v[6], v[7], w[6]);
  ibf<Q>(v[0], v[2], w[1]); ibf<Q>(v[1], v[3], w[1]);
  ibf<Q>(v[4], v[6], w[2]); ibf<Q>(v[5], v[7], w[2]);
  ibf<Q>(v[0], v[4], w[0]); ibf<Q>(v[1], v[5], w[0]);
  ibf<Q>(v[2], v[6], w[0]); ibf<Q>(v[3], v[7], w[0]);
}

// twiddles of a pass: base b, group g; constant memory when every index < 64
template <int L, bool FWD>
__device__ __forceinline__ void tw_const(ulonglong2 (&w)[7], int b, int g) {
  const ulonglong2 *T = FWD ? c4_fwt[L] : c4_iwt[L];
  w[0] = T[b + g];
  w[1] = T[2 * b + 2 * g];
  w[2] = T[2 * b + 2 * g + 1];
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = T[4 * b + 4 * g + i];
}
__device__ __forceinline__ void tw_global(ulonglong2 (&w)[7], const ulonglong2 *T, int b, int g) {
  w[0] = __ldg(T + b + g);
  w[1] = __ldg(T + 2 * b + 2 * g);
  w[2] = __ldg(T + 2 * b + 2 * g + 1);
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = __ldg(T + 4 * b + 4 * g + i);
}

template <int P>
__device__ __forceinline__ int posP(int t, int k) {
  return P == 0 ? posA(t, k) : P == 1 ? posB(t, k) : P == 2 ? posC(t, k) : posD(t, k);
}
template <int P>
__device__ __forceinline__ void st_plane(uint64_t *pl, const uint64_t (&v)[8], int t) {
#pragma unroll
  for (int k = 0; k < 8; ++k) pl[pad(posP<P>(t, k))] = v[k];
}
template <int P>
__device__ __forceinline__ void ld_plane(const uint64_t *pl, uint64_t (&v)[8], int t) {
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = pl[pad(posP<P>(t, k))];
}

// forward pass A on canonical inputs (A-order in registers)
template <int L>
__device__ __forceinline__ void fA(uint64_t (&v)[8]) {
  ulonglong2 w[7];
  tw_const<L, true>(w, 1, 0);
  fpass<Limb<L>::q, false, false, false>(v, w);
}
// Forward passes B and C over np planes stored in A-order (after fA), up to
// a __syncthreads; ends synchronised. Then: ld_plane<3> + fD.
template <int L>
__device__ __forceinline__ void fwd_mid(uint64_t *sm, int np, const Tables &T) {
  constexpr uint64_t Q = Limb<L>::q;
  const int t = threadIdx.x;
  {
    ulonglong2 w[7];
    tw_const<L, true>(w, 8, t >> 6);
#pragma unroll
    for (int i = 0; i < np; ++i) {
      uint64_t v[8];
      ld_plane<1>(sm + i * kPad, v, t);
      fpass<Q, true, false, true>(v, w);
      st_plane<1>(sm + i * kPad, v, t);
    }
  }
  __syncthreads();
  {
    ulonglong2 w[7];
    tw_global(w, T.fwt[L], 64, t >> 3);
#pragma unroll
    for (int i = 0; i < np; ++i) {
      uint64_t v[8];
      ld_plane<2>(sm + i * kPad, v, t);
      fpass<Q, false, true, false>(v, w);
      st_plane<2>(sm + i * kPad, v, t);
    }
  }
  __syncthreads();
}
// forward pass D (stages 10-12, D-order values), output in [0, 6q)
template <int L>
__device__ __forceinline__ void fD(uint64_t (&v)[8], const ulonglong2 (&w)[7]) {
  fpass<Limb<L>::q, true, false, true>(v, w);
}
template <int L>
__device__ __forceinline__ void fload_d(ulonglong2 (&w)[7], const Tables &T) {
  tw_global(w, T.fwt[L], 512, threadIdx.x);
}

// inverse: pass D first (D-order, inputs in [0, 2q))
template <int L>
__device__ __forceinline__ void iload_d(ulonglong2 (&w)[7], const Tables &T) {
  tw_global(w, T.iwt[L], 512, threadIdx.x);
}
template <int L>
__device__ __forceinline__ void iD(uint64_t (&v)[8], const ulonglong2 (&w)[7]) {
  ipass<Limb<L>::q>(v, w);
}
// Inverse passes C and B over np planes stored in D-order after iD, up to a
// __syncthreads; ends synchronised. Then: ld_plane<0> + iA.
template <int L>
__device__ __forceinline__ void inv_mid(uint64_t *sm, int np, const Tables &T) {
  constexpr uint64_t Q = Limb<L>::q;
  const int t = threadIdx.x;
  {
    ulonglong2 w[7];
    tw_global(w, T.iwt[L], 64, t >> 3);
#pragma unroll
    for (int i = 0; i < np; ++i) {
      uint64_t v[8];
      ld_plane<2>(sm + i * kPad, v, t);
      ipass<Q>(v, w);
      st_plane<2>(sm + i * kPad, v, t);
    }
  }
  __syncthreads();
  {
    ulonglong2 w[7];
    tw_const<L, false>(w, 8, t >> 6);
#pragma unroll
    for (int i = 0; i < np; ++i) {
      uint64_t v[8];
      ld_plane<1>(sm + i * kPad, v, t);
      ipass<Q>(v, w);
      st_plane<1>(sm + i * kPad, v, t);
    }
  }
  __syncthreads();
}
// last inverse pass (A-order): stages with twiddles 4..7 and 2, 3, then the
// distance-2048 stage with N^-1 folded in; output canonical
template <int L>
__device__ __forceinline__ void iA(uint64_t (&v)[8]) {
  constexpr uint64_t Q = Limb<L>::q;
  ibf<Q>(v[0], v[1], c4_iwt[L][4]); ibf<Q>(v[2], v[3], c4_iwt[L][5]);
  ibf<Q>(v[4], v[5], c4_iwt[L][6]); ibf<Q>(v[6], v[7], c4_iwt[L][7]);
  ibf<Q>(v[0], v[2], c4_iwt[L][2]); ibf<Q>(v[1], v[3], c4_iwt[L][2]);
  ibf<Q>(v[4], v[6], c4_iwt[L][3]); ibf<Q>(v[5], v[7], c4_iwt[L][3]);
  const ulonglong2 a = c4_ninv[L], b = c4_w1ninv[L];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint64_t X = v[k], Y = v[k + 4];
    const uint64_t ra = mul_shoup<Q>(X + Y, a.x, a.y);
    const uint64_t rb = mul_shoup<Q>(X - Y + 2 * Q, b.x, b.y);
    v[k] = min(ra, ra - Q);
    v[k + 4] = min(rb, rb - Q);
  }
}

// floor(w 2^64 / q) for w < q = 2^60 - c: w 2^64 = w (16 q + 16 c), so the
// quotient is 16 w + floor(x / q) with x = 16 c w < 2^81, and floor(x / q) is
// t0 = floor(x / 2^60) or t0 + 1 (x / q - x / 2^60 < 2^-22); the remainder
// x - t0 q = (x mod 2^60) + t0 c decides.
template <uint64_t Q>
__device__ __forceinline__ uint64_t shoup_of(uint64_t w) {
  constexpr uint64_t c = (1ull << 60) - Q;
  const unsigned __int128 x = static_cast<unsigned __int128>(w) * (16 * c);
  const uint64_t hi = static_cast<uint64_t>(x >> 64), lo = static_cast<uint64_t>(x);
  const uint64_t t0 = (hi << 4) | (lo >> 60);
  const uint64_t r0 = (lo & ((1ull << 60) - 1)) + t0 * c;
  return 16 * w + t0 + (r0 >= Q ? 1 : 0);
}
// [0, 16q) -> [0, 2q)
template <uint64_t Q>
__device__ __forceinline__ uint64_t fold16(uint64_t x) {
  x = min(x, x - 8 * Q);
  x = min(x, x - 4 * Q);
  return min(x, x - 2 * Q);
}

// ------------------------------------------------------ RNS <-> integer
// Garner compose of canonical limbs into [0, q0 q1) (gsw.cpp:22-53)
__device__ __forceinline__ unsigned __int128 compose(uint64_t r0, uint64_t r1, uint64_t q0inv,
                                                     uint64_t q0inv_sh) {
  const uint64_t r0m = min(r0, r0 - kQ1);  // q0 < 2 q1
  const uint64_t diff = r1 - r0m + kQ1;    // (0, 2 q1)
  uint64_t s = mul_shoup<kQ1>(diff, q0inv, q0inv_sh);
  s = min(s, s - kQ1);
  return static_cast<unsigned __int128>(kQ0) * s + r0;
}

}  // namespace opir4
