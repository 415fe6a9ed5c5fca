// Residue-specialised register NTT for the query-path kernels.
//
// Same transform, layout and positions as the register-resident NTT of
// opir_device.cuh (radix 8/8/8/4, A/B/C/D thread positions, padded planes),
// with three changes that cut instructions per butterfly:
//   * the residue is a template parameter, so q is an immediate;
//   * twiddles with index < 64 (passes A and B, uniform over a warp) and the
//     inverse scaling constants live in constant memory; the per-thread
//     twiddles of passes C and D are loaded once per plane loop instead of
//     once per plane;
//   * forward butterflies correct X only where the bound needs it. With
//     inputs below 2q (canonical values, or gadget digits as r + q) and
//     Shoup products t in [0, 2q), an uncorrected butterfly maps [0, b q)
//     to [0, (b + 2) q) and a corrected one (X taken to [0, 4q) first) maps
//     [0, 8q) to [0, 6q); the three uncorrected stages of the first pass end
//     below 8q, and correcting stages 4, 6, 8 and 10 keeps every later value
//     below 8q < 2^32 (8 q1 = 4294508552), so the output lies in [0, 8q).
// This header defines constant-memory arrays and is included by one
// translation unit only (opir_kernels.cu), which uploads them per device.
#pragma once

#include "opir_device.cuh"

namespace opir {

constexpr uint32_t kQ1 = 536813569u;  // CONFIG_N2048_K1_COMP composite limbs
constexpr uint32_t kQ2 = 536752129u;

template <int RES>
struct Res {
  static constexpr uint32_t q = RES ? kQ2 : kQ1;
  static constexpr uint64_t mu = ~0ull / q;  // floor(2^64 / q) (q odd, > 1)
};

// (w, floor(w 2^32 / q)) for twiddle indices < 64: [residue][index]
static __constant__ uint2 c_fwt[2][64];
static __constant__ uint2 c_iwt[2][64];
// {N^-1, its Shoup companion, iw[1] N^-1, its Shoup companion} per residue
static __constant__ uint4 c_nscale[2];

// floor(x mu / 2^64) - e with 0 <= e < 3, mod 2^32, from one high product:
// mu = floor((2^64 - 1) / q) = 8 2^32 + ml for both residues, so with x =
// xh 2^32 + xl, x mu / 2^64 = 8 xh + xh ml / 2^32 + xl / 2^29 + xl ml / 2^64,
// and the estimate drops three fractions, each below 1.
template <int RES>
__device__ __forceinline__ uint32_t quot64(uint64_t x) {
  constexpr uint64_t mu = Res<RES>::mu;
  static_assert((mu >> 32) == 8, "quot64 assumes floor(2^64 / q) = 8 2^32 + ml");
  const uint32_t xh = static_cast<uint32_t>(x >> 32), xl = static_cast<uint32_t>(x);
  return (xh << 3) + __umulhi(xh, static_cast<uint32_t>(mu)) + (xl >> 29);
}
// any x -> [0, 2q]: x mu / 2^64 > x / q - 1 - 1/q, so the estimate exceeds
// x / q - 4 - 1/q and x - quot64(x) q <= 4q (< 2^32, so 32-bit arithmetic is
// exact); one correction maps [0, 4q] to [0, 2q]. The inverse NTT's passes
// take inputs up to 2q inclusive (X + Y <= 4q < 2^32; their min correction
// maps [0, 4q] to [0, 2q]).
template <int RES>
__device__ __forceinline__ uint32_t red64_lazy(uint64_t x) {
  constexpr uint32_t Q = Res<RES>::q;
  const uint32_t r = static_cast<uint32_t>(x) - quot64<RES>(x) * Q;
  return min(r, r - 2 * Q);
}
template <int RES>
__device__ __forceinline__ uint32_t red64(uint64_t x) {  // any x -> [0, q)
  constexpr uint32_t Q = Res<RES>::q;
  uint32_t r = red64_lazy<RES>(x);  // [0, 2q]
  r = min(r, r - Q);                // [0, q]
  return min(r, r - Q);
}
template <int RES>
__device__ __forceinline__ uint32_t canon8(uint32_t x) {  // [0, 8q) -> [0, q)
  constexpr uint32_t Q = Res<RES>::q;
  x = min(x, x - 4 * Q);
  x = min(x, x - 2 * Q);
  return min(x, x - Q);
}
template <int RES>
__device__ __forceinline__ uint32_t to4q(uint32_t x) {  // [0, 8q) -> [0, 4q)
  return min(x, x - 4 * Res<RES>::q);
}
// A digit NTT value leaves the forward transform in [0, 8q) and enters a
// 64-bit multiply-accumulate with canonical key / RGSW values. P products
// (plus a carried value below 2q) stay below 2^64 uncorrected when P <= 8
// (8 8q q < 64 q1^2 = 0.99979 2^64), with values taken to [0, 4q) when
// P <= 16, and canonical beyond.
template <int RES, int P>
__device__ __forceinline__ uint32_t mac_in(uint32_t v) {
  if (P <= 8) return v;
  if (P <= 16) return to4q<RES>(v);
  return canon8<RES>(v);
}

// ------------------------------------------------------ gadget digits
// Gadget shapes (digits x log2 base) and digit kinds of the two parameter
// sets whose ring is the residue pair (q1, q2):
//   CONFIG_N2048_K1_COMP: data RGSW (L_EP 6 x 10), key RGSW (L_KEY 10 x 6)
//     and BV key switching (L_KS 8 x 8), all balanced digits of the centred
//     value mod q1 q2 in [-B/2, B/2) (gsw.cpp:252-295, bv_keyswitch.cpp:20-40);
//   CONFIG_N2048_K2_MP: data RGSW (5 x 12) and key RGSW (8 x 8) as unsigned
//     digits of the composed value in [0, q1 q2) (gsw.cpp:184-250), BV key
//     switching (8 x 8) as balanced digits in (-B/2, B/2] of the centred
//     composed value (bv_keyswitch.cpp:42-62, 373-481).
enum DigitKind { kDigitsLow = 0, kDigitsHigh = 1, kDigitsUnsigned = 2 };
template <int LEp, int BEp, int KEp, int LKey, int BKey, int KKey, int LKs, int BKs, int KKs>
struct Gadgets {
  static constexpr int lep = LEp, bep = BEp, kep = KEp;
  static constexpr int lkey = LKey, bkey = BKey, kkey = KKey;
  static constexpr int lks = LKs, bks = BKs, kks = KKs;
};
using GadgetsK1Comp = Gadgets<6, 10, kDigitsLow, 10, 6, kDigitsLow, 8, 8, kDigitsLow>;
using GadgetsK2Mp = Gadgets<5, 12, kDigitsUnsigned, 8, 8, kDigitsUnsigned, 8, 8, kDigitsHigh>;
constexpr int kLEp = GadgetsK1Comp::lep, kBaseEp = GadgetsK1Comp::bep;
constexpr int kLKey = GadgetsK1Comp::lkey, kBaseKey = GadgetsK1Comp::bkey;
constexpr int kLKs = GadgetsK1Comp::lks, kBaseKs = GadgetsK1Comp::bks;

constexpr uint32_t inv_mod_c(uint64_t a, uint64_t m) {  // a^-1 mod m (gcd 1)
  int64_t t = 0, nt = 1, r = static_cast<int64_t>(m), nr = static_cast<int64_t>(a % m);
  while (nr != 0) {
    const int64_t qq = r / nr, tt = t - qq * nt, rr = r - qq * nr;
    t = nt; nt = tt; r = nr; nr = rr;
  }
  return static_cast<uint32_t>(t < 0 ? t + static_cast<int64_t>(m) : t);
}
constexpr uint32_t kQ1InvQ2 = inv_mod_c(kQ1, kQ2);
constexpr uint32_t kQ1InvQ2Sh = static_cast<uint32_t>((static_cast<uint64_t>(kQ1InvQ2) << 32) / kQ2);
constexpr uint64_t kQ = static_cast<uint64_t>(kQ1) * kQ2;

// Garner compose of a canonical residue pair into [0, q1 q2).
__device__ __forceinline__ uint64_t compose_c(uint32_t r1, uint32_t r2) {
  const uint32_t r1m = min(r1, r1 - kQ2);                 // q1 < 2 q2
  const uint32_t diff = r2 - r1m + kQ2;                     // [1, 2 q2)
  uint32_t k = diff * kQ1InvQ2 - __umulhi(diff, kQ1InvQ2Sh) * kQ2;
  k = min(k, k - kQ2);
  return static_cast<uint64_t>(r1) + static_cast<uint64_t>(kQ1) * k;
}
// Per-digit offset of a digit kind: balanced digits r_i in [-o, B - o).
template <int B, int KIND>
__host__ __device__ constexpr uint32_t digit_offset() {
  return KIND == kDigitsLow ? (1u << (B - 1)) : KIND == kDigitsHigh ? (1u << (B - 1)) - 1u : 0u;
}
// Base-2^B digits, LSB first, as the plain base-2^B digits u_i of one 64-bit
// word. Balanced kinds: v in [0, q) is centred to c in (-q/2, q/2], and
// c + C with C = o sum_{i<L} 2^(B i) (o the kind's offset) has plain digits
// u_i = r_i + o, where r_i in [-o, B - o) are the balanced digits (the
// balanced expansion of |c| < 2^(B L) / 2 ends within L digits, and the
// base-2^B expansion of c + C is unique). Unsigned kind: u_i are the digits
// of v itself.
template <int L, int B, int KIND = kDigitsLow>
__device__ __forceinline__ uint64_t digit_source(uint64_t v) {
  if (KIND == kDigitsUnsigned) return v;
  uint64_t C = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) C += static_cast<uint64_t>(digit_offset<B, KIND>()) << (B * i);
  return v + C - (v > kQ / 2 ? kQ : 0);
}
// r_i as a residue mod Q below 2Q: r_i + Q for every balanced digit (in
// [Q - o, Q - o + 2^B), not reduced: the forward NTT's first pass takes
// inputs below 2q), the digit itself for unsigned digits.
template <uint32_t Q, int B, int KIND = kDigitsLow>
__device__ __forceinline__ uint32_t digit_res(uint64_t u, int i) {
  const int o = B * i;  // a constant once the caller's digit loop is unrolled
  const uint32_t lo = static_cast<uint32_t>(u), hi = static_cast<uint32_t>(u >> 32);
  uint32_t f;
  if (o + B <= 32) f = lo >> o;
  else if (o >= 32) f = hi >> (o - 32);
  else f = __funnelshift_r(lo, hi, o);
  f &= (1u << B) - 1;
  if (KIND == kDigitsUnsigned) return f;  // f < 2^B < Q
  return f + (Q - digit_offset<B, KIND>());
}

// --------------------------------------------------------------- forward
template <uint32_t Q, bool C>
__device__ __forceinline__ void fbf(uint32_t &X, uint32_t &Y, uint2 w) {
  uint32_t x = X;
  if (C) x = min(x, x - 4 * Q);
  const uint32_t t = Y * w.x - __umulhi(Y, w.y) * Q;
  X = x + t;
  Y = x - t + 2 * Q;
}
template <uint32_t Q, bool C1, bool C2, bool C3>
__device__ __forceinline__ void fpass8(uint32_t (&v)[8], const uint2 (&w)[7]) {
  fbf<Q, C1>(v[0], v[4], w[0]); fbf<Q, C1>(v[1], v[5], w[0]);
  fbf<Q, C1>(v[2], v[6], w[0]); fbf<Q, C1>(v[3], v[7], w[0]);
  fbf<Q, C2>(v[0], v[2], w[1]); fbf<Q, C2>(v[1], v[3], w[1]);
  fbf<Q, C2>(v[4], v[6], w[2]); fbf<Q, C2>(v[5], v[7], w[2]);
  fbf<Q, C3>(v[0], v[1], w[3]); fbf<Q, C3>(v[2], v[3], w[4]);
  fbf<Q, C3>(v[4], v[5], w[5]); fbf<Q, C3>(v[6], v[7], w[6]);
}
// pass A (stages 1-3), inputs below 2q, outputs below 8q; twiddles 1..7
// from constant memory
template <int RES>
__device__ __forceinline__ void fA(uint32_t (&v)[8]) {
  const uint2 w[7] = {c_fwt[RES][1], c_fwt[RES][2], c_fwt[RES][3], c_fwt[RES][4],
                      c_fwt[RES][5], c_fwt[RES][6], c_fwt[RES][7]};
  fpass8<Res<RES>::q, false, false, false>(v, w);
}
// per-thread twiddles of passes B (warp-uniform, constant memory), C and D
template <int RES>
__device__ __forceinline__ void fload_b(uint2 (&w)[7], int t) {
  const int g = t >> 5;
  w[0] = c_fwt[RES][8 + g];
  w[1] = c_fwt[RES][16 + 2 * g];
  w[2] = c_fwt[RES][17 + 2 * g];
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = c_fwt[RES][32 + 4 * g + i];
}
__device__ __forceinline__ void fload_c(uint2 (&w)[7], const uint2 *fwt, int t) {
  const int g = t & 63;
  w[0] = __ldg(fwt + 64 + g);
  w[1] = __ldg(fwt + 128 + 2 * g);
  w[2] = __ldg(fwt + 129 + 2 * g);
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = __ldg(fwt + 256 + 4 * g + i);
}
__device__ __forceinline__ void fload_d(uint2 (&w)[6], const uint2 *fwt, int t) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int b4 = t + 256 * h;
    w[3 * h] = __ldg(fwt + 512 + b4);
    w[3 * h + 1] = __ldg(fwt + 1024 + 2 * b4);
    w[3 * h + 2] = __ldg(fwt + 1025 + 2 * b4);
  }
}
// pass D (stages 10-11): output in [0, 8q)
template <int RES>
__device__ __forceinline__ void fD(uint32_t (&v)[8], const uint2 (&w)[6]) {
  constexpr uint32_t Q = Res<RES>::q;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t *u = v + 4 * h;
    fbf<Q, true>(u[0], u[2], w[3 * h]);
    fbf<Q, true>(u[1], u[3], w[3 * h]);
    fbf<Q, false>(u[0], u[1], w[3 * h + 1]);
    fbf<Q, false>(u[2], u[3], w[3 * h + 2]);
  }
}
template <uint32_t Q>
__device__ __forceinline__ void ipass8(uint32_t (&v)[8], const uint2 (&w)[7]);
// One radix-8 pass over the padded plane `pl`: load in pass order PASS,
// butterflies, store back.
template <int RES, int PASS, bool FWD>
__device__ __forceinline__ void mid_plane_r(uint32_t *pl, const uint2 (&w)[7], int t) {
  constexpr uint32_t Q = Res<RES>::q;
  uint32_t v[8];
  ld_plane<PASS>(pl, v, t);
  if (!FWD) ipass8<Q>(v, w);
  else if (PASS == 1) fpass8<Q, true, false, true>(v, w);
  else fpass8<Q, false, true, false>(v, w);
  st_plane<PASS>(pl, v, t);
}
// Passes B and C over `np` padded planes stored in A-order after fA, up to a
// __syncthreads; ends synchronised. The caller then loads D-order and runs fD.
// Full = true unrolls the plane loops (faster in the one-CTA-per-step
// kernels; the cluster-split kernels, with 1 to 4 planes per CTA, keep the
// compiler's choice, which is faster there).
template <int RES, bool Full = true>
__device__ __forceinline__ void fwd_mid_r(uint32_t *sm, int np, const uint2 *fwt) {
  const int t = threadIdx.x;
  {
    uint2 w[7];
    fload_b<RES>(w, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 1, true>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 1, true>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
  {
    uint2 w[7];
    fload_c(w, fwt, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 2, true>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 2, true>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
}

// --------------------------------------------------------------- inverse
// Gentleman-Sande, inputs and outputs in [0, 2q] between passes (X + Y and
// X - Y + 2q stay within [0, 4q], and the min maps [0, 4q] to [0, 2q]).
template <uint32_t Q>
__device__ __forceinline__ void ibf(uint32_t &X, uint32_t &Y, uint2 w) {
  uint32_t u = X + Y;
  u = min(u, u - 2 * Q);
  const uint32_t d = X - Y + 2 * Q;
  Y = d * w.x - __umulhi(d, w.y) * Q;
  X = u;
}
template <uint32_t Q>
__device__ __forceinline__ void ipass8(uint32_t (&v)[8], const uint2 (&w)[7]) {
  ibf<Q>(v[0], v[1], w[3]); ibf<Q>(v[2], v[3], w[4]);
  ibf<Q>(v[4], v[5], w[5]); ibf<Q>(v[6], v[7], w[6]);
  ibf<Q>(v[0], v[2], w[1]); ibf<Q>(v[1], v[3], w[1]);
  ibf<Q>(v[4], v[6], w[2]); ibf<Q>(v[5], v[7], w[2]);
  ibf<Q>(v[0], v[4], w[0]); ibf<Q>(v[1], v[5], w[0]);
  ibf<Q>(v[2], v[6], w[0]); ibf<Q>(v[3], v[7], w[0]);
}
// twiddles of the inverse passes in the same [base + g, 2 base + 2 g (+1),
// 4 base + 4 g (+0..3)] arrangement as the forward ones
template <int RES>
__device__ __forceinline__ void iload_b(uint2 (&w)[7], int t) {
  const int g = t >> 5;
  w[0] = c_iwt[RES][8 + g];
  w[1] = c_iwt[RES][16 + 2 * g];
  w[2] = c_iwt[RES][17 + 2 * g];
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = c_iwt[RES][32 + 4 * g + i];
}
__device__ __forceinline__ void iload_c(uint2 (&w)[7], const uint2 *iwt, int t) {
  const int g = t & 63;
  w[0] = __ldg(iwt + 64 + g);
  w[1] = __ldg(iwt + 128 + 2 * g);
  w[2] = __ldg(iwt + 129 + 2 * g);
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = __ldg(iwt + 256 + 4 * g + i);
}
__device__ __forceinline__ void iload_d(uint2 (&w)[6], const uint2 *iwt, int t) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int b4 = t + 256 * h;
    w[3 * h] = __ldg(iwt + 512 + b4);
    w[3 * h + 1] = __ldg(iwt + 1024 + 2 * b4);
    w[3 * h + 2] = __ldg(iwt + 1025 + 2 * b4);
  }
}
// first inverse pass (stages t = 1, 2) on D-order values in [0, 2q)
template <int RES>
__device__ __forceinline__ void iD(uint32_t (&v)[8], const uint2 (&w)[6]) {
  constexpr uint32_t Q = Res<RES>::q;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t *u = v + 4 * h;
    ibf<Q>(u[0], u[1], w[3 * h + 1]);
    ibf<Q>(u[2], u[3], w[3 * h + 2]);
    ibf<Q>(u[0], u[2], w[3 * h]);
    ibf<Q>(u[1], u[3], w[3 * h]);
  }
}
// last inverse pass (t = 256, 512, then 1024 with N^-1 folded in); canonical
template <int RES>
__device__ __forceinline__ void iA(uint32_t (&v)[8]) {
  constexpr uint32_t Q = Res<RES>::q;
  ibf<Q>(v[0], v[1], c_iwt[RES][4]); ibf<Q>(v[2], v[3], c_iwt[RES][5]);
  ibf<Q>(v[4], v[5], c_iwt[RES][6]); ibf<Q>(v[6], v[7], c_iwt[RES][7]);
  ibf<Q>(v[0], v[2], c_iwt[RES][2]); ibf<Q>(v[1], v[3], c_iwt[RES][2]);
  ibf<Q>(v[4], v[6], c_iwt[RES][3]); ibf<Q>(v[5], v[7], c_iwt[RES][3]);
  const uint4 s = c_nscale[RES];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t X = v[k], Y = v[k + 4];
    const uint32_t a = X + Y, d = X - Y + 2 * Q;
    const uint32_t ra = a * s.x - __umulhi(a, s.y) * Q;
    const uint32_t rb = d * s.z - __umulhi(d, s.w) * Q;
    v[k] = min(ra, ra - Q);
    v[k + 4] = min(rb, rb - Q);
  }
}
// Passes C and B over `np` planes holding D-order values after iD, up to a
// __syncthreads; ends synchronised. The caller then loads A-order and runs iA.
template <int RES, bool Full = true>
__device__ __forceinline__ void inv_mid_r(uint32_t *sm, int np, const uint2 *iwt) {
  const int t = threadIdx.x;
  {
    uint2 w[7];
    iload_c(w, iwt, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 2, false>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 2, false>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
  {
    uint2 w[7];
    iload_b<RES>(w, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 1, false>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane_r<RES, 1, false>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
}

}  // namespace opir
