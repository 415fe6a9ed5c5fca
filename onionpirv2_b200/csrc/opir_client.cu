// Client-side batch operations: query packing (PirClient::fast_generate_query,
// src/client.cpp:107-225), response decryption (PirClient::decrypt_mod_q,
// src/client.cpp:364-410) for many queries or responses of one client, and
// its session keys (create_session_keys, src/client.cpp:40-45).
//
// Both are dominated by one negacyclic product x * s with the client's ternary
// secret s. The reference multiplies in the NTT domain mod the target modulus;
// here s is held as two index lists, P (coefficients equal to 1) and M (equal
// to -1), and the product is the exact integer sum
//     (x*s)_i = sum_{j in P} xe[N+i-j] - sum_{j in M} xe[N+i-j]
// over the sign-extended copy xe[N+m] = x[m], xe[m] = -x[m] (m < N) staged in
// shared memory; only the epilogue reduces, so the result equals the NTT
// product mod the same modulus exactly. x is split into parts of at most 31
// bits so each shared word is an int32 and each partial sum fits an int64.
// Two forms of the product: the index-list form (list_product: one shared
// load per nonzero secret coefficient, output and part) for any batch, and
// for decryption batches that fill the GPU the window form (window_product:
// register windows reused across secret coefficients one block apart, int32
// partial sums). One CTA of kBlock threads per (item, output slice).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/onionpir_b200.h"
#include "opir_client.h"
#include "opir_host.h"
#include "opir_kernels.h"
#include "opir_params.h"
#include "opir_scan_tc.h"

namespace {

using opir::ck;
using opir::DevBuf;
using opir::DeviceGuard;

constexpr int kBlock = 256;
constexpr uint32_t kNoPos = 0xFFFFFFFFu;

// One plaintext-constant addition of a query: c0[limb k][pos] += val[k].
struct ConstEntry {
  uint32_t pos;
  uint32_t pad;
  uint64_t val[2];
};

// xe for one polynomial in NP parts of PB bits, part p at ext + p 2n.
template <int NP, int PB>
__device__ __forceinline__ void stage_ext(const uint64_t *__restrict__ x, uint64_t mod, uint32_t n,
                                          int32_t *ext) {
  constexpr uint64_t kMask = (1ull << PB) - 1;
  for (uint32_t m = threadIdx.x; m < n; m += blockDim.x) {
    const uint64_t v = x[m] % mod;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int32_t part = static_cast<int32_t>(p + 1 < NP ? (v >> (PB * p)) & kMask : v >> (PB * p));
      ext[2 * n * p + n + m] = part;
      ext[2 * n * p + m] = -part;
    }
  }
}

// Index-list product: acc[p][r] = part p of (x*s)_i for i = i0 + kBlock r,
// one shared load per nonzero secret coefficient, output and part.
template <int NP, int R>
__device__ __forceinline__ void list_product(const int32_t *ext, const uint16_t *sl,
                                             uint32_t npos, uint32_t nneg, uint32_t n,
                                             uint32_t i0, int64_t (&acc)[NP][R]) {
#pragma unroll
  for (int p = 0; p < NP; ++p)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[p][r] = 0;
  const int32_t *e0 = ext + n + i0;
#pragma unroll 4
  for (uint32_t u = 0; u < npos; ++u) {
    const int j = sl[u];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < NP; ++p) acc[p][r] += e0[2 * n * p + kBlock * r - j];
  }
#pragma unroll 4
  for (uint32_t u = npos; u < npos + nneg; ++u) {
    const int j = sl[u];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < NP; ++p) acc[p][r] -= e0[2 * n * p + kBlock * r - j];
  }
}

// Window product for n = kBlock J: with j = jl + kBlock jh, the term of output
// i_r = i0 + kBlock r is xe[n + i0 - jl + kBlock (r - jh)], so for one jl the
// thread loads the R + J - 1 window values once into registers and applies
// all J secret coefficients s[jl + kBlock jh] (packed 2 bits each in cs[jl]:
// 1 = +1, 2 = -1, 0 = 0; the same word for every thread, so the branches are
// uniform) to all R outputs. Partial sums run in int32 for F = 2^(31 - PB -
// log2 J) values of jl (each adds at most J terms below 2^PB per output) and
// are then folded into the int64 totals.
template <int NP, int PB, int R, int J>
__device__ __forceinline__ void window_product(const int32_t *ext, const uint32_t *cs, uint32_t n,
                                               uint32_t i0, int64_t (&acc)[NP][R]) {
  constexpr int W = R + J - 1;
  constexpr int kLogJ = J == 16 ? 4 : J == 8 ? 3 : J == 4 ? 2 : J == 2 ? 1 : 0;
  constexpr int F = 1 << (31 - PB - kLogJ);
  static_assert(31 - PB - kLogJ >= 0, "partial sums must fit an int32");
  static_assert((1 << kLogJ) == J, "J is a power of two up to 16");
  int32_t a32[NP][R];
#pragma unroll
  for (int p = 0; p < NP; ++p)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[p][r] = 0, a32[p][r] = 0;
  const int32_t *base = ext + n + i0 - kBlock * (J - 1);
  for (int jl0 = 0; jl0 < kBlock; jl0 += F) {
    const int jend = jl0 + F < kBlock ? jl0 + F : kBlock;
#pragma unroll 1
    for (int jl = jl0; jl < jend; ++jl) {
      const uint32_t c = cs[jl];
      if (c == 0) continue;
      int32_t w[NP][W];
#pragma unroll
      for (int p = 0; p < NP; ++p)
#pragma unroll
        for (int d = 0; d < W; ++d) w[p][d] = base[2 * n * p - jl + kBlock * d];
#pragma unroll
      for (int jh = 0; jh < J; ++jh) {
        const uint32_t cc = (c >> (2 * jh)) & 3u;
        if (cc == 1u) {
#pragma unroll
          for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int r = 0; r < R; ++r) a32[p][r] += w[p][r - jh + J - 1];
        } else if (cc == 2u) {
#pragma unroll
          for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int r = 0; r < R; ++r) a32[p][r] -= w[p][r - jh + J - 1];
        }
      }
    }
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
      for (int r = 0; r < R; ++r) acc[p][r] += a32[p][r], a32[p][r] = 0;
  }
}

// sum_p acc[p] 2^(PB p) mod m, canonical.
template <int NP, int PB, int R>
__device__ __forceinline__ uint64_t reduce_parts(const int64_t (&acc)[NP][R], int r, uint64_t m) {
  __int128 v = acc[NP - 1][r];
#pragma unroll
  for (int p = NP - 2; p >= 0; --p) v = v * (static_cast<__int128>(1) << PB) + acc[p][r];
  __int128 x = v % static_cast<__int128>(m);
  if (x < 0) x += m;
  return static_cast<uint64_t>(x);
}

// Constants of the decryption epilogue. When sq t < 2^63 every product fits
// 64 bits and the divisions use Barrett reciprocals mu = floor(2^64 / d):
// mulhi(x, mu) is floor(x / d) or one less (x mu / 2^64 lies in (x/d - 1,
// x/d]), so one correction makes it exact; otherwise (wide) 128-bit division.
struct DecConst {
  uint64_t sq, t, mu_sq, mu_t;
  double inv_sq, inv_t;  // 1/sq, 1/t (wide form)
  uint32_t wide, pad;
};

// floor(x / d) for x < 2^104 whose quotient is below 2^52: the double
// estimate x (1/d) carries a relative error of a few 2^-53, so it is off by
// at most a small integer, which the exact remainder x - q d corrects
// (long division by an estimated reciprocal with integer correction).
__device__ __forceinline__ uint64_t div_est(unsigned __int128 x, uint64_t d, double inv_d) {
  const double xd = static_cast<double>(static_cast<uint64_t>(x >> 64)) * 18446744073709551616.0 +
                    static_cast<double>(static_cast<uint64_t>(x));
  double qd = xd * inv_d;
  uint64_t q = qd <= 0.0 ? 0 : static_cast<uint64_t>(qd);
  __int128 r = static_cast<__int128>(x) - static_cast<__int128>(static_cast<unsigned __int128>(q) * d);
  for (int it = 0; it < 4 && r < 0; ++it) { --q; r += d; }
  for (int it = 0; it < 4 && r >= static_cast<__int128>(d); ++it) { ++q; r -= d; }
  return q;
}

// v mod q (canonical) for |v| < 2^104 with |v| / q below 2^52.
__device__ __forceinline__ uint64_t mod_est(__int128 v, uint64_t q, double inv_q) {
  const bool neg = v < 0;
  const unsigned __int128 a = static_cast<unsigned __int128>(neg ? -v : v);
  const uint64_t r = static_cast<uint64_t>(a - static_cast<unsigned __int128>(div_est(a, q, inv_q)) * q);
  return neg && r ? q - r : r;
}

__device__ __forceinline__ uint64_t div_barrett(uint64_t x, uint64_t d, uint64_t mu) {
  uint64_t q = __umul64hi(x, mu);
  if (x - q * d >= d) ++q;
  return q;
}

// decrypt_mod_q of one coefficient from prod = (c1 s mod sq): pt =
// round((c0 + prod mod sq) t / sq) mod t; *worst tracks the max noise
// |phase - round(sq m / t)| the reference reports as its noise budget
// (client.cpp:389-407).
__device__ __forceinline__ uint64_t decrypt_coeff(uint64_t prod, uint64_t c0, const DecConst &dc,
                                                  uint64_t &worst) {
  const uint64_t sq = dc.sq, t = dc.t;
  uint64_t m, approx, phase;
  if (!dc.wide) {
    phase = prod + (c0 - div_barrett(c0, sq, dc.mu_sq) * sq);
    if (phase >= sq) phase -= sq;
    m = div_barrett(phase * t + (sq >> 1), sq, dc.mu_sq);
    if (m >= t) m -= t;
    approx = div_barrett(sq * m + (t >> 1), t, dc.mu_t);
    if (approx >= sq) approx -= sq;
  } else {
    phase = prod + c0 % sq;
    if (phase >= sq) phase -= sq;
    m = div_est(static_cast<unsigned __int128>(phase) * t + (sq >> 1), sq, dc.inv_sq);
    if (m >= t) m -= t;
    approx = div_est(static_cast<unsigned __int128>(sq) * m + (t >> 1), t, dc.inv_t);
    if (approx >= sq) approx -= sq;
  }
  const uint64_t pos = phase >= approx ? phase - approx : sq - approx + phase;
  const uint64_t nabs = pos > (sq >> 1) ? sq - pos : pos;
  worst = nabs > worst ? nabs : worst;
  return m;
}

__device__ __forceinline__ void publish_noise(uint64_t worst, unsigned long long *max_noise) {
  if (!max_noise) return;
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t w = __shfl_xor_sync(0xFFFFFFFFu, worst, o);
    worst = w > worst ? w : worst;
  }
  if ((threadIdx.x & 31) == 0)
    atomicMax(max_noise + blockIdx.x, static_cast<unsigned long long>(worst));
}

// c0 of one coefficient: -(prod + e) mod q (prod = a s mod q, e any int64).
__device__ __forceinline__ uint64_t pack_coeff(uint64_t prod, int64_t ei, uint64_t q) {
  const uint64_t em = ei >= 0 ? static_cast<uint64_t>(ei) % q
                              : (q - static_cast<uint64_t>(-(ei + 1)) % q - 1);
  uint64_t v = prod + em;
  if (v >= q) v -= q;
  return v ? q - v : 0;
}

// The query's plaintext constants that fall in this CTA's output slice
// [o0, o0 + span), after every thread's c0 store (caller synchronises).
__device__ __forceinline__ void add_constants(const ConstEntry *ce, uint32_t nconst, uint32_t limb,
                                              uint32_t o0, uint32_t span, uint64_t q,
                                              uint64_t *c0) {
  for (uint32_t u = threadIdx.x; u < nconst; u += blockDim.x) {
    const uint32_t pos = ce[u].pos;
    if (pos == kNoPos || pos < o0 || pos >= o0 + span) continue;
    const uint64_t v = c0[pos] + ce[u].val[limb];
    c0[pos] = v >= q ? v - q : v;
  }
}

// decrypt_mod_q for response blockIdx.x, output slice blockIdx.y: index-list
// product (any batch) with 31-bit parts.
template <int NP, int R>
__global__ void __launch_bounds__(kBlock) k_client_decrypt(
    const uint64_t *__restrict__ resp, const uint16_t *__restrict__ sidx, uint32_t npos,
    uint32_t nneg, uint32_t n, DecConst dc, uint64_t *__restrict__ pt,
    unsigned long long *__restrict__ max_noise) {
  const uint64_t sq = dc.sq;
  extern __shared__ __align__(16) int32_t smem[];
  int32_t *ext = smem;
  uint16_t *sl = reinterpret_cast<uint16_t *>(smem + NP * 2 * n);
  const uint64_t b = blockIdx.x;
  const uint64_t *c0 = resp + b * 2 * n, *c1 = c0 + n;
  stage_ext<NP, 31>(c1, sq, n, ext);
  for (uint32_t u = threadIdx.x; u < npos + nneg; u += blockDim.x) sl[u] = sidx[u];
  __syncthreads();
  const uint32_t i0 = blockIdx.y * (n / gridDim.y) + threadIdx.x;
  int64_t acc[NP][R];
  list_product<NP, R>(ext, sl, npos, nneg, n, i0, acc);
  uint64_t worst = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t i = i0 + kBlock * r;
    pt[b * n + i] = decrypt_coeff(reduce_parts<NP, 31, R>(acc, r, sq), c0[i], dc, worst);
  }
  publish_noise(worst, max_noise);
}

// The same with the window product (n = kBlock J, PB-bit parts).
template <int NP, int PB, int R, int J>
__global__ void __launch_bounds__(kBlock) k_client_decrypt_w(
    const uint64_t *__restrict__ resp, const uint32_t *__restrict__ code, uint32_t n, DecConst dc,
    uint64_t *__restrict__ pt, unsigned long long *__restrict__ max_noise) {
  const uint64_t sq = dc.sq;
  extern __shared__ __align__(16) int32_t smem[];
  int32_t *ext = smem;
  uint32_t *cs = reinterpret_cast<uint32_t *>(smem + NP * 2 * n);
  const uint64_t b = blockIdx.x;
  const uint64_t *c0 = resp + b * 2 * n, *c1 = c0 + n;
  stage_ext<NP, PB>(c1, sq, n, ext);
  for (uint32_t u = threadIdx.x; u < kBlock; u += blockDim.x) cs[u] = code[u];
  __syncthreads();
  const uint32_t i0 = blockIdx.y * (n / gridDim.y) + threadIdx.x;
  int64_t acc[NP][R];
  window_product<NP, PB, R, J>(ext, cs, n, i0, acc);
  uint64_t worst = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t i = i0 + kBlock * r;
    pt[b * n + i] = decrypt_coeff(reduce_parts<NP, PB, R>(acc, r, sq), c0[i], dc, worst);
  }
  publish_noise(worst, max_noise);
}

// fast_generate_query for item = (query, limb) = blockIdx.x, output slice
// blockIdx.y: c0 = -(a s + e) mod q_k plus the query's plaintext constants,
// c1 = a as given. a and the output are limb-major per query: a [K n], out
// [c0 (K n)][c1 (K n)]. Index-list product with 31-bit parts.
template <int R>
__global__ void __launch_bounds__(kBlock) k_client_pack(
    const uint64_t *__restrict__ a, const int64_t *__restrict__ e,
    const ConstEntry *__restrict__ consts, uint32_t nconst, const uint16_t *__restrict__ sidx,
    uint32_t npos, uint32_t nneg, uint32_t n, uint32_t limbs, uint64_t q0, uint64_t q1,
    uint64_t *__restrict__ out) {
  extern __shared__ __align__(16) int32_t smem[];
  int32_t *ext = smem;
  uint16_t *sl = reinterpret_cast<uint16_t *>(smem + 2 * 2 * n);
  const uint64_t query = blockIdx.x / limbs;
  const uint32_t limb = blockIdx.x % limbs;
  const uint64_t q = limb ? q1 : q0;
  const uint64_t kn = static_cast<uint64_t>(limbs) * n;
  const uint64_t *x = a + query * kn + static_cast<uint64_t>(limb) * n;
  stage_ext<2, 31>(x, q, n, ext);
  for (uint32_t u = threadIdx.x; u < npos + nneg; u += blockDim.x) sl[u] = sidx[u];
  __syncthreads();
  const uint32_t span = n / gridDim.y, o0 = blockIdx.y * span;
  const uint32_t i0 = o0 + threadIdx.x;
  int64_t acc[2][R];
  list_product<2, R>(ext, sl, npos, nneg, n, i0, acc);
  uint64_t *c0 = out + query * 2 * kn + static_cast<uint64_t>(limb) * n;
  uint64_t *c1 = c0 + kn;
  const int64_t *eq = e + query * n;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t i = i0 + kBlock * r;
    c0[i] = pack_coeff(reduce_parts<2, 31, R>(acc, r, q), eq[i], q);
    c1[i] = x[i];
  }
  __syncthreads();
  add_constants(consts + query * nconst, nconst, limb, o0, span, q, c0);
}

// One ciphertext row of the client's session keys (create_session_keys,
// client.cpp:40-45), before the NTT: c0 = -(a s) + esign e + [half = 0] msg,
// c1 = a + [half = 1] msg, msg = scale_k * m for a ternary polynomial m (s for
// the RGSW rows, sigma_k(s) for the BV rows).
struct KeyRow {
  const uint64_t *a;  // K n, coefficient form, limb k below q_k
  const int64_t *e;   // n
  uint64_t *out;      // [c0 (K n)][c1 (K n)]
  uint32_t msg;       // ternary message polynomial: 0 = s, 1 + i = sigma_{N/2^i + 1}(s)
  uint32_t half;      // message in c0 (0) or c1 (1)
  int32_t esign;      // +1: BV row (b = msg - a s + e), -1: encryption of zero
  uint32_t pad;
  uint64_t scale[2];  // message scale per limb, below q_k
};

__device__ __forceinline__ uint64_t signed_mod(int64_t v, uint64_t q) {
  return v >= 0 ? static_cast<uint64_t>(v) % q : (q - static_cast<uint64_t>(-(v + 1)) % q - 1);
}

// Coefficient-form key rows, item = (row, limb) = blockIdx.x, output slice
// blockIdx.y; index-list product with 31-bit parts.
template <int R>
__global__ void __launch_bounds__(kBlock) k_client_keyrows(
    const KeyRow *__restrict__ rows, const int8_t *__restrict__ msgs,
    const uint16_t *__restrict__ sidx, uint32_t npos, uint32_t nneg, uint32_t n, uint32_t limbs,
    uint64_t q0, uint64_t q1) {
  extern __shared__ __align__(16) int32_t smem[];
  int32_t *ext = smem;
  uint16_t *sl = reinterpret_cast<uint16_t *>(smem + 2 * 2 * n);
  const KeyRow row = rows[blockIdx.x / limbs];
  const uint32_t limb = blockIdx.x % limbs;
  const uint64_t q = limb ? q1 : q0;
  const uint64_t kn = static_cast<uint64_t>(limbs) * n;
  const uint64_t *x = row.a + static_cast<uint64_t>(limb) * n;
  stage_ext<2, 31>(x, q, n, ext);
  for (uint32_t u = threadIdx.x; u < npos + nneg; u += blockDim.x) sl[u] = sidx[u];
  __syncthreads();
  const uint32_t i0 = blockIdx.y * (n / gridDim.y) + threadIdx.x;
  int64_t acc[2][R];
  list_product<2, R>(ext, sl, npos, nneg, n, i0, acc);
  uint64_t *c0 = row.out + static_cast<uint64_t>(limb) * n;
  uint64_t *c1 = c0 + kn;
  const int8_t *m = msgs + static_cast<uint64_t>(row.msg) * n;
  const uint64_t sc = row.scale[limb];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t i = i0 + kBlock * r;
    const uint64_t prod = reduce_parts<2, 31, R>(acc, r, q);
    const uint64_t em = signed_mod(row.e[i], q);
    const uint64_t term = m[i] == 1 ? sc : (m[i] == -1 && sc ? q - sc : 0);
    uint64_t v = prod ? q - prod : 0;                        // -(a s)
    if (row.esign > 0) {
      v += em;
      if (v >= q) v -= q;
    } else {
      v = v >= em ? v - em : v + (q - em);
    }
    uint64_t w = x[i] % q;
    if (row.half == 0) {
      v += term;
      if (v >= q) v -= q;
    } else {
      w += term;
      if (w >= q) w -= q;
    }
    c0[i] = v;
    c1[i] = w;
  }
}

// In-place forward negacyclic NTT of polynomial blockIdx.x (limb = index % K)
// in the reference's convention: Cooley-Tukey from natural order, output in
// bit-reversed order, twiddle at butterfly group m + i = root^BitRev(m + i)
// (fw, per limb), every value canonical in [0, q).
__global__ void __launch_bounds__(kBlock) k_client_ntt(uint64_t *__restrict__ polys, uint32_t n,
                                                       uint32_t limbs, const uint64_t *__restrict__ fw,
                                                       uint64_t q0, uint64_t q1) {
  extern __shared__ __align__(16) uint64_t sp[];
  const uint32_t limb = blockIdx.x % limbs;
  const uint64_t q = limb ? q1 : q0;
  const uint64_t *w = fw + static_cast<uint64_t>(limb) * n;
  uint64_t *a = polys + static_cast<uint64_t>(blockIdx.x) * n;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sp[i] = a[i];
  __syncthreads();
  for (uint32_t m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1) {
    for (uint32_t b = threadIdx.x; b < n / 2; b += blockDim.x) {
      const uint32_t g = b / t, j = b % t;
      const uint32_t xi = 2 * g * t + j, yi = xi + t;
      const uint64_t u = sp[xi];
      const uint64_t v = static_cast<uint64_t>(static_cast<unsigned __int128>(sp[yi]) * w[m + g] % q);
      const uint64_t s = u + v;
      sp[xi] = s >= q ? s - q : s;
      sp[yi] = u >= v ? u - v : u + (q - v);
    }
    __syncthreads();
  }
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) a[i] = sp[i];
}

// Tensor-core decryption (single-modulus set, small_q < 2^29): (c1 s)_i =
// sum_j S[i][j] x_j with S[i][j] = s[i - j] (i >= j) or -s[N + i - j], so with
// A = S + 1 (entries 0, 1, 2: one unsigned byte plane) y = A x - sum_j x_j.
// A x mod small_q is the tensor-core scan (opir_scan_tc.h) with one residue
// and one level: A [4 planes (1..3 zero)][N rows][N bytes], x as the four byte
// planes of each response's c1 mod small_q, Q [4][n][N].
__global__ void __launch_bounds__(kBlock) k_client_secret_matrix(const int8_t *__restrict__ s,
                                                                 uint32_t n,
                                                                 uint8_t *__restrict__ a) {
  const uint32_t i = blockIdx.x;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const int v = i >= j ? s[i - j] : -s[n + i - j];
    a[static_cast<uint64_t>(i) * n + j] = static_cast<uint8_t>(v + 1);
  }
}

// Q planes and sum_j x_j mod small_q of response blockIdx.x.
__global__ void __launch_bounds__(kBlock) k_client_tc_prep(const uint64_t *__restrict__ resp,
                                                           uint32_t n, uint32_t nresp, uint64_t sq,
                                                           uint8_t *__restrict__ qpl,
                                                           uint64_t *__restrict__ colsum) {
  __shared__ uint64_t part[kBlock / 32];
  const uint64_t b = blockIdx.x;
  const uint64_t *c1 = resp + b * 2 * n + n;
  uint64_t sum = 0;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint64_t x = c1[j] % sq;
    sum += x;
#pragma unroll
    for (int pl = 0; pl < 4; ++pl)
      qpl[(static_cast<uint64_t>(pl) * nresp + b) * n + j] = static_cast<uint8_t>(x >> (8 * pl));
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
    for (int w = 0; w < kBlock / 32; ++w) t += part[w];
    colsum[b] = t % sq;
  }
}

// Two-limb decryption (small_q < 2^50): x = c1 mod small_q splits into 25-bit
// halves; A x_half < 2 N 2^25 <= 2^38 is exact from its residues mod two
// primes P1 P2 > 2^38 (four scans). Planes [half][4][nr][n], sums [half][nr].
__global__ void __launch_bounds__(kBlock) k_client_tc_prep_split(const uint64_t *__restrict__ resp,
                                                                 uint32_t n, uint32_t nr,
                                                                 uint64_t sq,
                                                                 uint8_t *__restrict__ qpl,
                                                                 uint64_t *__restrict__ colsum) {
  __shared__ uint64_t part[2][kBlock / 32];
  const uint64_t b = blockIdx.x;
  const uint64_t *c1 = resp + b * 2 * n + n;
  const uint64_t plane = static_cast<uint64_t>(nr) * n;
  uint64_t sum[2] = {0, 0};
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint64_t x = c1[j] % sq;
    const uint64_t h[2] = {x & ((1ull << 25) - 1), x >> 25};
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      sum[hf] += h[hf];
#pragma unroll
      for (int pl = 0; pl < 4; ++pl)
        qpl[(4ull * hf + pl) * plane + b * n + j] = static_cast<uint8_t>(h[hf] >> (8 * pl));
    }
  }
#pragma unroll
  for (int hf = 0; hf < 2; ++hf) {
    for (int o = 16; o > 0; o >>= 1) sum[hf] += __shfl_xor_sync(0xFFFFFFFFu, sum[hf], o);
    if ((threadIdx.x & 31) == 0) part[hf][threadIdx.x >> 5] = sum[hf];
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    uint64_t tot = 0;
    for (int w = 0; w < kBlock / 32; ++w) tot += part[threadIdx.x][w];
    colsum[static_cast<uint64_t>(threadIdx.x) * nr + b] = tot;
  }
}

// pt from the four scans ax [half][prime][nr][n]: u_half = CRT(mod P1, mod
// P2) = A x_half exactly, y = (u_lo - sum_lo) + 2^25 (u_hi - sum_hi) = c1 s
// (|y| < 2^62), then the decryption epilogue on y mod small_q.
__global__ void __launch_bounds__(kBlock) k_client_tc_finish_split(
    const uint64_t *__restrict__ resp, const uint32_t *__restrict__ ax,
    const uint64_t *__restrict__ colsum, uint32_t n, uint32_t nr, uint64_t p1, uint64_t p2,
    uint64_t p1_inv_mod_p2, DecConst dc, uint64_t *__restrict__ pt,
    unsigned long long *__restrict__ max_noise) {
  const uint64_t b = blockIdx.x;
  const uint64_t *c0 = resp + b * 2 * n;
  const uint64_t plane = static_cast<uint64_t>(nr) * n;
  uint64_t worst = 0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    int64_t y[2];
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      const uint64_t v1 = ax[(2ull * hf) * plane + b * n + i];
      const uint64_t v2 = ax[(2ull * hf + 1) * plane + b * n + i];
      const uint64_t v1m = v1 >= p2 ? v1 - p2 : v1;  // p1 < 2 p2
      const uint64_t d = v2 >= v1m ? v2 - v1m : v2 + (p2 - v1m);
      const uint64_t u = v1 + p1 * (d * p1_inv_mod_p2 % p2);
      y[hf] = static_cast<int64_t>(u) - static_cast<int64_t>(colsum[static_cast<uint64_t>(hf) * nr + b]);
    }
    const int64_t v = y[0] + y[1] * (int64_t{1} << 25);
    const int64_t r = v % static_cast<int64_t>(dc.sq);
    const uint64_t prod = static_cast<uint64_t>(r < 0 ? r + static_cast<int64_t>(dc.sq) : r);
    pt[b * n + i] = decrypt_coeff(prod, c0[i], dc, worst);
  }
  publish_noise(worst, max_noise);
}

// pt from the scan's (A x mod small_q), laid out [response][i].
__global__ void __launch_bounds__(kBlock) k_client_tc_finish(
    const uint64_t *__restrict__ resp, const uint32_t *__restrict__ ax,
    const uint64_t *__restrict__ colsum, uint32_t n, DecConst dc,
    uint64_t *__restrict__ pt, unsigned long long *__restrict__ max_noise) {
  const uint64_t sq = dc.sq;
  const uint64_t b = blockIdx.x;
  const uint64_t *c0 = resp + b * 2 * n;
  const uint64_t cs = colsum[b];
  uint64_t worst = 0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint64_t v = ax[b * n + i];
    const uint64_t prod = v >= cs ? v - cs : v + (sq - cs);
    pt[b * n + i] = decrypt_coeff(prod, c0[i], dc, worst);
  }
  publish_noise(worst, max_noise);
}

// Tensor-core packing (single-modulus set, q = q1 q2): a s mod q is the CRT
// of a s mod q1 and mod q2, each the scan of the same A = S + 1 against the
// byte planes of a mod q_r. Planes [r][4][nq][n], sums [r][nq].
__global__ void __launch_bounds__(kBlock) k_client_tc_pack_prep(const uint64_t *__restrict__ a,
                                                                uint32_t n, uint32_t nq,
                                                                uint64_t q1, uint64_t q2,
                                                                uint8_t *__restrict__ qpl,
                                                                uint64_t *__restrict__ colsum) {
  __shared__ uint64_t part[2][kBlock / 32];
  const uint64_t b = blockIdx.x;
  const uint64_t *x = a + b * n;
  uint64_t sum[2] = {0, 0};
  const uint64_t plane = static_cast<uint64_t>(nq) * n;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint64_t r[2] = {x[j] % q1, x[j] % q2};
#pragma unroll
    for (int res = 0; res < 2; ++res) {
      sum[res] += r[res];
#pragma unroll
      for (int pl = 0; pl < 4; ++pl)
        qpl[(4ull * res + pl) * plane + b * n + j] = static_cast<uint8_t>(r[res] >> (8 * pl));
    }
  }
#pragma unroll
  for (int res = 0; res < 2; ++res) {
    for (int o = 16; o > 0; o >>= 1) sum[res] += __shfl_xor_sync(0xFFFFFFFFu, sum[res], o);
    if ((threadIdx.x & 31) == 0) part[res][threadIdx.x >> 5] = sum[res];
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    uint64_t tot = 0;
    for (int w = 0; w < kBlock / 32; ++w) tot += part[threadIdx.x][w];
    colsum[static_cast<uint64_t>(threadIdx.x) * nq + b] = tot % (threadIdx.x ? q2 : q1);
  }
}

// What the device needs to place a query's plaintext constants itself.
struct PackLayout {
  uint64_t n0, other;      // first-dimension size, rows
  uint32_t num_dims, h;    // dimensions, expansion height
  uint32_t l_ep, pad;
  uint64_t one[2];         // the one-hot's value per limb
  uint64_t gadget[16][2];  // B^(L_EP-1-k) (2^h)^-1 mod q_limb
};

__device__ __forceinline__ uint32_t bitrev_dev(uint64_t x, uint32_t bits) {
  return bits ? static_cast<uint32_t>(__brevll(x) >> (64 - bits)) : 0u;
}

// get_query_indices (src/client.cpp:48-98) for selector bit i >= 1 of index
// idx: the leaf's parity on the incomplete last level, then the perfect-tree
// path MSB first.
__device__ __forceinline__ uint32_t selector_bit(const PackLayout &L, uint64_t idx, uint32_t i) {
  const uint64_t row = idx / L.n0;
  const uint64_t hd = L.num_dims - 1;
  const uint64_t r = 2 * L.other - (1ull << hd), sl = L.other - r;
  uint64_t perfect, first;
  if (row < sl) {
    first = 0;
    perfect = row;
  } else {
    first = (row - sl) % 2;
    perfect = sl + (row - sl) / 2;
  }
  return static_cast<uint32_t>(i == 1 ? first : (perfect >> (hd - i)) & 1ull);
}

// c0 = -(a s + e) mod q plus the query's constants, c1 = a, from the two
// scans' (A x_r mod q_r) [r][nq][n]: y_r = A x_r - sum_j x_r,j mod q_r, then
// Garner: a s mod q = y_1 + q1 ((y_2 - y_1) q1^-1 mod q2). The constants
// (client.cpp:128-225) are placed from the index: the one-hot at
// BitRev(col, h), and for each set selector bit i the L_EP gadget rows at
// BitRev(N0 + (i-1) L_EP + k, h).
__global__ void __launch_bounds__(kBlock) k_client_tc_pack_finish(
    const uint64_t *__restrict__ a, const int64_t *__restrict__ e,
    const uint64_t *__restrict__ pt_idx, PackLayout L, const uint32_t *__restrict__ ax,
    const uint64_t *__restrict__ colsum, uint32_t n, uint32_t nq, uint64_t q1, uint64_t q2,
    uint64_t q1_inv_mod_q2, uint64_t *__restrict__ out) {
  const uint64_t b = blockIdx.x, q = q1 * q2;
  const uint64_t cs1 = colsum[b], cs2 = colsum[static_cast<uint64_t>(nq) + b];
  const uint32_t *ax1 = ax + b * n, *ax2 = ax + (static_cast<uint64_t>(nq) + b) * n;
  uint64_t *c0 = out + b * 2 * n, *c1 = c0 + n;
  const uint64_t *x = a + b * n;
  const int64_t *eq = e + b * n;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const uint64_t v1 = ax1[i], v2 = ax2[i];
    const uint64_t y1 = v1 >= cs1 ? v1 - cs1 : v1 + (q1 - cs1);
    const uint64_t y2 = v2 >= cs2 ? v2 - cs2 : v2 + (q2 - cs2);
    const uint64_t y1m = y1 >= q2 ? y1 - q2 : y1;  // q1 < 2 q2
    const uint64_t d = y2 >= y1m ? y2 - y1m : y2 + (q2 - y1m);
    const uint64_t k = d * q1_inv_mod_q2 % q2;
    c0[i] = pack_coeff(y1 + q1 * k, eq[i], q);
    c1[i] = x[i];
  }
  __syncthreads();
  const uint64_t idx = pt_idx[b];
  const uint32_t nconst = 1 + (L.num_dims - 1) * L.l_ep;
  for (uint32_t u = threadIdx.x; u < nconst; u += blockDim.x) {
    uint32_t pos;
    uint64_t val;
    if (u == 0) {
      pos = bitrev_dev(idx % L.n0, L.h);
      val = L.one[0];
    } else {
      const uint32_t i = 1 + (u - 1) / L.l_ep, k = (u - 1) % L.l_ep;
      if (!selector_bit(L, idx, i)) continue;
      pos = bitrev_dev(L.n0 + static_cast<uint64_t>(i - 1) * L.l_ep + k, L.h);
      val = L.gadget[k][0];
    }
    const uint64_t v = c0[pos] + val;
    c0[pos] = v >= q ? v - q : v;
  }
}

// Two-limb packing: every (query, limb) is one column x = a_limb mod q_limb
// (< 2^60), split into 30-bit halves; A x_half < 2 N 2^30 <= 2^43 comes back
// exactly from its residues mod P1 and P2. Planes [half][4][cols][n], sums
// [half][cols], cols = queries x 2.
__global__ void __launch_bounds__(kBlock) k_client_tc_pack_prep_split(
    const uint64_t *__restrict__ a, uint32_t n, uint32_t cols, uint64_t q0, uint64_t q1,
    uint8_t *__restrict__ qpl, uint64_t *__restrict__ colsum) {
  __shared__ uint64_t part[2][kBlock / 32];
  const uint64_t col = blockIdx.x;
  const uint64_t q = (col & 1) ? q1 : q0;
  const uint64_t *x = a + col * n;
  const uint64_t plane = static_cast<uint64_t>(cols) * n;
  uint64_t sum[2] = {0, 0};
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    const uint64_t v = x[j] % q;
    const uint64_t h[2] = {v & ((1ull << 30) - 1), v >> 30};
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      sum[hf] += h[hf];
#pragma unroll
      for (int pl = 0; pl < 4; ++pl)
        qpl[(4ull * hf + pl) * plane + col * n + j] = static_cast<uint8_t>(h[hf] >> (8 * pl));
    }
  }
#pragma unroll
  for (int hf = 0; hf < 2; ++hf) {
    for (int o = 16; o > 0; o >>= 1) sum[hf] += __shfl_xor_sync(0xFFFFFFFFu, sum[hf], o);
    if ((threadIdx.x & 31) == 0) part[hf][threadIdx.x >> 5] = sum[hf];
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    uint64_t tot = 0;
    for (int w = 0; w < kBlock / 32; ++w) tot += part[threadIdx.x][w];
    colsum[static_cast<uint64_t>(threadIdx.x) * cols + col] = tot;
  }
}

// Query blockIdx.x: per limb k, a_k s = (A x_lo - sum_lo) + 2^30 (A x_hi -
// sum_hi) (|.| < 2^73, 128-bit) mod q_k, c0 = -(a_k s + e) plus the constants
// placed from the index, c1 = a.
__global__ void __launch_bounds__(kBlock) k_client_tc_pack_finish_split(
    const uint64_t *__restrict__ a, const int64_t *__restrict__ e,
    const uint64_t *__restrict__ pt_idx, PackLayout L, const uint32_t *__restrict__ ax,
    const uint64_t *__restrict__ colsum, uint32_t n, uint32_t cols, uint64_t p1, uint64_t p2,
    uint64_t p1_inv_mod_p2, uint64_t q0, uint64_t q1, double inv_q0, double inv_q1,
    uint64_t *__restrict__ out) {
  const uint64_t b = blockIdx.x;
  const uint64_t plane = static_cast<uint64_t>(cols) * n;
  uint64_t *c0 = out + b * 4 * n, *c1 = c0 + 2 * n;
  const int64_t *eq = e + b * n;
  for (uint32_t w = threadIdx.x; w < 2 * n; w += blockDim.x) {
    const uint32_t k = w / n, i = w % n;
    const uint64_t col = 2 * b + k, q = k ? q1 : q0;
    __int128 y[2];
#pragma unroll
    for (int hf = 0; hf < 2; ++hf) {
      const uint64_t v1 = ax[(2ull * hf) * plane + col * n + i];
      const uint64_t v2 = ax[(2ull * hf + 1) * plane + col * n + i];
      const uint64_t v1m = v1 >= p2 ? v1 - p2 : v1;
      const uint64_t d = v2 >= v1m ? v2 - v1m : v2 + (p2 - v1m);
      const uint64_t u = v1 + p1 * (d * p1_inv_mod_p2 % p2);
      y[hf] = static_cast<__int128>(u) - static_cast<__int128>(colsum[static_cast<uint64_t>(hf) * cols + col]);
    }
    const uint64_t v = mod_est(y[0] + y[1] * (static_cast<__int128>(1) << 30), q,
                               k ? inv_q1 : inv_q0);
    c0[w] = pack_coeff(v, eq[i], q);
    c1[w] = a[col * n + i];
  }
  __syncthreads();
  const uint64_t idx = pt_idx[b];
  const uint32_t nconst = 1 + (L.num_dims - 1) * L.l_ep;
  for (uint32_t u = threadIdx.x; u < 2 * nconst; u += blockDim.x) {
    const uint32_t k = u / nconst, cu = u % nconst;
    const uint64_t q = k ? q1 : q0;
    uint32_t pos;
    uint64_t val;
    if (cu == 0) {
      pos = bitrev_dev(idx % L.n0, L.h);
      val = L.one[k];
    } else {
      const uint32_t i = 1 + (cu - 1) / L.l_ep, r = (cu - 1) % L.l_ep;
      if (!selector_bit(L, idx, i)) continue;
      pos = bitrev_dev(L.n0 + static_cast<uint64_t>(i - 1) * L.l_ep + r, L.h);
      val = L.gadget[r][k];
    }
    uint64_t *cell = c0 + static_cast<uint64_t>(k) * n + pos;
    const uint64_t s2 = *cell + val;
    *cell = s2 >= q ? s2 - q : s2;
  }
}


uint64_t bitrev(uint64_t x, uint32_t bits) {
  uint64_t r = 0;
  for (uint32_t i = 0; i < bits; ++i) r |= ((x >> i) & 1ull) << (bits - 1 - i);
  return r;
}

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) {
  return static_cast<uint64_t>(static_cast<unsigned __int128>(a) * b % m);
}

}  // namespace

struct opir_client {
  opir_params params{};
  int device = 0;
  int sms = 148;
  uint32_t n = 0, limbs = 1;
  uint64_t mods[2]{};        // ciphertext moduli: the logical q (K = 1) or the two limbs
  DevBuf<uint16_t> sidx;     // [P | M] secret index lists
  uint32_t npos = 0, nneg = 0;
  DevBuf<uint32_t> code;     // [kBlock]: s[jl + kBlock jh] 2 bits each (window product)
  DevBuf<int8_t> msgs;       // [1 + h][n]: s, then sigma_{N/2^i + 1}(s) for i < h
  DevBuf<uint64_t> fw;       // [K][n]: forward NTT twiddles per limb
  DevBuf<KeyRow> keyrows;
  // tensor-core decryption: A = S + 1 (built on first use), per-call scratch
  DevBuf<uint8_t> tc_a, tc_q;
  DevBuf<uint64_t> tc_colsum, pk_colsum;
  DevBuf<uint32_t> tc_ax, tc_err, pk_ax;
  DevBuf<uint8_t> pk_q;
  DevBuf<uint64_t> pk_idx;
  uint64_t *idx_staging = nullptr;   // pinned copy of the last call's indices
  size_t idx_staging_cap = 0;
  // host-buffer calls: the handle's stream and device copies of their buffers
  cudaStream_t io_stream = nullptr;
  DevBuf<uint64_t> io_u0, io_u1, io_out, io_noise;
  DevBuf<int64_t> io_e0, io_e1;
  uint32_t nconst = 1;       // constant slots per query
  uint64_t one_val[2]{};     // the one-hot's value per limb
  std::vector<uint64_t> gadget_val;  // [k][limb]: B^(L_EP-1-k) (2^h)^-1 mod q_limb
  DevBuf<ConstEntry> consts;
  ConstEntry *staging = nullptr;     // pinned host copy of the last call's constants
  size_t staging_cap = 0;
  cudaEvent_t staged = nullptr;      // that copy has been consumed
  std::string last_error;
};

namespace {

template <typename F>
opir_status client_guarded(opir_client *c, F &&f) {
  std::string msg;
  opir_status st = OPIR_OK;
  try {
    f();
  } catch (const std::invalid_argument &e) {
    st = OPIR_ERR_INVALID_ARGUMENT, msg = e.what();
  } catch (const std::out_of_range &e) {
    st = OPIR_ERR_OUT_OF_RANGE, msg = e.what();
  } catch (const std::bad_alloc &) {
    st = OPIR_ERR_NO_MEMORY, msg = "device or host allocation failed";
  } catch (const opir::CudaError &e) {
    cudaGetLastError();
    st = OPIR_ERR_CUDA, msg = e.what();
  } catch (const std::exception &e) {
    cudaGetLastError();
    st = OPIR_ERR_RUNTIME, msg = e.what();
  } catch (...) {
    st = OPIR_ERR_RUNTIME, msg = "unknown error";
  }
  if (c) c->last_error = msg;
  return st;
}

// The layout must be one opir_params_init[_config] produces.
opir_params checked_layout(const opir_params &p) {
  const bool c4 = p.num_limbs == 2 && p.poly_degree == 4096;
  if (!c4 && !(p.num_limbs == 1 && p.poly_degree == 2048 && p.q1 != 0))
    throw std::invalid_argument("unsupported parameter set (CONFIG_N2048_K1_COMP or CONFIG_N4096_K2_MP)");
  if (p.view != OPIR_VIEW_LAYOUT)
    throw std::invalid_argument("a client needs a database layout (opir_params_init[_config])");
  const opir_layout lay{p.target_num_pt, p.expansion_height, p.fst_dim_pow2};
  const opir_params d = c4 ? opir::derive_params_c4(lay) : opir::derive_params(lay);
  if (d.num_pt != p.num_pt || d.q != p.q || d.q1 != p.q1 || d.q2 != p.q2 ||
      d.fst_dim_sz != p.fst_dim_sz || d.num_dims != p.num_dims)
    throw std::invalid_argument("params do not match their layout");
  return d;
}

// get_query_indices (src/client.cpp:48-98): the first-dimension column, then
// one selector bit per further dimension (the leaf's parity on the
// incomplete last level, then the perfect-tree path MSB first).
std::vector<uint64_t> query_indices(const opir_params &p, uint64_t idx) {
  std::vector<uint64_t> out;
  const uint64_t col = idx % p.fst_dim_sz, row = idx / p.fst_dim_sz;
  out.push_back(col);
  if (p.num_dims == 1) return out;
  const uint64_t h = p.num_dims - 1, other = p.other_dim_sz;
  const uint64_t r = 2 * other - (1ull << h), sl = other - r;
  uint64_t perfect;
  if (row < sl) {
    out.push_back(0);
    perfect = row;
  } else {
    const uint64_t corr = row - sl;
    out.push_back(corr % 2);
    perfect = sl + corr / 2;
  }
  for (uint64_t k = h - 1; k-- > 0;) out.push_back((perfect >> k) & 1ull);
  return out;
}

// The values of a query's plaintext constants (client.cpp:128-225), fixed
// per parameter set: the first dimension's one-hot is the BFV lift of
// (2^h)^-1 mod t (under Q = q0 q1 when K = 2, reduced per limb), and selector
// gadget row k is B^(L_EP-1-k) (2^h)^-1 mod q_k.
void prepare_constants(opir_client &c) {
  const opir_params &p = c.params;
  const uint32_t h = p.expansion_height;
  const uint64_t t = p.plain_mod, cap = 1ull << h;
  uint64_t inv_t = 0;
  if (!opir::invert_mod(cap % t, t, inv_t)) throw std::invalid_argument("2^h is not invertible mod t");
  if (c.limbs == 1) {
    const uint64_t q = c.mods[0];
    c.one_val[0] = static_cast<uint64_t>(
        ((static_cast<unsigned __int128>(q) * inv_t + (t >> 1)) / t) % q);
  } else {
    const unsigned __int128 Q = static_cast<unsigned __int128>(c.mods[0]) * c.mods[1];
    const unsigned __int128 delta = Q / t;
    const uint64_t rem = static_cast<uint64_t>(Q - delta * t);
    const uint64_t rem_round =
        static_cast<uint64_t>((static_cast<unsigned __int128>(rem) * inv_t + (t >> 1)) / t);
    const unsigned __int128 scaled = delta * inv_t + rem_round;
    for (uint32_t k = 0; k < 2; ++k) c.one_val[k] = static_cast<uint64_t>(scaled % c.mods[k]);
  }
  c.gadget_val.assign(static_cast<size_t>(p.l_ep) * 2, 0);
  for (uint32_t m = 0; m < c.limbs; ++m) {
    const uint64_t q = c.mods[m];
    uint64_t inv_q = 0;
    if (!opir::invert_mod(cap % q, q, inv_q)) throw std::invalid_argument("2^h is not invertible mod q");
    uint64_t g = 1;  // B^(L_EP-1-k) mod q, k from L_EP - 1 down
    for (uint32_t k = p.l_ep; k-- > 0;) {
      c.gadget_val[2 * k + m] = mulmod(g, inv_q, q);
      g = static_cast<uint64_t>((static_cast<unsigned __int128>(g) << p.base_log2) % q);
    }
  }
}

// The constants of one query: the one-hot at BitRev(col, h), and for each set
// selector bit i the L_EP gadget rows at BitRev(N0 + (i-1) L_EP + k, h).
void query_constants(const opir_client &c, uint64_t idx, ConstEntry *out) {
  const opir_params &p = c.params;
  for (uint32_t u = 0; u < c.nconst; ++u) out[u] = ConstEntry{kNoPos, 0, {0, 0}};
  const std::vector<uint64_t> qi = query_indices(p, idx);
  const uint32_t h = p.expansion_height;
  out[0].pos = static_cast<uint32_t>(bitrev(qi[0], h));
  out[0].val[0] = c.one_val[0];
  out[0].val[1] = c.one_val[1];
  uint32_t at = 1;
  for (size_t i = 1; i < qi.size(); ++i) {
    if (qi[i] != 1) continue;
    for (uint32_t k = 0; k < p.l_ep; ++k) {
      ConstEntry &ce = out[at++];
      ce.pos = static_cast<uint32_t>(bitrev(p.fst_dim_sz + (i - 1) * p.l_ep + k, h));
      ce.val[0] = c.gadget_val[2 * k];
      ce.val[1] = c.gadget_val[2 * k + 1];
    }
  }
}

// make_tree_query's plaintext constants (tree_query.cpp:70-140) for one
// query, W = 2^h_q: the alpha one-hot as the BFV lift of W^-1 mod t at
// BitRev(alpha, h_q) (add_bfv_query_constant), and for every set bit of group
// g (b beta bits, then r gamma bits) the L_EP gadget rows times W^-1 mod q_k
// at BitRev(N0 + g L_EP + row, h_q) (add_rlwe_star_constant).
void tree_query_constants(const opir_client &c, uint64_t n0, uint32_t h_q, uint64_t alpha,
                          const uint8_t *bits, uint32_t groups, ConstEntry *out) {
  const opir_params &p = c.params;
  const uint32_t nconst = 1 + groups * p.l_ep;
  for (uint32_t u = 0; u < nconst; ++u) out[u] = ConstEntry{kNoPos, 0, {0, 0}};
  const uint64_t t = p.plain_mod, W = 1ull << h_q;
  uint64_t w_inv_t = 0;
  if (!opir::invert_mod(W % t, t, w_inv_t)) throw std::invalid_argument("W is not invertible mod t");
  out[0].pos = static_cast<uint32_t>(bitrev(alpha, h_q));
  if (c.limbs == 1) {
    const uint64_t q = c.mods[0];
    out[0].val[0] = static_cast<uint64_t>(
        ((static_cast<unsigned __int128>(q) * w_inv_t + (t >> 1)) / t) % q);
  } else {
    const unsigned __int128 Q = static_cast<unsigned __int128>(c.mods[0]) * c.mods[1];
    const unsigned __int128 delta = Q / t;
    const uint64_t rem = static_cast<uint64_t>(Q - delta * t);
    const uint64_t rem_round =
        static_cast<uint64_t>((static_cast<unsigned __int128>(rem) * w_inv_t + (t >> 1)) / t);
    const unsigned __int128 scaled = delta * w_inv_t + rem_round;
    for (uint32_t k = 0; k < 2; ++k) out[0].val[k] = static_cast<uint64_t>(scaled % c.mods[k]);
  }
  uint64_t w_inv_q[2] = {0, 0};
  for (uint32_t m = 0; m < c.limbs; ++m)
    if (!opir::invert_mod(W % c.mods[m], c.mods[m], w_inv_q[m]))
      throw std::invalid_argument("W is not invertible mod q");
  uint32_t at = 1;
  for (uint32_t g = 0; g < groups; ++g) {
    if (!bits[g]) continue;
    for (uint32_t row = 0; row < p.l_ep; ++row) {
      ConstEntry &ce = out[at++];
      ce.pos = static_cast<uint32_t>(bitrev(n0 + static_cast<uint64_t>(g) * p.l_ep + row, h_q));
      for (uint32_t m = 0; m < c.limbs; ++m) {
        uint64_t gd = 1;  // B^(L_EP-1-row) mod q_m
        for (uint32_t s2 = 0; s2 + 1 + row < p.l_ep; ++s2)
          gd = static_cast<uint64_t>((static_cast<unsigned __int128>(gd) << p.base_log2) % c.mods[m]);
        ce.val[m] = mulmod(gd, w_inv_q[m], c.mods[m]);
      }
    }
  }
}

// Output slices per item so that a batch fills the GPU (index-list
// product); R = n / (s kBlock) outputs per thread, at most kMaxR.
constexpr uint32_t kMaxR = 8;
uint32_t slices_for(uint64_t items, uint32_t n, int sms) {
  uint32_t s = 1;
  while (n / (s * kBlock) > kMaxR) s *= 2;
  while (items * s < 2ull * sms && s * 2 * kBlock <= n) s *= 2;
  return s;
}

// The window product pays when each thread keeps R >= 4 outputs (R + J - 1
// loads serve R J terms); decryption uses it when those slices still give
// every SM a CTA. Query packing keeps the index-list product: its moduli need
// three 20-bit parts in the window form, which issued as many instructions
// per term as the list form at half the occupancy. OPIR_CLIENT_WINDOW=0 keeps
// the index-list product everywhere.
bool window_enabled() {
  const char *v = std::getenv("OPIR_CLIENT_WINDOW");
  return !(v && v[0] == '0');
}
uint32_t window_r(uint64_t items, uint32_t n, int sms) {
  if (!window_enabled() || (n != 2048 && n != 4096)) return 0;
  for (uint32_t R : {8u, 4u})
    if (items * (n / (kBlock * R)) >= static_cast<uint64_t>(sms)) return R;
  return 0;
}

template <typename K>
void set_smem(K kernel, size_t smem, const char *what) {
  ck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          static_cast<int>(smem)),
     what);
}

void launched(const char *what) {
  ck(cudaGetLastError(), what);
  opir::note_launches(1);
}

DecConst dec_const(const opir_params &p) {
  DecConst dc{};
  dc.sq = p.small_q;
  dc.t = p.plain_mod;
  dc.mu_sq = static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) / dc.sq);
  dc.mu_t = static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) / dc.t);
  dc.wide = static_cast<unsigned __int128>(dc.sq) * dc.t + dc.sq >= (static_cast<unsigned __int128>(1) << 63);
  dc.inv_sq = 1.0 / static_cast<double>(dc.sq);
  dc.inv_t = 1.0 / static_cast<double>(dc.t);
  return dc;
}

// The tensor-core form serves single-modulus decryption batches of at least
// kTcMinResponses (OPIR_CLIENT_TC=0 turns it off).
constexpr uint64_t kTcMinResponses = 32;
// any_limbs: decryption, whose modulus (small_q) is one prime for both sets.
bool tc_enabled(const opir_client &c, uint64_t items, uint64_t modulus_bound,
                bool any_limbs = false) {
  const char *v = std::getenv("OPIR_CLIENT_TC");
  if ((v && v[0] == '0') || !window_enabled()) return false;
  return (any_limbs || c.limbs == 1) && c.n % 128 == 0 && c.n <= 8192 &&
         modulus_bound < (1ull << 29) && items >= kTcMinResponses;
}

void ensure_secret_matrix(opir_client &c, cudaStream_t st) {
  if (c.tc_a.p) return;
  const uint32_t n = c.n;
  c.tc_a.alloc(4ull * n * n);
  ck(cudaMemsetAsync(c.tc_a.p, 0, 4ull * n * n, st), "secret matrix clear");
  k_client_secret_matrix<<<n, kBlock, 0, st>>>(c.msgs.p, n, c.tc_a.p);
  launched("secret matrix launch");
  c.tc_err.alloc(1);
}

// One scan C = A x mod q (< 2^29) over nr columns of byte planes `planes`
// ([4][nr][n]) into cmat [nr][n].
void scan_secret_matrix(const opir_client &c, uint32_t nr, uint64_t q, const uint8_t *planes,
                        uint32_t *cmat, cudaStream_t st) {
  const uint32_t n = c.n;
  opir::TcScanArgs a{};
  a.ntile = nr <= 16 ? 16 : nr <= 32 ? 32 : 64;
  a.kt = 128;
  a.stages = opir::scan_tc_max_stages(a.ntile, a.kt);
  a.col_tiles = (nr + a.ntile - 1) / a.ntile;
  a.k_tiles = n / a.kt;
  a.other = n;
  a.m_tiles = n / 128;
  a.ncols = nr;
  a.zcount = 1;
  a.levels_per_res = 1;
  a.q[0] = a.q[1] = static_cast<uint32_t>(q);
  a.mu[0] = a.mu[1] = static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) / q);
  uint64_t w = 1;
  for (int sft = 0; sft < 7; ++sft) {
    a.w[0][sft] = a.w[1][sft] = static_cast<uint32_t>(w);
    w = (w << 8) % q;
  }
  a.cmat = cmat;
  a.err = c.tc_err.p;
  CUtensorMap map_a, map_q;
  opir::make_plane_map(&map_a, c.tc_a.p, n, n, 4, 128, 128);
  opir::make_plane_map(&map_q, planes, n, nr, 4, a.ntile, 128);
  opir::launch_scan_tc(map_a, map_q, a, c.sms, st);
}

// Reads the scans' error word (synchronises the stream).
void check_scan_error(const opir_client &c, cudaStream_t st, const char *what) {
  uint32_t err = 0;
  ck(cudaMemcpyAsync(&err, c.tc_err.p, sizeof(err), cudaMemcpyDeviceToHost, st), "scan error read");
  ck(cudaStreamSynchronize(st), what);
  if (err) throw std::runtime_error(std::string(what) + ": tensor-core scan gave up (error bits " +
                                    std::to_string(err) + ")");
}

// The two primes of the split forms (29-bit, product above 2^57).
constexpr uint64_t kSplitP1 = 536813569, kSplitP2 = 536752129;

void launch_pack_tc(uint64_t n_q, const uint64_t *pt_idx, cudaStream_t st, const uint64_t *a,
                    const int64_t *e, opir_client &c, uint64_t *out) {
  const uint32_t n = c.n, nq = static_cast<uint32_t>(n_q);
  const opir_params &p = c.params;
  if (p.l_ep > 16) throw std::runtime_error("client pack: L_EP above 16");
  ensure_secret_matrix(c, st);
  // columns: one per query (single modulus: two residue sets) or one per
  // (query, limb) (two limbs: two 30-bit halves); both need 8 plane sets'
  // worth of room per column pair
  const uint64_t cols = n_q * c.limbs;
  if (c.pk_colsum.n < 2 * cols) {
    ck(cudaStreamSynchronize(st), "client sync");
    c.pk_q.alloc(8ull * cols * n);
    c.pk_colsum.alloc(2 * cols);
    c.pk_ax.alloc((c.limbs == 2 ? 4 : 2) * cols * n);
    c.pk_idx.alloc(n_q);
  }
  // the previous call's index upload must have left the staging buffer
  ck(cudaEventSynchronize(c.staged), "client staging wait");
  if (c.idx_staging_cap < n_q) {
    if (c.idx_staging) cudaFreeHost(c.idx_staging);
    c.idx_staging = nullptr;
    c.idx_staging_cap = 0;
    ck(cudaMallocHost(&c.idx_staging, n_q * sizeof(uint64_t)), "client index staging");
    c.idx_staging_cap = n_q;
  }
  std::memcpy(c.idx_staging, pt_idx, n_q * sizeof(uint64_t));
  ck(cudaMemcpyAsync(c.pk_idx.p, c.idx_staging, n_q * sizeof(uint64_t), cudaMemcpyHostToDevice, st),
     "client index upload");
  ck(cudaEventRecord(c.staged, st), "client staging record");
  PackLayout L{};
  L.n0 = p.fst_dim_sz;
  L.other = p.other_dim_sz;
  L.num_dims = p.num_dims;
  L.h = p.expansion_height;
  L.l_ep = p.l_ep;
  L.one[0] = c.one_val[0];
  L.one[1] = c.one_val[1];
  for (uint32_t k = 0; k < p.l_ep; ++k) {
    L.gadget[k][0] = c.gadget_val[2 * k];
    L.gadget[k][1] = c.gadget_val[2 * k + 1];
  }
  ck(cudaMemsetAsync(c.tc_err.p, 0, sizeof(uint32_t), st), "scan error reset");
  if (c.limbs == 2) {
    const uint32_t nc = static_cast<uint32_t>(cols);
    uint64_t inv = 0;
    if (!opir::invert_mod(kSplitP1 % kSplitP2, kSplitP2, inv)) throw std::runtime_error("split primes");
    k_client_tc_pack_prep_split<<<nc, kBlock, 0, st>>>(a, n, nc, p.q1, p.q2, c.pk_q.p,
                                                       c.pk_colsum.p);
    launched("client pack prep launch");
    const uint64_t set = 4ull * cols * n, outw = cols * n;
    for (int hf = 0; hf < 2; ++hf)
      for (int pr = 0; pr < 2; ++pr)
        scan_secret_matrix(c, nc, pr ? kSplitP2 : kSplitP1, c.pk_q.p + hf * set,
                           c.pk_ax.p + (2 * hf + pr) * outw, st);
    k_client_tc_pack_finish_split<<<nq, kBlock, 0, st>>>(a, e, c.pk_idx.p, L, c.pk_ax.p,
                                                         c.pk_colsum.p, n, nc, kSplitP1, kSplitP2,
                                                         inv, p.q1, p.q2, 1.0 / static_cast<double>(p.q1),
                                                         1.0 / static_cast<double>(p.q2), out);
    launched("client pack finish launch");
    check_scan_error(c, st, "client pack");
    return;
  }
  k_client_tc_pack_prep<<<nq, kBlock, 0, st>>>(a, n, nq, p.q1, p.q2, c.pk_q.p, c.pk_colsum.p);
  launched("client pack prep launch");
  const uint64_t plane_set = 4ull * n_q * n;
  scan_secret_matrix(c, nq, p.q1, c.pk_q.p, c.pk_ax.p, st);
  scan_secret_matrix(c, nq, p.q2, c.pk_q.p + plane_set, c.pk_ax.p + n_q * n, st);
  k_client_tc_pack_finish<<<nq, kBlock, 0, st>>>(a, e, c.pk_idx.p, L, c.pk_ax.p,
                                                 c.pk_colsum.p, n, nq, p.q1, p.q2,
                                                 p.q1_inv_mod_q2, out);
  launched("client pack finish launch");
  check_scan_error(c, st, "client pack");
}

void launch_decrypt_tc_split(uint64_t n_resp, cudaStream_t st, const uint64_t *resp,
                             opir_client &c, uint64_t *pt, unsigned long long *noise) {
  const uint32_t n = c.n, nr = static_cast<uint32_t>(n_resp);
  ensure_secret_matrix(c, st);
  if (c.tc_colsum.n < 2 * n_resp) {
    ck(cudaStreamSynchronize(st), "client sync");
    c.tc_q.alloc(8ull * n_resp * n);
    c.tc_colsum.alloc(2 * n_resp);
    c.tc_ax.alloc(4 * n_resp * n);
  }
  uint64_t inv = 0;
  if (!opir::invert_mod(kSplitP1 % kSplitP2, kSplitP2, inv)) throw std::runtime_error("split primes");
  ck(cudaMemsetAsync(c.tc_err.p, 0, sizeof(uint32_t), st), "scan error reset");
  k_client_tc_prep_split<<<nr, kBlock, 0, st>>>(resp, n, nr, c.params.small_q, c.tc_q.p,
                                                c.tc_colsum.p);
  launched("client prep launch");
  const uint64_t plane_set = 4ull * n_resp * n, out = n_resp * n;
  for (int hf = 0; hf < 2; ++hf)
    for (int pr = 0; pr < 2; ++pr)
      scan_secret_matrix(c, nr, pr ? kSplitP2 : kSplitP1, c.tc_q.p + hf * plane_set,
                         c.tc_ax.p + (2 * hf + pr) * out, st);
  k_client_tc_finish_split<<<nr, kBlock, 0, st>>>(resp, c.tc_ax.p, c.tc_colsum.p, n, nr, kSplitP1,
                                                  kSplitP2, inv, dec_const(c.params), pt, noise);
  launched("client finish launch");
  check_scan_error(c, st, "client decrypt");
}

void launch_decrypt_tc(uint64_t n_resp, cudaStream_t st, const uint64_t *resp, opir_client &c,
                       uint64_t *pt, unsigned long long *noise) {
  if (c.params.small_q >= (1ull << 29))
    return launch_decrypt_tc_split(n_resp, st, resp, c, pt, noise);
  const uint32_t n = c.n, nr = static_cast<uint32_t>(n_resp);
  const uint64_t sq = c.params.small_q;
  ensure_secret_matrix(c, st);
  if (c.tc_colsum.n < n_resp) {
    ck(cudaStreamSynchronize(st), "client sync");
    c.tc_q.alloc(4ull * n_resp * n);
    c.tc_colsum.alloc(n_resp);
    c.tc_ax.alloc(n_resp * n);
  }
  ck(cudaMemsetAsync(c.tc_err.p, 0, sizeof(uint32_t), st), "scan error reset");
  k_client_tc_prep<<<nr, kBlock, 0, st>>>(resp, n, nr, sq, c.tc_q.p, c.tc_colsum.p);
  launched("client prep launch");
  scan_secret_matrix(c, nr, sq, c.tc_q.p, c.tc_ax.p, st);
  k_client_tc_finish<<<nr, kBlock, 0, st>>>(resp, c.tc_ax.p, c.tc_colsum.p, n,
                                            dec_const(c.params), pt, noise);
  launched("client finish launch");
  // the scan's bounded waits report through its error word
  check_scan_error(c, st, "client decrypt");
}

void launch_decrypt(uint64_t n_resp, cudaStream_t st, const uint64_t *resp, const opir_client &c,
                    uint64_t *pt, unsigned long long *noise) {
  const uint32_t n = c.n;
  const uint64_t sq = c.params.small_q;
  const DecConst dc = dec_const(c.params);
  const uint32_t nb = static_cast<uint32_t>(n_resp);
  const uint32_t R = sq < (1ull << 50) ? window_r(n_resp, n, c.sms) : 0;
  if (R) {
    const int np = sq < (1ull << 25) ? 1 : 2;
    const dim3 grid(nb, n / (kBlock * R));
    const size_t smem = np * 2 * n * sizeof(int32_t) + kBlock * sizeof(uint32_t);
#define OPIR_DECW(NP, RR, JJ)                                                                  \
  if (np == NP && R == RR && n == kBlock * JJ) {                                              \
    set_smem(k_client_decrypt_w<NP, 25, RR, JJ>, smem, "client decrypt smem");               \
    k_client_decrypt_w<NP, 25, RR, JJ><<<grid, kBlock, smem, st>>>(resp, c.code.p, n, dc, pt, \
                                                                   noise);                    \
    return launched("client decrypt launch");                                                 \
  }
    OPIR_DECW(1, 8, 8) OPIR_DECW(1, 4, 8) OPIR_DECW(1, 8, 16) OPIR_DECW(1, 4, 16)
    OPIR_DECW(2, 8, 8) OPIR_DECW(2, 4, 8) OPIR_DECW(2, 8, 16) OPIR_DECW(2, 4, 16)
#undef OPIR_DECW
    throw std::runtime_error("client decrypt: no window kernel for this shape");
  }
  const uint32_t s = slices_for(n_resp, n, c.sms);
  const uint32_t Rl = n / (s * kBlock);
  const dim3 grid(nb, s);
  const size_t lists = (c.npos + c.nneg + 8) * sizeof(uint16_t);
  const int np = sq < (1ull << 31) ? 1 : 2;
  const size_t smem = np * 2 * n * sizeof(int32_t) + lists;
#define OPIR_DEC(NP, RR)                                                                      \
  if (np == NP && Rl == RR) {                                                                 \
    set_smem(k_client_decrypt<NP, RR>, smem, "client decrypt smem");                          \
    k_client_decrypt<NP, RR><<<grid, kBlock, smem, st>>>(resp, c.sidx.p, c.npos, c.nneg, n,   \
                                                         dc, pt, noise);                      \
    return launched("client decrypt launch");                                                 \
  }
  OPIR_DEC(1, 1) OPIR_DEC(1, 2) OPIR_DEC(1, 4) OPIR_DEC(1, 8)
  OPIR_DEC(2, 1) OPIR_DEC(2, 2) OPIR_DEC(2, 4) OPIR_DEC(2, 8)
#undef OPIR_DEC
  throw std::runtime_error("client decrypt: unsupported slice width");
}

void launch_pack(uint64_t items, cudaStream_t st, const uint64_t *a, const int64_t *e,
                 const opir_client &c, const ConstEntry *consts, uint32_t nconst, uint64_t *out) {
  const uint32_t n = c.n;
  const uint32_t ni = static_cast<uint32_t>(items);
  const uint32_t s = slices_for(items, n, c.sms);
  const uint32_t Rl = n / (s * kBlock);
  const dim3 grid(ni, s);
  const size_t smem = 2 * 2 * n * sizeof(int32_t) + (c.npos + c.nneg + 8) * sizeof(uint16_t);
#define OPIR_PACK(RR)                                                                         \
  if (Rl == RR) {                                                                             \
    set_smem(k_client_pack<RR>, smem, "client pack smem");                                    \
    k_client_pack<RR><<<grid, kBlock, smem, st>>>(a, e, consts, nconst, c.sidx.p,             \
                                                  c.npos, c.nneg, n, c.limbs, c.mods[0],      \
                                                  c.mods[1], out);                            \
    return launched("client pack launch");                                                    \
  }
  OPIR_PACK(1) OPIR_PACK(2) OPIR_PACK(4) OPIR_PACK(8)
#undef OPIR_PACK
  throw std::runtime_error("client pack: unsupported slice width");
}

void launch_keygen(const opir_client &c, const std::vector<KeyRow> &rows, uint64_t *bv,
                   uint64_t bv_polys, uint64_t *gsw, uint64_t gsw_polys, cudaStream_t st) {
  const uint32_t n = c.n;
  const uint64_t items = rows.size() * c.limbs;
  const uint32_t s = slices_for(items, n, c.sms);
  const uint32_t Rl = n / (s * kBlock);
  const dim3 grid(static_cast<uint32_t>(items), s);
  const size_t smem = 2 * 2 * n * sizeof(int32_t) + (c.npos + c.nneg + 8) * sizeof(uint16_t);
  bool done = false;
#define OPIR_KEYROWS(RR)                                                                      \
  if (!done && Rl == RR) {                                                                    \
    set_smem(k_client_keyrows<RR>, smem, "client keygen smem");                               \
    k_client_keyrows<RR><<<grid, kBlock, smem, st>>>(c.keyrows.p, c.msgs.p, c.sidx.p, c.npos, \
                                                     c.nneg, n, c.limbs, c.mods[0],          \
                                                     c.mods[1]);                              \
    launched("client keygen launch");                                                         \
    done = true;                                                                              \
  }
  OPIR_KEYROWS(1) OPIR_KEYROWS(2) OPIR_KEYROWS(4) OPIR_KEYROWS(8)
#undef OPIR_KEYROWS
  if (!done) throw std::runtime_error("client keygen: unsupported slice width");
  for (const auto &part : {std::make_pair(bv, bv_polys), std::make_pair(gsw, gsw_polys)}) {
    if (part.second == 0) continue;
    k_client_ntt<<<static_cast<uint32_t>(part.second), kBlock, n * sizeof(uint64_t), st>>>(
        part.first, n, c.limbs, c.fw.p, c.mods[0], c.mods[1]);
    launched("client keygen NTT launch");
  }
}

}  // namespace

namespace opir {

std::vector<uint64_t> forward_twiddles(const opir_params &p) {
  const uint32_t n = p.poly_degree, limbs = p.num_limbs;
  uint32_t lg = 0;
  while ((1u << lg) < n) ++lg;
  std::vector<uint64_t> fw(static_cast<size_t>(limbs) * n);
  for (uint32_t m = 0; m < limbs; ++m) {
    const uint64_t q = limbs == 1 ? p.q : (m == 0 ? p.q1 : p.q2);
    const uint64_t root = limbs == 1 ? p.w_crt % q : (m == 0 ? p.w1 : p.w2);
    std::vector<uint64_t> pw(n);
    pw[0] = 1 % q;
    for (uint32_t e = 1; e < n; ++e) pw[e] = mulmod(pw[e - 1], root, q);
    for (uint32_t k = 0; k < n; ++k) fw[static_cast<size_t>(m) * n + k] = pw[bitrev(k, lg)];
  }
  return fw;
}

void forward_ntt_polys(uint64_t *d_polys, uint64_t count, const opir_params &p,
                       const uint64_t *d_fw, cudaStream_t st) {
  if (count == 0) return;
  const uint32_t n = p.poly_degree, limbs = p.num_limbs;
  const uint64_t q0 = limbs == 1 ? p.q : p.q1, q1 = limbs == 1 ? 0 : p.q2;
  for (uint64_t done = 0; done < count;) {
    const uint32_t chunk = static_cast<uint32_t>(std::min<uint64_t>(count - done, 1u << 30));
    // chunks keep the limb of polynomial i at i % limbs (chunk sizes are multiples of limbs)
    k_client_ntt<<<chunk, kBlock, n * sizeof(uint64_t), st>>>(d_polys + done * n, n, limbs, d_fw,
                                                            q0, q1);
    launched("NTT launch");
    done += chunk;
  }
}

}  // namespace opir

// Helpers of the host-buffer calls.
namespace {

template <typename T>
T *upload(DevBuf<T> &buf, const T *host, size_t count, cudaStream_t st) {
  buf.alloc(std::max<size_t>(count, 1));
  if (count)
    ck(cudaMemcpyAsync(buf.p, host, count * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
  return buf.p;
}

void ensure_io_stream(opir_client &c) {
  if (!c.io_stream) ck(cudaStreamCreateWithFlags(&c.io_stream, cudaStreamNonBlocking), "client stream");
}

void download(void *host, const void *dev, size_t bytes, cudaStream_t st) {
  ck(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st), "download");
  ck(cudaStreamSynchronize(st), "client call");
}

}  // namespace

extern "C" {

opir_status opir_client_create(const opir_params *params, const int8_t *secret, int device,
                               opir_client **out) {
  if (!params || !secret || !out) return OPIR_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  opir_client *c = new (std::nothrow) opir_client();
  if (!c) return OPIR_ERR_NO_MEMORY;
  const opir_status st = client_guarded(c, [&] {
    c->params = checked_layout(*params);
    c->device = device;
    c->n = c->params.poly_degree;
    c->limbs = c->params.num_limbs;
    if (c->limbs == 1) {
      c->mods[0] = c->params.q;
    } else {
      c->mods[0] = c->params.q1;
      c->mods[1] = c->params.q2;
    }
    std::vector<uint16_t> lists;
    lists.reserve(c->n);
    for (uint32_t j = 0; j < c->n; ++j) {
      if (secret[j] < -1 || secret[j] > 1)
        throw std::invalid_argument("secret coefficients must be -1, 0 or 1");
      if (secret[j] == 1) lists.push_back(static_cast<uint16_t>(j));
    }
    c->npos = static_cast<uint32_t>(lists.size());
    for (uint32_t j = 0; j < c->n; ++j)
      if (secret[j] == -1) lists.push_back(static_cast<uint16_t>(j));
    c->nneg = static_cast<uint32_t>(lists.size()) - c->npos;
    std::vector<uint32_t> code(kBlock, 0);
    if (c->n % kBlock == 0 && c->n / kBlock <= 16)
      for (uint32_t j = 0; j < c->n; ++j)
        if (secret[j] != 0)
          code[j % kBlock] |= (secret[j] == 1 ? 1u : 2u) << (2 * (j / kBlock));
    c->nconst = 1 + (c->params.num_dims - 1) * c->params.l_ep;
    prepare_constants(*c);
    DeviceGuard g(device);
    ck(cudaEventCreateWithFlags(&c->staged, cudaEventDisableTiming), "client event");
    ck(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    c->sidx.alloc(std::max<size_t>(lists.size(), 1));
    if (!lists.empty())
      ck(cudaMemcpy(c->sidx.p, lists.data(), lists.size() * sizeof(uint16_t),
                    cudaMemcpyHostToDevice),
         "secret upload");
    c->code.alloc(kBlock);
    ck(cudaMemcpy(c->code.p, code.data(), kBlock * sizeof(uint32_t), cudaMemcpyHostToDevice),
       "secret code upload");
    // key generation: s and its automorphisms sigma_k(s), k = N/2^i + 1
    // (utils.cpp:58-72: coefficient j moves to j k mod 2N, negated past N)
    const uint32_t h = c->params.expansion_height;
    std::vector<int8_t> msgs(static_cast<size_t>(1 + h) * c->n, 0);
    std::copy(secret, secret + c->n, msgs.begin());
    for (uint32_t i = 0; i < h; ++i) {
      const uint64_t k = (c->n >> i) + 1, two_n = 2ull * c->n;
      int8_t *o = msgs.data() + static_cast<size_t>(1 + i) * c->n;
      for (uint64_t j = 0; j < c->n; ++j) {
        const uint64_t dest = j * k % two_n;
        if (dest < c->n) o[dest] = secret[j];
        else o[dest - c->n] = static_cast<int8_t>(-secret[j]);
      }
    }
    c->msgs.alloc(msgs.size());
    ck(cudaMemcpy(c->msgs.p, msgs.data(), msgs.size(), cudaMemcpyHostToDevice), "message upload");
    const std::vector<uint64_t> fw = opir::forward_twiddles(c->params);
    c->fw.alloc(fw.size());
    ck(cudaMemcpy(c->fw.p, fw.data(), fw.size() * sizeof(uint64_t), cudaMemcpyHostToDevice),
       "twiddle upload");
  });
  if (st != OPIR_OK) {
    // device resources exist once the event does; release them on their device
    if (c->staged) opir_client_destroy(c);
    else delete c;
    return st;
  }
  *out = c;
  return OPIR_OK;
}

void opir_client_destroy(opir_client *c) {
  if (!c) return;
  {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    c->sidx.reset();
    c->code.reset();
    c->msgs.reset();
    c->fw.reset();
    c->keyrows.reset();
    c->tc_a.reset();
    c->tc_q.reset();
    c->tc_colsum.reset();
    c->tc_ax.reset();
    c->tc_err.reset();
    c->pk_q.reset();
    c->pk_idx.reset();
    if (c->idx_staging) cudaFreeHost(c->idx_staging);
    c->pk_colsum.reset();
    c->pk_ax.reset();
    c->consts.reset();
    if (c->staging) cudaFreeHost(c->staging);
    if (c->staged) cudaEventDestroy(c->staged);
    c->io_u0.reset();
    c->io_u1.reset();
    c->io_out.reset();
    c->io_noise.reset();
    c->io_e0.reset();
    c->io_e1.reset();
    if (c->io_stream) cudaStreamDestroy(c->io_stream);
    if (prev >= 0) cudaSetDevice(prev);
  }
  delete c;
}

const char *opir_client_last_error(const opir_client *c) {
  return c ? c->last_error.c_str() : "null client handle";
}

opir_status opir_client_generate_queries_device(opir_client *c, uint32_t n,
                                                const uint64_t *pt_idx, const uint64_t *d_a,
                                                const int64_t *d_e, uint64_t *d_queries,
                                                void *stream) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  return client_guarded(c, [&] {
    if (n == 0) return;
    if (!pt_idx || !d_a || !d_e || !d_queries) throw std::invalid_argument("null buffer");
    for (uint32_t i = 0; i < n; ++i)
      if (pt_idx[i] >= c->params.num_pt)
        throw std::out_of_range("PIR plaintext index exceeds the runtime layout");
    DeviceGuard g(c->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t qmax = std::max(c->params.q1, c->params.q2);
    const bool tc = c->limbs == 1 ? tc_enabled(*c, n, qmax)
                                  : tc_enabled(*c, n, 0, true) && qmax < (1ull << 60);
    if (tc) {
      launch_pack_tc(n, pt_idx, st, d_a, d_e, *c, d_queries);
      return;
    }
    const size_t count = static_cast<size_t>(n) * c->nconst;
    // the previous call's upload must have left the staging buffer
    ck(cudaEventSynchronize(c->staged), "client staging wait");
    if (c->staging_cap < count) {
      if (c->staging) cudaFreeHost(c->staging);
      c->staging = nullptr;
      c->staging_cap = 0;
      ck(cudaMallocHost(&c->staging, count * sizeof(ConstEntry)), "client staging");
      c->staging_cap = count;
    }
    for (uint32_t i = 0; i < n; ++i)
      query_constants(*c, pt_idx[i], c->staging + static_cast<size_t>(i) * c->nconst);
    if (c->consts.n < count) {
      ck(cudaStreamSynchronize(st), "client sync");
      c->consts.alloc(count);
    }
    ck(cudaMemcpyAsync(c->consts.p, c->staging, count * sizeof(ConstEntry),
                       cudaMemcpyHostToDevice, st),
       "client constants upload");
    ck(cudaEventRecord(c->staged, st), "client staging record");
    launch_pack(static_cast<uint64_t>(n) * c->limbs, st, d_a, d_e, *c, c->consts.p, c->nconst,
                d_queries);
  });
}

opir_status opir_client_decrypt_device(opir_client *c, uint32_t n, const uint64_t *d_responses,
                                       uint64_t *d_plaintexts, uint64_t *d_max_noise,
                                       void *stream) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  return client_guarded(c, [&] {
    if (n == 0) return;
    if (!d_responses || !d_plaintexts) throw std::invalid_argument("null buffer");
    DeviceGuard g(c->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (d_max_noise)
      ck(cudaMemsetAsync(d_max_noise, 0, static_cast<size_t>(n) * sizeof(uint64_t), st),
         "noise reset");
    auto *noise = reinterpret_cast<unsigned long long *>(d_max_noise);
    const uint64_t sq = c->params.small_q;
    if (tc_enabled(*c, n, sq < (1ull << 29) ? sq : 0, true) && sq < (1ull << 50))
      launch_decrypt_tc(n, st, d_responses, *c, d_plaintexts, noise);
    else
      launch_decrypt(n, st, d_responses, *c, d_plaintexts, noise);
  });
}

opir_status opir_client_keygen_device(opir_client *c, const uint64_t *d_bv_a,
                                      const int64_t *d_bv_e, const uint64_t *d_gsw_a,
                                      const int64_t *d_gsw_e, uint64_t *d_bv_keys,
                                      uint64_t *d_gsw_key, void *stream) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  return client_guarded(c, [&] {
    const opir_params &p = c->params;
    const uint32_t h = p.expansion_height, K = c->limbs, n = c->n;
    if (h && (!d_bv_a || !d_bv_e || !d_bv_keys)) throw std::invalid_argument("null BV buffer");
    if (!d_gsw_a || !d_gsw_e || !d_gsw_key) throw std::invalid_argument("null RGSW buffer");
    const uint64_t kn = static_cast<uint64_t>(K) * n;
    auto power = [&](uint32_t bits, uint32_t m) {  // 2^bits mod q_m
      uint64_t v = 1 % c->mods[m];
      for (uint32_t b = 0; b < bits; ++b) v = mulmod(v, 2, c->mods[m]);
      return v;
    };
    std::vector<KeyRow> rows;
    for (uint32_t i = 0; i < h; ++i)
      for (uint32_t r = 0; r < p.l_ks; ++r) {
        const uint64_t at = static_cast<uint64_t>(i) * p.l_ks + r;
        KeyRow kr{d_bv_a + at * kn, d_bv_e + at * n, d_bv_keys + at * 2 * kn, 1 + i, 0, 1, 0, {0, 0}};
        for (uint32_t m = 0; m < K; ++m) kr.scale[m] = power(r * p.base_log2_ks, m);
        rows.push_back(kr);
      }
    for (uint32_t half = 0; half < 2; ++half)
      for (uint32_t r = 0; r < p.l_key; ++r) {
        const uint64_t at = static_cast<uint64_t>(half) * p.l_key + r;
        KeyRow kr{d_gsw_a + at * kn, d_gsw_e + at * n, d_gsw_key + at * 2 * kn, 0, half, -1, 0, {0, 0}};
        for (uint32_t m = 0; m < K; ++m) kr.scale[m] = power(p.base_log2_key * (p.l_key - 1 - r), m);
        rows.push_back(kr);
      }
    DeviceGuard g(c->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (c->keyrows.n < rows.size()) {
      ck(cudaStreamSynchronize(st), "client sync");
      c->keyrows.alloc(rows.size());
    }
    ck(cudaMemcpyAsync(c->keyrows.p, rows.data(), rows.size() * sizeof(KeyRow),
                       cudaMemcpyHostToDevice, st),
       "key row upload");
    launch_keygen(*c, rows, d_bv_keys, static_cast<uint64_t>(h) * p.l_ks * 2 * K, d_gsw_key,
                  2ull * p.l_key * 2 * K, st);
  });
}

// ---- host-buffer forms: the same calls on host arrays (same layouts), on
// the handle's own stream; each returns when its results are in host memory.

opir_status opir_client_generate_queries(opir_client *c, uint32_t n, const uint64_t *pt_idx,
                                         const uint64_t *a, const int64_t *e,
                                         uint64_t *queries) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  if (n == 0) return OPIR_OK;
  const size_t kn = static_cast<size_t>(c->limbs) * c->n;
  opir_status st = client_guarded(c, [&] {
    if (!pt_idx || !a || !e || !queries) throw std::invalid_argument("null buffer");
    DeviceGuard g(c->device);
    ensure_io_stream(*c);
    upload(c->io_u0, a, n * kn, c->io_stream);
    upload(c->io_e0, e, static_cast<size_t>(n) * c->n, c->io_stream);
    c->io_out.alloc(n * 2 * kn);
  });
  if (st != OPIR_OK) return st;
  st = opir_client_generate_queries_device(c, n, pt_idx, c->io_u0.p, c->io_e0.p, c->io_out.p,
                                           c->io_stream);
  if (st != OPIR_OK) return st;
  return client_guarded(c, [&] {
    DeviceGuard g(c->device);
    download(queries, c->io_out.p, n * 2 * kn * sizeof(uint64_t), c->io_stream);
  });
}

opir_status opir_client_decrypt(opir_client *c, uint32_t n, const uint64_t *responses,
                                uint64_t *plaintexts, uint64_t *max_noise) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  if (n == 0) return OPIR_OK;
  opir_status st = client_guarded(c, [&] {
    if (!responses || !plaintexts) throw std::invalid_argument("null buffer");
    DeviceGuard g(c->device);
    ensure_io_stream(*c);
    upload(c->io_u0, responses, static_cast<size_t>(n) * 2 * c->n, c->io_stream);
    c->io_out.alloc(static_cast<size_t>(n) * c->n);
    if (max_noise) c->io_noise.alloc(n);
  });
  if (st != OPIR_OK) return st;
  st = opir_client_decrypt_device(c, n, c->io_u0.p, c->io_out.p, max_noise ? c->io_noise.p : nullptr,
                                  c->io_stream);
  if (st != OPIR_OK) return st;
  return client_guarded(c, [&] {
    DeviceGuard g(c->device);
    if (max_noise)
      ck(cudaMemcpyAsync(max_noise, c->io_noise.p, n * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                         c->io_stream),
         "download");
    download(plaintexts, c->io_out.p, static_cast<size_t>(n) * c->n * sizeof(uint64_t),
             c->io_stream);
  });
}

opir_status opir_client_keygen(opir_client *c, const uint64_t *bv_a, const int64_t *bv_e,
                               const uint64_t *gsw_a, const int64_t *gsw_e, uint64_t *bv_keys,
                               uint64_t *gsw_key) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  const opir_params &p = c->params;
  const size_t kn = static_cast<size_t>(c->limbs) * c->n;
  const size_t bv_rows = static_cast<size_t>(p.expansion_height) * p.l_ks;
  const size_t gsw_rows = 2ull * p.l_key;
  opir_status st = client_guarded(c, [&] {
    if (bv_rows && (!bv_a || !bv_e || !bv_keys)) throw std::invalid_argument("null BV buffer");
    if (!gsw_a || !gsw_e || !gsw_key) throw std::invalid_argument("null RGSW buffer");
    DeviceGuard g(c->device);
    ensure_io_stream(*c);
    upload(c->io_u0, bv_a, bv_rows * kn, c->io_stream);
    upload(c->io_e0, bv_e, bv_rows * c->n, c->io_stream);
    upload(c->io_u1, gsw_a, gsw_rows * kn, c->io_stream);
    upload(c->io_e1, gsw_e, gsw_rows * c->n, c->io_stream);
    c->io_out.alloc((bv_rows + gsw_rows) * 2 * kn);
  });
  if (st != OPIR_OK) return st;
  st = opir_client_keygen_device(c, bv_rows ? c->io_u0.p : nullptr, bv_rows ? c->io_e0.p : nullptr,
                                 c->io_u1.p, c->io_e1.p, bv_rows ? c->io_out.p : nullptr,
                                 c->io_out.p + bv_rows * 2 * kn, c->io_stream);
  if (st != OPIR_OK) return st;
  return client_guarded(c, [&] {
    DeviceGuard g(c->device);
    if (bv_rows)
      ck(cudaMemcpyAsync(bv_keys, c->io_out.p, bv_rows * 2 * kn * sizeof(uint64_t),
                         cudaMemcpyDeviceToHost, c->io_stream),
         "download");
    download(gsw_key, c->io_out.p + bv_rows * 2 * kn, gsw_rows * 2 * kn * sizeof(uint64_t),
             c->io_stream);
  });
}

opir_status opir_client_generate_tree_queries(opir_client *c, const opir_tree_params *tree,
                                              uint32_t n, const uint64_t *alpha,
                                              const uint8_t *bits, uint32_t groups,
                                              const uint64_t *a, const int64_t *e,
                                              uint64_t *queries) {
  if (!c) return OPIR_ERR_INVALID_ARGUMENT;
  return client_guarded(c, [&] {
    if (n == 0) return;
    if (!tree || !alpha || (groups && !bits) || !a || !e || !queries)
      throw std::invalid_argument("null buffer");
    const opir_params &p = c->params;
    const uint64_t n0 = tree->N0;
    const uint32_t h_q = static_cast<uint32_t>(tree->h_q);
    if ((1ull << h_q) > c->n || n0 + static_cast<uint64_t>(groups) * p.l_ep > (1ull << h_q))
      throw std::invalid_argument("tree query shape does not fit the polynomial");
    for (uint32_t i = 0; i < n; ++i)
      if (alpha[i] >= n0) throw std::out_of_range("tree query alpha exceeds N0");
    const uint32_t nconst = 1 + groups * p.l_ep;
    const size_t count = static_cast<size_t>(n) * nconst;
    const size_t kn = static_cast<size_t>(c->limbs) * c->n;
    DeviceGuard g(c->device);
    ensure_io_stream(*c);
    cudaStream_t st = c->io_stream;
    ck(cudaEventSynchronize(c->staged), "client staging wait");
    if (c->staging_cap < count) {
      if (c->staging) cudaFreeHost(c->staging);
      c->staging = nullptr;
      c->staging_cap = 0;
      ck(cudaMallocHost(&c->staging, count * sizeof(ConstEntry)), "client staging");
      c->staging_cap = count;
    }
    for (uint32_t i = 0; i < n; ++i)
      tree_query_constants(*c, n0, h_q, alpha[i], bits + static_cast<size_t>(i) * groups, groups,
                           c->staging + static_cast<size_t>(i) * nconst);
    if (c->consts.n < count) {
      ck(cudaStreamSynchronize(st), "client sync");
      c->consts.alloc(count);
    }
    ck(cudaMemcpyAsync(c->consts.p, c->staging, count * sizeof(ConstEntry),
                       cudaMemcpyHostToDevice, st),
       "client constants upload");
    ck(cudaEventRecord(c->staged, st), "client staging record");
    upload(c->io_u0, a, n * kn, st);
    upload(c->io_e0, e, static_cast<size_t>(n) * c->n, st);
    c->io_out.alloc(n * 2 * kn);
    launch_pack(static_cast<uint64_t>(n) * c->limbs, st, c->io_u0.p, c->io_e0.p, *c, c->consts.p,
                nconst, c->io_out.p);
    download(queries, c->io_out.p, n * 2 * kn * sizeof(uint64_t), st);
  });
}

}  // extern "C"
