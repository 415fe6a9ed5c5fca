// Kernels of the CONFIG_N2048_K1 query path (opir_k1p_kernels.h): one 60-bit
// NTT prime at N = 2048, every polynomial one plane of N u64.
//
// NTT: the register-resident radix-8/8/8/4 form of the CONFIG_N2048_K1_COMP
// kernels (opir_device.cuh: 256 threads x 8 coefficients, thread positions
// A/B/C/D, shared planes padded by one word per 32) in 64-bit arithmetic:
// Harvey/Shoup lazy butterflies with w' = floor(w 2^64 / q), forward values
// below 8q < 2^63 with X corrected on stages 4, 6, 8 and 10, inverse values
// in [0, 2q). Merged Cooley-Tukey forward with bit-reversed output,
// Gentleman-Sande inverse scaled by N^-1 (the HEXL convention the reference
// registers, utils.cpp:26-56). Key and selector rows carry Shoup companions,
// so every key product is three 64-bit multiplies landing in [0, 2q).
#include "opir_k1p_kernels.h"

#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

namespace opir1 {

namespace {

using u128 = unsigned __int128;

constexpr int kThreads = 256;
constexpr int kPad = kN + kN / 32;  // u64 words per padded plane
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

// (w, Shoup) for twiddle indices < 64, forward and inverse; {N^-1, its
// Shoup companion} and {iw[1] N^-1, Shoup}
static __constant__ ulonglong2 c1_fwt[64];
static __constant__ ulonglong2 c1_iwt[64];
static __constant__ ulonglong2 c1_nscale[2];

void check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
  opir4::note_launches(1);
}

template <typename K>
void set_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> granted;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(dev, reinterpret_cast<const void *>(kernel));
  std::lock_guard<std::mutex> lock(mu);
  auto it = granted.find(key);
  if (it != granted.end() && it->second >= bytes) return;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(bytes));
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  granted[key] = bytes;
}

constexpr size_t plane_bytes(int np) { return static_cast<size_t>(np) * kPad * sizeof(uint64_t); }

// SMs of the current device (cached per device).
int sms() {
  static std::mutex mu;
  static std::map<int, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    n = 1;
  }
  cache[dev] = n;
  return n;
}

// ------------------------------------------------------------ arithmetic
__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// a w mod q in [0, 2q) for any 64-bit a (Shoup)
__device__ __forceinline__ uint64_t mulsh(uint64_t a, uint64_t w, uint64_t ws) {
  return a * w - __umul64hi(a, ws) * kQ;
}
__device__ __forceinline__ uint64_t canon8(uint64_t x) {  // [0, 8q) -> [0, q)
  x = min(x, x - 4 * kQ);
  x = min(x, x - 2 * kQ);
  return min(x, x - kQ);
}
__device__ __forceinline__ uint64_t fold2(uint64_t x) { return min(x, x - kQ); }  // [0, 2q)
__device__ __forceinline__ uint64_t add_q(uint64_t a, uint64_t b) {
  const uint64_t s = a + b;
  return min(s, s - kQ);
}
__device__ __forceinline__ uint64_t sub_q(uint64_t a, uint64_t b) {
  const uint64_t d = a - b + kQ;
  return min(d, d - kQ);
}
__device__ __forceinline__ uint64_t neg_q(uint64_t a) { return a ? kQ - a : 0; }
__device__ __forceinline__ uint64_t shoup_of(uint64_t w) {
  return static_cast<uint64_t>((static_cast<u128>(w) << 64) / kQ);
}
// Balanced base-2^B digits, LSB first (gsw.cpp:277-293, bv_keyswitch.cpp:
// 20-40): v in [0, q) is centred to c in (-q/2, q/2]; c + C with
// C = 2^(B-1) sum_{i<L} 2^(B i) has plain base-2^B digits u_i = r_i + 2^(B-1)
// in its low L B bits (r_i in [-2^(B-1), 2^(B-1)) the balanced digits; a
// carry out of digit L - 1, which the reference drops, only touches bits
// above L B).
template <int L, int B>
__device__ __forceinline__ uint64_t digit_source(uint64_t v) {
  uint64_t C = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) C += (1ull << (B - 1)) << (B * i);
  return v + C - (v > kQ / 2 ? kQ : 0);
}
template <int B>
__device__ __forceinline__ uint64_t digit_res(uint64_t u, int i) {  // r_i mod q
  const int64_t r = static_cast<int64_t>((u >> (B * i)) & ((1ull << B) - 1)) - (1ll << (B - 1));
  return r >= 0 ? static_cast<uint64_t>(r) : static_cast<uint64_t>(r + static_cast<int64_t>(kQ));
}

// ------------------------------------------------------------ NTT
__device__ __forceinline__ int padi(int p) { return p + (p >> 5); }
__device__ __forceinline__ int posA(int t, int k) { return t + 256 * k; }
__device__ __forceinline__ int posB(int t, int k) { return ((t >> 5) << 8) + (t & 31) + 32 * k; }
__device__ __forceinline__ int posC(int t, int k) { return ((t & 63) << 5) + (t >> 6) + 4 * k; }
__device__ __forceinline__ int posD(int t, int k) { return ((t + ((k >> 2) << 8)) << 2) + (k & 3); }

template <int P>
__device__ __forceinline__ void st_plane(uint64_t *pl, const uint64_t (&v)[8], int t) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int p = P == 0 ? posA(t, k) : P == 1 ? posB(t, k) : P == 2 ? posC(t, k) : posD(t, k);
    pl[padi(p)] = v[k];
  }
}
template <int P>
__device__ __forceinline__ void ld_plane(const uint64_t *pl, uint64_t (&v)[8], int t) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int p = P == 0 ? posA(t, k) : P == 1 ? posB(t, k) : P == 2 ? posC(t, k) : posD(t, k);
    v[k] = pl[padi(p)];
  }
}

template <bool C>
__device__ __forceinline__ void fbf(uint64_t &X, uint64_t &Y, ulonglong2 w) {
  uint64_t x = X;
  if (C) x = min(x, x - 4 * kQ);
  const uint64_t t = mulsh(Y, w.x, w.y);
  X = x + t;
  Y = x - t + 2 * kQ;
}
template <bool C1, bool C2, bool C3>
__device__ __forceinline__ void fpass8(uint64_t (&v)[8], const ulonglong2 (&w)[7]) {
  fbf<C1>(v[0], v[4], w[0]); fbf<C1>(v[1], v[5], w[0]);
  fbf<C1>(v[2], v[6], w[0]); fbf<C1>(v[3], v[7], w[0]);
  fbf<C2>(v[0], v[2], w[1]); fbf<C2>(v[1], v[3], w[1]);
  fbf<C2>(v[4], v[6], w[2]); fbf<C2>(v[5], v[7], w[2]);
  fbf<C3>(v[0], v[1], w[3]); fbf<C3>(v[2], v[3], w[4]);
  fbf<C3>(v[4], v[5], w[5]); fbf<C3>(v[6], v[7], w[6]);
}
// pass A (stages 1-3), canonical input
__device__ __forceinline__ void fA(uint64_t (&v)[8]) {
  const ulonglong2 w[7] = {c1_fwt[1], c1_fwt[2], c1_fwt[3], c1_fwt[4],
                           c1_fwt[5], c1_fwt[6], c1_fwt[7]};
  fpass8<false, false, false>(v, w);
}
__device__ __forceinline__ void load_b(ulonglong2 (&w)[7], const ulonglong2 *c, int t) {
  const int g = t >> 5;
  w[0] = c[8 + g];
  w[1] = c[16 + 2 * g];
  w[2] = c[17 + 2 * g];
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = c[32 + 4 * g + i];
}
__device__ __forceinline__ void load_c(ulonglong2 (&w)[7], const ulonglong2 *tw, int t) {
  const int g = t & 63;
  w[0] = __ldg(tw + 64 + g);
  w[1] = __ldg(tw + 128 + 2 * g);
  w[2] = __ldg(tw + 129 + 2 * g);
#pragma unroll
  for (int i = 0; i < 4; ++i) w[3 + i] = __ldg(tw + 256 + 4 * g + i);
}
__device__ __forceinline__ void load_d(ulonglong2 (&w)[6], const ulonglong2 *tw, int t) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int b4 = t + 256 * h;
    w[3 * h] = __ldg(tw + 512 + b4);
    w[3 * h + 1] = __ldg(tw + 1024 + 2 * b4);
    w[3 * h + 2] = __ldg(tw + 1025 + 2 * b4);
  }
}
// pass D (stages 10-11): output in [0, 8q)
__device__ __forceinline__ void fD(uint64_t (&v)[8], const ulonglong2 (&w)[6]) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint64_t *u = v + 4 * h;
    fbf<true>(u[0], u[2], w[3 * h]);
    fbf<true>(u[1], u[3], w[3 * h]);
    fbf<false>(u[0], u[1], w[3 * h + 1]);
    fbf<false>(u[2], u[3], w[3 * h + 2]);
  }
}
// passes B and C over np planes stored in A-order after fA (up to a
// __syncthreads); ends synchronised. Full = true unrolls the plane loops
// (faster in the expansion and MUX levels; the selector kernel keeps the
// compiler's choice, which is faster there).
__device__ __forceinline__ void ipass8(uint64_t (&v)[8], const ulonglong2 (&w)[7]);
template <int PASS, bool FWD>
__device__ __forceinline__ void mid_plane(uint64_t *pl, const ulonglong2 (&w)[7], int t) {
  uint64_t v[8];
  ld_plane<PASS>(pl, v, t);
  if (FWD) {
    if (PASS == 1) fpass8<true, false, true>(v, w);
    else fpass8<false, true, false>(v, w);
  } else {
    ipass8(v, w);
  }
  st_plane<PASS>(pl, v, t);
}
template <bool Full = true>
__device__ __forceinline__ void fwd_mid(uint64_t *sm, int np, const ulonglong2 *fwt) {
  const int t = threadIdx.x;
  {
    ulonglong2 w[7];
    load_b(w, c1_fwt, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane<1, true>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane<1, true>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
  {
    ulonglong2 w[7];
    load_c(w, fwt, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane<2, true>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane<2, true>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void ibf(uint64_t &X, uint64_t &Y, ulonglong2 w) {
  uint64_t u = X + Y;
  u = min(u, u - 2 * kQ);
  const uint64_t d = X - Y + 2 * kQ;
  Y = mulsh(d, w.x, w.y);
  X = u;
}
__device__ __forceinline__ void ipass8(uint64_t (&v)[8], const ulonglong2 (&w)[7]) {
  ibf(v[0], v[1], w[3]); ibf(v[2], v[3], w[4]);
  ibf(v[4], v[5], w[5]); ibf(v[6], v[7], w[6]);
  ibf(v[0], v[2], w[1]); ibf(v[1], v[3], w[1]);
  ibf(v[4], v[6], w[2]); ibf(v[5], v[7], w[2]);
  ibf(v[0], v[4], w[0]); ibf(v[1], v[5], w[0]);
  ibf(v[2], v[6], w[0]); ibf(v[3], v[7], w[0]);
}
// first inverse pass (stages t = 1, 2) on D-order values in [0, 2q)
__device__ __forceinline__ void iD(uint64_t (&v)[8], const ulonglong2 (&w)[6]) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint64_t *u = v + 4 * h;
    ibf(u[0], u[1], w[3 * h + 1]);
    ibf(u[2], u[3], w[3 * h + 2]);
    ibf(u[0], u[2], w[3 * h]);
    ibf(u[1], u[3], w[3 * h]);
  }
}
// passes C and B over np planes holding D-order values after iD (up to a
// __syncthreads); ends synchronised. Full as in fwd_mid.
template <bool Full = true>
__device__ __forceinline__ void inv_mid(uint64_t *sm, int np, const ulonglong2 *iwt) {
  const int t = threadIdx.x;
  {
    ulonglong2 w[7];
    load_c(w, iwt, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane<2, false>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane<2, false>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
  {
    ulonglong2 w[7];
    load_b(w, c1_iwt, t);
    if constexpr (Full) {
#pragma unroll
      for (int i = 0; i < np; ++i) mid_plane<1, false>(sm + i * kPad, w, t);
    } else {
      for (int i = 0; i < np; ++i) mid_plane<1, false>(sm + i * kPad, w, t);
    }
  }
  __syncthreads();
}
// last inverse pass (t = 256, 512, then 1024 with N^-1 folded in); canonical
__device__ __forceinline__ void iA(uint64_t (&v)[8]) {
  ibf(v[0], v[1], c1_iwt[4]); ibf(v[2], v[3], c1_iwt[5]);
  ibf(v[4], v[5], c1_iwt[6]); ibf(v[6], v[7], c1_iwt[7]);
  ibf(v[0], v[2], c1_iwt[2]); ibf(v[1], v[3], c1_iwt[2]);
  ibf(v[4], v[6], c1_iwt[3]); ibf(v[5], v[7], c1_iwt[3]);
  const ulonglong2 ni = c1_nscale[0], wn = c1_nscale[1];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint64_t X = v[k], Y = v[k + 4];
    v[k] = fold2(mulsh(X + Y, ni.x, ni.y));
    v[k + 4] = fold2(mulsh(X - Y + 2 * kQ, wn.x, wn.y));
  }
}

// Four consecutive u64 of a row at D-order positions 4 (t + 256 h) .. + 3.
__device__ __forceinline__ void ld4(const uint64_t *p, uint64_t *v) {
  const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2 *>(p));
  const ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2 *>(p + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// acc_k += v_k * row polynomial `part` (of a row [p0][p1][p0'][p1'], each N),
// each product in [0, 2q)
__device__ __forceinline__ void mac_part(const uint64_t *row, int part, const uint64_t (&v)[8],
                                         uint64_t (&acc)[8], int tid) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int j0 = 4 * (tid + 256 * h);
    uint64_t w[4], ws[4];
    ld4(row + part * kN + j0, w);
    ld4(row + (2 + part) * kN + j0, ws);
#pragma unroll
    for (int m = 0; m < 4; ++m) acc[4 * h + m] += mulsh(v[4 * h + m], w[m], ws[m]);
  }
}
// [0, 2q G) -> [0, 2q) for the running sums (G <= 7 products of [0, 2q)
// plus a folded sum, below 16q < 2^64)
__device__ __forceinline__ uint64_t fold16(uint64_t x) {
  x = min(x, x - 8 * kQ);
  x = min(x, x - 4 * kQ);
  return min(x, x - 2 * kQ);
}

// ------------------------------------------------------------ DB preprocessing
// server.cpp:80-203 with one prime: pt mod q, NTT, the coefficient-major
// transpose as eight byte planes per NTT level, db8[(z 8 + plane)][row][n0p].
constexpr int kDbTile = 4;  // plaintexts per CTA (one plane each)

__global__ void __launch_bounds__(kThreads)
k1p_db_preprocess(Dev1 P, const uint64_t *__restrict__ coeffs, uint64_t coeff_pt_begin,
                  uint64_t seed, uint64_t t, uint64_t logical, uint32_t n0, uint32_t n0p,
                  uint32_t other, uint64_t pt_begin, uint64_t pt_end, uint8_t *__restrict__ db8) {
  extern __shared__ uint64_t sm1[];
  const int tid = threadIdx.x;
  const uint64_t pt0 = pt_begin + static_cast<uint64_t>(blockIdx.x) * kDbTile;
  for (int e = 0; e < kDbTile; ++e) {
    const uint64_t pt = pt0 + e;
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int c = posA(tid, k);
      uint64_t x = 0;
      if (pt < pt_end && pt < logical)
        x = coeffs ? coeffs[(pt - coeff_pt_begin) * kN + c] : mix64(seed + (pt * kN + c + 1) * kGolden) % t;
      v[k] = x;  // x < t < q
    }
    fA(v);
    st_plane<0>(sm1 + e * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid(sm1, kDbTile, P.fwt);
  ulonglong2 wd[6];
  load_d(wd, P.fwt, tid);
  uint64_t out[kDbTile][8];
#pragma unroll
  for (int e = 0; e < kDbTile; ++e) {
    ld_plane<3>(sm1 + e * kPad, out[e], tid);
    fD(out[e], wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) out[e][k] = canon8(out[e][k]);
  }
  const uint64_t row = pt0 / n0, col = pt0 % n0;
  const uint64_t pb = static_cast<uint64_t>(other) * n0p;  // bytes per plane
  if (pt0 + kDbTile <= pt_end && col + kDbTile <= n0 && (col & 3) == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      uint8_t *dst = db8 + static_cast<uint64_t>(posD(tid, k)) * 8 * pb + row * n0p + col;
#pragma unroll
      for (int pl = 0; pl < 8; ++pl) {
        uint32_t w = 0;
#pragma unroll
        for (int e = 0; e < kDbTile; ++e)
          w |= static_cast<uint32_t>((out[e][k] >> (8 * pl)) & 0xFF) << (8 * e);
        *reinterpret_cast<uint32_t *>(dst + pl * pb) = w;
      }
    }
  } else {
#pragma unroll
    for (int e = 0; e < kDbTile; ++e) {
      const uint64_t pt = pt0 + e;
      if (pt >= pt_end) break;
      const uint64_t r = pt / n0, c = pt % n0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        uint8_t *dst = db8 + static_cast<uint64_t>(posD(tid, k)) * 8 * pb + r * n0p + c;
#pragma unroll
        for (int pl = 0; pl < 8; ++pl) dst[pl * pb] = static_cast<uint8_t>(out[e][k] >> (8 * pl));
      }
    }
  }
}

// ------------------------------------------------------------ expansion level
// One heap node per CTA: the BV key switch (bv_keyswitch.cpp:296-367) of the
// node and its two children (server.cpp:794-809): left = c + c', right =
// (c - c') X^-k, sigma_k(c)[j] = +-c[j k^-1 mod 2N]. Digits in groups of 4
// planes; Shoup key products summed below 2q after each group.
constexpr int kGroup = 4;

// Children of the last level in NTT form (the first-dimension leaves), from
// the key switch's sums still in NTT form: with NTT slot i holding the value
// at psi^e_i, e_i = 2 brev(i) + 1 (the reference's bit-reversed order),
// sigma_g(c)^[i] = c^[j] for e_j = e_i g mod 2N, and (f X^-k)^[i] =
// psi^(-k e_i) f^[i]. So left = c^ + sigma(c0)^ + delta^ and right =
// (c^ - sigma(c0)^ - delta^) psi^(-k e), the values k1p_fst_ntt would
// compute from the coefficient-form children; the key switch's two inverse
// NTTs are replaced by forward NTTs of the parent's c0 and c1.
__device__ __forceinline__ void expand_tail_ntt(const Dev1 &P, uint32_t galois, uint32_t kshift,
                                                const uint64_t *ct, const uint64_t (&vb)[8],
                                                const uint64_t (&va)[8], uint64_t *outL,
                                                uint64_t *outR) {
  extern __shared__ uint64_t sm1[];
  const int tid = threadIdx.x;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = ct[p * kN + posA(tid, k)];
    fA(v);
    st_plane<0>(sm1 + p * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid(sm1, 2, P.fwt);
  uint64_t h0[8], h1[8];
  {
    ulonglong2 wd[6];
    load_d(wd, P.fwt, tid);
    ld_plane<3>(sm1, h0, tid);
    ld_plane<3>(sm1 + kPad, h1, tid);
    fD(h0, wd);
    fD(h1, wd);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    h0[k] = canon8(h0[k]);
    h1[k] = canon8(h1[k]);
  }
  st_plane<3>(sm1 + 2 * kPad, h0, tid);  // c0^ by slot, for the sigma gather
  __syncthreads();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint64_t l0[4], l1[4], r0[4], r1[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int k = 4 * h + c;
      const uint32_t i = posD(tid, k);
      const uint32_t e = 2 * (__brev(i) >> 21) + 1;  // 11-bit reversal (N = 2048)
      const uint32_t j = __brev(((e * galois) & (2 * kN - 1)) >> 1) >> 21;
      const uint64_t n0v = add_q(sm1[2 * kPad + padi(j)], vb[k]), n1v = va[k];
      l0[c] = add_q(h0[k], n0v);
      l1[c] = add_q(h1[k], n1v);
      const ulonglong2 lam =
          __ldg(P.pwt + ((2 * kN - ((kshift * e) & (2 * kN - 1))) & (2 * kN - 1)));
      r0[c] = fold2(mulsh(sub_q(h0[k], n0v), lam.x, lam.y));
      r1[c] = fold2(mulsh(sub_q(h1[k], n1v), lam.x, lam.y));
    }
    const int j0 = posD(tid, 4 * h);  // four consecutive slots
    *reinterpret_cast<ulonglong2 *>(outL + j0) = make_ulonglong2(l0[0], l0[1]);
    *reinterpret_cast<ulonglong2 *>(outL + j0 + 2) = make_ulonglong2(l0[2], l0[3]);
    *reinterpret_cast<ulonglong2 *>(outL + kN + j0) = make_ulonglong2(l1[0], l1[1]);
    *reinterpret_cast<ulonglong2 *>(outL + kN + j0 + 2) = make_ulonglong2(l1[2], l1[3]);
    *reinterpret_cast<ulonglong2 *>(outR + j0) = make_ulonglong2(r0[0], r0[1]);
    *reinterpret_cast<ulonglong2 *>(outR + j0 + 2) = make_ulonglong2(r0[2], r0[3]);
    *reinterpret_cast<ulonglong2 *>(outR + kN + j0) = make_ulonglong2(r1[0], r1[1]);
    *reinterpret_cast<ulonglong2 *>(outR + kN + j0 + 2) = make_ulonglong2(r1[2], r1[3]);
  }
}

// One key switch (node node0 + blockIdx.x); NTT_OUT: children in NTT form.
template <bool NTT_OUT>
__device__ __forceinline__ void expand_body(const Dev1 &P, uint32_t galois_inv, uint32_t kshift,
                                            uint32_t galois, uint32_t node0, const uint64_t *in,
                                            uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                                            const uint64_t *const *bv_keys,
                                            uint64_t bv_level_off) {
  extern __shared__ uint64_t sm1[];
  const int node = node0 + blockIdx.x, b = blockIdx.z, tid = threadIdx.x;
  const uint64_t *ct = in + (static_cast<uint64_t>(b) * in_stride + node) * kCtWords;
  const uint64_t *key = bv_keys[b] + bv_level_off;  // rows [b][a][b'][a']
  uint64_t u[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t j = posA(tid, k);
    const uint32_t w = (j * galois_inv) & (2 * kN - 1);
    const uint64_t a = ct[kN + (w & (kN - 1))];
    u[k] = digit_source<kLKs, kBaseKs>(w >= kN ? neg_q(a) : a);  // sigma_k(c1)
  }
  uint64_t ab[8], aa[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) ab[k] = aa[k] = 0;
  for (int g = 0; g < kLKs / kGroup; ++g) {
#pragma unroll
    for (int e = 0; e < kGroup; ++e) {
      uint64_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = digit_res<kBaseKs>(u[k], g * kGroup + e);
      fA(v);
      st_plane<0>(sm1 + e * kPad, v, tid);
    }
    __syncthreads();
    fwd_mid(sm1, kGroup, P.fwt);
    ulonglong2 wd[6];
    load_d(wd, P.fwt, tid);
    for (int e = 0; e < kGroup; ++e) {
      const uint64_t *R = key + static_cast<uint64_t>(g * kGroup + e) * kRowWords;
      uint64_t v[8];
      ld_plane<3>(sm1 + e * kPad, v, tid);
      fD(v, wd);
      mac_part(R, 0, v, ab, tid);
      mac_part(R, 1, v, aa, tid);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) { ab[k] = fold16(ab[k]); aa[k] = fold16(aa[k]); }
    __syncthreads();
  }
  uint64_t *outL = out + (static_cast<uint64_t>(b) * out_stride + 2ull * node) * kCtWords;
  uint64_t *outR = outL + kCtWords;
  if constexpr (NTT_OUT) {
    uint64_t vb[8], va[8];  // the key switch's delta in NTT form, canonical
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      vb[k] = fold2(ab[k]);
      va[k] = fold2(aa[k]);
    }
    expand_tail_ntt(P, galois, kshift, ct, vb, va, outL, outR);
    return;
  }
  {
    ulonglong2 wd[6];
    load_d(wd, P.iwt, tid);
    iD(ab, wd);  // [0, 2q) in
    iD(aa, wd);
    st_plane<3>(sm1, ab, tid);
    st_plane<3>(sm1 + kPad, aa, tid);
  }
  __syncthreads();
  inv_mid(sm1, 2, P.iwt);
  uint64_t db_[8], da[8];
  ld_plane<0>(sm1, db_, tid);
  ld_plane<0>(sm1 + kPad, da, tid);
  iA(db_);
  iA(da);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t j = posA(tid, k);
    const uint32_t w = (j * galois_inv) & (2 * kN - 1);
    const uint64_t z = ct[w & (kN - 1)];
    const uint64_t s0 = w >= kN ? neg_q(z) : z;  // sigma_k(c0)
    const uint64_t n0v = add_q(s0, db_[k]), n1v = da[k];
    const uint64_t o0 = ct[j], o1 = ct[kN + j];
    outL[j] = add_q(o0, n0v);
    outL[kN + j] = add_q(o1, n1v);
    const uint64_t d0 = sub_q(o0, n0v), d1 = sub_q(o1, n1v);
    int dst = static_cast<int>(j) - static_cast<int>(kshift);
    const bool wrap = dst < 0;
    if (wrap) dst += kN;
    outR[dst] = wrap ? neg_q(d0) : d0;
    outR[kN + dst] = wrap ? neg_q(d1) : d1;
  }
}

// MINB CTAs per SM: 2 (128 registers, a few spilled) when a level fills
// the GPU twice over, else 1 (no spills, lower latency per CTA).
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
k1p_expand_level(Dev1 P, uint32_t galois_inv, uint32_t kshift, const uint64_t *__restrict__ in,
                 uint64_t in_stride, uint64_t *__restrict__ out, uint64_t out_stride,
                 const uint64_t *const *__restrict__ bv_keys, uint64_t bv_level_off,
                 uint32_t node0) {
  expand_body<false>(P, galois_inv, kshift, 0, node0, in, in_stride, out, out_stride, bv_keys,
                     bv_level_off);
}
// The last level's nodes below ntt_nodes when the first-dimension leaves are
// wanted in NTT form (expand_tail_ntt); k1p_expand_level takes the others.
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
k1p_expand_level_ntt(Dev1 P, uint32_t galois, uint32_t galois_inv, uint32_t kshift,
                     const uint64_t *__restrict__ in, uint64_t in_stride,
                     uint64_t *__restrict__ out, uint64_t out_stride,
                     const uint64_t *const *__restrict__ bv_keys, uint64_t bv_level_off) {
  expand_body<true>(P, galois_inv, kshift, galois, 0, in, in_stride, out, out_stride, bv_keys,
                    bv_level_off);
}

// ------------------------------------------------------------ gadget product
// The external product's decomposition and MAC (gsw.cpp:119-182, 252-295):
// each polynomial p of the decomposed ciphertext (y - x, or x when y is
// null) split into L balanced base-2^B digits; digit d of poly p meets row
// p L + (L - 1 - d) (MSB-first rows). Digit planes in groups of up to 5;
// sums folded below 2q after each group.
template <int L, int B, bool Full = true>
__device__ __forceinline__ void gadget_mac(const Dev1 &P, const uint64_t *x, const uint64_t *y,
                                           const uint64_t *rgsw, uint64_t *sm,
                                           uint64_t (&acc0)[8], uint64_t (&acc1)[8]) {
  constexpr int G = L <= 5 ? L : kGroup;
  static_assert(L % G == 0, "digit groups of equal size");
  const int tid = threadIdx.x;
#pragma unroll 1
  for (int p = 0; p < 2; ++p) {
    uint64_t u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posA(tid, k);
      uint64_t v = x[p * kN + j];
      if (y != nullptr) v = sub_q(y[p * kN + j], v);
      u[k] = digit_source<L, B>(v);
    }
#pragma unroll 1
    for (int g = 0; g < L / G; ++g) {
#pragma unroll
      for (int e = 0; e < G; ++e) {
        uint64_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = digit_res<B>(u[k], g * G + e);
        fA(v);
        st_plane<0>(sm + e * kPad, v, tid);
      }
      __syncthreads();
      fwd_mid<Full>(sm, G, P.fwt);
      ulonglong2 wd[6];
      load_d(wd, P.fwt, tid);
      for (int e = 0; e < G; ++e) {
        const int d = g * G + e;
        const uint64_t *R = rgsw + static_cast<uint64_t>(p * L + (L - 1 - d)) * kRowWords;
        uint64_t v[8];
        ld_plane<3>(sm + e * kPad, v, tid);
        fD(v, wd);
        mac_part(R, 0, v, acc0, tid);  // row [c0][c1][c0'][c1']
        mac_part(R, 1, v, acc1, tid);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) { acc0[k] = fold16(acc0[k]); acc1[k] = fold16(acc1[k]); }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ selectors
// complete_selectors / query_to_gsw (server.cpp:823-855, gsw.cpp:317-357):
// the top row is the expanded row itself in NTT form, the bottom row its
// external product with RGSW(s); both stored with Shoup companions.
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
k1p_selectors(Dev1 P, Shape1 S, const uint64_t *__restrict__ leaves, uint64_t leaf_stride,
              const uint64_t *const *__restrict__ gsw_keys, uint64_t *__restrict__ sel) {
  extern __shared__ uint64_t sm1[];
  const int row_id = blockIdx.x, b = blockIdx.z, tid = threadIdx.x;
  const int selno = row_id / S.l_ep, r = row_id % S.l_ep;
  const uint64_t *ct = leaves + (static_cast<uint64_t>(b) * leaf_stride + S.n0 + row_id) * kCtWords;
  uint64_t *outs = sel + (static_cast<uint64_t>(b) * (S.num_dims - 1) + selno) * 2 * S.l_ep * kRowWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  gadget_mac<kLKey, kBaseKey, false>(P, ct, nullptr, gsw_keys[b], sm1, acc0, acc1);
  uint64_t *bot = outs + static_cast<uint64_t>(S.l_ep + r) * kRowWords;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int j = posD(tid, k);
    const uint64_t v0 = fold2(acc0[k]), v1 = fold2(acc1[k]);
    bot[j] = v0;
    bot[kN + j] = v1;
    bot[2 * kN + j] = shoup_of(v0);
    bot[3 * kN + j] = shoup_of(v1);
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = ct[p * kN + posA(tid, k)];
    fA(v);
    st_plane<0>(sm1 + p * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid<false>(sm1, 2, P.fwt);
  ulonglong2 wd[6];
  load_d(wd, P.fwt, tid);
  uint64_t *top = outs + static_cast<uint64_t>(r) * kRowWords;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
    ld_plane<3>(sm1 + p * kPad, v, tid);
    fD(v, wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posD(tid, k);
      const uint64_t c = canon8(v[k]);
      top[p * kN + j] = c;
      top[2 * kN + p * kN + j] = shoup_of(c);
    }
  }
}

// ------------------------------------------------------------ first-dim query
// Forward NTT of the first n0 leaves (server.cpp:313-361) into qm[col][k][z]
// (col = 2 query + poly), then k1p_fst_pack transposes it through shared
// memory into the scan's eight byte planes qb[(z 8 + plane)][col][n0p].
constexpr int kFstTile = 2;  // leaves per CTA (4 planes)

__global__ void __launch_bounds__(kThreads)
k1p_fst_ntt(Dev1 P, Shape1 S, const uint64_t *__restrict__ leaves, uint64_t leaf_stride,
            uint64_t *__restrict__ qm) {
  extern __shared__ uint64_t sm1[];
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t k0 = blockIdx.x * kFstTile;
  for (int e = 0; e < 2 * kFstTile; ++e) {
    const uint32_t kk = k0 + (e >> 1);
    const int p = e & 1;
    const uint64_t *src = leaves + (static_cast<uint64_t>(b) * leaf_stride + kk) * kCtWords + p * kN;
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = kk < S.n0 ? src[posA(tid, k)] : 0;
    fA(v);
    st_plane<0>(sm1 + e * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid(sm1, 2 * kFstTile, P.fwt);
  ulonglong2 wd[6];
  load_d(wd, P.fwt, tid);
  for (int e = 0; e < 2 * kFstTile; ++e) {
    const uint32_t kk = k0 + (e >> 1);
    if (kk >= S.n0) continue;  // uniform over the CTA
    const int p = e & 1;
    uint64_t v[8];
    ld_plane<3>(sm1 + e * kPad, v, tid);
    fD(v, wd);
    uint64_t *dst = qm + (static_cast<uint64_t>(2 * b + p) * S.n0 + kk) * kN;
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // D-order positions 4 (tid + 256 h) .. + 3
      const int j0 = posD(tid, 4 * h);
      *reinterpret_cast<ulonglong2 *>(dst + j0) =
          make_ulonglong2(canon8(v[4 * h + 0]), canon8(v[4 * h + 1]));
      *reinterpret_cast<ulonglong2 *>(dst + j0 + 2) =
          make_ulonglong2(canon8(v[4 * h + 2]), canon8(v[4 * h + 3]));
    }
  }
}

// A CTA transposes 32 coefficients z x 128 leaves k of one column through
// shared memory (z-major tile, 16-k runs 18 words apart, rows 145 apart),
// then one thread per (z, 16 consecutive k) writes that run's eight byte
// planes, 16 bytes each; k in [n0, n0p) reads as zero.
constexpr int kPackZ = 32, kPackK = 128, kRunPitch = 18, kRowPitch = 145;
__global__ void __launch_bounds__(256)
k1p_fst_pack(const uint64_t *__restrict__ qm, uint64_t q_stride, uint64_t p_stride,
             uint64_t k_stride, uint32_t n0, uint32_t n0p, uint32_t ncols,
             uint8_t *__restrict__ qb) {
  __shared__ uint64_t tile[(kPackZ - 1) * kRowPitch + (kPackK / 16 - 1) * kRunPitch + 16];
  const uint32_t z0 = blockIdx.x * kPackZ, col = blockIdx.y, k0 = blockIdx.z * kPackK;
  const int t = threadIdx.x;
  // column col = 2 query + poly: qm (q_stride = 2 p_stride, p_stride = n0 N,
  // k_stride = N) or NTT-form leaves (q_stride = slots 2N, p_stride = N,
  // k_stride = 2N)
  const uint64_t *src = qm + (col >> 1) * q_stride + (col & 1) * p_stride + z0;
#pragma unroll 4
  for (int i = t; i < kPackK * kPackZ; i += 256) {
    const int kk = i / kPackZ, zz = i % kPackZ;
    const uint32_t k = k0 + kk;
    tile[zz * kRowPitch + (kk / 16) * kRunPitch + kk % 16] =
        k < n0 ? src[static_cast<uint64_t>(k) * k_stride + zz] : 0;
  }
  __syncthreads();
  const int chunk = t % (kPackK / 16), zz = t / (kPackK / 16);
  const uint64_t *run = tile + zz * kRowPitch + chunk * kRunPitch;
  uint32_t w[8][4];
#pragma unroll
  for (int pl = 0; pl < 8; ++pl)
#pragma unroll
    for (int j = 0; j < 4; ++j) w[pl][j] = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const uint64_t v = run[i];
#pragma unroll
    for (int pl = 0; pl < 8; ++pl)
      w[pl][i >> 2] |= static_cast<uint32_t>((v >> (8 * pl)) & 0xFF) << (8 * (i & 3));
  }
  const uint64_t pb = static_cast<uint64_t>(ncols) * n0p;
  const uint64_t z = z0 + zz;
  const uint32_t k = k0 + chunk * 16;
  if (k >= n0p) return;
  uint8_t *dst = qb + z * 8 * pb + static_cast<uint64_t>(col) * n0p + k;
#pragma unroll
  for (int pl = 0; pl < 8; ++pl)
    *reinterpret_cast<uint4 *>(dst + pl * pb) = make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
}

// ------------------------------------------------------------ scan epilogue
// inter_to_cts (server.cpp:408-527): the scan's cmat[z][col][row] gathered
// into candidate ciphertexts and INTT'd. A CTA transforms 4 consecutive
// rows of one column.
constexpr int kEpiRows = 4;

__global__ void __launch_bounds__(kThreads)
k1p_epilogue(Dev1 P, Shape1 S, const uint64_t *__restrict__ cmat, uint32_t ncols,
             uint64_t *__restrict__ mid, uint64_t mid_stride) {
  extern __shared__ uint64_t sm1[];
  const int tid = threadIdx.x;
  const uint32_t r0 = blockIdx.x * kEpiRows, c = blockIdx.z;
  {
    uint64_t v[kEpiRows][8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint64_t z = posD(tid, k);
      const uint64_t *src = cmat + (z * ncols + c) * S.other + r0;
#pragma unroll
      for (int e = 0; e < kEpiRows; ++e) v[e][k] = r0 + e < S.other ? src[e] : 0;
    }
    ulonglong2 wd[6];
    load_d(wd, P.iwt, tid);
#pragma unroll
    for (int e = 0; e < kEpiRows; ++e) {
      iD(v[e], wd);
      st_plane<3>(sm1 + e * kPad, v[e], tid);
    }
  }
  __syncthreads();
  inv_mid(sm1, kEpiRows, P.iwt);
  for (int e = 0; e < kEpiRows; ++e) {
    const uint32_t r = r0 + e;
    if (r >= S.other) break;  // uniform over the CTA
    uint64_t w[8];
    ld_plane<0>(sm1 + e * kPad, w, tid);
    iA(w);
    uint64_t *dst = mid + (static_cast<uint64_t>(c >> 1) * mid_stride + r) * kCtWords + (c & 1) * kN;
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[posA(tid, k)] = w[k];
  }
}

// ------------------------------------------------------------ MUX level
// ext_prod_mux (server.cpp:652-722): out = x + INTT(ExtProd(sel, y - x)).
__global__ void __launch_bounds__(kThreads)
k1p_mux_level(Dev1 P, Shape1 S, uint32_t level, uint32_t n_pairs, uint32_t offset, uint32_t half,
              const uint64_t *__restrict__ in, uint64_t *__restrict__ out, uint64_t mid_stride,
              const uint64_t *__restrict__ sel) {
  extern __shared__ uint64_t sm1[];
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t i = blockIdx.x;
  const uint64_t *base_in = in + static_cast<uint64_t>(b) * mid_stride * kCtWords;
  uint64_t *base_out = out + static_cast<uint64_t>(b) * mid_stride * kCtWords;
  if (i >= n_pairs) {  // level 0: carry the unpaired prefix over unchanged
    const uint64_t c = i - n_pairs;
    for (int j = tid; j < kCtWords; j += kThreads) base_out[c * kCtWords + j] = base_in[c * kCtWords + j];
    return;
  }
  uint32_t xi, yi, oi;
  if (level == 0) { xi = offset + 2 * i; yi = xi + 1; oi = offset + i; }
  else { xi = i; yi = i + half; oi = i; }
  const uint64_t *x = base_in + static_cast<uint64_t>(xi) * kCtWords;
  const uint64_t *y = base_in + static_cast<uint64_t>(yi) * kCtWords;
  const uint64_t *rgsw =
      sel + (static_cast<uint64_t>(b) * (S.num_dims - 1) + level) * 2 * kLEp * kRowWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  gadget_mac<kLEp, kBaseEp>(P, x, y, rgsw, sm1, acc0, acc1);
  {
    ulonglong2 wd[6];
    load_d(wd, P.iwt, tid);
    iD(acc0, wd);  // [0, 2q) in
    iD(acc1, wd);
    st_plane<3>(sm1, acc0, tid);
    st_plane<3>(sm1 + kPad, acc1, tid);
  }
  __syncthreads();
  inv_mid(sm1, 2, P.iwt);
  uint64_t *o = base_out + static_cast<uint64_t>(oi) * kCtWords;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
    ld_plane<0>(sm1 + p * kPad, v, tid);
    iA(v);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posA(tid, k);
      o[p * kN + j] = add_q(x[p * kN + j], v[k]);
    }
  }
}

// ------------------------------------------------------------ modulus switch
// mod_switch_inplace (server.cpp:1025-1043) with utils::rescale
// (utils.cpp:445-462): centred round(v small_q / q), then the response bit
// packing of save_resp_to_stream (server.cpp:950-1009).
__device__ __forceinline__ uint64_t rescale_q(uint64_t v, uint64_t outm) {
  const int64_t inp = static_cast<int64_t>(kQ);
  int64_t c = static_cast<int64_t>(v);
  if (c >= inp / 2) c -= inp;
  const bool neg = c < 0;
  const uint64_t mag = neg ? static_cast<uint64_t>(-c) : static_cast<uint64_t>(c);
  const u128 num = static_cast<u128>(mag) * outm + static_cast<uint64_t>(inp / 2);
  const uint64_t quo = static_cast<uint64_t>(num / kQ) % outm;
  return neg ? (quo ? outm - quo : 0) : quo;
}

__global__ void __launch_bounds__(256)
k1p_modswitch(Dev1 P, const uint64_t *__restrict__ ct_all, uint64_t ct_stride,
              uint64_t *__restrict__ resp, uint8_t *__restrict__ bytes, uint32_t resp_bytes) {
  extern __shared__ uint64_t vals[];  // 2N when packing
  const int b = blockIdx.x;
  const uint64_t *ct = ct_all + static_cast<uint64_t>(b) * ct_stride * kCtWords;
  for (int idx = threadIdx.x; idx < 2 * kN; idx += blockDim.x) {
    const uint64_t r = rescale_q(ct[idx], P.small_q);
    resp[static_cast<uint64_t>(b) * 2 * kN + idx] = r;
    if (bytes) vals[idx] = r;
  }
  if (bytes == nullptr) return;
  __syncthreads();
  const uint32_t w = P.small_q_width;
  for (uint32_t B = threadIdx.x; B < resp_bytes; B += blockDim.x) {
    const uint64_t bit0 = 8ull * B;
    const uint32_t i = static_cast<uint32_t>(bit0 / w), o = static_cast<uint32_t>(bit0 % w);
    uint64_t v = vals[i] >> o;
    const uint32_t have = w - o;
    if (have < 8 && i + 1 < 2 * kN) v |= vals[i + 1] << have;
    bytes[static_cast<uint64_t>(b) * resp_bytes + B] = static_cast<uint8_t>(v & 0xFF);
  }
}

}  // namespace

// ===================================================================== launchers
void upload_constants(const uint64_t *fw, const uint64_t *fw_sh, const uint64_t *iw,
                      const uint64_t *iw_sh, const uint64_t ninv[2], const uint64_t w1ninv[2]) {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return;
  ulonglong2 f[64], i[64], sc[2];
  for (int k = 0; k < 64; ++k) {
    f[k] = make_ulonglong2(fw[k], fw_sh[k]);
    i[k] = make_ulonglong2(iw[k], iw_sh[k]);
  }
  sc[0] = make_ulonglong2(ninv[0], ninv[1]);
  sc[1] = make_ulonglong2(w1ninv[0], w1ninv[1]);
  cudaError_t e = cudaMemcpyToSymbol(c1_fwt, f, sizeof(f));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c1_iwt, i, sizeof(i));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c1_nscale, sc, sizeof(sc));
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("CONFIG_N2048_K1 NTT constants: ") + cudaGetErrorString(e));
  done.insert(dev);
}

void launch_db_preprocess(const Dev1 &P, const Shape1 &s, const uint64_t *coeffs,
                          uint64_t coeff_pt_begin, uint64_t seed, uint64_t t, uint64_t logical,
                          uint64_t pt_begin, uint64_t pt_end, uint8_t *db8, cudaStream_t st) {
  if (pt_end <= pt_begin) return;
  if (pt_end > static_cast<uint64_t>(s.other) * s.n0) throw std::invalid_argument("db tile beyond the layout");
  const size_t smem = plane_bytes(kDbTile);
  set_smem(k1p_db_preprocess, smem);
  const uint64_t tiles = (pt_end - pt_begin + kDbTile - 1) / kDbTile;
  k1p_db_preprocess<<<static_cast<unsigned>(tiles), kThreads, smem, st>>>(
      P, coeffs, coeff_pt_begin, seed, t, logical, s.n0, s.n0p, s.other, pt_begin, pt_end, db8);
  check_launch("k1p_db_preprocess");
}

void launch_expand_level(const Dev1 &P, const Shape1 &s, uint32_t d, const uint64_t *in,
                         uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                         const uint64_t *const *bv_keys, uint64_t bv_level_stride, uint32_t batch,
                         cudaStream_t st, uint32_t ntt_nodes) {
  const uint32_t nodes = opir4::expand_nodes(s, d);
  const size_t smem = plane_bytes(kGroup);
  const uint32_t k = 1u << d;
  const uint32_t galois = kN / k + 1;
  uint32_t galois_inv = 1;  // galois^-1 mod 2N (galois is odd)
  while (((galois_inv * galois) & (2 * kN - 1)) != 1) galois_inv += 2;
  const uint64_t koff = d * bv_level_stride;
  static_assert(kGroup >= 3, "the NTT-form tail uses three planes");
  if (ntt_nodes > nodes || (ntt_nodes > 0 && d + 1 != s.h))
    throw std::invalid_argument("NTT-form children only at the last expansion level");
  if (ntt_nodes > 0) {
    const dim3 grid(ntt_nodes, 1, batch);
    if (static_cast<uint64_t>(ntt_nodes) * batch >= 2ull * sms()) {
      set_smem(k1p_expand_level_ntt<2>, smem);
      k1p_expand_level_ntt<2><<<grid, kThreads, smem, st>>>(P, galois, galois_inv, k, in,
                                                             in_stride, out, out_stride, bv_keys,
                                                             koff);
    } else {
      set_smem(k1p_expand_level_ntt<1>, smem);
      k1p_expand_level_ntt<1><<<grid, kThreads, smem, st>>>(P, galois, galois_inv, k, in,
                                                             in_stride, out, out_stride, bv_keys,
                                                             koff);
    }
    check_launch("k1p_expand_level_ntt");
  }
  const uint32_t rest = nodes - ntt_nodes;  // coefficient-form children
  if (rest == 0) return;
  const dim3 grid(rest, 1, batch);
  if (static_cast<uint64_t>(rest) * batch >= 2ull * sms()) {
    set_smem(k1p_expand_level<2>, smem);
    k1p_expand_level<2><<<grid, kThreads, smem, st>>>(P, galois_inv, k, in, in_stride, out,
                                                       out_stride, bv_keys, koff, ntt_nodes);
  } else {
    set_smem(k1p_expand_level<1>, smem);
    k1p_expand_level<1><<<grid, kThreads, smem, st>>>(P, galois_inv, k, in, in_stride, out,
                                                       out_stride, bv_keys, koff, ntt_nodes);
  }
  check_launch("k1p_expand_level");
}

void launch_selectors(const Dev1 &P, const Shape1 &s, const uint64_t *leaves, uint64_t leaf_stride,
                      const uint64_t *const *gsw_keys, uint64_t *sel, uint32_t batch,
                      cudaStream_t st) {
  if (s.num_dims <= 1) return;
  const size_t smem = plane_bytes(kGroup);
  const uint32_t rows = (s.num_dims - 1) * s.l_ep;
  const dim3 grid(rows, 1, batch);
  if (static_cast<uint64_t>(rows) * batch >= 2ull * sms()) {
    set_smem(k1p_selectors<2>, smem);
    k1p_selectors<2><<<grid, kThreads, smem, st>>>(P, s, leaves, leaf_stride, gsw_keys, sel);
  } else {
    set_smem(k1p_selectors<1>, smem);
    k1p_selectors<1><<<grid, kThreads, smem, st>>>(P, s, leaves, leaf_stride, gsw_keys, sel);
  }
  check_launch("k1p_selectors");
}

void launch_fst_ntt(const Dev1 &P, const Shape1 &s, const uint64_t *leaves, uint64_t leaf_stride,
                    uint64_t *qm, uint32_t batch, cudaStream_t st) {
  const size_t smem = plane_bytes(2 * kFstTile);
  set_smem(k1p_fst_ntt, smem);
  k1p_fst_ntt<<<dim3((s.n0 + kFstTile - 1) / kFstTile, 1, batch), kThreads, smem, st>>>(
      P, s, leaves, leaf_stride, qm);
  check_launch("k1p_fst_ntt");
}

void launch_fst_pack(const Shape1 &s, const uint64_t *qm, uint8_t *qb, uint32_t batch,
                     cudaStream_t st) {
  const uint32_t ncols = 2 * batch;
  const dim3 grid(kN / kPackZ, ncols, (s.n0p + kPackK - 1) / kPackK);
  const uint64_t p_stride = static_cast<uint64_t>(s.n0) * kN;
  k1p_fst_pack<<<grid, 256, 0, st>>>(qm, 2 * p_stride, p_stride, kN, s.n0, s.n0p, ncols, qb);
  check_launch("k1p_fst_pack");
}

void launch_fst_pack_leaves(const Shape1 &s, const uint64_t *leaves, uint64_t leaf_stride,
                            uint8_t *qb, uint32_t batch, cudaStream_t st) {
  const uint32_t ncols = 2 * batch;
  const dim3 grid(kN / kPackZ, ncols, (s.n0p + kPackK - 1) / kPackK);
  k1p_fst_pack<<<grid, 256, 0, st>>>(leaves, leaf_stride * kCtWords, kN, kCtWords, s.n0, s.n0p,
                                      ncols, qb);
  check_launch("k1p_fst_pack");
}

void launch_epilogue(const Dev1 &P, const Shape1 &s, const uint64_t *cmat, uint64_t *mid,
                     uint64_t mid_stride, uint32_t batch, cudaStream_t st) {
  const size_t smem = plane_bytes(kEpiRows);
  set_smem(k1p_epilogue, smem);
  const uint32_t ncols = 2 * batch;
  k1p_epilogue<<<dim3((s.other + kEpiRows - 1) / kEpiRows, 1, ncols), kThreads, smem, st>>>(
      P, s, cmat, ncols, mid, mid_stride);
  check_launch("k1p_epilogue");
}

void launch_mux_level(const Dev1 &P, const Shape1 &s, uint32_t level, uint32_t tree_h,
                      const uint64_t *in, uint64_t *out, uint64_t mid_stride, const uint64_t *sel,
                      uint32_t batch, cudaStream_t st) {
  const uint32_t h = tree_h;
  if (h == 0 || h > 31 || level >= h || h > s.num_dims - 1)
    throw std::invalid_argument("MUX level outside its selector tree");
  uint32_t n_pairs, offset = 0, half = 0, copies = 0;
  if (level == 0 && (s.other > (1u << h) || 2ull * s.other < (1ull << h)))
    throw std::invalid_argument("MUX tree: candidate count outside (2^(d-2), 2^(d-1)]");
  if (level == 0) {
    const uint32_t last = 2 * s.other - (1u << h);
    offset = s.other - last;
    n_pairs = last / 2;
    copies = offset;
  } else {
    half = (1u << (h - level)) >> 1;
    n_pairs = half;
  }
  const size_t smem = plane_bytes(kLEp);
  set_smem(k1p_mux_level, smem);
  k1p_mux_level<<<dim3(n_pairs + copies, 1, batch), kThreads, smem, st>>>(
      P, s, level, n_pairs, offset, half, in, out, mid_stride, sel);
  check_launch("k1p_mux_level");
}

void launch_modswitch(const Dev1 &P, const uint64_t *ct, uint64_t ct_stride, uint64_t *resp,
                      uint8_t *bytes, uint32_t resp_bytes, uint32_t batch, cudaStream_t st) {
  const size_t smem = bytes ? 2 * kN * sizeof(uint64_t) : 0;
  if (smem) set_smem(k1p_modswitch, smem);
  k1p_modswitch<<<batch, 256, smem, st>>>(P, ct, ct_stride, resp, bytes, resp_bytes);
  check_launch("k1p_modswitch");
}

}  // namespace opir1
