// sm_100a kernels of the server path for CONFIG_N4096_K2_MP (N = 4096, two
// 60-bit RNS limbs, includes/database_constants.h:111-125). Every polynomial
// kernel runs 512 threads and one CTA per (item, limb, query); limb-major
// ciphertexts [c0 l0][c0 l1][c1 l0][c1 l1] u64 stay in the reference's own
// layout (rlwe.h:17-31), so no split or compose is needed at the boundary.
#include "opir_c4_kernels.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

#include "opir_c4_device.cuh"

#include <cooperative_groups.h>

namespace opir4 {

namespace {

using u128 = unsigned __int128;
using i128 = __int128;

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;
constexpr u128 kQQ = static_cast<u128>(kQ0) * kQ1;
constexpr int kLKs = 8, kBaseKs = 16, kLKey = 8, kBaseKey = 15, kLEp = 5, kBaseEp = 24;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

std::atomic<uint64_t> g_launches4{0};

void check_launch(const char *what) {
  g_launches4.fetch_add(1, std::memory_order_relaxed);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// SMs of the current device (cached per device).
int sm_count() {
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
    n = 148;
  }
  cache[dev] = n;
  return n;
}

// Cluster-split levels (k4_expand_level_split, k4_mux_level_split): on
// unless OPIR_SPLIT=0.
bool split_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("OPIR_SPLIT");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

// Launch with a 1-D cluster of `c` CTAs along x.
template <typename Kern, typename... Args>
void launch_cluster(Kern kernel, int c, dim3 grid, size_t smem, cudaStream_t st, const char *what,
                    Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = c;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, args...);
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
  check_launch(what);
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

// 8 consecutive u64 (D-order positions 8t .. 8t+7) as four 16-byte loads
__device__ __forceinline__ void ld8(const uint64_t *p, uint64_t (&v)[8]) {
  const ulonglong2 *q = reinterpret_cast<const ulonglong2 *>(p);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const ulonglong2 x = __ldg(q + i);
    v[2 * i] = x.x;
    v[2 * i + 1] = x.y;
  }
}

// ------------------------------------------------------------ gadget digits
// Balanced BV digits (bv_keyswitch.cpp:42-62) lie in (-B/2, B/2]: the
// centred value plus C = (B/2 - 1) sum_i B^i has plain base-B digits
// u_i = r_i + B/2 - 1 (|c| < Q/2 < 2^119 < B^L / 2).
template <int L, int B>
__device__ __forceinline__ u128 bv_digit_source(u128 x) {
  u128 C = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) C += static_cast<u128>((1ull << (B - 1)) - 1) << (B * i);
  return x + C - (x > kQQ / 2 ? kQQ : 0);
}
template <int B>
__device__ __forceinline__ uint64_t field(u128 u, int i) {
  return static_cast<uint64_t>(u >> (B * i)) & ((1ull << B) - 1);
}

// ------------------------------------------------------------ DB preprocessing
// server.cpp:80-203 per limb: pt mod q_k, NTT, transpose into the
// coefficient-major layout -- here as eight byte planes per NTT level,
// db8[(z 8 + plane)][row][n0p] (z = limb N + level), the tensor-core scan's
// A operand. A CTA transforms 4 consecutive plaintexts; when they are 4
// consecutive columns of one row their bytes go out as one 32-bit store.
constexpr int kDbTile = 4;  // plaintexts per CTA (one padded plane each)

template <int L>
__device__ __forceinline__ void db_body(const Dev4 &P, const uint64_t *coeffs,
                                        uint64_t coeff_pt_begin, uint64_t seed, uint64_t t,
                                        uint64_t logical, uint32_t n0, uint32_t n0p,
                                        uint32_t other, uint64_t pt_begin, uint64_t pt_end,
                                        const uint32_t *row_map, uint8_t *db8) {
  extern __shared__ uint64_t sm4[];
  const int tid = threadIdx.x;
  const uint64_t pt0 = pt_begin + static_cast<uint64_t>(blockIdx.x) * kDbTile;
  for (int e = 0; e < kDbTile; ++e) {
    const uint64_t pt = pt0 + e;
    // the database plaintext stored at local position pt (a row shard keeps
    // some of the rows; pt < pt_end keeps pt / n0 below the shard's rows)
    const uint64_t gpt = (row_map && pt < pt_end) ? static_cast<uint64_t>(row_map[pt / n0]) * n0 + pt % n0 : pt;
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int c = posA(tid, k);
      uint64_t x = 0;
      if (pt < pt_end && gpt < logical)
        x = coeffs ? coeffs[(pt - coeff_pt_begin) * kN + c] : mix64(seed + (gpt * kN + c + 1) * kGolden) % t;
      v[k] = x;  // x < t < q: canonical (server.cpp:172-180 reduces pt mod q_k)
    }
    fA<L>(v);
    st_plane<0>(sm4 + e * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid<L>(sm4, kDbTile, P.T);
  ulonglong2 wd[7];
  fload_d<L>(wd, P.T);
  uint64_t out[kDbTile][8];
#pragma unroll
  for (int e = 0; e < kDbTile; ++e) {
    ld_plane<3>(sm4 + e * kPad, out[e], tid);
    fD<L>(out[e], wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) out[e][k] = canon8<Limb<L>::q>(out[e][k]);
  }
  const uint64_t row = pt0 / n0, col = pt0 % n0;
  const uint64_t plane_bytes = static_cast<uint64_t>(other) * n0p;
  // 4 plaintexts in one row from a column that is a multiple of 4: the
  // address (n0p and every plane size are multiples of 16) is 4-byte aligned
  if (pt0 + kDbTile <= pt_end && col + kDbTile <= n0 && (col & 3) == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint64_t z = static_cast<uint64_t>(L) * kN + posD(tid, k);
      uint8_t *dst = db8 + z * 8 * plane_bytes + row * n0p + col;
#pragma unroll
      for (int pl = 0; pl < 8; ++pl) {
        uint32_t w = 0;
#pragma unroll
        for (int e = 0; e < kDbTile; ++e)
          w |= static_cast<uint32_t>((out[e][k] >> (8 * pl)) & 0xFF) << (8 * e);
        *reinterpret_cast<uint32_t *>(dst + pl * plane_bytes) = w;
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
        const uint64_t z = static_cast<uint64_t>(L) * kN + posD(tid, k);
        uint8_t *dst = db8 + z * 8 * plane_bytes + r * n0p + c;
#pragma unroll
        for (int pl = 0; pl < 8; ++pl) dst[pl * plane_bytes] = static_cast<uint8_t>(out[e][k] >> (8 * pl));
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1)
k4_db_preprocess(Dev4 P, const uint64_t *__restrict__ coeffs, uint64_t coeff_pt_begin,
                 uint64_t seed, uint64_t t, uint64_t logical, uint32_t n0, uint32_t n0p,
                 uint32_t other, uint64_t pt_begin, uint64_t pt_end,
                 const uint32_t *__restrict__ row_map, uint8_t *__restrict__ db8) {
  if (blockIdx.y == 0)
    db_body<0>(P, coeffs, coeff_pt_begin, seed, t, logical, n0, n0p, other, pt_begin, pt_end, row_map, db8);
  else
    db_body<1>(P, coeffs, coeff_pt_begin, seed, t, logical, n0, n0p, other, pt_begin, pt_end, row_map, db8);
}

// ------------------------------------------------------------ expansion level
// One heap node, one limb per CTA: the K = 2 BV key switch of the node
// (bv_keyswitch.cpp:373-481) and its two children (server.cpp:794-809).
// Digits come from the CRT composition of sigma_k(c1) over both limbs. Key
// products are Shoup products in [0, 2q) with the rows' stored companions,
// so eight rows sum below 16q in 64 bits.
constexpr int kExpGroup = 4;  // digit planes per group

// Children of the last level in NTT form (the first-dimension leaves), from
// the key switch's sums still in NTT form: with NTT slot i holding the value
// at psi^e_i, e_i = 2 brev(i) + 1 (the reference's bit-reversed order),
// sigma_g(c)^[i] = c^[j] for e_j = e_i g mod 2N, and (f X^-k)^[i] =
// psi^(-k e_i) f^[i]. So left = c^ + sigma(c0)^ + delta^ and right =
// (c^ - sigma(c0)^ - delta^) psi^(-k e), the values k4_fst_ntt would compute
// from the coefficient-form children; the key switch's two inverse NTTs are
// replaced by forward NTTs of the parent's c0 and c1 (this limb).
template <int L>
__device__ __forceinline__ void expand_tail_ntt(const Dev4 &P, uint32_t galois, uint32_t kshift,
                                                const uint64_t *ct, const uint64_t (&vb)[8],
                                                const uint64_t (&va)[8], uint64_t *outL,
                                                uint64_t *outR) {
  extern __shared__ uint64_t sm4[];
  constexpr uint64_t Q = Limb<L>::q;
  const int tid = threadIdx.x;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = ct[p * 2 * kN + L * kN + posA(tid, k)];
    fA<L>(v);
    st_plane<0>(sm4 + p * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid<L>(sm4, 2, P.T);
  uint64_t h0[8], h1[8];
  {
    ulonglong2 wd[7];
    fload_d<L>(wd, P.T);
    ld_plane<3>(sm4, h0, tid);
    ld_plane<3>(sm4 + kPad, h1, tid);
    fD<L>(h0, wd);
    fD<L>(h1, wd);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    h0[k] = canon8<Q>(h0[k]);
    h1[k] = canon8<Q>(h1[k]);
  }
  st_plane<3>(sm4 + 2 * kPad, h0, tid);  // c0^ by slot, for the sigma gather
  __syncthreads();
  uint64_t l0[8], l1[8], r0[8], r1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t i = posD(tid, k);
    const uint32_t e = 2 * (__brev(i) >> 20) + 1;  // 12-bit reversal (N = 4096)
    const uint32_t j = __brev(((e * galois) & (2 * kN - 1)) >> 1) >> 20;
    const uint64_t n0v = add_mod<Q>(sm4[2 * kPad + pad(j)], vb[k]), n1v = va[k];
    l0[k] = add_mod<Q>(h0[k], n0v);
    l1[k] = add_mod<Q>(h1[k], n1v);
    const ulonglong2 lam =
        __ldg(P.T.pwt[L] + ((2 * kN - ((kshift * e) & (2 * kN - 1))) & (2 * kN - 1)));
    const uint64_t t0 = mul_shoup<Q>(sub_mod<Q>(h0[k], n0v), lam.x, lam.y);
    const uint64_t t1 = mul_shoup<Q>(sub_mod<Q>(h1[k], n1v), lam.x, lam.y);
    r0[k] = min(t0, t0 - Q);
    r1[k] = min(t1, t1 - Q);
  }
  const int j0 = posD(tid, 0);  // eight consecutive slots
#pragma unroll
  for (int c = 0; c < 8; c += 2) {
    *reinterpret_cast<ulonglong2 *>(outL + L * kN + j0 + c) = make_ulonglong2(l0[c], l0[c + 1]);
    *reinterpret_cast<ulonglong2 *>(outL + 2 * kN + L * kN + j0 + c) =
        make_ulonglong2(l1[c], l1[c + 1]);
    *reinterpret_cast<ulonglong2 *>(outR + L * kN + j0 + c) = make_ulonglong2(r0[c], r0[c + 1]);
    *reinterpret_cast<ulonglong2 *>(outR + 2 * kN + L * kN + j0 + c) =
        make_ulonglong2(r1[c], r1[c + 1]);
  }
}

template <int L, bool NTT_OUT = false>
__device__ __forceinline__ void expand_body(const Dev4 &P, uint32_t galois_inv, uint32_t kshift,
                                            const uint64_t *in, uint64_t in_stride, uint64_t *out,
                                            uint64_t out_stride, const uint64_t *const *bv_keys,
                                            uint64_t bv_level_off, uint32_t node0 = 0,
                                            uint32_t galois = 0) {
  extern __shared__ uint64_t sm4[];
  constexpr uint64_t Q = Limb<L>::q;
  const int node = node0 + blockIdx.x, b = blockIdx.z, tid = threadIdx.x;
  const uint64_t *ct = in + (static_cast<uint64_t>(b) * in_stride + node) * kCtWords;
  const uint64_t *key = bv_keys[b] + bv_level_off;  // [row][b][a][b'][a']
  uint64_t ab[8], aa[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) ab[k] = aa[k] = 0;
  for (int g = 0; g < kLKs / kExpGroup; ++g) {
    u128 u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t j = posA(tid, k);
      const uint32_t w = (j * galois_inv) & (2 * kN - 1);
      const bool neg = w >= kN;
      const uint32_t src = w & (kN - 1);
      uint64_t a0 = ct[2 * kN + src], a1 = ct[3 * kN + src];
      if (neg) { a0 = neg_mod<kQ0>(a0); a1 = neg_mod<kQ1>(a1); }
      u[k] = bv_digit_source<kLKs, kBaseKs>(compose(a0, a1, P.q0inv, P.q0inv_sh));
    }
#pragma unroll
    for (int e = 0; e < kExpGroup; ++e) {
      uint64_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int64_t r = static_cast<int64_t>(field<kBaseKs>(u[k], g * kExpGroup + e)) -
                          ((1ll << (kBaseKs - 1)) - 1);
        v[k] = r >= 0 ? static_cast<uint64_t>(r) : static_cast<uint64_t>(r + static_cast<int64_t>(Q));
      }
      fA<L>(v);
      st_plane<0>(sm4 + e * kPad, v, tid);
    }
    __syncthreads();
    fwd_mid<L>(sm4, kExpGroup, P.T);
    for (int e = 0; e < kExpGroup; ++e) {
      const int i = g * kExpGroup + e;
      uint64_t v[8];
      {
        ulonglong2 wd[7];
        fload_d<L>(wd, P.T);
        ld_plane<3>(sm4 + e * kPad, v, tid);
        fD<L>(v, wd);  // [0, 6q)
      }
      const uint64_t *R = key + static_cast<uint64_t>(i) * kRowWords + L * kN + 8 * tid;
      {
        uint64_t w[8], ws[8];
        ld8(R, w);
        ld8(R + 4 * kN, ws);
#pragma unroll
        for (int k = 0; k < 8; ++k) ab[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
      }
      {
        uint64_t w[8], ws[8];
        ld8(R + 2 * kN, w);
        ld8(R + 6 * kN, ws);
#pragma unroll
        for (int k = 0; k < 8; ++k) aa[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
      }
    }
    __syncthreads();
  }
  uint64_t *outL = out + (static_cast<uint64_t>(b) * out_stride + 2ull * node) * kCtWords;
  uint64_t *outR = outL + kCtWords;
  if constexpr (NTT_OUT) {
    uint64_t vb[8], va[8];  // the key switch's delta in NTT form, canonical
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      vb[k] = fold16<Q>(ab[k]);
      vb[k] = min(vb[k], vb[k] - Q);
      va[k] = fold16<Q>(aa[k]);
      va[k] = min(va[k], va[k] - Q);
    }
    expand_tail_ntt<L>(P, galois, kshift, ct, vb, va, outL, outR);
    return;
  }
  {
    ulonglong2 wd[7];
    iload_d<L>(wd, P.T);
    uint64_t vb[8], va[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { vb[k] = fold16<Q>(ab[k]); va[k] = fold16<Q>(aa[k]); }
    iD<L>(vb, wd);
    iD<L>(va, wd);
    st_plane<3>(sm4, vb, tid);
    st_plane<3>(sm4 + kPad, va, tid);
  }
  __syncthreads();
  inv_mid<L>(sm4, 2, P.T);
  uint64_t db_[8], da[8];
  ld_plane<0>(sm4, db_, tid);
  ld_plane<0>(sm4 + kPad, da, tid);
  iA<L>(db_);
  iA<L>(da);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t j = posA(tid, k);
    const uint32_t w = (j * galois_inv) & (2 * kN - 1);
    const uint64_t z = ct[L * kN + (w & (kN - 1))];
    const uint64_t s0 = w >= kN ? neg_mod<Q>(z) : z;        // sigma_k(c0), own limb
    const uint64_t n0v = add_mod<Q>(s0, db_[k]), n1v = da[k];
    const uint64_t o0 = ct[L * kN + j], o1 = ct[2 * kN + L * kN + j];
    outL[L * kN + j] = add_mod<Q>(o0, n0v);
    outL[2 * kN + L * kN + j] = add_mod<Q>(o1, n1v);
    const uint64_t d0 = sub_mod<Q>(o0, n0v), d1 = sub_mod<Q>(o1, n1v);
    int dst = static_cast<int>(j) - static_cast<int>(kshift);
    const bool wrap = dst < 0;
    if (wrap) dst += kN;
    outR[L * kN + dst] = wrap ? neg_mod<Q>(d0) : d0;
    outR[2 * kN + L * kN + dst] = wrap ? neg_mod<Q>(d1) : d1;
  }
}

__global__ void __launch_bounds__(kThreads, 1)
k4_expand_level(Dev4 P, uint32_t galois_inv, uint32_t kshift, const uint64_t *__restrict__ in,
                uint64_t in_stride, uint64_t *__restrict__ out, uint64_t out_stride,
                const uint64_t *const *__restrict__ bv_keys, uint64_t bv_level_off,
                uint32_t node0) {
  if (blockIdx.y == 0)
    expand_body<0>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys, bv_level_off,
                   node0);
  else
    expand_body<1>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys, bv_level_off,
                   node0);
}

// The last level's nodes below ntt_nodes when the first-dimension leaves are
// wanted in NTT form (expand_tail_ntt); k4_expand_level takes the others.
__global__ void __launch_bounds__(kThreads, 1)
k4_expand_level_ntt(Dev4 P, uint32_t galois, uint32_t galois_inv, uint32_t kshift,
                    const uint64_t *__restrict__ in, uint64_t in_stride,
                    uint64_t *__restrict__ out, uint64_t out_stride,
                    const uint64_t *const *__restrict__ bv_keys, uint64_t bv_level_off) {
  if (blockIdx.y == 0)
    expand_body<0, true>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys,
                         bv_level_off, 0, galois);
  else
    expand_body<1, true>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys,
                         bv_level_off, 0, galois);
}

// Expansion level, cluster split: with fewer nodes than SMs (the top of the
// heap, and most levels of a single query) each node's key switch runs on a
// cluster of C CTAs. CTA r NTTs digits [r D, (r + 1) D) (D = L_KS / C) of
// sigma_k(c1) and accumulates their Shoup products with the key rows; the
// partial sums (below 2q D each, their total below 16q as in the single-CTA
// sum) meet in distributed shared memory; CTA 0 finishes the b part (c0 of
// both children), CTA 1 the a part (c1 of both children). Same children bit
// for bit.
template <int L, int C>
__device__ __forceinline__ void expand_split_body(const Dev4 &P, uint32_t galois_inv,
                                                  uint32_t kshift, const uint64_t *in,
                                                  uint64_t in_stride, uint64_t *out,
                                                  uint64_t out_stride,
                                                  const uint64_t *const *bv_keys,
                                                  uint64_t bv_level_off) {
  static_assert(kLKs % C == 0 && kLKs / C <= kExpGroup, "digits per CTA fit the planes");
  constexpr int D = kLKs / C;
  extern __shared__ uint64_t sm4[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  constexpr uint64_t Q = Limb<L>::q;
  const int rank = static_cast<int>(cluster.block_rank());
  const int node = blockIdx.x / C, b = blockIdx.z, tid = threadIdx.x;
  const uint64_t *ct = in + (static_cast<uint64_t>(b) * in_stride + node) * kCtWords;
  const uint64_t *key = bv_keys[b] + bv_level_off;
  uint64_t ab[8], aa[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) ab[k] = aa[k] = 0;
  {
    u128 u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t j = posA(tid, k);
      const uint32_t w = (j * galois_inv) & (2 * kN - 1);
      const bool neg = w >= kN;
      const uint32_t src = w & (kN - 1);
      uint64_t a0 = ct[2 * kN + src], a1 = ct[3 * kN + src];
      if (neg) { a0 = neg_mod<kQ0>(a0); a1 = neg_mod<kQ1>(a1); }
      u[k] = bv_digit_source<kLKs, kBaseKs>(compose(a0, a1, P.q0inv, P.q0inv_sh));
    }
#pragma unroll
    for (int e = 0; e < D; ++e) {
      uint64_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int64_t r = static_cast<int64_t>(field<kBaseKs>(u[k], rank * D + e)) -
                          ((1ll << (kBaseKs - 1)) - 1);
        v[k] = r >= 0 ? static_cast<uint64_t>(r) : static_cast<uint64_t>(r + static_cast<int64_t>(Q));
      }
      fA<L>(v);
      st_plane<0>(sm4 + e * kPad, v, tid);
    }
  }
  __syncthreads();
  fwd_mid<L>(sm4, D, P.T);
  for (int e = 0; e < D; ++e) {
    const int i = rank * D + e;
    uint64_t v[8];
    {
      ulonglong2 wd[7];
      fload_d<L>(wd, P.T);
      ld_plane<3>(sm4 + e * kPad, v, tid);
      fD<L>(v, wd);  // [0, 6q)
    }
    const uint64_t *R = key + static_cast<uint64_t>(i) * kRowWords + L * kN + 8 * tid;
    {
      uint64_t w[8], ws[8];
      ld8(R, w);
      ld8(R + 4 * kN, ws);
#pragma unroll
      for (int k = 0; k < 8; ++k) ab[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
    }
    {
      uint64_t w[8], ws[8];
      ld8(R + 2 * kN, w);
      ld8(R + 6 * kN, ws);
#pragma unroll
      for (int k = 0; k < 8; ++k) aa[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
    }
  }
  __syncthreads();
  uint64_t *ex = sm4;  // [b / a][k][tid]
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    ex[(0 * 8 + k) * kThreads + tid] = ab[k];
    ex[(1 * 8 + k) * kThreads + tid] = aa[k];
  }
  cluster.sync();
  uint64_t tot[8];
  if (rank < 2) {
#pragma unroll
    for (int k = 0; k < 8; ++k) tot[k] = rank == 0 ? ab[k] : aa[k];
    for (int r = 0; r < C; ++r) {
      if (r == rank) continue;
      const uint64_t *rex = cluster.map_shared_rank(ex, r);
#pragma unroll
      for (int k = 0; k < 8; ++k) tot[k] += rex[(rank * 8 + k) * kThreads + tid];
    }
  }
  cluster.sync();  // every remote read is done before shared memory is reused
  if (rank >= 2) return;
  {
    ulonglong2 wd[7];
    iload_d<L>(wd, P.T);
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = fold16<Q>(tot[k]);
    iD<L>(v, wd);
    st_plane<3>(sm4, v, tid);
  }
  __syncthreads();
  inv_mid<L>(sm4, 1, P.T);
  uint64_t dv[8];
  ld_plane<0>(sm4, dv, tid);
  iA<L>(dv);
  uint64_t *outL = out + (static_cast<uint64_t>(b) * out_stride + 2ull * node) * kCtWords;
  uint64_t *outR = outL + kCtWords;
  const uint64_t off = static_cast<uint64_t>(rank) * 2 * kN + L * kN;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t j = posA(tid, k);
    uint64_t nv = dv[k];
    if (rank == 0) {  // c0' = sigma_k(c0) + delta_b
      const uint32_t w = (j * galois_inv) & (2 * kN - 1);
      const uint64_t z = ct[L * kN + (w & (kN - 1))];
      nv = add_mod<Q>(w >= kN ? neg_mod<Q>(z) : z, nv);
    }
    const uint64_t o = ct[off + j];
    outL[off + j] = add_mod<Q>(o, nv);
    const uint64_t dd = sub_mod<Q>(o, nv);
    int dst = static_cast<int>(j) - static_cast<int>(kshift);
    const bool wrap = dst < 0;
    if (wrap) dst += kN;
    outR[off + dst] = wrap ? neg_mod<Q>(dd) : dd;
  }
}

template <int C>
__global__ void __launch_bounds__(kThreads, 1)
k4_expand_level_split(Dev4 P, uint32_t galois_inv, uint32_t kshift,
                      const uint64_t *__restrict__ in, uint64_t in_stride,
                      uint64_t *__restrict__ out, uint64_t out_stride,
                      const uint64_t *const *__restrict__ bv_keys, uint64_t bv_level_off) {
  if (blockIdx.y == 0)
    expand_split_body<0, C>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys,
                            bv_level_off);
  else
    expand_split_body<1, C>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys,
                            bv_level_off);
}

// ------------------------------------------------------------ gadget product
// acc += sum over the 2 l digit rows of NTT(digit) x rgsw[row] for one limb
// (gsw.cpp:119-182, decomp_rlwe_mp gsw.cpp:184-250): each polynomial of the
// decomposed ciphertext (both limbs read: y - x, or x when y is null) is
// CRT-composed and split into l unsigned base-2^B digits; digit d of poly p
// meets row p l + (l - 1 - d). Uses G planes (G = l when l <= 5, else 4).
// Products are Shoup products in [0, 2q) with the rows' companions; the
// sums are folded below 2q after each group (< 2q + 5 x 2q in between).
template <int L, int NL, int B>
__device__ __forceinline__ void gadget_mac(const Dev4 &P, const uint64_t *x, const uint64_t *y,
                                           const uint64_t *rgsw, uint64_t *sm, uint64_t (&acc0)[8],
                                           uint64_t (&acc1)[8]) {
  constexpr int G = NL <= 5 ? NL : 4;
  constexpr uint64_t Q = Limb<L>::q;
  const int tid = threadIdx.x;
#pragma unroll 1
  for (int p = 0; p < 2; ++p) {
#pragma unroll 1
    for (int g = 0; g < NL / G; ++g) {
      u128 u[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int j = posA(tid, k);
        uint64_t v0 = x[p * 2 * kN + j], v1 = x[p * 2 * kN + kN + j];
        if (y != nullptr) {
          v0 = sub_mod<kQ0>(y[p * 2 * kN + j], v0);
          v1 = sub_mod<kQ1>(y[p * 2 * kN + kN + j], v1);
        }
        u[k] = compose(v0, v1, P.q0inv, P.q0inv_sh);
      }
#pragma unroll
      for (int e = 0; e < G; ++e) {
        uint64_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = field<B>(u[k], g * G + e);  // < 2^B < q
        fA<L>(v);
        st_plane<0>(sm + e * kPad, v, tid);
      }
      __syncthreads();
      fwd_mid<L>(sm, G, P.T);
      for (int e = 0; e < G; ++e) {
        const int d = g * G + e;
        const int row = p * NL + (NL - 1 - d);
        uint64_t v[8];
        {
          ulonglong2 wd[7];
          fload_d<L>(wd, P.T);
          ld_plane<3>(sm + e * kPad, v, tid);
          fD<L>(v, wd);
        }
        const uint64_t *R = rgsw + static_cast<uint64_t>(row) * kRowWords + L * kN + 8 * tid;
        {
          uint64_t w[8], ws[8];
          ld8(R, w);
          ld8(R + 4 * kN, ws);
#pragma unroll
          for (int k = 0; k < 8; ++k) acc0[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
        }
        {
          uint64_t w[8], ws[8];
          ld8(R + 2 * kN, w);
          ld8(R + 6 * kN, ws);
#pragma unroll
          for (int k = 0; k < 8; ++k) acc1[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) { acc0[k] = fold16<Q>(acc0[k]); acc1[k] = fold16<Q>(acc1[k]); }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ selectors
template <int L>
__device__ __forceinline__ void selectors_body(const Dev4 &P, const Shape4 &S,
                                               const uint64_t *leaves, uint64_t leaf_stride,
                                               const uint64_t *const *gsw_keys, uint64_t *sel) {
  extern __shared__ uint64_t sm4[];
  constexpr uint64_t Q = Limb<L>::q;
  const int row_id = blockIdx.x, b = blockIdx.z, tid = threadIdx.x;
  const int selno = row_id / S.l_ep, r = row_id % S.l_ep;
  const uint64_t *ct = leaves + (static_cast<uint64_t>(b) * leaf_stride + S.n0 + row_id) * kCtWords;
  uint64_t *outs = sel + (static_cast<uint64_t>(b) * (S.num_dims - 1) + selno) * 2 * S.l_ep * kRowWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  // bottom row: ExtProd(RGSW(s), row) with the key gadget; each selector row
  // is stored with its Shoup companions (the MUX multiplies by it)
  gadget_mac<L, kLKey, kBaseKey>(P, ct, nullptr, gsw_keys[b], sm4, acc0, acc1);
  uint64_t *bot = outs + static_cast<uint64_t>(S.l_ep + r) * kRowWords + L * kN + 8 * tid;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint64_t v0 = min(acc0[k], acc0[k] - Q), v1 = min(acc1[k], acc1[k] - Q);
    bot[k] = v0;
    bot[2 * kN + k] = v1;
    bot[4 * kN + k] = shoup_of<Q>(v0);
    bot[6 * kN + k] = shoup_of<Q>(v1);
  }
  // top row: the expanded row itself in NTT form (gsw.cpp:330-338)
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = ct[p * 2 * kN + L * kN + posA(tid, k)];
    fA<L>(v);
    st_plane<0>(sm4 + p * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid<L>(sm4, 2, P.T);
  ulonglong2 wd[7];
  fload_d<L>(wd, P.T);
  uint64_t *top = outs + static_cast<uint64_t>(r) * kRowWords + L * kN + 8 * tid;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
    ld_plane<3>(sm4 + p * kPad, v, tid);
    fD<L>(v, wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint64_t c = canon8<Q>(v[k]);
      top[p * 2 * kN + k] = c;
      top[4 * kN + p * 2 * kN + k] = shoup_of<Q>(c);
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1)
k4_selectors(Dev4 P, Shape4 S, const uint64_t *__restrict__ leaves, uint64_t leaf_stride,
             const uint64_t *const *__restrict__ gsw_keys, uint64_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    selectors_body<0>(P, S, leaves, leaf_stride, gsw_keys, sel);
  else
    selectors_body<1>(P, S, leaves, leaf_stride, gsw_keys, sel);
}

// ------------------------------------------------------------ first-dim query
// Forward NTT per limb of the first n0 leaves (server.cpp:205-262) into
// qm[col][k][z] (col = 2 query + poly, k < n0, z = limb N + coefficient:
// each thread stores its 4-coefficient runs, so the stores are coalesced),
// then k4_fst_pack transposes it through shared memory into the scan's eight
// byte planes qb[(z 8 + plane)][col][n0p].
constexpr int kFstTile = 2;  // leaves per CTA (4 planes)

template <int L>
__device__ __forceinline__ void fst_body(const Dev4 &P, const Shape4 &S, const uint64_t *leaves,
                                         uint64_t leaf_stride, uint64_t *qm, uint32_t ncols) {
  extern __shared__ uint64_t sm4[];
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t k0 = blockIdx.x * kFstTile;
  for (int e = 0; e < 2 * kFstTile; ++e) {
    const uint32_t kk = k0 + (e >> 1);
    const int p = e & 1;
    uint64_t v[8];
    const uint64_t *src =
        leaves + (static_cast<uint64_t>(b) * leaf_stride + kk) * kCtWords + p * 2 * kN + L * kN;
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = kk < S.n0 ? src[posA(tid, k)] : 0;
    fA<L>(v);
    st_plane<0>(sm4 + e * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid<L>(sm4, 2 * kFstTile, P.T);
  ulonglong2 wd[7];
  fload_d<L>(wd, P.T);
  for (int e = 0; e < 2 * kFstTile; ++e) {
    const uint32_t kk = k0 + (e >> 1);
    if (kk >= S.n0) continue;  // uniform over the CTA
    const int p = e & 1;
    uint64_t v[8];
    ld_plane<3>(sm4 + e * kPad, v, tid);
    fD<L>(v, wd);
    uint64_t *dst = qm + ((static_cast<uint64_t>(2 * b + p)) * S.n0 + kk) * (2 * kN) +
                    static_cast<uint64_t>(L) * kN;
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // D-order positions 4 (tid + 512 h) .. + 3
      const int j0 = posD(tid, 4 * h);
      *reinterpret_cast<ulonglong2 *>(dst + j0) =
          make_ulonglong2(canon8<Limb<L>::q>(v[4 * h + 0]), canon8<Limb<L>::q>(v[4 * h + 1]));
      *reinterpret_cast<ulonglong2 *>(dst + j0 + 2) =
          make_ulonglong2(canon8<Limb<L>::q>(v[4 * h + 2]), canon8<Limb<L>::q>(v[4 * h + 3]));
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1)
k4_fst_ntt(Dev4 P, Shape4 S, const uint64_t *__restrict__ leaves, uint64_t leaf_stride,
           uint64_t *__restrict__ qm, uint32_t ncols) {
  if (blockIdx.y == 0)
    fst_body<0>(P, S, leaves, leaf_stride, qm, ncols);
  else
    fst_body<1>(P, S, leaves, leaf_stride, qm, ncols);
}

// A CTA transposes a tile of 32 coefficients z x 128 leaves k of one column
// through shared memory: 128 rows of 32 consecutive z in (256-byte reads),
// then one thread per (z, 16 consecutive k) builds that run's eight byte
// planes and writes 16 bytes per plane (8 threads cover a 128-byte row);
// k in [n0, n0p) reads as zero. The tile is z-major with 16-k runs 18 words
// apart and rows 145 words apart, so both the fill (32 z of one k) and the
// run reads (8 runs x 4 z) touch every bank pair at most twice.
constexpr int kPackZ = 32, kPackK = 128, kRunPitch = 18, kRowPitch = 145;
__global__ void __launch_bounds__(256)
k4_fst_pack(const uint64_t *__restrict__ qm, uint64_t q_stride, uint64_t p_stride,
            uint64_t k_stride, uint32_t n0, uint32_t n0p, uint32_t ncols,
            uint8_t *__restrict__ qb) {
  __shared__ uint64_t tile[(kPackZ - 1) * kRowPitch + (kPackK / 16 - 1) * kRunPitch + 16];
  const uint32_t z0 = blockIdx.x * kPackZ, col = blockIdx.y, k0 = blockIdx.z * kPackK;
  const int t = threadIdx.x;
  // column col = 2 query + poly: qm (q_stride = 2 p_stride, p_stride = n0 2N,
  // k_stride = 2N) or NTT-form leaves (q_stride = slots 4N, p_stride = 2N,
  // k_stride = 4N)
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
  const uint64_t plane_bytes = static_cast<uint64_t>(ncols) * n0p;
  const uint64_t z = z0 + zz;
  const uint32_t k = k0 + chunk * 16;
  if (k >= n0p) return;
  uint8_t *dst = qb + z * 8 * plane_bytes + static_cast<uint64_t>(col) * n0p + k;
#pragma unroll
  for (int pl = 0; pl < 8; ++pl)
    *reinterpret_cast<uint4 *>(dst + pl * plane_bytes) = make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
}

// ------------------------------------------------------------ scan epilogue
// inter_to_cts (server.cpp:405-527): INTT per limb of every candidate. A CTA
// transforms 4 consecutive rows of one column and one limb, reading the
// scan's cmat[z][col][row] as 32-byte row groups (two 16-byte loads each
// when the row count is even, so that every group is 16-byte aligned).
constexpr int kEpiRows = 4;

template <int L, bool VEC>
__device__ __forceinline__ void epi_body(const Dev4 &P, const Shape4 &S, const uint64_t *cmat,
                                         uint32_t ncols, uint64_t *mid, uint64_t mid_stride) {
  extern __shared__ uint64_t sm4[];
  const int tid = threadIdx.x;
  const uint32_t r0 = blockIdx.x * kEpiRows, c = blockIdx.z;
  {
    uint64_t v[kEpiRows][8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint64_t z = static_cast<uint64_t>(L) * kN + posD(tid, k);
      const uint64_t *src = cmat + (z * ncols + c) * S.other + r0;
      if (VEC && r0 + kEpiRows <= S.other) {
        const ulonglong2 a = *reinterpret_cast<const ulonglong2 *>(src);
        const ulonglong2 b = *reinterpret_cast<const ulonglong2 *>(src + 2);
        v[0][k] = a.x; v[1][k] = a.y; v[2][k] = b.x; v[3][k] = b.y;
      } else {
#pragma unroll
        for (int e = 0; e < kEpiRows; ++e) v[e][k] = r0 + e < S.other ? src[e] : 0;
      }
    }
    ulonglong2 wd[7];
    iload_d<L>(wd, P.T);
#pragma unroll
    for (int e = 0; e < kEpiRows; ++e) {
      iD<L>(v[e], wd);
      st_plane<3>(sm4 + e * kPad, v[e], tid);
    }
  }
  __syncthreads();
  inv_mid<L>(sm4, kEpiRows, P.T);
  for (int e = 0; e < kEpiRows; ++e) {
    const uint32_t r = r0 + e;
    if (r >= S.other) break;  // uniform over the CTA
    uint64_t w[8];
    ld_plane<0>(sm4 + e * kPad, w, tid);
    iA<L>(w);
    uint64_t *dst = mid + (static_cast<uint64_t>(c >> 1) * mid_stride + r) * kCtWords +
                    (c & 1) * 2 * kN + L * kN;
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[posA(tid, k)] = w[k];
  }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads, 1)
k4_epilogue(Dev4 P, Shape4 S, const uint64_t *__restrict__ cmat, uint32_t ncols,
            uint64_t *__restrict__ mid, uint64_t mid_stride) {
  if (blockIdx.y == 0)
    epi_body<0, VEC>(P, S, cmat, ncols, mid, mid_stride);
  else
    epi_body<1, VEC>(P, S, cmat, ncols, mid, mid_stride);
}

// ------------------------------------------------------------ MUX level
// ext_prod_mux (server.cpp:652-722): out = x + INTT(ExtProd(sel, y - x)).
template <int L>
__device__ __forceinline__ void mux_body(const Dev4 &P, const Shape4 &S, uint32_t level,
                                         uint32_t n_pairs, uint32_t offset, uint32_t half,
                                         const uint64_t *in, uint64_t *out, uint64_t mid_stride,
                                         const uint64_t *sel) {
  extern __shared__ uint64_t sm4[];
  constexpr uint64_t Q = Limb<L>::q;
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t i = blockIdx.x;
  const uint64_t *base_in = in + static_cast<uint64_t>(b) * mid_stride * kCtWords;
  uint64_t *base_out = out + static_cast<uint64_t>(b) * mid_stride * kCtWords;
  if (i >= n_pairs) {  // level 0: carry the unpaired prefix over unchanged
    const uint64_t c = i - n_pairs;
    for (int j = tid; j < kN; j += kThreads) {
      base_out[c * kCtWords + L * kN + j] = base_in[c * kCtWords + L * kN + j];
      base_out[c * kCtWords + 2 * kN + L * kN + j] = base_in[c * kCtWords + 2 * kN + L * kN + j];
    }
    return;
  }
  uint32_t xi, yi, oi;
  if (level == 0) { xi = offset + 2 * i; yi = xi + 1; oi = offset + i; }
  else { xi = i; yi = i + half; oi = i; }
  const uint64_t *x = base_in + static_cast<uint64_t>(xi) * kCtWords;
  const uint64_t *y = base_in + static_cast<uint64_t>(yi) * kCtWords;
  const uint64_t *rgsw = sel + (static_cast<uint64_t>(b) * (S.num_dims - 1) + level) * 2 * kLEp * kRowWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  gadget_mac<L, kLEp, kBaseEp>(P, x, y, rgsw, sm4, acc0, acc1);
  {
    ulonglong2 wd[7];
    iload_d<L>(wd, P.T);
    uint64_t v[8], w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { v[k] = acc0[k]; w[k] = acc1[k]; }  // [0, 2q)
    iD<L>(v, wd);
    iD<L>(w, wd);
    st_plane<3>(sm4, v, tid);
    st_plane<3>(sm4 + kPad, w, tid);
  }
  __syncthreads();
  inv_mid<L>(sm4, 2, P.T);
  uint64_t *o = base_out + static_cast<uint64_t>(oi) * kCtWords;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint64_t v[8];
    ld_plane<0>(sm4 + p * kPad, v, tid);
    iA<L>(v);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posA(tid, k);
      o[p * 2 * kN + L * kN + j] = add_mod<Q>(x[p * 2 * kN + L * kN + j], v[k]);
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1)
k4_mux_level(Dev4 P, Shape4 S, uint32_t level, uint32_t n_pairs, uint32_t offset, uint32_t half,
             const uint64_t *__restrict__ in, uint64_t *__restrict__ out, uint64_t mid_stride,
             const uint64_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    mux_body<0>(P, S, level, n_pairs, offset, half, in, out, mid_stride, sel);
  else
    mux_body<1>(P, S, level, n_pairs, offset, half, in, out, mid_stride, sel);
}

// MUX level, cluster split: with fewer pairs than SMs each MUX runs on a
// cluster of C CTAs. CTA r takes digits [d0, d0 + dn) of polynomial p of
// y - x (C = 2: p = r, all l digits; C = 4: p = r / 2, digits 0-2 or 3-4),
// accumulates their Shoup products with the RGSW rows and folds them below
// 2q; CTAs 0 and 1 add the partials (below 2q C) through distributed shared
// memory, fold them below 2q and finish output polynomial c0 / c1 (INTT,
// + x). The same residues enter the same INTT: bit for bit the single-CTA
// MUX.
template <int L>
__device__ __forceinline__ void gadget_part(const Dev4 &P, const uint64_t *x, const uint64_t *y,
                                            const uint64_t *rgsw, uint64_t *sm, int p, int d0,
                                            int dn, uint64_t (&acc0)[8], uint64_t (&acc1)[8]) {
  constexpr uint64_t Q = Limb<L>::q;
  const int tid = threadIdx.x;
  {
    u128 u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posA(tid, k);
      const uint64_t v0 = sub_mod<kQ0>(y[p * 2 * kN + j], x[p * 2 * kN + j]);
      const uint64_t v1 = sub_mod<kQ1>(y[p * 2 * kN + kN + j], x[p * 2 * kN + kN + j]);
      u[k] = compose(v0, v1, P.q0inv, P.q0inv_sh);
    }
    for (int e = 0; e < dn; ++e) {
      uint64_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = field<kBaseEp>(u[k], d0 + e);  // < 2^B < q
      fA<L>(v);
      st_plane<0>(sm + e * kPad, v, tid);
    }
  }
  __syncthreads();
  fwd_mid<L>(sm, dn, P.T);
  for (int e = 0; e < dn; ++e) {
    const int row = p * kLEp + (kLEp - 1 - (d0 + e));
    uint64_t v[8];
    {
      ulonglong2 wd[7];
      fload_d<L>(wd, P.T);
      ld_plane<3>(sm + e * kPad, v, tid);
      fD<L>(v, wd);
    }
    const uint64_t *R = rgsw + static_cast<uint64_t>(row) * kRowWords + L * kN + 8 * tid;
    {
      uint64_t w[8], ws[8];
      ld8(R, w);
      ld8(R + 4 * kN, ws);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc0[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
    }
    {
      uint64_t w[8], ws[8];
      ld8(R + 2 * kN, w);
      ld8(R + 6 * kN, ws);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc1[k] += mul_shoup<Q>(v[k], w[k], ws[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) { acc0[k] = fold16<Q>(acc0[k]); acc1[k] = fold16<Q>(acc1[k]); }
  __syncthreads();
}

// Pair i reads x = in[i xs], y = in[i xs + yoff] and writes out[i] (level 0
// without a carried prefix: xs = 2, yoff = 1; level a >= 1: xs = 1,
// yoff = half).
template <int L, int C>
__device__ __forceinline__ void mux_split_body(const Dev4 &P, const Shape4 &S, uint32_t level,
                                               uint32_t xs, uint32_t yoff, const uint64_t *in,
                                               uint64_t *out, uint64_t mid_stride,
                                               const uint64_t *sel) {
  static_assert(C == 2 || C == 4, "cluster of 2 or 4 CTAs");
  extern __shared__ uint64_t sm4[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  constexpr uint64_t Q = Limb<L>::q;
  const int rank = static_cast<int>(cluster.block_rank());
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t i = blockIdx.x / C;
  const uint64_t *base_in = in + static_cast<uint64_t>(b) * mid_stride * kCtWords;
  const uint64_t *x = base_in + static_cast<uint64_t>(i) * xs * kCtWords;
  const uint64_t *y = base_in + (static_cast<uint64_t>(i) * xs + yoff) * kCtWords;
  const uint64_t *rgsw = sel + (static_cast<uint64_t>(b) * (S.num_dims - 1) + level) * 2 * kLEp * kRowWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  constexpr int kHalf = (kLEp + 1) / 2;
  const int p = C == 2 ? rank : rank >> 1;
  const int d0 = C == 2 ? 0 : (rank & 1) * kHalf;
  const int dn = C == 2 ? kLEp : ((rank & 1) ? kLEp - kHalf : kHalf);
  gadget_part<L>(P, x, y, rgsw, sm4, p, d0, dn, acc0, acc1);
  uint64_t *ex = sm4;  // [output poly][k][tid]
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    ex[(0 * 8 + k) * kThreads + tid] = acc0[k];
    ex[(1 * 8 + k) * kThreads + tid] = acc1[k];
  }
  cluster.sync();
  uint64_t tot[8];
  if (rank < 2) {
#pragma unroll
    for (int k = 0; k < 8; ++k) tot[k] = rank == 0 ? acc0[k] : acc1[k];
    for (int r = 0; r < C; ++r) {
      if (r == rank) continue;
      const uint64_t *rex = cluster.map_shared_rank(ex, r);
#pragma unroll
      for (int k = 0; k < 8; ++k) tot[k] += rex[(rank * 8 + k) * kThreads + tid];
    }
  }
  cluster.sync();  // every remote read is done before shared memory is reused
  if (rank >= 2) return;
  {
    ulonglong2 wd[7];
    iload_d<L>(wd, P.T);
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = fold16<Q>(tot[k]);  // < 2q C <= 8q -> [0, 2q)
    iD<L>(v, wd);
    st_plane<3>(sm4, v, tid);
  }
  __syncthreads();
  inv_mid<L>(sm4, 1, P.T);
  uint64_t v[8];
  ld_plane<0>(sm4, v, tid);
  iA<L>(v);
  uint64_t *o = out + static_cast<uint64_t>(b) * mid_stride * kCtWords + static_cast<uint64_t>(i) * kCtWords;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int j = posA(tid, k);
    o[rank * 2 * kN + L * kN + j] = add_mod<Q>(x[rank * 2 * kN + L * kN + j], v[k]);
  }
}

template <int C>
__global__ void __launch_bounds__(kThreads, 1)
k4_mux_level_split(Dev4 P, Shape4 S, uint32_t level, uint32_t xs, uint32_t yoff,
                   const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                   uint64_t mid_stride, const uint64_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    mux_split_body<0, C>(P, S, level, xs, yoff, in, out, mid_stride, sel);
  else
    mux_split_body<1, C>(P, S, level, xs, yoff, in, out, mid_stride, sel);
}

// ------------------------------------------------------------ modulus switch
// server.cpp:1044-1075: drop q1 with rounding, then utils::rescale
// (utils.cpp:445-462) q0 -> small_q; bit packing as save_resp_to_stream
// (server.cpp:950-1009).
__device__ __forceinline__ uint64_t rescale_dev(uint64_t a, uint64_t inp, uint64_t outm) {
  const int64_t inp_i = static_cast<int64_t>(inp);
  const i128 out_i = static_cast<i128>(outm);
  int64_t v = static_cast<int64_t>(a % inp);
  if (v >= inp_i / 2) v -= inp_i;
  const int64_t sign = v >= 0 ? 1 : -1;
  const i128 val = static_cast<i128>(v) * static_cast<i128>(outm);
  i128 r = (val + static_cast<i128>(sign * (inp_i / 2))) / static_cast<i128>(inp);
  r = (r + static_cast<i128>((inp / outm) * outm) + 2 * out_i) % out_i;
  return static_cast<uint64_t>((r + out_i) % out_i);
}

__global__ void __launch_bounds__(256)
k4_modswitch(Dev4 P, const uint64_t *__restrict__ ct_all, uint64_t ct_stride,
             uint64_t *__restrict__ resp, uint8_t *__restrict__ bytes, uint32_t resp_bytes) {
  extern __shared__ uint64_t vals[];  // 2N
  const int b = blockIdx.x;
  const uint64_t *ct = ct_all + static_cast<uint64_t>(b) * ct_stride * kCtWords;
  for (int idx = threadIdx.x; idx < 2 * kN; idx += blockDim.x) {
    const int p = idx >> 12, j = idx & (kN - 1);
    const u128 x = compose(ct[p * 2 * kN + j], ct[p * 2 * kN + kN + j], P.q0inv, P.q0inv_sh);
    uint64_t v = static_cast<uint64_t>((x + (static_cast<u128>(kQ1) >> 1)) / kQ1);
    if (v >= kQ0) v -= kQ0;
    const uint64_t r = rescale_dev(v, kQ0, P.small_q);
    resp[static_cast<uint64_t>(b) * 2 * kN + idx] = r;
    vals[idx] = r & ((1ull << P.small_q_width) - 1);
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

// ============================================================== launchers
uint64_t launch_count() { return g_launches4.load(std::memory_order_relaxed); }
void note_launches(int64_t delta) {
  g_launches4.fetch_add(static_cast<uint64_t>(delta), std::memory_order_relaxed);
}

void upload_constants(const uint64_t *const fw[2], const uint64_t *const fw_sh[2],
                      const uint64_t *const iw[2], const uint64_t *const iw_sh[2],
                      const uint64_t ninv[2][2], const uint64_t w1ninv[2][2]) {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return;
  ulonglong2 f[2][64], i[2][64], a[2], b[2];
  for (int r = 0; r < 2; ++r) {
    for (int k = 0; k < 64; ++k) {
      f[r][k] = make_ulonglong2(fw[r][k], fw_sh[r][k]);
      i[r][k] = make_ulonglong2(iw[r][k], iw_sh[r][k]);
    }
    a[r] = make_ulonglong2(ninv[r][0], ninv[r][1]);
    b[r] = make_ulonglong2(w1ninv[r][0], w1ninv[r][1]);
  }
  cudaError_t e = cudaMemcpyToSymbol(c4_fwt, f, sizeof(f));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c4_iwt, i, sizeof(i));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c4_ninv, a, sizeof(a));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c4_w1ninv, b, sizeof(b));
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("NTT constants: ") + cudaGetErrorString(e));
  done.insert(dev);
}

void launch_db_preprocess(const Dev4 &P, const Shape4 &s, const uint64_t *coeffs,
                          uint64_t coeff_pt_begin, uint64_t seed, uint64_t t, uint64_t logical,
                          uint64_t pt_begin, uint64_t pt_end, const uint32_t *row_map,
                          uint8_t *db8, cudaStream_t st) {
  if (pt_begin % kDbTile != 0) throw std::invalid_argument("db tiles start at a multiple of 4");
  if (pt_end > static_cast<uint64_t>(s.other) * s.n0) throw std::invalid_argument("db tile beyond the layout");
  const size_t smem = plane_bytes(kDbTile);
  set_smem(k4_db_preprocess, smem);
  const uint64_t tiles = (pt_end - pt_begin + kDbTile - 1) / kDbTile;
  dim3 grid(static_cast<unsigned>(tiles), 2);
  k4_db_preprocess<<<grid, kThreads, smem, st>>>(P, coeffs, coeff_pt_begin, seed, t, logical, s.n0,
                                                   s.n0p, s.other, pt_begin, pt_end, row_map, db8);
  check_launch("k4_db_preprocess");
}

uint32_t expand_nodes(const Shape4 &s, uint32_t d) {
  const uint64_t span = 1ull << (s.h - d);  // leaves under one node of level d
  return static_cast<uint32_t>((s.useful + span - 1) / span);
}

void launch_expand_level(const Dev4 &P, const Shape4 &s, uint32_t d, const uint64_t *in,
                         uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                         const uint64_t *const *bv_keys, uint64_t bv_level_stride, uint32_t batch,
                         cudaStream_t st, uint32_t ntt_nodes) {
  const uint32_t nodes = expand_nodes(s, d);
  if (nodes == 0) return;
  const size_t smem = plane_bytes(kExpGroup);
  set_smem(k4_expand_level, smem);
  const uint32_t k = 1u << d;
  const uint32_t galois = kN / k + 1;
  // sigma_k as a gather: sigma(c)[j] = +-c[j k^-1 mod 2N] (utils.cpp:58-72)
  uint32_t inv = 1;
  for (uint32_t e = 0; e < 2 * kN; ++e)
    if ((static_cast<uint64_t>(galois) * e) % (2 * kN) == 1) { inv = e; break; }
  // nodes of level d are heap slots k .. k + nodes - 1, stored from slot 0;
  // children of node i go to slots 2 i, 2 i + 1 of the next buffer
  const uint64_t koff = static_cast<uint64_t>(d) * bv_level_stride;
  if (ntt_nodes > 0) {  // NTT tail: planes 0..2 of the kExpGroup-plane area
    static_assert(kExpGroup >= 3, "the NTT-form tail uses three planes");
    if (d + 1 != s.h || ntt_nodes > nodes)
      throw std::invalid_argument("NTT-form children only at the last expansion level");
    set_smem(k4_expand_level_ntt, smem);
    k4_expand_level_ntt<<<dim3(ntt_nodes, 2, batch), kThreads, smem, st>>>(
        P, galois, inv, k, in, in_stride, out, out_stride, bv_keys, koff);
    check_launch("k4_expand_level_ntt");
    if (ntt_nodes < nodes) {
      k4_expand_level<<<dim3(nodes - ntt_nodes, 2, batch), kThreads, smem, st>>>(
          P, inv, k, in, in_stride, out, out_stride, bv_keys, koff, ntt_nodes);
      check_launch("k4_expand_level");
    }
    return;
  }
  // fewer nodes than SMs (one CTA each): a cluster of 2, 4 or 8 CTAs per node
  const uint64_t ctas = 2ull * nodes * batch, slots = sm_count();
  const int split = !split_enabled() ? 1
                    : 8 * ctas <= slots ? 8 : 4 * ctas <= slots ? 4 : 2 * ctas <= slots ? 2 : 1;
  if (split == 1) {
    dim3 grid(nodes, 2, batch);
    k4_expand_level<<<grid, kThreads, smem, st>>>(P, inv, k, in, in_stride, out, out_stride,
                                                   bv_keys, koff, 0u);
    check_launch("k4_expand_level");
    return;
  }
  const dim3 grid(nodes * split, 2, batch);
  if (split == 8) {
    set_smem(k4_expand_level_split<8>, smem);
    launch_cluster(k4_expand_level_split<8>, 8, grid, smem, st, "k4_expand_level_split", P, inv, k,
                   in, in_stride, out, out_stride, bv_keys, koff);
  } else if (split == 4) {
    set_smem(k4_expand_level_split<4>, smem);
    launch_cluster(k4_expand_level_split<4>, 4, grid, smem, st, "k4_expand_level_split", P, inv, k,
                   in, in_stride, out, out_stride, bv_keys, koff);
  } else {
    set_smem(k4_expand_level_split<2>, smem);
    launch_cluster(k4_expand_level_split<2>, 2, grid, smem, st, "k4_expand_level_split", P, inv, k,
                   in, in_stride, out, out_stride, bv_keys, koff);
  }
}

void launch_selectors(const Dev4 &P, const Shape4 &s, const uint64_t *leaves, uint64_t leaf_stride,
                      const uint64_t *const *gsw_keys, uint64_t *sel, uint32_t batch,
                      cudaStream_t st) {
  if (s.num_dims <= 1) return;
  const size_t smem = plane_bytes(4);
  set_smem(k4_selectors, smem);
  dim3 grid((s.num_dims - 1) * s.l_ep, 2, batch);
  k4_selectors<<<grid, kThreads, smem, st>>>(P, s, leaves, leaf_stride, gsw_keys, sel);
  check_launch("k4_selectors");
}

void launch_fst_ntt(const Dev4 &P, const Shape4 &s, const uint64_t *leaves, uint64_t leaf_stride,
                    uint64_t *qm, uint32_t batch, cudaStream_t st) {
  const size_t smem = plane_bytes(2 * kFstTile);
  set_smem(k4_fst_ntt, smem);
  dim3 grid((s.n0 + kFstTile - 1) / kFstTile, 2, batch);
  k4_fst_ntt<<<grid, kThreads, smem, st>>>(P, s, leaves, leaf_stride, qm, 2 * batch);
  check_launch("k4_fst_ntt");
}

void launch_fst_pack(const Shape4 &s, const uint64_t *qm, uint8_t *qb, uint32_t batch,
                     cudaStream_t st) {
  const uint32_t ncols = 2 * batch;
  const dim3 grid(2 * kN / kPackZ, ncols, (s.n0p + kPackK - 1) / kPackK);
  const uint64_t p_stride = static_cast<uint64_t>(s.n0) * 2 * kN;
  k4_fst_pack<<<grid, 256, 0, st>>>(qm, 2 * p_stride, p_stride, 2 * kN, s.n0, s.n0p, ncols, qb);
  check_launch("k4_fst_pack");
}

void launch_fst_pack_leaves(const Shape4 &s, const uint64_t *leaves, uint64_t leaf_stride,
                            uint8_t *qb, uint32_t batch, cudaStream_t st) {
  const uint32_t ncols = 2 * batch;
  const dim3 grid(2 * kN / kPackZ, ncols, (s.n0p + kPackK - 1) / kPackK);
  k4_fst_pack<<<grid, 256, 0, st>>>(leaves, leaf_stride * kCtWords, 2 * kN, kCtWords, s.n0, s.n0p,
                                     ncols, qb);
  check_launch("k4_fst_pack");
}

void launch_epilogue(const Dev4 &P, const Shape4 &s, const uint64_t *cmat, uint64_t *mid,
                     uint64_t mid_stride, uint32_t batch, cudaStream_t st) {
  const size_t smem = plane_bytes(kEpiRows);
  dim3 grid((s.other + kEpiRows - 1) / kEpiRows, 2, 2 * batch);
  // an even row count keeps every 4-row group (r0 a multiple of 4) 16-byte aligned
  if (s.other % 2 == 0) {
    set_smem(k4_epilogue<true>, smem);
    k4_epilogue<true><<<grid, kThreads, smem, st>>>(P, s, cmat, 2 * batch, mid, mid_stride);
  } else {
    set_smem(k4_epilogue<false>, smem);
    k4_epilogue<false><<<grid, kThreads, smem, st>>>(P, s, cmat, 2 * batch, mid, mid_stride);
  }
  check_launch("k4_epilogue");
}

void launch_mux_level(const Dev4 &P, const Shape4 &s, uint32_t level, uint32_t tree_h,
                      const uint64_t *in, uint64_t *out, uint64_t mid_stride, const uint64_t *sel,
                      uint32_t batch, cudaStream_t st) {
  const uint32_t h = tree_h;
  if (h == 0 || h > 31 || level >= h || h > s.num_dims - 1)
    throw std::invalid_argument("MUX level outside its selector tree");
  const uint32_t other = s.other;
  uint32_t n_pairs, offset = 0, half = 0, extra = 0;
  if (level == 0 && (other > (1u << h) || 2ull * other < (1ull << h)))
    throw std::invalid_argument("MUX tree: candidate count outside (2^(d-2), 2^(d-1)]");
  if (level == 0) {
    const uint32_t last = 2 * other - (1u << h);
    offset = other - last;
    n_pairs = last / 2;
    extra = offset;  // carried prefix
  } else {
    half = ((1u << (h - level)) >> 1);
    n_pairs = half;
  }
  if (n_pairs + extra == 0) return;
  const size_t smem = plane_bytes(kLEp);
  // fewer pairs than SMs (one CTA each): a cluster of 2 or 4 CTAs per pair
  const uint64_t ctas = 2ull * n_pairs * batch, slots = sm_count();
  const int split = (extra != 0 || !split_enabled()) ? 1
                    : 4 * ctas <= slots ? 4 : 2 * ctas <= slots ? 2 : 1;
  if (split != 1) {
    // offset == extra == 0 here, so level 0 pairs (2i, 2i + 1) into i
    const uint32_t xs = level == 0 ? 2 : 1, yoff = level == 0 ? 1 : half;
    const dim3 g(n_pairs * split, 2, batch);
    if (split == 4) {
      set_smem(k4_mux_level_split<4>, smem);
      launch_cluster(k4_mux_level_split<4>, 4, g, smem, st, "k4_mux_level_split", P, s, level, xs,
                     yoff, in, out, mid_stride, sel);
    } else {
      set_smem(k4_mux_level_split<2>, smem);
      launch_cluster(k4_mux_level_split<2>, 2, g, smem, st, "k4_mux_level_split", P, s, level, xs,
                     yoff, in, out, mid_stride, sel);
    }
    return;
  }
  set_smem(k4_mux_level, smem);
  dim3 grid(n_pairs + extra, 2, batch);
  k4_mux_level<<<grid, kThreads, smem, st>>>(P, s, level, n_pairs, offset, half, in, out,
                                              mid_stride, sel);
  check_launch("k4_mux_level");
}

void launch_modswitch(const Dev4 &P, const uint64_t *ct, uint64_t ct_stride, uint64_t *resp,
                      uint8_t *bytes, uint32_t resp_bytes, uint32_t batch, cudaStream_t st) {
  const size_t smem = 2 * kN * sizeof(uint64_t);
  set_smem(k4_modswitch, smem);
  k4_modswitch<<<batch, 256, smem, st>>>(P, ct, ct_stride, resp, bytes, resp_bytes);
  check_launch("k4_modswitch");
}

// ------------------------------------------------- butterfly-rate probe
// The two-limb NTT's forward radix-8 pass (fpass, limb 0) on register values
// and twiddles, three passes per iteration with one pass's corrections per
// stage pattern of the kernels; see the single-modulus probe.
__global__ void __launch_bounds__(256)
k4_bfly_rate(uint64_t *__restrict__ sink, uint32_t iters, ulonglong2 w0) {
  uint64_t v[8];
  ulonglong2 w[7];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = (threadIdx.x * 8ull + k + blockIdx.x) % kQ0;
#pragma unroll
  for (int k = 0; k < 7; ++k) w[k] = make_ulonglong2(w0.x + 2 * k, w0.y + k);
  for (uint32_t it = 0; it < iters; ++it) {
    fpass<kQ0, false, false, false>(v, w);
    fpass<kQ0, true, false, true>(v, w);
    fpass<kQ0, false, true, false>(v, w);
  }
  uint64_t acc = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) acc ^= v[k];
  sink[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

uint32_t bfly_rate_blocks(int sms) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k4_bfly_rate, 256, 0) != cudaSuccess || occ < 1)
    occ = 1;
  return static_cast<uint32_t>(sms) * static_cast<uint32_t>(occ);
}

uint64_t launch_bfly_rate(uint64_t *sink, uint32_t blocks, uint32_t iters, cudaStream_t st) {
  const uint64_t w = 1234567890123456789ull % kQ0;
  const ulonglong2 w0 = make_ulonglong2(
      w, static_cast<uint64_t>((static_cast<unsigned __int128>(w) << 64) / kQ0));
  k4_bfly_rate<<<blocks, 256, 0, st>>>(sink, iters, w0);
  check_launch("k4_bfly_rate");
  return static_cast<uint64_t>(blocks) * 256 * iters * 36;
}

}  // namespace opir4
