// sm_100a kernels of the OnionPIRv2 server path. Every kernel runs 256
// threads per block; polynomial kernels keep their working planes in shared
// memory (8 KiB per residue plane) and run the block-cooperative NTT of
// opir_device.cuh. Thread t owns coefficient positions t + 256 s, s < 8, for
// every per-coefficient step, so global reads of planes are coalesced.
#include "opir_kernels.h"
#include "opir_ntt.cuh"

#include <cooperative_groups.h>

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

namespace opir {

namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

std::atomic<uint64_t> g_launches{0};

void check_launch(const char *what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
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

// Cluster-split MUX levels (k_mux_level_split): on unless OPIR_SPLIT=0.
bool split_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("OPIR_SPLIT");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

// Raise a kernel's dynamic shared-memory limit once per (device, kernel,
// size); cudaFuncSetAttribute applies to the current device.
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
  const cudaError_t e = cudaFuncSetAttribute(
      kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  granted[key] = bytes;
}

// ------------------------------------------------------------ split/compose
// Boundary polynomials -> residue pairs. One boundary polynomial is N u64
// mod q1 q2 (limbs <= 1) or 2N u64, limb q1 then limb q2 (limbs == 2).
__global__ void k_split_u64(DevParams P, const uint64_t *__restrict__ in,
                            uint32_t *__restrict__ out, uint64_t n, uint64_t per_item,
                            uint64_t stride) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i >> kLogN, j = i & (kN - 1);
    const uint64_t item = p / per_item, pp = p % per_item;
    uint32_t *o = out + item * stride + pp * 2 * kN + j;
    if (P.limbs == 2) {
      const uint64_t *src = in + p * 2 * kN + j;
      o[0] = reduce64(src[0], P.q1, P.r[0].mu);
      o[kN] = reduce64(src[kN], P.q2, P.r[1].mu);
    } else {
      const uint64_t v = in[i];
      o[0] = reduce64(v, P.q1, P.r[0].mu);
      o[kN] = reduce64(v, P.q2, P.r[1].mu);
    }
  }
}

// Residue pairs -> boundary polynomials (the inverse of k_split_u64).
__global__ void k_compose_u64(DevParams P, const uint32_t *__restrict__ in, uint64_t stride,
                              uint64_t *__restrict__ out, uint64_t n, uint64_t per_item) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i >> kLogN, j = i & (kN - 1);
    const uint64_t item = p / per_item, pp = p % per_item;
    const uint32_t *s = in + item * stride + pp * 2 * kN + j;
    if (P.limbs == 2) {
      out[p * 2 * kN + j] = s[0];
      out[p * 2 * kN + kN + j] = s[kN];
    } else {
      out[i] = crt_compose(s[0], s[kN], P);
    }
  }
}

// --------------------------------------------------------- DB preprocessing
constexpr int kDbTile = 8;  // plaintexts per block (one padded plane each)

template <int RES>
__device__ __forceinline__ void db_preprocess_body(const DevParams &P, const uint16_t *coeffs,
                                                   uint64_t coeff_pt_begin, uint64_t seed,
                                                   uint64_t t, uint64_t logical, uint32_t n0,
                                                   uint32_t n0p, uint32_t other, uint64_t pt_begin,
                                                   uint64_t pt_end, const uint32_t *row_map,
                                                   uint8_t *db8) {
  extern __shared__ uint32_t sm[];
  const int tid = threadIdx.x;
  const ResidueTables &T = P.r[RES];
  const uint64_t pt0 = pt_begin + (uint64_t)blockIdx.x * kDbTile;
  for (int e = 0; e < kDbTile; ++e) {
    const uint64_t pt = pt0 + e;
    // the database plaintext stored at local position pt (a row shard keeps
    // some of the rows; pt < pt_end keeps pt / n0 below the shard's rows)
    const uint64_t gpt = (row_map && pt < pt_end) ? (uint64_t)row_map[pt / n0] * n0 + pt % n0 : pt;
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int c = posA(tid, k);
      uint32_t x = 0;
      if (pt < pt_end && gpt < logical) {
        if (coeffs != nullptr)
          x = coeffs[(pt - coeff_pt_begin) * kN + c];
        else
          x = static_cast<uint32_t>(mix64(seed + (gpt * kN + c + 1) * kGolden) % t);
      }
      v[k] = x;  // x < t < q_res: canonical
    }
    fA<RES>(v);
    st_plane<0>(sm + e * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid_r<RES>(sm, kDbTile, T.fwt);
  uint32_t out[kDbTile][8];
  {
    uint2 wd[6];
    fload_d(wd, T.fwt, tid);
#pragma unroll
    for (int e = 0; e < kDbTile; ++e) {
      ld_plane<3>(sm + e * kPad, out[e], tid);
      fD<RES>(out[e], wd);
#pragma unroll
      for (int k = 0; k < 8; ++k) out[e][k] = canon8<RES>(out[e][k]);
    }
  }
  // byte planes: db8[((res N + level) 4 + plane) other + row][n0p], pt = row n0 + k
  const bool packed = (n0 % kDbTile) == 0 && pt0 + kDbTile <= pt_end;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint64_t zl = (uint64_t)RES * kN + posD(tid, k);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uint8_t *plane = db8 + (zl * 4 + j) * (uint64_t)other * n0p;
      if (packed) {
        const uint64_t row = pt0 / n0, col = pt0 % n0;
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          lo |= ((out[e][k] >> (8 * j)) & 0xFFu) << (8 * e);
          hi |= ((out[e + 4][k] >> (8 * j)) & 0xFFu) << (8 * e);
        }
        *reinterpret_cast<uint2 *>(plane + row * n0p + col) = make_uint2(lo, hi);
      } else {
        for (int e = 0; e < kDbTile; ++e) {
          const uint64_t pt = pt0 + e;
          if (pt < pt_end)
            plane[(pt / n0) * n0p + pt % n0] = static_cast<uint8_t>(out[e][k] >> (8 * j));
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads, 2)
k_db_preprocess(DevParams P, const uint16_t *__restrict__ coeffs,
                uint64_t coeff_pt_begin, uint64_t seed, uint64_t t,
                uint64_t logical, uint32_t n0, uint32_t n0p, uint32_t other,
                uint64_t pt_begin, uint64_t pt_end, const uint32_t *__restrict__ row_map,
                uint8_t *__restrict__ db8) {
  if (blockIdx.y == 0)
    db_preprocess_body<0>(P, coeffs, coeff_pt_begin, seed, t, logical, n0, n0p, other, pt_begin,
                          pt_end, row_map, db8);
  else
    db_preprocess_body<1>(P, coeffs, coeff_pt_begin, seed, t, logical, n0, n0p, other, pt_begin,
                          pt_end, row_map, db8);
}

// ----------------------------------------------------------- expansion level
// One heap node (and one residue) per block: BV key switch of the node's
// ciphertext (bv_keyswitch.cpp:296-367) then the two children
// (server.cpp:794-809): left = c + c', right = (c - c') X^-k.
// sigma_k is applied as a gather: sigma(c)[j] = +-c[j k^-1 mod 2N].
// Children of the last level in NTT form (the first-dimension leaves), from
// the key switch's sums still in NTT form: with NTT slot i holding the value
// at psi^e_i, e_i = 2 brev(i) + 1 (the reference's bit-reversed order),
// sigma_g(c)^[i] = c^[j] for e_j = e_i g mod 2N, and (f X^-k)^[i] =
// psi^(-k e_i) f^[i]. So left = c^ + sigma(c0)^ + delta^ and right =
// (c^ - sigma(c0)^ - delta^) psi^(-k e), the same values fst_ntt would
// compute from the coefficient-form children, with the two inverse NTTs of
// the key switch replaced by forward NTTs of the parent (c0, c1).
template <int RES>
__device__ __forceinline__ void expand_tail_ntt(const ResidueTables &T, uint32_t galois,
                                                uint32_t kshift, const uint32_t *ct,
                                                const uint32_t (&vb)[8], const uint32_t (&va)[8],
                                                uint32_t *sm, uint32_t *out, uint64_t out_stride,
                                                uint32_t node) {
  constexpr uint32_t q = Res<RES>::q;
  const int tid = threadIdx.x;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = ct[(p * 2 + RES) * kN + posA(tid, k)];
    fA<RES>(v);
    st_plane<0>(sm + p * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid_r<RES>(sm, 2, T.fwt);
  uint32_t h0[8], h1[8];
  {
    uint2 wd[6];
    fload_d(wd, T.fwt, tid);
    ld_plane<3>(sm, h0, tid);
    ld_plane<3>(sm + kPad, h1, tid);
    fD<RES>(h0, wd);
    fD<RES>(h1, wd);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    h0[k] = canon8<RES>(h0[k]);
    h1[k] = canon8<RES>(h1[k]);
  }
  st_plane<3>(sm + 2 * kPad, h0, tid);  // c0^ by slot, for the sigma gather
  __syncthreads();
  // children, four coefficients (one uint4 per polynomial) at a time
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint32_t l0[4], l1[4], r0[4], r1[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int k = 4 * h + c;
      const uint32_t i = posD(tid, k);
      const uint32_t e = 2 * (__brev(i) >> 21) + 1;  // 11-bit reversal (N = 2048)
      const uint32_t j = __brev(((e * galois) & (2 * kN - 1)) >> 1) >> 21;
      const uint32_t n0v = add_mod(sm[2 * kPad + padi(j)], vb[k], q);
      const uint32_t n1v = va[k];
      l0[c] = add_mod(h0[k], n0v, q);
      l1[c] = add_mod(h1[k], n1v, q);
      const uint2 lam = __ldg(T.pwt + ((2 * kN - ((kshift * e) & (2 * kN - 1))) & (2 * kN - 1)));
      const uint32_t d0 = sub_mod(h0[k], n0v, q), d1 = sub_mod(h1[k], n1v, q);
      const uint32_t t0 = d0 * lam.x - __umulhi(d0, lam.y) * q;
      const uint32_t t1 = d1 * lam.x - __umulhi(d1, lam.y) * q;
      r0[c] = min(t0, t0 - q);
      r1[c] = min(t1, t1 - q);
    }
    const int j0 = 4 * (tid + 256 * h);
    uint32_t *outL = out + ((uint64_t)blockIdx.z * out_stride + 2 * (uint64_t)node) * kCtWords;
    uint32_t *outR = outL + kCtWords;
    *reinterpret_cast<uint4 *>(outL + RES * kN + j0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
    *reinterpret_cast<uint4 *>(outL + 2 * kN + RES * kN + j0) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
    *reinterpret_cast<uint4 *>(outR + RES * kN + j0) = make_uint4(r0[0], r0[1], r0[2], r0[3]);
    *reinterpret_cast<uint4 *>(outR + 2 * kN + RES * kN + j0) = make_uint4(r1[0], r1[1], r1[2], r1[3]);
  }
}

template <int RES, class G, bool NTT_OUT = false>
__device__ __forceinline__ void expand_level_body(const DevParams &P, uint32_t galois_inv,
                                                  uint32_t kshift, int base_ks, int l_ks,
                                                  const uint32_t *in, uint64_t in_stride,
                                                  uint32_t *out, uint64_t out_stride,
                                                  const uint32_t *const *bv_keys,
                                                  uint64_t bv_level_off, uint32_t galois = 0,
                                                  uint32_t node0 = 0) {
  extern __shared__ uint32_t sm[];
  constexpr uint32_t q = Res<RES>::q;
  const int node = node0 + blockIdx.x, b = blockIdx.z, tid = threadIdx.x;
  const ResidueTables &T = P.r[RES];
  const uint32_t *ct = in + ((uint64_t)b * in_stride + node) * kCtWords;
  const uint32_t *c0 = ct + RES * kN;
  const uint32_t *c1 = ct + 2 * kN + RES * kN;

  // sigma_k(c0) (own residue) and the centred sigma_k(c1) at A-order positions
  uint32_t s0[8];
  uint64_t d[8];  // centred sigma_k(c1) + digit offset
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t j = posA(tid, k);
    const uint32_t u = (j * galois_inv) & (2 * kN - 1);
    const bool neg = u >= kN;
    const uint32_t src = u & (kN - 1);
    const uint32_t z = c0[src], a0 = ct[2 * kN + src], a1 = ct[3 * kN + src];
    s0[k] = neg ? neg_mod(z, q) : z;
    d[k] = digit_source<G::lks, G::bks, G::kks>(compose_c(neg ? neg_mod(a0, kQ1) : a0,
                                                          neg ? neg_mod(a1, kQ2) : a1));
  }
  // digit planes: decompose, pass A in registers
#pragma unroll
  for (int i = 0; i < G::lks; ++i) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = digit_res<q, G::bks, G::kks>(d[k], i);
    fA<RES>(v);
    st_plane<0>(sm + i * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid_r<RES>(sm, G::lks, T.fwt);
  // inner product with the key rows (row t encrypts sigma(s) B^t), D-order;
  // L_KS products per coefficient (mac_in)
  const uint32_t *key = bv_keys[b] + bv_level_off + RES * kN;
  uint64_t ab[8], aa[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) ab[k] = aa[k] = 0;
  {
    uint2 wd[6];
    fload_d(wd, T.fwt, tid);
#pragma unroll
    for (int i = 0; i < G::lks; ++i) {
      uint32_t v[8];
      ld_plane<3>(sm + i * kPad, v, tid);
      fD<RES>(v, wd);
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = mac_in<RES, G::lks>(v[k]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j0 = 4 * (tid + 256 * h);
        const uint4 kb = __ldg(reinterpret_cast<const uint4 *>(key + (uint64_t)(i * 4 + 0) * kN + j0));
        const uint4 ka = __ldg(reinterpret_cast<const uint4 *>(key + (uint64_t)(i * 4 + 2) * kN + j0));
        ab[4 * h + 0] += (uint64_t)v[4 * h + 0] * kb.x; aa[4 * h + 0] += (uint64_t)v[4 * h + 0] * ka.x;
        ab[4 * h + 1] += (uint64_t)v[4 * h + 1] * kb.y; aa[4 * h + 1] += (uint64_t)v[4 * h + 1] * ka.y;
        ab[4 * h + 2] += (uint64_t)v[4 * h + 2] * kb.z; aa[4 * h + 2] += (uint64_t)v[4 * h + 2] * ka.z;
        ab[4 * h + 3] += (uint64_t)v[4 * h + 3] * kb.w; aa[4 * h + 3] += (uint64_t)v[4 * h + 3] * ka.w;
      }
    }
  }
  __syncthreads();
  if constexpr (NTT_OUT) {
    uint32_t vb[8], va[8];  // the key switch's delta in NTT form, canonical
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      vb[k] = red64<RES>(ab[k]);
      va[k] = red64<RES>(aa[k]);
    }
    expand_tail_ntt<RES>(T, galois, kshift, ct, vb, va, sm, out, out_stride, node);
    return;
  }
  uint32_t *outL = out + ((uint64_t)b * out_stride + 2 * (uint64_t)node) * kCtWords;
  uint32_t *outR = outL + kCtWords;
  {
    uint2 wd[6];
    iload_d(wd, T.iwt, tid);
    uint32_t v[8], w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { v[k] = red64_lazy<RES>(ab[k]); w[k] = red64_lazy<RES>(aa[k]); }
    iD<RES>(v, wd);
    iD<RES>(w, wd);
    st_plane<3>(sm, v, tid);
    st_plane<3>(sm + kPad, w, tid);
  }
  __syncthreads();
  inv_mid_r<RES>(sm, 2, T.iwt);
  uint32_t db_[8], da[8];
  ld_plane<0>(sm, db_, tid);
  ld_plane<0>(sm + kPad, da, tid);
  iA<RES>(db_);
  iA<RES>(da);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int j = posA(tid, k);
    const uint32_t n0v = add_mod(s0[k], db_[k], q);  // c0' = sigma(c0) + delta_b
    const uint32_t n1v = da[k];                      // c1' = delta_a
    const uint32_t o0 = c0[j], o1 = c1[j];
    outL[RES * kN + j] = add_mod(o0, n0v, q);
    outL[2 * kN + RES * kN + j] = add_mod(o1, n1v, q);
    const uint32_t d0 = sub_mod(o0, n0v, q), d1 = sub_mod(o1, n1v, q);
    int dst = j - static_cast<int>(kshift);
    const bool wrap = dst < 0;
    if (wrap) dst += kN;
    outR[RES * kN + dst] = wrap ? neg_mod(d0, q) : d0;
    outR[2 * kN + RES * kN + dst] = wrap ? neg_mod(d1, q) : d1;
  }
}

template <class G>
__global__ void __launch_bounds__(kThreads, 2)
k_expand_level(DevParams P, uint32_t galois_inv, uint32_t kshift, int base_ks, int l_ks,
               const uint32_t *__restrict__ in, uint64_t in_stride,
               uint32_t *__restrict__ out, uint64_t out_stride,
               const uint32_t *const *__restrict__ bv_keys, uint64_t bv_level_off,
               uint32_t node0) {
  if (blockIdx.y == 0)
    expand_level_body<0, G>(P, galois_inv, kshift, base_ks, l_ks, in, in_stride, out, out_stride,
                            bv_keys, bv_level_off, 0, node0);
  else
    expand_level_body<1, G>(P, galois_inv, kshift, base_ks, l_ks, in, in_stride, out, out_stride,
                            bv_keys, bv_level_off, 0, node0);
}

// The last expansion level's nodes below ntt_nodes when the
// first-dimension leaves are wanted in NTT form: their children (leaves
// < n0) are written in NTT form (expand_tail_ntt); k_expand_level takes the
// remaining nodes.
template <class G>
__global__ void __launch_bounds__(kThreads, 2)
k_expand_level_ntt(DevParams P, uint32_t galois, uint32_t galois_inv, uint32_t kshift,
                   const uint32_t *__restrict__ in, uint64_t in_stride,
                   uint32_t *__restrict__ out, uint64_t out_stride,
                   const uint32_t *const *__restrict__ bv_keys, uint64_t bv_level_off) {
  if (blockIdx.y == 0)
    expand_level_body<0, G, true>(P, galois_inv, kshift, 0, 0, in, in_stride, out, out_stride,
                                  bv_keys, bv_level_off, galois);
  else
    expand_level_body<1, G, true>(P, galois_inv, kshift, 0, 0, in, in_stride, out, out_stride,
                                  bv_keys, bv_level_off, galois);
}

// Expansion level, cluster split: a level with fewer nodes than the GPU
// has CTA slots (the top of the heap, and most levels of a single query)
// runs each node's key switch on a cluster of C CTAs. CTA r NTTs digits
// [r D, (r + 1) D) (D = L_KS / C) of sigma_k(c1) and multiplies them with
// their key rows; the partial sums meet in distributed shared memory; CTA 0
// then finishes the b part (c0 of both children) and CTA 1 the a part (c1 of
// both children). Every partial and their total are exact 64-bit sums below
// the single-CTA bound, so the children are the same bit for bit.
template <int RES, int C, class G>
__device__ __forceinline__ void expand_split_body(const DevParams &P, uint32_t galois_inv,
                                                  uint32_t kshift, const uint32_t *in,
                                                  uint64_t in_stride, uint32_t *out,
                                                  uint64_t out_stride,
                                                  const uint32_t *const *bv_keys,
                                                  uint64_t bv_level_off) {
  static_assert(G::lks % C == 0, "digits split evenly over the cluster");
  constexpr int D = G::lks / C;
  extern __shared__ uint32_t sm[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  constexpr uint32_t q = Res<RES>::q;
  const int rank = static_cast<int>(cluster.block_rank());
  const int node = blockIdx.x / C, b = blockIdx.z, tid = threadIdx.x;
  const ResidueTables &T = P.r[RES];
  const uint32_t *ct = in + ((uint64_t)b * in_stride + node) * kCtWords;
  const uint32_t *c0 = ct + RES * kN;
  const uint32_t *c1 = ct + 2 * kN + RES * kN;

  uint64_t d[8];  // centred sigma_k(c1) + digit offset
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t j = posA(tid, k);
    const uint32_t u = (j * galois_inv) & (2 * kN - 1);
    const bool neg = u >= kN;
    const uint32_t src = u & (kN - 1);
    const uint32_t a0 = ct[2 * kN + src], a1 = ct[3 * kN + src];
    d[k] = digit_source<G::lks, G::bks, G::kks>(compose_c(neg ? neg_mod(a0, kQ1) : a0,
                                                          neg ? neg_mod(a1, kQ2) : a1));
  }
  const int i0 = rank * D;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = digit_res<q, G::bks, G::kks>(d[k], i0 + i);
    fA<RES>(v);
    st_plane<0>(sm + i * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid_r<RES, false>(sm, D, T.fwt);
  const uint32_t *key = bv_keys[b] + bv_level_off + RES * kN;
  uint64_t ab[8], aa[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) ab[k] = aa[k] = 0;
  {
    uint2 wd[6];
    fload_d(wd, T.fwt, tid);
    for (int i = 0; i < D; ++i) {
      uint32_t v[8];
      ld_plane<3>(sm + i * kPad, v, tid);
      fD<RES>(v, wd);
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = mac_in<RES, G::lks>(v[k]);  // L_KS products over the cluster
      const int row = i0 + i;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j0 = 4 * (tid + 256 * h);
        const uint4 kb = __ldg(reinterpret_cast<const uint4 *>(key + (uint64_t)(row * 4 + 0) * kN + j0));
        const uint4 ka = __ldg(reinterpret_cast<const uint4 *>(key + (uint64_t)(row * 4 + 2) * kN + j0));
        ab[4 * h + 0] += (uint64_t)v[4 * h + 0] * kb.x; aa[4 * h + 0] += (uint64_t)v[4 * h + 0] * ka.x;
        ab[4 * h + 1] += (uint64_t)v[4 * h + 1] * kb.y; aa[4 * h + 1] += (uint64_t)v[4 * h + 1] * ka.y;
        ab[4 * h + 2] += (uint64_t)v[4 * h + 2] * kb.z; aa[4 * h + 2] += (uint64_t)v[4 * h + 2] * ka.z;
        ab[4 * h + 3] += (uint64_t)v[4 * h + 3] * kb.w; aa[4 * h + 3] += (uint64_t)v[4 * h + 3] * ka.w;
      }
    }
  }
  __syncthreads();
  // partial sums out to shared memory: [b / a][k][tid]
  uint64_t *ex = reinterpret_cast<uint64_t *>(sm);
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
    uint2 wd[6];
    iload_d(wd, T.iwt, tid);
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = red64_lazy<RES>(tot[k]);
    iD<RES>(v, wd);
    st_plane<3>(sm, v, tid);
  }
  __syncthreads();
  inv_mid_r<RES>(sm, 1, T.iwt);
  uint32_t dv[8];
  ld_plane<0>(sm, dv, tid);
  iA<RES>(dv);
  // rank 0: c0 of both children (with sigma_k(c0)); rank 1: c1 of both
  uint32_t *outL = out + ((uint64_t)b * out_stride + 2 * (uint64_t)node) * kCtWords;
  uint32_t *outR = outL + kCtWords;
  const uint32_t *src_poly = rank == 0 ? c0 : c1;
  const uint64_t off = (uint64_t)rank * 2 * kN + RES * kN;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int j = posA(tid, k);
    uint32_t nv = dv[k];
    if (rank == 0) {  // c0' = sigma(c0) + delta_b
      const uint32_t u = (j * galois_inv) & (2 * kN - 1);
      const uint32_t z = c0[u & (kN - 1)];
      nv = add_mod(u >= kN ? neg_mod(z, q) : z, nv, q);
    }
    const uint32_t o = src_poly[j];
    outL[off + j] = add_mod(o, nv, q);
    const uint32_t dd = sub_mod(o, nv, q);
    int dst = j - static_cast<int>(kshift);
    const bool wrap = dst < 0;
    if (wrap) dst += kN;
    outR[off + dst] = wrap ? neg_mod(dd, q) : dd;
  }
}

template <int C, class G>
__global__ void __launch_bounds__(kThreads, 2)
k_expand_level_split(DevParams P, uint32_t galois_inv, uint32_t kshift,
                     const uint32_t *__restrict__ in, uint64_t in_stride,
                     uint32_t *__restrict__ out, uint64_t out_stride,
                     const uint32_t *const *__restrict__ bv_keys, uint64_t bv_level_off) {
  if (blockIdx.y == 0)
    expand_split_body<0, C, G>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys,
                               bv_level_off);
  else
    expand_split_body<1, C, G>(P, galois_inv, kshift, in, in_stride, out, out_stride, bv_keys,
                               bv_level_off);
}

// Shared gadget product of a coefficient-form ciphertext (both residues read
// from `x` / optional `y`: the decomposed value is y - x, or x when y is
// null) against NTT-form RGSW rows: acc_k += sum_rows digit * rgsw[row][k],
// accumulated at this thread's D-order positions. Digit i (LSB first) of
// poly p meets row p*l + (l - 1 - i) (gsw.cpp:283-293). Uses l padded planes.
// The accumulators start at zero and take 2 l products of mac_in values;
// when 2 l > 16 they are reduced to [0, 2q] after the first polynomial, so
// at most 16 products (plus that carry) build up between reductions, below
// 2^64.
template <int RES, int L, int B, int KIND>
__device__ __forceinline__ void gadget_mac(const DevParams &P, const uint32_t *x,
                                           const uint32_t *y, const uint32_t *rgsw,
                                           uint32_t *sm, uint64_t (&acc0)[8],
                                           uint64_t (&acc1)[8]) {
  constexpr uint32_t q = Res<RES>::q;
  constexpr int l = L;
  constexpr bool mid = 2 * L > 16;            // reduce after the first polynomial
  constexpr int kProducts = mid ? L : 2 * L;  // products between reductions
  const ResidueTables &T = P.r[RES];
  const int tid = threadIdx.x;
#pragma unroll 1
  for (int p = 0; p < 2; ++p) {
    uint64_t d[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posA(tid, k);
      uint32_t v1 = x[(p * 2 + 0) * kN + j], v2 = x[(p * 2 + 1) * kN + j];
      if (y != nullptr) {
        v1 = sub_mod(y[(p * 2 + 0) * kN + j], v1, kQ1);
        v2 = sub_mod(y[(p * 2 + 1) * kN + j], v2, kQ2);
      }
      d[k] = digit_source<L, B, KIND>(compose_c(v1, v2));
    }
#pragma unroll
    for (int i = 0; i < l; ++i) {
      uint32_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = digit_res<q, B, KIND>(d[k], i);
      fA<RES>(v);
      st_plane<0>(sm + i * kPad, v, tid);
    }
    __syncthreads();
    fwd_mid_r<RES>(sm, l, T.fwt);
    uint2 wd[6];
    fload_d(wd, T.fwt, tid);
#pragma unroll
    for (int i = 0; i < l; ++i) {
      uint32_t v[8];
      ld_plane<3>(sm + i * kPad, v, tid);
      fD<RES>(v, wd);
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = mac_in<RES, kProducts>(v[k]);
      const int row = p * l + (l - 1 - i);
      const uint32_t *R0 = rgsw + (uint64_t)row * kCtWords + RES * kN;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j0 = 4 * (tid + 256 * h);
        const uint4 r0 = __ldg(reinterpret_cast<const uint4 *>(R0 + j0));
        const uint4 r1 = __ldg(reinterpret_cast<const uint4 *>(R0 + 2 * kN + j0));
        acc0[4 * h + 0] += (uint64_t)v[4 * h + 0] * r0.x; acc1[4 * h + 0] += (uint64_t)v[4 * h + 0] * r1.x;
        acc0[4 * h + 1] += (uint64_t)v[4 * h + 1] * r0.y; acc1[4 * h + 1] += (uint64_t)v[4 * h + 1] * r1.y;
        acc0[4 * h + 2] += (uint64_t)v[4 * h + 2] * r0.z; acc1[4 * h + 2] += (uint64_t)v[4 * h + 2] * r1.z;
        acc0[4 * h + 3] += (uint64_t)v[4 * h + 3] * r0.w; acc1[4 * h + 3] += (uint64_t)v[4 * h + 3] * r1.w;
      }
    }
    if (mid && p == 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        acc0[k] = red64_lazy<RES>(acc0[k]);
        acc1[k] = red64_lazy<RES>(acc1[k]);
      }
    }
    __syncthreads();
  }
}

// -------------------------------------------------------- selector completion
template <int RES, class G>
__device__ __forceinline__ void selectors_body(const DevParams &P, const Shape &S,
                                               const uint32_t *leaves, uint64_t leaf_stride,
                                               const uint32_t *const *gsw_keys, uint32_t *sel) {
  extern __shared__ uint32_t sm[];
  const int row_id = blockIdx.x, b = blockIdx.z, tid = threadIdx.x;
  const int selno = row_id / S.l_ep, r = row_id % S.l_ep;
  const ResidueTables &T = P.r[RES];
  const uint32_t *ct = leaves + ((uint64_t)b * leaf_stride + S.n0 + row_id) * kCtWords;
  uint32_t *out = sel + ((uint64_t)b * (S.num_dims - 1) + selno) * 2 * S.l_ep * kCtWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  // bottom row: ExtProd(RGSW(s), row) with the key gadget (gsw.cpp:119-182)
  gadget_mac<RES, G::lkey, G::bkey, G::kkey>(P, ct, nullptr, gsw_keys[b], sm, acc0, acc1);
  uint32_t *bot = out + (uint64_t)(S.l_ep + r) * kCtWords + RES * kN;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int j0 = 4 * (tid + 256 * h);
    uint4 o0, o1;
    o0.x = red64<RES>(acc0[4 * h + 0]); o0.y = red64<RES>(acc0[4 * h + 1]);
    o0.z = red64<RES>(acc0[4 * h + 2]); o0.w = red64<RES>(acc0[4 * h + 3]);
    o1.x = red64<RES>(acc1[4 * h + 0]); o1.y = red64<RES>(acc1[4 * h + 1]);
    o1.z = red64<RES>(acc1[4 * h + 2]); o1.w = red64<RES>(acc1[4 * h + 3]);
    *reinterpret_cast<uint4 *>(bot + j0) = o0;
    *reinterpret_cast<uint4 *>(bot + 2 * kN + j0) = o1;
  }
  // top row: the expanded row itself in NTT form (gsw.cpp:330-338)
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = ct[(p * 2 + RES) * kN + posA(tid, k)];
    fA<RES>(v);
    st_plane<0>(sm + p * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid_r<RES>(sm, 2, T.fwt);
  uint32_t *top = out + (uint64_t)r * kCtWords + RES * kN;
  uint2 wd[6];
  fload_d(wd, T.fwt, tid);
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint32_t v[8];
    ld_plane<3>(sm + p * kPad, v, tid);
    fD<RES>(v, wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = canon8<RES>(v[k]);
#pragma unroll
    for (int h = 0; h < 2; ++h)
      *reinterpret_cast<uint4 *>(top + p * 2 * kN + 4 * (tid + 256 * h)) =
          make_uint4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
  }
}

template <class G>
__global__ void __launch_bounds__(kThreads, 2)
k_selectors(DevParams P, Shape S, const uint32_t *__restrict__ leaves, uint64_t leaf_stride,
            const uint32_t *const *__restrict__ gsw_keys, uint32_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    selectors_body<0, G>(P, S, leaves, leaf_stride, gsw_keys, sel);
  else
    selectors_body<1, G>(P, S, leaves, leaf_stride, gsw_keys, sel);
}

// ------------------------------------------------------- first-dim query prep
// Forward NTT of the first n0 leaves (prep_query_composite, server.cpp:
// 264-304) into `out`, same ciphertext layout as the leaves, stored as
// coalesced quads; k_fst_pack then turns them into byte planes.
constexpr int kFstTile = 4;  // ciphertexts per block (8 planes)

template <int RES>
__device__ __forceinline__ void fst_ntt_body(const DevParams &P, const Shape &S,
                                             const uint32_t *leaves, uint64_t leaf_stride,
                                             uint32_t *out, uint64_t out_stride) {
  extern __shared__ uint32_t sm[];
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t k0 = blockIdx.x * kFstTile;
  const ResidueTables &T = P.r[RES];
  {
    // every plane's loads first (more loads in flight), then the first pass
    uint32_t v[2 * kFstTile][8];
#pragma unroll
    for (int e = 0; e < 2 * kFstTile; ++e) {
      const uint32_t kk = k0 + (e >> 1);
      const int p = e & 1;
      const uint32_t *src = leaves + ((uint64_t)b * leaf_stride + kk) * kCtWords + (p * 2 + RES) * kN;
#pragma unroll
      for (int k = 0; k < 8; ++k) v[e][k] = kk < S.n0 ? src[posA(tid, k)] : 0u;
    }
#pragma unroll
    for (int e = 0; e < 2 * kFstTile; ++e) {
      fA<RES>(v[e]);
      st_plane<0>(sm + e * kPad, v[e], tid);
    }
  }
  __syncthreads();
  fwd_mid_r<RES>(sm, 2 * kFstTile, T.fwt);
  uint2 wd[6];
  fload_d(wd, T.fwt, tid);
#pragma unroll
  for (int e = 0; e < 2 * kFstTile; ++e) {
    const uint32_t kk = k0 + (e >> 1);
    if (kk >= S.n0) continue;  // uniform over the block
    const int p = e & 1;
    uint32_t v[8];
    ld_plane<3>(sm + e * kPad, v, tid);
    fD<RES>(v, wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = canon8<RES>(v[k]);
    uint32_t *dst = out + ((uint64_t)b * out_stride + kk) * kCtWords + (p * 2 + RES) * kN;
#pragma unroll
    for (int h = 0; h < 2; ++h)
      *reinterpret_cast<uint4 *>(dst + 4 * (tid + 256 * h)) =
          make_uint4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
  }
}

__global__ void __launch_bounds__(kThreads, 2)
k_fst_ntt(DevParams P, Shape S, const uint32_t *__restrict__ leaves, uint64_t leaf_stride,
          uint32_t *__restrict__ out, uint64_t out_stride) {
  if (blockIdx.y == 0)
    fst_ntt_body<0>(P, S, leaves, leaf_stride, out, out_stride);
  else
    fst_ntt_body<1>(P, S, leaves, leaf_stride, out, out_stride);
}

// Byte-plane packing of the NTT-form query matrix:
//   qb[((res N + z) 4 + j) ncols + col][k] = byte j of ntt[b][k][p][res][z],
//   col = 2 b + p, zero for n0 <= k < n0p.
// Block = (128 leaves, 32 levels of one residue, one column). Reads are 128-B
// rows of 32 levels per leaf; the tile is transposed through shared memory
// (33-word pitch: conflict-free both ways) and written as 128-B rows of
// leaves per (level, byte plane).
constexpr int kPackK = 128, kPackZ = 32, kPackPitch = kPackK / 4 + 1;

__global__ void __launch_bounds__(kThreads)
k_fst_pack(const uint32_t *__restrict__ ntt, uint64_t ntt_stride, uint32_t n0, uint32_t n0p,
           uint8_t *__restrict__ qb, uint32_t ncols) {
  __shared__ uint32_t sw[4][kPackZ][kPackPitch];
  const uint32_t k0 = blockIdx.x * kPackK;
  const uint32_t zt = blockIdx.y;
  const int res = zt >= kN / kPackZ ? 1 : 0;
  const uint32_t z0 = (zt - res * (kN / kPackZ)) * kPackZ;
  const uint32_t col = blockIdx.z, b = col >> 1, p = col & 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t *src = ntt + (uint64_t)b * ntt_stride * kCtWords + (p * 2 + res) * kN + z0 + lane;
  // warp w packs leaves 4w' .. 4w'+3 (w' = w, w + 8, ...) of level z0 + lane
  for (int kq = warp; kq < kPackK / 4; kq += kThreads / 32) {
    uint32_t v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t k = k0 + 4 * kq + i;
      v[i] = k < n0 ? src[(uint64_t)k * kCtWords] : 0u;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      sw[j][lane][kq] = __byte_perm(__byte_perm(v[0], v[1], 0x40 + 0x11 * j),
                                    __byte_perm(v[2], v[3], 0x40 + 0x11 * j), 0x5410);
  }
  __syncthreads();
  // each thread writes 16 leaves (one uint4) of one (byte plane, level) row
  for (int i = tid; i < 4 * kPackZ * (kPackK / 16); i += kThreads) {
    const int c = i & 7, row = i >> 3, j = row / kPackZ, z = row % kPackZ;
    const uint32_t k = k0 + 16 * c;
    if (k >= n0p) continue;
    const uint32_t *w = &sw[j][z][4 * c];
    *reinterpret_cast<uint4 *>(qb + (((uint64_t)(res * kN + z0 + z) * 4 + j) * ncols + col) * n0p + k) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// ------------------------------------------------------------ first-dim scan
// CUDA-core form (used for small batches): block = (column tile, residue x
// level); a warp owns one database row at a time, its lanes split the first
// dimension, accumulate exact 64-bit sums of 29x29-bit products (at most 64
// per lane, so no overflow), reduce mod q and finish with a shuffle tree of
// modular adds. Operands are the byte planes also used by the tensor-core
// form; values are rebuilt with byte permutes.
__device__ __forceinline__ void unpack16(const uint4 &p0, const uint4 &p1, const uint4 &p2,
                                         const uint4 &p3, uint32_t (&a)[16]) {
  const uint32_t x0[4] = {p0.x, p0.y, p0.z, p0.w}, x1[4] = {p1.x, p1.y, p1.z, p1.w};
  const uint32_t x2[4] = {p2.x, p2.y, p2.z, p2.w}, x3[4] = {p3.x, p3.y, p3.z, p3.w};
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const uint32_t lo01 = __byte_perm(x0[w], x1[w], 0x5140), lo23 = __byte_perm(x2[w], x3[w], 0x5140);
    const uint32_t hi01 = __byte_perm(x0[w], x1[w], 0x7362), hi23 = __byte_perm(x2[w], x3[w], 0x7362);
    a[4 * w + 0] = __byte_perm(lo01, lo23, 0x5410);
    a[4 * w + 1] = __byte_perm(lo01, lo23, 0x7632);
    a[4 * w + 2] = __byte_perm(hi01, hi23, 0x5410);
    a[4 * w + 3] = __byte_perm(hi01, hi23, 0x7632);
  }
}

template <int NCT, bool VEC>
__global__ void __launch_bounds__(kThreads)
k_scan(DevParams P, uint32_t n0, uint32_t n0p, uint32_t m, const uint8_t *__restrict__ db8,
       const uint8_t *__restrict__ qb, uint32_t ncols, uint32_t *__restrict__ cmat) {
  extern __shared__ __align__(16) uint32_t qs[];  // [NCT][n0p]
  const int ct0 = blockIdx.x * NCT;
  const uint32_t z = blockIdx.y;
  const int res = z >= kN ? 1 : 0;
  const uint32_t q = res ? P.q2 : P.q1;
  const uint64_t mu = res ? P.r[1].mu : P.r[0].mu;
  for (uint32_t idx = threadIdx.x; idx < n0p * NCT; idx += kThreads) {
    const uint32_t c = idx / n0p, k = idx % n0p;
    uint32_t v = 0;
    if (ct0 + c < ncols && k < n0) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        v |= static_cast<uint32_t>(qb[(((uint64_t)z * 4 + j) * ncols + ct0 + c) * n0p + k]) << (8 * j);
    }
    qs[c * n0p + k] = v;
  }
  __syncthreads();
  const uint64_t plane_stride = (uint64_t)m * n0p;
  const uint8_t *A = db8 + (uint64_t)z * 4 * plane_stride;
  uint32_t *C = cmat + (uint64_t)z * m * ncols;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t r = warp; r < m; r += kThreads / 32) {
    const uint8_t *Ar = A + (uint64_t)r * n0p;
    uint64_t acc[NCT];
#pragma unroll
    for (int c = 0; c < NCT; ++c) acc[c] = 0;
    if (VEC) {
      for (uint32_t k = 16 * lane; k < n0p; k += 512) {
        const uint4 p0 = __ldg(reinterpret_cast<const uint4 *>(Ar + k));
        const uint4 p1 = __ldg(reinterpret_cast<const uint4 *>(Ar + plane_stride + k));
        const uint4 p2 = __ldg(reinterpret_cast<const uint4 *>(Ar + 2 * plane_stride + k));
        const uint4 p3 = __ldg(reinterpret_cast<const uint4 *>(Ar + 3 * plane_stride + k));
        uint32_t a[16];
        unpack16(p0, p1, p2, p3, a);
#pragma unroll
        for (int c = 0; c < NCT; ++c) {
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            const uint4 b = *reinterpret_cast<const uint4 *>(qs + c * n0p + k + 4 * w);
            acc[c] += (uint64_t)a[4 * w] * b.x + (uint64_t)a[4 * w + 1] * b.y;
            acc[c] += (uint64_t)a[4 * w + 2] * b.z + (uint64_t)a[4 * w + 3] * b.w;
          }
        }
      }
    } else {
      for (uint32_t k = lane; k < n0; k += 32) {
        const uint64_t a = Ar[k] | (uint32_t)Ar[plane_stride + k] << 8 |
                           (uint32_t)Ar[2 * plane_stride + k] << 16 |
                           (uint32_t)Ar[3 * plane_stride + k] << 24;
#pragma unroll
        for (int c = 0; c < NCT; ++c) acc[c] += a * qs[c * n0p + k];
      }
    }
#pragma unroll
    for (int c = 0; c < NCT; ++c) {
      uint32_t v = reduce64(acc[c], q, mu);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v = add_mod(v, __shfl_xor_sync(0xffffffffu, v, off), q);
      if (lane == c && ct0 + c < (int)ncols) C[(uint64_t)(ct0 + c) * m + r] = v;
    }
  }
}

// ----------------------------------------------------------- scan epilogue
// inter_to_cts_composite (server.cpp:529-597): INTT of every candidate of
// the scan. cmat is [residue x level][column][row]; a block transforms 8
// adjacent rows of one column and one residue, so the 8 words it reads per
// level are one contiguous 32-byte sector.
template <int RES, bool VEC>
__device__ __forceinline__ void scan_epilogue_body(const DevParams &P, const Shape &S,
                                                   const uint32_t *cmat, uint32_t ncols,
                                                   uint32_t *mid, uint64_t mid_stride) {
  extern __shared__ uint32_t sm[];
  const int tid = threadIdx.x;
  const uint32_t r0 = blockIdx.x * 8, c = blockIdx.z;
  const ResidueTables &T = P.r[RES];
  uint32_t v[8][8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t *src = cmat + (((uint64_t)RES * kN + posD(tid, k)) * ncols + c) * S.other + r0;
    if (VEC && r0 + 8 <= S.other) {
      const uint4 lo = __ldg(reinterpret_cast<const uint4 *>(src));
      const uint4 hi = __ldg(reinterpret_cast<const uint4 *>(src + 4));
      v[0][k] = lo.x; v[1][k] = lo.y; v[2][k] = lo.z; v[3][k] = lo.w;
      v[4][k] = hi.x; v[5][k] = hi.y; v[6][k] = hi.z; v[7][k] = hi.w;
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e) v[e][k] = r0 + e < S.other ? __ldg(src + e) : 0u;
    }
  }
  {
    uint2 wd[6];
    iload_d(wd, T.iwt, tid);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      iD<RES>(v[e], wd);
      st_plane<3>(sm + e * kPad, v[e], tid);
    }
  }
  __syncthreads();
  inv_mid_r<RES>(sm, 8, T.iwt);
  uint32_t *dst0 = mid + (uint64_t)(c >> 1) * mid_stride * kCtWords + ((c & 1) * 2 + RES) * kN;
  for (int e = 0; e < 8; ++e) {
    const uint32_t r = r0 + e;
    if (r >= S.other) break;  // uniform over the block
    uint32_t w[8];
    ld_plane<0>(sm + e * kPad, w, tid);
    iA<RES>(w);
    uint32_t *dst = dst0 + (uint64_t)r * kCtWords;
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[posA(tid, k)] = w[k];
  }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads, 2)
k_scan_epilogue(DevParams P, Shape S, const uint32_t *__restrict__ cmat, uint32_t ncols,
                uint32_t *__restrict__ mid, uint64_t mid_stride) {
  if (blockIdx.y == 0)
    scan_epilogue_body<0, VEC>(P, S, cmat, ncols, mid, mid_stride);
  else
    scan_epilogue_body<1, VEC>(P, S, cmat, ncols, mid, mid_stride);
}

// --------------------------------------------------------------- MUX level
// ext_prod_mux (server.cpp:652-722): out = x + INTT(ExtProd(sel, y - x)).
template <int RES, class G>
__device__ __forceinline__ void mux_level_body(const DevParams &P, const Shape &S, uint32_t level,
                                               uint32_t n_pairs, uint32_t offset, uint32_t half,
                                               const uint32_t *in, uint32_t *out,
                                               uint64_t mid_stride, const uint32_t *sel) {
  extern __shared__ uint32_t sm[];
  constexpr uint32_t q = Res<RES>::q;
  const int b = blockIdx.z, tid = threadIdx.x;
  const uint32_t i = blockIdx.x;
  const uint32_t *base_in = in + (uint64_t)b * mid_stride * kCtWords;
  uint32_t *base_out = out + (uint64_t)b * mid_stride * kCtWords;
  if (i >= n_pairs) {  // level 0: carry the unpaired prefix over unchanged
    const uint32_t c = i - n_pairs;
    for (int j = tid; j < kN; j += kThreads) {
      base_out[(uint64_t)c * kCtWords + RES * kN + j] = base_in[(uint64_t)c * kCtWords + RES * kN + j];
      base_out[(uint64_t)c * kCtWords + 2 * kN + RES * kN + j] =
          base_in[(uint64_t)c * kCtWords + 2 * kN + RES * kN + j];
    }
    return;
  }
  uint32_t xi, yi, oi;
  if (level == 0) { xi = offset + 2 * i; yi = xi + 1; oi = offset + i; }
  else { xi = i; yi = i + half; oi = i; }
  const ResidueTables &T = P.r[RES];
  const uint32_t *x = base_in + (uint64_t)xi * kCtWords;
  const uint32_t *y = base_in + (uint64_t)yi * kCtWords;
  const uint32_t *rgsw = sel + ((uint64_t)b * (S.num_dims - 1) + level) * 2 * S.l_ep * kCtWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  gadget_mac<RES, G::lep, G::bep, G::kep>(P, x, y, rgsw, sm, acc0, acc1);
  {
    uint2 wd[6];
    iload_d(wd, T.iwt, tid);
    uint32_t v[8], w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { v[k] = red64_lazy<RES>(acc0[k]); w[k] = red64_lazy<RES>(acc1[k]); }
    iD<RES>(v, wd);
    iD<RES>(w, wd);
    st_plane<3>(sm, v, tid);
    st_plane<3>(sm + kPad, w, tid);
  }
  __syncthreads();
  inv_mid_r<RES>(sm, 2, T.iwt);
  uint32_t *o = base_out + (uint64_t)oi * kCtWords;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    uint32_t v[8];
    ld_plane<0>(sm + p * kPad, v, tid);
    iA<RES>(v);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int j = posA(tid, k);
      o[(p * 2 + RES) * kN + j] = add_mod(x[(p * 2 + RES) * kN + j], v[k], q);
    }
  }
}

template <class G>
__global__ void __launch_bounds__(kThreads, 2)
k_mux_level(DevParams P, Shape S, uint32_t level, uint32_t n_pairs, uint32_t offset,
            uint32_t half, const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
            uint64_t mid_stride, const uint32_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    mux_level_body<0, G>(P, S, level, n_pairs, offset, half, in, out, mid_stride, sel);
  else
    mux_level_body<1, G>(P, S, level, n_pairs, offset, half, in, out, mid_stride, sel);
}

// ------------------------------------------------- MUX level, cluster split
// A MUX level with fewer pairs than the GPU has CTA slots (the upper levels
// of the tree, and most levels of a single query) runs each MUX on a
// cluster of C CTAs instead of one: CTA r takes D = 2 l / C of the 2 l
// gadget rows (C = 2: polynomial r; C = 4: half of polynomial r / 2's
// digits) through their digit NTTs and key products, the partial sums meet
// in distributed shared memory, and CTAs 0 and 1 finish output polynomials
// c0 and c1 (sum, reduction, INTT, + x). Every partial and their total are
// exact 64-bit sums below the single-CTA bound (2 l products < 4q x q each),
// so the result is the same bit for bit.
// gadget_mac restricted to digits [i0, i0 + D) of polynomial p (decomposed
// value y - x, or x when y is null).
template <int RES, int L, int B, int KIND, int D>
__device__ __forceinline__ void gadget_mac_part(const DevParams &P, const uint32_t *x,
                                                const uint32_t *y, const uint32_t *rgsw,
                                                uint32_t *sm, int p, int i0,
                                                uint64_t (&acc0)[8], uint64_t (&acc1)[8]) {
  constexpr uint32_t q = Res<RES>::q;
  constexpr int l = L;
  const ResidueTables &T = P.r[RES];
  const int tid = threadIdx.x;
  uint64_t d[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int j = posA(tid, k);
    uint32_t v1 = x[(p * 2 + 0) * kN + j], v2 = x[(p * 2 + 1) * kN + j];
    if (y != nullptr) {
      v1 = sub_mod(y[(p * 2 + 0) * kN + j], v1, kQ1);
      v2 = sub_mod(y[(p * 2 + 1) * kN + j], v2, kQ2);
    }
    d[k] = digit_source<l, B, KIND>(compose_c(v1, v2));
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = digit_res<q, B, KIND>(d[k], i0 + i);
    fA<RES>(v);
    st_plane<0>(sm + i * kPad, v, tid);
  }
  __syncthreads();
  fwd_mid_r<RES, false>(sm, D, T.fwt);
  uint2 wd[6];
  fload_d(wd, T.fwt, tid);
  for (int i = 0; i < D; ++i) {
    uint32_t v[8];
    ld_plane<3>(sm + i * kPad, v, tid);
    fD<RES>(v, wd);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = mac_in<RES, 2 * L>(v[k]);  // 2 l products over the cluster
    const int row = p * l + (l - 1 - (i0 + i));
    const uint32_t *R0 = rgsw + (uint64_t)row * kCtWords + RES * kN;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j0 = 4 * (tid + 256 * h);
      const uint4 r0 = __ldg(reinterpret_cast<const uint4 *>(R0 + j0));
      const uint4 r1 = __ldg(reinterpret_cast<const uint4 *>(R0 + 2 * kN + j0));
      acc0[4 * h + 0] += (uint64_t)v[4 * h + 0] * r0.x; acc1[4 * h + 0] += (uint64_t)v[4 * h + 0] * r1.x;
      acc0[4 * h + 1] += (uint64_t)v[4 * h + 1] * r0.y; acc1[4 * h + 1] += (uint64_t)v[4 * h + 1] * r1.y;
      acc0[4 * h + 2] += (uint64_t)v[4 * h + 2] * r0.z; acc1[4 * h + 2] += (uint64_t)v[4 * h + 2] * r1.z;
      acc0[4 * h + 3] += (uint64_t)v[4 * h + 3] * r0.w; acc1[4 * h + 3] += (uint64_t)v[4 * h + 3] * r1.w;
    }
  }
  __syncthreads();
}

// Pair i reads x = in[i xs], y = in[i xs + yoff] and writes out[i]: level 0
// without a carried prefix has xs = 2, yoff = 1; level a >= 1 has xs = 1,
// yoff = half.
template <int RES, int C, class G>
__device__ __forceinline__ void mux_split_body(const DevParams &P, const Shape &S, uint32_t level,
                                               uint32_t xs, uint32_t yoff, const uint32_t *in,
                                               uint32_t *out, uint64_t mid_stride,
                                               const uint32_t *sel) {
  static_assert(C == 2 || C == 4, "cluster of 2 or 4 CTAs");
  static_assert((2 * G::lep) % C == 0 && (C == 2 || G::lep % 2 == 0),
                "gadget rows split evenly, within one polynomial per CTA");
  constexpr int D = 2 * G::lep / C;  // gadget rows per CTA
  extern __shared__ uint32_t sm[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  constexpr uint32_t q = Res<RES>::q;
  const int tid = threadIdx.x, b = blockIdx.z;
  const int rank = static_cast<int>(cluster.block_rank());
  const uint32_t i = blockIdx.x / C;
  const uint32_t *base_in = in + (uint64_t)b * mid_stride * kCtWords;
  const uint32_t *x = base_in + (uint64_t)i * xs * kCtWords;
  const uint32_t *y = base_in + ((uint64_t)i * xs + yoff) * kCtWords;
  const uint32_t *rgsw = sel + ((uint64_t)b * (S.num_dims - 1) + level) * 2 * S.l_ep * kCtWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  const int p = C == 2 ? rank : rank >> 1;
  const int i0 = C == 2 ? 0 : (rank & 1) * D;
  gadget_mac_part<RES, G::lep, G::bep, G::kep, D>(P, x, y, rgsw, sm, p, i0, acc0, acc1);
  // partial sums out to shared memory: [output poly][k][tid]
  uint64_t *ex = reinterpret_cast<uint64_t *>(sm);
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
  const ResidueTables &T = P.r[RES];
  {
    uint2 wd[6];
    iload_d(wd, T.iwt, tid);
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = red64_lazy<RES>(tot[k]);
    iD<RES>(v, wd);
    st_plane<3>(sm, v, tid);
  }
  __syncthreads();
  inv_mid_r<RES>(sm, 1, T.iwt);
  uint32_t v[8];
  ld_plane<0>(sm, v, tid);
  iA<RES>(v);
  uint32_t *o = out + (uint64_t)b * mid_stride * kCtWords + (uint64_t)i * kCtWords;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int j = posA(tid, k);
    o[(rank * 2 + RES) * kN + j] = add_mod(x[(rank * 2 + RES) * kN + j], v[k], q);
  }
}

// Selector completion, cluster split: with fewer rows than CTA slots each
// row runs on a pair of CTAs, CTA r decomposing polynomial r of the
// expanded row (l_key digits) against RGSW(s); the two partial sums meet in
// distributed shared memory and CTA r writes polynomial r of the bottom row
// (sum, reduction) and of the top row (the row's own NTT). Exact 64-bit
// partial sums: the same rows bit for bit.
template <int RES, class G>
__device__ __forceinline__ void selectors_split_body(const DevParams &P, const Shape &S,
                                                     const uint32_t *leaves, uint64_t leaf_stride,
                                                     const uint32_t *const *gsw_keys,
                                                     uint32_t *sel) {
  extern __shared__ uint32_t sm[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank());
  const int row_id = blockIdx.x / 2, b = blockIdx.z, tid = threadIdx.x;
  const int selno = row_id / S.l_ep, r = row_id % S.l_ep;
  const ResidueTables &T = P.r[RES];
  const uint32_t *ct = leaves + ((uint64_t)b * leaf_stride + S.n0 + row_id) * kCtWords;
  uint32_t *out = sel + ((uint64_t)b * (S.num_dims - 1) + selno) * 2 * S.l_ep * kCtWords;
  uint64_t acc0[8], acc1[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc0[k] = acc1[k] = 0;
  gadget_mac_part<RES, G::lkey, G::bkey, G::kkey, G::lkey>(P, ct, nullptr, gsw_keys[b], sm, rank,
                                                            0, acc0, acc1);
  uint64_t *ex = reinterpret_cast<uint64_t *>(sm);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    ex[(0 * 8 + k) * kThreads + tid] = acc0[k];
    ex[(1 * 8 + k) * kThreads + tid] = acc1[k];
  }
  cluster.sync();
  uint64_t tot[8];
  {
    const uint64_t *rex = cluster.map_shared_rank(ex, rank ^ 1);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      tot[k] = (rank == 0 ? acc0[k] : acc1[k]) + rex[(rank * 8 + k) * kThreads + tid];
  }
  cluster.sync();  // every remote read is done before shared memory is reused
  // bottom row, polynomial `rank`: ExtProd(RGSW(s), row) (gsw.cpp:119-182)
  uint32_t *bot = out + (uint64_t)(S.l_ep + r) * kCtWords + RES * kN + rank * 2 * kN;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int j0 = 4 * (tid + 256 * h);
    *reinterpret_cast<uint4 *>(bot + j0) =
        make_uint4(red64<RES>(tot[4 * h + 0]), red64<RES>(tot[4 * h + 1]),
                   red64<RES>(tot[4 * h + 2]), red64<RES>(tot[4 * h + 3]));
  }
  // top row, polynomial `rank`: the expanded row in NTT form (gsw.cpp:330-338)
  uint32_t v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = ct[(rank * 2 + RES) * kN + posA(tid, k)];
  fA<RES>(v);
  st_plane<0>(sm, v, tid);
  __syncthreads();
  fwd_mid_r<RES>(sm, 1, T.fwt);
  uint2 wd[6];
  fload_d(wd, T.fwt, tid);
  ld_plane<3>(sm, v, tid);
  fD<RES>(v, wd);
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = canon8<RES>(v[k]);
  uint32_t *top = out + (uint64_t)r * kCtWords + RES * kN + rank * 2 * kN;
#pragma unroll
  for (int h = 0; h < 2; ++h)
    *reinterpret_cast<uint4 *>(top + 4 * (tid + 256 * h)) =
        make_uint4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
}

template <class G>
__global__ void __launch_bounds__(kThreads, 2)
k_selectors_split(DevParams P, Shape S, const uint32_t *__restrict__ leaves, uint64_t leaf_stride,
                  const uint32_t *const *__restrict__ gsw_keys, uint32_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    selectors_split_body<0, G>(P, S, leaves, leaf_stride, gsw_keys, sel);
  else
    selectors_split_body<1, G>(P, S, leaves, leaf_stride, gsw_keys, sel);
}

template <int C, class G>
__global__ void __launch_bounds__(kThreads, 2)
k_mux_level_split(DevParams P, Shape S, uint32_t level, uint32_t xs, uint32_t yoff,
                  const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                  uint64_t mid_stride, const uint32_t *__restrict__ sel) {
  if (blockIdx.y == 0)
    mux_split_body<0, C, G>(P, S, level, xs, yoff, in, out, mid_stride, sel);
  else
    mux_split_body<1, C, G>(P, S, level, xs, yoff, in, out, mid_stride, sel);
}

// ------------------------------------------------ modulus switch + packing
// utils.cpp:445-462: centred round(v * out / inp), inp = q (or q1 after the
// high limb is dropped), out = small_q.
__device__ __forceinline__ uint64_t rescale_dev(uint64_t v, uint64_t inp, uint64_t outm) {
  const int64_t inp_i = static_cast<int64_t>(inp);
  int64_t c = static_cast<int64_t>(v);
  if (c >= inp_i / 2) c -= inp_i;
  const bool neg = c < 0;
  const uint64_t mag = neg ? static_cast<uint64_t>(-c) : static_cast<uint64_t>(c);
  const unsigned __int128 num =
      static_cast<unsigned __int128>(mag) * outm + static_cast<uint64_t>(inp_i / 2);
  const uint64_t quo = static_cast<uint64_t>(num / inp) % outm;
  return neg ? (quo ? outm - quo : 0) : quo;
}

__global__ void __launch_bounds__(kThreads)
k_modswitch(DevParams P, const uint32_t *__restrict__ ct_all, uint64_t ct_stride,
            uint64_t *__restrict__ resp, uint8_t *__restrict__ bytes, uint32_t resp_bytes) {
  __shared__ uint32_t vals[2 * kN];
  const int b = blockIdx.x;
  const uint32_t *ct = ct_all + (uint64_t)b * ct_stride * kCtWords;
  // gridDim.y blocks share a query's coefficients (one block when packing)
  const int per = 2 * kN / gridDim.y;
  for (int idx = blockIdx.y * per + threadIdx.x; idx < (int)(blockIdx.y + 1) * per;
       idx += kThreads) {
    const int p = idx >> kLogN, j = idx & (kN - 1);
    const uint64_t v = crt_compose(ct[(p * 2 + 0) * kN + j], ct[(p * 2 + 1) * kN + j], P);
    uint64_t r;
    if (P.limbs == 2) {
      // two RNS limbs (server.cpp:1044-1075): round the composed value's
      // high limb q2 away (mod q1), then rescale q1 -> small_q
      uint64_t d = (v + (P.q2 >> 1)) / P.q2;
      if (d >= P.q1) d -= P.q1;
      r = rescale_dev(d, P.q1, P.small_q);
    } else {
      r = rescale_dev(v, P.q, P.small_q);
    }
    resp[(uint64_t)b * 2 * kN + idx] = r;
    vals[idx] = static_cast<uint32_t>(r & ((1ull << P.small_q_width) - 1));
  }
  if (bytes == nullptr) return;
  __syncthreads();
  const uint32_t w = P.small_q_width;
  for (uint32_t B = threadIdx.x; B < resp_bytes; B += kThreads) {
    const uint64_t bit0 = 8ull * B;
    const uint32_t i = static_cast<uint32_t>(bit0 / w), o = static_cast<uint32_t>(bit0 % w);
    uint64_t v = vals[i] >> o;
    const uint32_t have = w - o;
    if (have < 8 && i + 1 < 2 * kN) v |= static_cast<uint64_t>(vals[i + 1]) << have;
    bytes[(uint64_t)b * resp_bytes + B] = static_cast<uint8_t>(v & 0xFF);
  }
}

inline unsigned grid1d(uint64_t n) {
  const uint64_t g = (n + kThreads - 1) / kThreads;
  return static_cast<unsigned>(g < 65535ull * 16 ? g : 65535ull * 16);
}

}  // namespace

// ===================================================================== launchers
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }
void note_launches(int64_t delta) {
  g_launches.fetch_add(static_cast<uint64_t>(delta), std::memory_order_relaxed);
}

void upload_ntt_constants(const uint32_t q[2], const uint32_t *const fw[2],
                          const uint32_t *const fw_sh[2], const uint32_t *const iw[2],
                          const uint32_t *const iw_sh[2], const uint32_t nscale[2][4]) {
  if (q[0] != kQ1 || q[1] != kQ2)
    throw std::invalid_argument("the kernels are compiled for the CONFIG_N2048_K1_COMP moduli");
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return;
  uint2 f[2][64], i[2][64];
  uint4 sc[2];
  for (int r = 0; r < 2; ++r) {
    for (int k = 0; k < 64; ++k) {
      f[r][k] = make_uint2(fw[r][k], fw_sh[r][k]);
      i[r][k] = make_uint2(iw[r][k], iw_sh[r][k]);
    }
    sc[r] = make_uint4(nscale[r][0], nscale[r][1], nscale[r][2], nscale[r][3]);
  }
  cudaError_t e = cudaMemcpyToSymbol(c_fwt, f, sizeof(f));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_iwt, i, sizeof(i));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_nscale, sc, sizeof(sc));
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("NTT constants: ") + cudaGetErrorString(e));
  done.insert(dev);
}

void launch_split_u64(const DevParams &P, const uint64_t *in, uint32_t *out, uint64_t n_items,
                      uint64_t per_item, uint64_t out_item_stride, cudaStream_t st) {
  const uint64_t n = n_items * per_item * kN;
  if (n == 0) return;
  k_split_u64<<<grid1d(n), kThreads, 0, st>>>(P, in, out, n, per_item, out_item_stride);
  check_launch("k_split_u64");
}

void launch_compose_u64(const DevParams &P, const uint32_t *in, uint64_t in_item_stride,
                        uint64_t *out, uint64_t n_items, uint64_t per_item, cudaStream_t st) {
  const uint64_t n = n_items * per_item * kN;
  if (n == 0) return;
  k_compose_u64<<<grid1d(n), kThreads, 0, st>>>(P, in, in_item_stride, out, n, per_item);
  check_launch("k_compose_u64");
}

void launch_db_preprocess(const DevParams &P, const Shape &s, const uint16_t *coeffs,
                          uint64_t coeff_pt_begin, uint64_t seed, uint64_t t, uint64_t logical,
                          uint64_t pt_begin, uint64_t pt_end, const uint32_t *row_map,
                          uint8_t *db8, cudaStream_t st) {
  if (pt_end <= pt_begin) return;
  if (pt_end > static_cast<uint64_t>(s.other) * s.n0) throw std::invalid_argument("db tile beyond the layout");
  const size_t smem = kDbTile * kPad * sizeof(uint32_t);
  set_smem(k_db_preprocess, smem);
  const uint64_t tiles = (pt_end - pt_begin + kDbTile - 1) / kDbTile;
  dim3 grid(static_cast<unsigned>(tiles), 2);
  k_db_preprocess<<<grid, kThreads, smem, st>>>(P, coeffs, coeff_pt_begin, seed, t, logical, s.n0,
                                                 s.n0p, s.other, pt_begin, pt_end, row_map, db8);
  check_launch("k_db_preprocess");
}

// The kernels are compiled for the gadget shapes of CONFIG_N2048_K1_COMP
// (s.gadget 0) and CONFIG_N2048_K2_MP (s.gadget 1).
template <class G>
static bool gadgets_match(const Shape &s) {
  return s.l_ep == static_cast<uint32_t>(G::lep) && s.base_ep == static_cast<uint32_t>(G::bep) &&
         s.l_key == static_cast<uint32_t>(G::lkey) && s.base_key == static_cast<uint32_t>(G::bkey) &&
         s.l_ks == static_cast<uint32_t>(G::lks) && s.base_ks == static_cast<uint32_t>(G::bks);
}
static void check_gadgets(const Shape &s) {
  if (s.gadget == 0 ? !gadgets_match<GadgetsK1Comp>(s)
                    : s.gadget != 1 || !gadgets_match<GadgetsK2Mp>(s))
    throw std::invalid_argument(
        "the kernels are compiled for the CONFIG_N2048_K1_COMP and CONFIG_N2048_K2_MP gadgets");
}

template <class G>
static void expand_level_impl(const DevParams &P, const Shape &s, uint32_t d, const uint32_t *in,
                              uint64_t in_stride, uint32_t *out, uint64_t out_stride,
                              const uint32_t *const *bv_keys, uint64_t bv_level_stride,
                              uint32_t batch, cudaStream_t st, uint32_t ntt_nodes) {
  const uint32_t nodes = expand_nodes(s, d);
  const size_t smem = s.l_ks * kPad * sizeof(uint32_t);
  const uint32_t k = 1u << d;
  const uint32_t galois = kN / k + 1;
  uint32_t galois_inv = 1;  // galois^-1 mod 2N (galois is odd)
  while (((galois_inv * galois) & (2 * kN - 1)) != 1) galois_inv += 2;
  if (ntt_nodes > 0) {
    if (d + 1 != s.h || ntt_nodes > nodes || G::lks < 3)  // NTT tail uses planes 0..2
      throw std::invalid_argument("NTT-form children only at the last expansion level");
    set_smem(k_expand_level_ntt<G>, smem);
    k_expand_level_ntt<G><<<dim3(ntt_nodes, 2, batch), kThreads, smem, st>>>(
        P, galois, galois_inv, k, in, in_stride, out, out_stride, bv_keys, d * bv_level_stride);
    check_launch("k_expand_level_ntt");
    if (ntt_nodes < nodes) {
      set_smem(k_expand_level<G>, smem);
      k_expand_level<G><<<dim3(nodes - ntt_nodes, 2, batch), kThreads, smem, st>>>(
          P, galois_inv, k, s.base_ks, s.l_ks, in, in_stride, out, out_stride, bv_keys,
          d * bv_level_stride, ntt_nodes);
      check_launch("k_expand_level");
    }
    return;
  }
  set_smem(k_expand_level<G>, smem);
  // levels with fewer nodes than CTA slots (2 per SM) split each key switch
  // over a cluster of 2, 4 or 8 CTAs (k_expand_level_split)
  const uint64_t ctas = 2ull * nodes * batch, slots = 2ull * sm_count();
  int split = !split_enabled() ? 1
              : 8 * ctas <= slots ? 8 : 4 * ctas <= slots ? 4 : 2 * ctas <= slots ? 2 : 1;
  if (d < 16 && s.split_exp[d]) {  // autotuned width
    split = s.split_exp[d];
    if (split != 1 && split != 2 && split != 4 && split != 8)
      throw std::invalid_argument("expansion cluster width must be 1, 2, 4 or 8");
  }
  if (split == 1) {
    dim3 grid(nodes, 2, batch);
    k_expand_level<G><<<grid, kThreads, smem, st>>>(P, galois_inv, k, s.base_ks, s.l_ks, in,
                                                     in_stride, out, out_stride, bv_keys,
                                                     d * bv_level_stride, 0u);
    check_launch("k_expand_level");
    return;
  }
  // the exchange area ([2][8][256] u64) reuses the digit planes
  const size_t smem_split = std::max<size_t>(G::lks / 2 * kPad * sizeof(uint32_t),
                                             2 * 8 * kThreads * sizeof(uint64_t));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(nodes * split, 2, batch);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem_split;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = split;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const uint64_t koff = d * bv_level_stride;
  cudaError_t e;
  if (split == 8) {
    set_smem(k_expand_level_split<8, G>, smem_split);
    e = cudaLaunchKernelEx(&cfg, k_expand_level_split<8, G>, P, galois_inv, k, in, in_stride, out,
                           out_stride, bv_keys, koff);
  } else if (split == 4) {
    set_smem(k_expand_level_split<4, G>, smem_split);
    e = cudaLaunchKernelEx(&cfg, k_expand_level_split<4, G>, P, galois_inv, k, in, in_stride, out,
                           out_stride, bv_keys, koff);
  } else {
    set_smem(k_expand_level_split<2, G>, smem_split);
    e = cudaLaunchKernelEx(&cfg, k_expand_level_split<2, G>, P, galois_inv, k, in, in_stride, out,
                           out_stride, bv_keys, koff);
  }
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("k_expand_level_split: ") + cudaGetErrorString(e));
  check_launch("k_expand_level_split");
}

void launch_expand_level(const DevParams &P, const Shape &s, uint32_t d, const uint32_t *in,
                         uint64_t in_stride, uint32_t *out, uint64_t out_stride,
                         const uint32_t *const *bv_keys, uint64_t bv_level_stride,
                         uint32_t batch, cudaStream_t st, uint32_t ntt_nodes) {
  check_gadgets(s);
  if (s.gadget == 1)
    expand_level_impl<GadgetsK2Mp>(P, s, d, in, in_stride, out, out_stride, bv_keys,
                                   bv_level_stride, batch, st, ntt_nodes);
  else
    expand_level_impl<GadgetsK1Comp>(P, s, d, in, in_stride, out, out_stride, bv_keys,
                                     bv_level_stride, batch, st, ntt_nodes);
}

template <class G>
static void selectors_impl(const DevParams &P, const Shape &s, const uint32_t *leaves,
                           uint64_t leaf_stride, const uint32_t *const *gsw_keys, uint32_t *sel,
                           uint32_t batch, cudaStream_t st) {
  const size_t smem = s.l_key * kPad * sizeof(uint32_t);
  const uint32_t rows = (s.num_dims - 1) * s.l_ep;
  // fewer rows than CTA slots (2 per SM): one pair of CTAs per row
  if (split_enabled() && 2ull * 2 * rows * batch <= 2ull * sm_count()) {
    const size_t smem_split = std::max<size_t>(smem, 2 * 8 * kThreads * sizeof(uint64_t));
    set_smem(k_selectors_split<G>, smem_split);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(rows * 2, 2, batch);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem_split;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e =
        cudaLaunchKernelEx(&cfg, k_selectors_split<G>, P, s, leaves, leaf_stride, gsw_keys, sel);
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("k_selectors_split: ") + cudaGetErrorString(e));
    check_launch("k_selectors_split");
    return;
  }
  set_smem(k_selectors<G>, smem);
  dim3 grid(rows, 2, batch);
  k_selectors<G><<<grid, kThreads, smem, st>>>(P, s, leaves, leaf_stride, gsw_keys, sel);
  check_launch("k_selectors");
}

void launch_selectors(const DevParams &P, const Shape &s, const uint32_t *leaves,
                      uint64_t leaf_stride, const uint32_t *const *gsw_keys, uint32_t *sel,
                      uint32_t batch, cudaStream_t st) {
  check_gadgets(s);
  if (s.num_dims <= 1) return;
  if (s.gadget == 1)
    selectors_impl<GadgetsK2Mp>(P, s, leaves, leaf_stride, gsw_keys, sel, batch, st);
  else
    selectors_impl<GadgetsK1Comp>(P, s, leaves, leaf_stride, gsw_keys, sel, batch, st);
}

void launch_fst_prep(const DevParams &P, const Shape &s, const uint32_t *leaves,
                     uint64_t leaf_stride, uint32_t *ntt, uint64_t ntt_stride, uint8_t *qb,
                     uint32_t batch, cudaStream_t st) {
  const size_t smem = 2 * kFstTile * kPad * sizeof(uint32_t);
  set_smem(k_fst_ntt, smem);
  dim3 grid((s.n0 + kFstTile - 1) / kFstTile, 2, batch);
  k_fst_ntt<<<grid, kThreads, smem, st>>>(P, s, leaves, leaf_stride, ntt, ntt_stride);
  check_launch("k_fst_ntt");
  launch_fst_pack(s, ntt, ntt_stride, qb, batch, st);
}

void launch_fst_pack(const Shape &s, const uint32_t *ntt, uint64_t ntt_stride, uint8_t *qb,
                     uint32_t batch, cudaStream_t st) {
  dim3 pgrid((s.n0p + kPackK - 1) / kPackK, 2 * kN / kPackZ, 2 * batch);
  k_fst_pack<<<pgrid, kThreads, 0, st>>>(ntt, ntt_stride, s.n0, s.n0p, qb, 2 * batch);
  check_launch("k_fst_pack");
}

template <int NCT>
static void scan_dispatch(const DevParams &P, const Shape &s, const uint8_t *db8, const uint8_t *qb,
                          uint32_t *cmat, uint32_t ncols, cudaStream_t st) {
  const size_t smem = (size_t)NCT * s.n0p * sizeof(uint32_t);
  dim3 grid((ncols + NCT - 1) / NCT, 2 * kN);
  if (s.n0 % 16 == 0) {
    set_smem(k_scan<NCT, true>, smem);
    k_scan<NCT, true><<<grid, kThreads, smem, st>>>(P, s.n0, s.n0p, s.other, db8, qb, ncols, cmat);
  } else {
    set_smem(k_scan<NCT, false>, smem);
    k_scan<NCT, false><<<grid, kThreads, smem, st>>>(P, s.n0, s.n0p, s.other, db8, qb, ncols, cmat);
  }
  check_launch("k_scan");
}

void launch_scan(const DevParams &P, const Shape &s, const uint8_t *db8, const uint8_t *qb,
                 uint32_t *cmat, uint32_t batch, cudaStream_t st) {
  const uint32_t ncols = 2 * batch;
  if (ncols <= 2) scan_dispatch<2>(P, s, db8, qb, cmat, ncols, st);
  else if (ncols <= 4) scan_dispatch<4>(P, s, db8, qb, cmat, ncols, st);
  else if (ncols <= 8) scan_dispatch<8>(P, s, db8, qb, cmat, ncols, st);
  else scan_dispatch<16>(P, s, db8, qb, cmat, ncols, st);
}

void launch_scan_epilogue(const DevParams &P, const Shape &s, const uint32_t *cmat, uint32_t *mid,
                          uint64_t mid_stride, uint32_t batch, cudaStream_t st) {
  const size_t smem = 8 * kPad * sizeof(uint32_t);
  const uint32_t ncols = 2 * batch;
  dim3 grid((s.other + 7) / 8, 2, ncols);
  if (s.other % 4 == 0) {
    set_smem(k_scan_epilogue<true>, smem);
    k_scan_epilogue<true><<<grid, kThreads, smem, st>>>(P, s, cmat, ncols, mid, mid_stride);
  } else {
    set_smem(k_scan_epilogue<false>, smem);
    k_scan_epilogue<false><<<grid, kThreads, smem, st>>>(P, s, cmat, ncols, mid, mid_stride);
  }
  check_launch("k_scan_epilogue");
}

template <class G>
static void mux_level_impl(const DevParams &P, const Shape &s, uint32_t level, uint32_t tree_h,
                           const uint32_t *in, uint32_t *out, uint64_t mid_stride,
                           const uint32_t *sel, uint32_t batch, cudaStream_t st) {
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
  const size_t smem = s.l_ep * kPad * sizeof(uint32_t);
  // levels with fewer MUX steps than CTA slots (2 per SM) split each step
  // over a cluster of 2 or 4 CTAs (k_mux_level_split); 4 only when each
  // polynomial's digits halve evenly
  constexpr bool four = G::lep % 2 == 0;
  const uint64_t ctas = 2ull * n_pairs * batch, slots = 2ull * sm_count();
  int split = (copies != 0 || !split_enabled()) ? 1
              : (four && 4 * ctas <= slots) ? 4 : 2 * ctas <= slots ? 2 : 1;
  if (level < 32 && s.split_mux[level] && copies == 0) {  // autotuned width
    split = s.split_mux[level];
    if (split != 1 && split != 2 && (split != 4 || !four))
      throw std::invalid_argument("MUX cluster width must be 1, 2 or (even digit counts) 4");
  }
  if (split == 1) {
    set_smem(k_mux_level<G>, smem);
    dim3 grid(n_pairs + copies, 2, batch);
    k_mux_level<G><<<grid, kThreads, smem, st>>>(P, s, level, n_pairs, offset, half, in, out,
                                                  mid_stride, sel);
    check_launch("k_mux_level");
    return;
  }
  // the exchange area ([2][8][256] u64) reuses the digit planes
  const size_t smem_split = std::max<size_t>(smem, 2 * 8 * kThreads * sizeof(uint64_t));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(n_pairs * split, 2, batch);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem_split;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = split;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // offset == copies == 0 here, so level 0 pairs (2i, 2i + 1) into i
  const uint32_t xs = level == 0 ? 2 : 1, yoff = level == 0 ? 1 : half;
  cudaError_t e = cudaSuccess;
  if constexpr (four) {
    if (split == 4) {
      set_smem(k_mux_level_split<4, G>, smem_split);
      e = cudaLaunchKernelEx(&cfg, k_mux_level_split<4, G>, P, s, level, xs, yoff, in, out,
                             mid_stride, sel);
    }
  }
  if (split == 2) {
    set_smem(k_mux_level_split<2, G>, smem_split);
    e = cudaLaunchKernelEx(&cfg, k_mux_level_split<2, G>, P, s, level, xs, yoff, in, out,
                           mid_stride, sel);
  }
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("k_mux_level_split: ") + cudaGetErrorString(e));
  check_launch("k_mux_level_split");
}

void launch_mux_level(const DevParams &P, const Shape &s, uint32_t level, uint32_t tree_h,
                      const uint32_t *in, uint32_t *out, uint64_t mid_stride, const uint32_t *sel,
                      uint32_t batch, cudaStream_t st) {
  check_gadgets(s);
  if (s.gadget == 1)
    mux_level_impl<GadgetsK2Mp>(P, s, level, tree_h, in, out, mid_stride, sel, batch, st);
  else
    mux_level_impl<GadgetsK1Comp>(P, s, level, tree_h, in, out, mid_stride, sel, batch, st);
}

void launch_modswitch(const DevParams &P, const uint32_t *ct, uint64_t ct_stride, uint64_t *resp,
                      uint8_t *bytes, uint32_t resp_bytes, uint32_t batch, cudaStream_t st) {
  // without packing, 8 blocks per query share the rescale (a 128-bit
  // division per coefficient); packing needs every value in one block
  k_modswitch<<<dim3(batch, bytes ? 1 : 8), kThreads, 0, st>>>(P, ct, ct_stride, resp, bytes,
                                                                resp_bytes);
  check_launch("k_modswitch");
}

// ------------------------------------------------- butterfly-rate probe
// The forward radix-8 pass of the NTT kernels (fpass8, the first residue's
// modulus) on register-resident values and twiddles, three passes per
// iteration with the kernels' correction pattern (stages 4, 6, 8 of 9
// corrected): the rate at which an SM retires NTT butterflies when nothing
// else (shared-memory exchanges, loads, digit work, MACs) is in the way.
// The values are not meaningful; `sink` keeps the work alive.
__global__ void __launch_bounds__(256)
k_bfly_rate(uint32_t *__restrict__ sink, uint32_t iters, uint2 w0) {
  uint32_t v[8];
  uint2 w[7];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = (threadIdx.x * 8 + k + blockIdx.x) % kQ1;
#pragma unroll
  for (int k = 0; k < 7; ++k) w[k] = make_uint2(w0.x + 2 * k, w0.y + k);
  for (uint32_t it = 0; it < iters; ++it) {
    fpass8<kQ1, false, false, false>(v, w);
    fpass8<kQ1, true, false, true>(v, w);
    fpass8<kQ1, false, true, false>(v, w);
  }
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) acc ^= v[k];
  sink[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

uint32_t bfly_rate_blocks(int sms) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bfly_rate, 256, 0) != cudaSuccess || occ < 1)
    occ = 1;
  return static_cast<uint32_t>(sms) * static_cast<uint32_t>(occ);
}

uint64_t launch_bfly_rate(uint32_t *sink, uint32_t blocks, uint32_t iters, cudaStream_t st) {
  const uint32_t w = 123456789u % kQ1;
  const uint2 w0 = make_uint2(w, static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / kQ1));
  k_bfly_rate<<<blocks, 256, 0, st>>>(sink, iters, w0);
  check_launch("k_bfly_rate");
  return static_cast<uint64_t>(blocks) * 256 * iters * 36;
}

}  // namespace opir
