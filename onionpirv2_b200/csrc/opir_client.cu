// Client-side batch operations: query packing (PirClient::fast_generate_query,
// src/client.cpp:107-225) and response decryption (PirClient::decrypt_mod_q,
// src/client.cpp:364-410) for many queries or responses of one client.
//
// Both are dominated by one negacyclic product x * s with the client's ternary
// secret s. The reference multiplies in the NTT domain mod the target modulus;
// here s is held as two index lists, P (coefficients equal to 1) and M (equal
// to -1), and the product is the exact integer sum
//     (x*s)_i = sum_{j in P} xe[N+i-j] - sum_{j in M} xe[N+i-j]
// over the sign-extended copy xe[N+m] = x[m], xe[m] = -x[m] (m < N) staged in
// shared memory; only the epilogue reduces, so the result equals the NTT
// product mod the same modulus exactly. x is split into 31-bit parts so each
// shared word is an int32 and each partial sum fits an int64 (N 2^31 < 2^43).
// Cost: |P|+|M| (about 2N/3) shared loads per output coefficient and part --
// shared-memory bandwidth bound, one CTA per (item, output slice).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/onionpir_b200.h"
#include "opir_host.h"
#include "opir_kernels.h"
#include "opir_params.h"

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

// xe for one polynomial, PARTS 31-bit parts, part p at ext + p 2n.
template <int PARTS>
__device__ __forceinline__ void stage_ext(const uint64_t *__restrict__ x, uint64_t mod, uint32_t n,
                                          int32_t *ext) {
  for (uint32_t m = threadIdx.x; m < n; m += blockDim.x) {
    const uint64_t v = x[m] % mod;
    const int32_t lo = static_cast<int32_t>(v & 0x7FFFFFFFull);
    ext[n + m] = lo;
    ext[m] = -lo;
    if (PARTS == 2) {
      const int32_t hi = static_cast<int32_t>(v >> 31);
      ext[3 * n + m] = hi;
      ext[2 * n + m] = -hi;
    }
  }
}

// acc[p][r] = part p of (x*s)_i for i = i0 + kBlock r.
template <int PARTS, int R>
__device__ __forceinline__ void ternary_product(const int32_t *ext, const uint16_t *sl,
                                                uint32_t npos, uint32_t nneg, uint32_t n,
                                                uint32_t i0, int64_t (&acc)[PARTS][R]) {
#pragma unroll
  for (int p = 0; p < PARTS; ++p)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[p][r] = 0;
  const int32_t *e0 = ext + n + i0;
  const int32_t *e1 = ext + 3 * n + i0;
#pragma unroll 4
  for (uint32_t u = 0; u < npos; ++u) {
    const int j = sl[u];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      acc[0][r] += e0[kBlock * r - j];
      if (PARTS == 2) acc[PARTS - 1][r] += e1[kBlock * r - j];
    }
  }
#pragma unroll 4
  for (uint32_t u = npos; u < npos + nneg; ++u) {
    const int j = sl[u];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      acc[0][r] -= e0[kBlock * r - j];
      if (PARTS == 2) acc[PARTS - 1][r] -= e1[kBlock * r - j];
    }
  }
}

template <int PARTS, int R>
__device__ __forceinline__ uint64_t reduce_part_sums(const int64_t (&acc)[PARTS][R], int r,
                                                     uint64_t mod) {
  if (PARTS == 1) {
    int64_t v = acc[0][r] % static_cast<int64_t>(mod);
    return static_cast<uint64_t>(v < 0 ? v + static_cast<int64_t>(mod) : v);
  }
  const __int128 v = (static_cast<__int128>(acc[PARTS - 1][r]) << 31) + acc[0][r];
  __int128 m = v % static_cast<__int128>(mod);
  if (m < 0) m += mod;
  return static_cast<uint64_t>(m);
}

__device__ __forceinline__ uint64_t round_div(unsigned __int128 a, uint64_t b) {
  return static_cast<uint64_t>((a + (b >> 1)) / b);
}

// decrypt_mod_q: pt = round((c0 + c1 s mod sq) t / sq) mod t per coefficient;
// max_noise (may be null, zeroed by the host) receives max |phase - round(sq m
// / t)| over the response, the figure the reference reports as its noise
// budget (client.cpp:389-407).
template <int PARTS, int R>
__global__ void __launch_bounds__(kBlock) k_client_decrypt(
    const uint64_t *__restrict__ resp, const uint16_t *__restrict__ sidx, uint32_t npos,
    uint32_t nneg, uint32_t n, uint64_t sq, uint64_t t, uint64_t *__restrict__ pt,
    unsigned long long *__restrict__ max_noise) {
  extern __shared__ __align__(16) int32_t smem[];
  int32_t *ext = smem;
  uint16_t *sl = reinterpret_cast<uint16_t *>(smem + PARTS * 2 * n);
  const uint64_t b = blockIdx.x;
  const uint64_t *c0 = resp + b * 2 * n, *c1 = c0 + n;
  stage_ext<PARTS>(c1, sq, n, ext);
  for (uint32_t u = threadIdx.x; u < npos + nneg; u += blockDim.x) sl[u] = sidx[u];
  __syncthreads();
  const uint32_t i0 = blockIdx.y * (n / gridDim.y) + threadIdx.x;
  int64_t acc[PARTS][R];
  ternary_product<PARTS, R>(ext, sl, npos, nneg, n, i0, acc);
  uint64_t worst = 0;
  const uint64_t half = sq >> 1;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t i = i0 + kBlock * r;
    uint64_t phase = reduce_part_sums<PARTS, R>(acc, r, sq) + c0[i] % sq;
    if (phase >= sq) phase -= sq;
    const uint64_t m = round_div(static_cast<unsigned __int128>(phase) * t, sq) % t;
    pt[b * n + i] = m;
    const uint64_t approx = round_div(static_cast<unsigned __int128>(sq) * m, t) % sq;
    const uint64_t npos_ = phase >= approx ? phase - approx : sq - approx + phase;
    const uint64_t nabs = npos_ > half ? sq - npos_ : npos_;
    worst = nabs > worst ? nabs : worst;
  }
  if (max_noise) {
    for (int o = 16; o > 0; o >>= 1) {
      const uint64_t w = __shfl_xor_sync(0xFFFFFFFFu, worst, o);
      worst = w > worst ? w : worst;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(max_noise + b, static_cast<unsigned long long>(worst));
  }
}

// fast_generate_query for item = (query, limb): c0 = -(a s + e) mod q_k plus
// the query's plaintext constants, c1 = a as given. a and the output are
// limb-major per query: a [K n], out [c0 (K n)][c1 (K n)].
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
  stage_ext<2>(x, q, n, ext);
  for (uint32_t u = threadIdx.x; u < npos + nneg; u += blockDim.x) sl[u] = sidx[u];
  __syncthreads();
  const uint32_t span = n / gridDim.y, o0 = blockIdx.y * span;
  const uint32_t i0 = o0 + threadIdx.x;
  int64_t acc[2][R];
  ternary_product<2, R>(ext, sl, npos, nneg, n, i0, acc);
  uint64_t *c0 = out + query * 2 * kn + static_cast<uint64_t>(limb) * n;
  uint64_t *c1 = c0 + kn;
  const int64_t *eq = e + query * n;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const uint32_t i = i0 + kBlock * r;
    const int64_t ei = eq[i];
    const uint64_t em = ei >= 0 ? static_cast<uint64_t>(ei) % q
                                : (q - static_cast<uint64_t>(-(ei + 1)) % q - 1);
    uint64_t v = reduce_part_sums<2, R>(acc, r, q) + em;
    if (v >= q) v -= q;
    c0[i] = v ? q - v : 0;
    c1[i] = x[i];
  }
  __syncthreads();
  const ConstEntry *ce = consts + query * nconst;
  for (uint32_t u = threadIdx.x; u < nconst; u += blockDim.x) {
    const uint32_t pos = ce[u].pos;
    if (pos == kNoPos || pos < o0 || pos >= o0 + span) continue;
    const uint64_t v = c0[pos] + ce[u].val[limb];
    c0[pos] = v >= q ? v - q : v;
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
  if (!c4 && !(p.num_limbs == 1 && p.poly_degree == 2048))
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

// Output slices per item so that a batch fills the GPU; R = n / (s kBlock)
// outputs per thread, at most kMaxR (registers: 2 kMaxR int64 accumulators,
// so that two or more CTAs stay resident per SM).
constexpr uint32_t kMaxR = 8;
uint32_t slices_for(uint64_t items, uint32_t n, int sms) {
  uint32_t s = 1;
  while (n / (s * kBlock) > kMaxR) s *= 2;
  while (items * s < 2ull * sms && s * 2 * kBlock <= n) s *= 2;
  return s;
}

template <int PARTS>
void launch_decrypt(uint32_t R, dim3 grid, size_t smem, cudaStream_t st, const uint64_t *resp,
                    const opir_client &c, uint64_t *pt, unsigned long long *noise) {
  const uint16_t *s = c.sidx.p;
  const uint32_t n = c.n;
  const uint64_t sq = c.params.small_q, t = c.params.plain_mod;
  switch (R) {
#define OPIR_DEC(RR)                                                                          \
  case RR:                                                                                    \
    ck(cudaFuncSetAttribute(k_client_decrypt<PARTS, RR>,                                      \
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),          \
       "client decrypt smem");                                                                \
    k_client_decrypt<PARTS, RR><<<grid, kBlock, smem, st>>>(resp, s, c.npos, c.nneg, n, sq, t, \
                                                            pt, noise);                       \
    break;
    OPIR_DEC(1) OPIR_DEC(2) OPIR_DEC(4) OPIR_DEC(8)
#undef OPIR_DEC
    default:
      throw std::runtime_error("client decrypt: unsupported slice width");
  }
  ck(cudaGetLastError(), "client decrypt launch");
  opir::note_launches(1);
}

void launch_pack(uint32_t R, dim3 grid, size_t smem, cudaStream_t st, const uint64_t *a,
                 const int64_t *e, const opir_client &c, uint64_t *out) {
  const uint16_t *s = c.sidx.p;
  switch (R) {
#define OPIR_PACK(RR)                                                                          \
  case RR:                                                                                     \
    ck(cudaFuncSetAttribute(k_client_pack<RR>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                            (int)smem),                                                        \
       "client pack smem");                                                                    \
    k_client_pack<RR><<<grid, kBlock, smem, st>>>(a, e, c.consts.p, c.nconst, s, c.npos,       \
                                                  c.nneg, c.n, c.limbs, c.mods[0], c.mods[1],  \
                                                  out);                                        \
    break;
    OPIR_PACK(1) OPIR_PACK(2) OPIR_PACK(4) OPIR_PACK(8)
#undef OPIR_PACK
    default:
      throw std::runtime_error("client pack: unsupported slice width");
  }
  ck(cudaGetLastError(), "client pack launch");
  opir::note_launches(1);
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
  });
  if (st != OPIR_OK) {
    delete c;
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
    c->consts.reset();
    if (c->staging) cudaFreeHost(c->staging);
    if (c->staged) cudaEventDestroy(c->staged);
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
    const size_t count = static_cast<size_t>(n) * c->nconst;
    DeviceGuard g(c->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
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
    const uint64_t items = static_cast<uint64_t>(n) * c->limbs;
    const uint32_t s = slices_for(items, c->n, c->sms);
    const size_t smem = 2 * 2 * c->n * sizeof(int32_t) + (c->npos + c->nneg + 8) * sizeof(uint16_t);
    launch_pack(c->n / (s * kBlock), dim3(static_cast<uint32_t>(items), s), smem, st, d_a, d_e, *c,
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
    const uint32_t s = slices_for(n, c->n, c->sms);
    const uint32_t R = c->n / (s * kBlock);
    const dim3 grid(n, s);
    auto *noise = reinterpret_cast<unsigned long long *>(d_max_noise);
    const size_t lists = (c->npos + c->nneg + 8) * sizeof(uint16_t);
    if (c->params.small_q < (1ull << 31))
      launch_decrypt<1>(R, grid, 2 * c->n * sizeof(int32_t) + lists, st, d_responses, *c,
                        d_plaintexts, noise);
    else
      launch_decrypt<2>(R, grid, 4 * c->n * sizeof(int32_t) + lists, st, d_responses, *c,
                        d_plaintexts, noise);
  });
}

}  // extern "C"
