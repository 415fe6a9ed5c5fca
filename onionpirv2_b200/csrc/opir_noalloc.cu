// Allocation-free entry point: opir_ext_prod_mux_noalloc. Each of its MUX
// steps computes what PirServer::ext_prod_mux (src/server.cpp:652-722)
// computes, x + INTT(ExtProd(sel, y - x)).
//
// Why it exists: some callers cannot call cudaMalloc at the point where they
// need a MUX step -- for example code running inside a host that owns and
// pre-budgets all device memory, or a request loop that must not touch the
// device allocator (an allocation can synchronise the device and stall every
// stream). This entry point takes only caller-provided inputs and outputs and
// keeps its working memory in one fixed array compiled into the library.
//
// The array g_mux_scratch is a file-scope __device__ array: every GPU that
// loads this library holds kScratchWords * 4 bytes (about 3.9 MiB) of it
// until the process exits. In host code its name is only a host-side stand-in
// for the symbol, never a device address, so the host obtains the real device
// address once per device with cudaGetSymbolAddress and passes that pointer
// to the kernels.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/onionpir_b200.h"
#include "opir_device.cuh"
#include "opir_params.h"

namespace {

using opir::kCtWords;
using opir::kN;
using opir::kPer;
using opir::kThreads;

constexpr int kMaxMux = OPIR_NOALLOC_MAX_MUX;  // MUX operations per call
constexpr int kSelRows = 12;                   // 2 L_EP gadget rows
constexpr uint64_t kTableWords = 8ull * kN;    // fw, fw_sh, iw, iw_sh x 2 residues
// per MUX: x, y, out residue pairs + selector rows in residue form
constexpr uint64_t kPerMuxWords = 3ull * kCtWords + kSelRows * (uint64_t)kCtWords;
constexpr uint64_t kScratchWords = kTableWords + kMaxMux * kPerMuxWords;

static __device__ __align__(256) uint32_t g_mux_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
uint32_t *g_scratch_ptr[kMaxDevices] = {nullptr};
opir::DevParams g_dev_params[kMaxDevices];

// u64 (mod q) polys -> residue pairs, item stride in u32 words.
__global__ void k_noalloc_split(opir::DevParams P, const uint64_t *__restrict__ in,
                                uint64_t polys_per_item, uint32_t *__restrict__ out,
                                uint64_t out_stride, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / kN, j = i % kN;
    const uint64_t item = p / polys_per_item, pp = p % polys_per_item;
    uint32_t *o = out + item * out_stride + pp * 2 * kN + j;
    const uint64_t v = in[i];
    o[0] = opir::reduce64(v, P.q1, P.r[0].mu);
    o[kN] = opir::reduce64(v, P.q2, P.r[1].mu);
  }
}

// out = x + INTT(ExtProd(sel, y - x)), one block per (MUX, residue); the same
// arithmetic as the MUX level of make_query (src/server.cpp:652-722).
__global__ void __launch_bounds__(kThreads)
k_noalloc_mux(opir::DevParams P, uint32_t *__restrict__ scratch, int l, int base_log2) {
  extern __shared__ uint32_t D[];
  const int m = blockIdx.x, res = blockIdx.y;
  const opir::ResidueTables T = res ? P.r[1] : P.r[0];
  const uint32_t q = T.q;
  uint32_t *item = scratch + kTableWords + (uint64_t)m * kPerMuxWords;
  const uint32_t *x = item, *y = item + kCtWords, *sel = item + 3 * kCtWords;
  uint32_t *out = item + 2 * kCtWords;
  uint64_t acc0[kPer], acc1[kPer];
#pragma unroll
  for (int s = 0; s < kPer; ++s) acc0[s] = acc1[s] = 0;
  for (int p = 0; p < 2; ++p) {
#pragma unroll
    for (int s = 0; s < kPer; ++s) {
      const int j = threadIdx.x + s * kThreads;
      const uint32_t v1 = opir::sub_mod(y[(p * 2 + 0) * kN + j], x[(p * 2 + 0) * kN + j], P.q1);
      const uint32_t v2 = opir::sub_mod(y[(p * 2 + 1) * kN + j], x[(p * 2 + 1) * kN + j], P.q2);
      int64_t d = opir::centre(opir::crt_compose(v1, v2, P), P);
      for (int i = 0; i < l; ++i)
        D[i * kN + j] = opir::digit_residue(opir::next_digit(d, base_log2), q);
    }
    __syncthreads();
    opir::ntt_fwd_planes(D, l, T);
#pragma unroll
    for (int s = 0; s < kPer; ++s) {
      const int j = threadIdx.x + s * kThreads;
      for (int i = 0; i < l; ++i) {
        const int row = p * l + (l - 1 - i);
        const uint64_t dv = D[i * kN + j];
        const uint32_t *R = sel + (uint64_t)row * kCtWords + res * kN + j;
        acc0[s] += dv * R[0];
        acc1[s] += dv * R[2 * kN];
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int s = 0; s < kPer; ++s) {
    const int j = threadIdx.x + s * kThreads;
    D[j] = opir::reduce64(acc0[s], q, T.mu);
    D[kN + j] = opir::reduce64(acc1[s], q, T.mu);
  }
  __syncthreads();
  opir::ntt_inv_planes(D, 2, T);
#pragma unroll
  for (int s = 0; s < kPer; ++s) {
    const int j = threadIdx.x + s * kThreads;
    out[res * kN + j] = opir::add_mod(x[res * kN + j], D[j], q);
    out[2 * kN + res * kN + j] = opir::add_mod(x[2 * kN + res * kN + j], D[kN + j], q);
  }
}

__global__ void k_noalloc_compose(opir::DevParams P, const uint32_t *__restrict__ scratch,
                                  uint64_t *__restrict__ out, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t m = i / (2 * kN), r = i % (2 * kN), p = r / kN, j = r % kN;
    const uint32_t *o = scratch + kTableWords + m * kPerMuxWords + 2 * kCtWords + p * 2 * kN + j;
    out[i] = opir::crt_compose(o[0], o[kN], P);
  }
}

// Once per device, with that device current: fetch the device address of
// g_mux_scratch and write the NTT tables into its head. Uses only a
// synchronous cudaMemcpy into the array (no device allocation).
opir_status setup_device(int dev, const opir_params &p) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (g_scratch_ptr[dev] != nullptr) return OPIR_OK;
  uint32_t *ptr = nullptr;
  if (cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_mux_scratch) != cudaSuccess) {
    cudaGetLastError();
    return OPIR_ERR_CUDA;
  }
  const opir::LimbTables t1 = opir::make_limb_tables(kN, (uint32_t)p.q1, (uint32_t)p.w1);
  const opir::LimbTables t2 = opir::make_limb_tables(kN, (uint32_t)p.q2, (uint32_t)p.w2);
  const opir::LimbTables *ts[2] = {&t1, &t2};
  opir::DevParams d{};
  for (int r = 0; r < 2; ++r) {
    const std::vector<uint32_t> *parts[4] = {&ts[r]->fw, &ts[r]->fw_sh, &ts[r]->iw, &ts[r]->iw_sh};
    for (int k = 0; k < 4; ++k) {
      uint32_t *dst = ptr + (r * 4 + k) * kN;
      if (cudaMemcpy(dst, parts[k]->data(), kN * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
        cudaGetLastError();
        return OPIR_ERR_CUDA;
      }
    }
    d.r[r].fw = ptr + (r * 4 + 0) * kN;
    d.r[r].fw_sh = ptr + (r * 4 + 1) * kN;
    d.r[r].iw = ptr + (r * 4 + 2) * kN;
    d.r[r].iw_sh = ptr + (r * 4 + 3) * kN;
    d.r[r].q = ts[r]->q;
    d.r[r].n_inv = ts[r]->n_inv;
    d.r[r].n_inv_sh = ts[r]->n_inv_sh;
    d.r[r].mu = ts[r]->mu;
  }
  d.q = p.q;
  d.half_q = p.q >> 1;
  d.q1 = (uint32_t)p.q1;
  d.q2 = (uint32_t)p.q2;
  d.q1_inv = (uint32_t)p.q1_inv_mod_q2;
  d.q1_inv_sh = (uint32_t)(((uint64_t)d.q1_inv << 32) / d.q2);
  d.small_q = p.small_q;
  d.small_q_width = p.small_q_width;
  g_dev_params[dev] = d;
  g_scratch_ptr[dev] = ptr;
  return OPIR_OK;
}

}  // namespace

extern "C" opir_status opir_ext_prod_mux_noalloc(const opir_params *params, uint32_t n,
                                                 const uint64_t *d_x, const uint64_t *d_y,
                                                 const uint64_t *d_selectors, uint64_t *d_out,
                                                 void *stream) {
  if (!params || !d_x || !d_y || !d_selectors || !d_out) return OPIR_ERR_INVALID_ARGUMENT;
  if (n == 0) return OPIR_OK;
  if (n > static_cast<uint32_t>(kMaxMux)) return OPIR_ERR_INVALID_ARGUMENT;  // beyond the fixed scratch
  if (params->poly_degree != static_cast<uint32_t>(kN) || params->num_limbs != 1 ||
      2 * params->l_ep != static_cast<uint32_t>(kSelRows) || params->base_log2 == 0 ||
      params->base_log2 > 32)
    return OPIR_ERR_INVALID_ARGUMENT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return OPIR_ERR_CUDA;
  }
  const opir_status st = setup_device(dev, *params);
  if (st != OPIR_OK) return st;
  if (g_dev_params[dev].q != params->q) return OPIR_ERR_INVALID_ARGUMENT;  // one parameter set
  uint32_t *scratch = g_scratch_ptr[dev];
  const opir::DevParams &P = g_dev_params[dev];
  cudaStream_t st_ = static_cast<cudaStream_t>(stream);
  const uint64_t ct_coeffs = 2ull * kN;
  const unsigned blocks = static_cast<unsigned>((n * ct_coeffs + kThreads - 1) / kThreads);
  // every scratch word the MUX kernel reads is written by these splits first,
  // so nothing depends on what an earlier call left in the array
  k_noalloc_split<<<blocks, kThreads, 0, st_>>>(P, d_x, 2, scratch + kTableWords, kPerMuxWords,
                                                n * ct_coeffs);
  k_noalloc_split<<<blocks, kThreads, 0, st_>>>(P, d_y, 2, scratch + kTableWords + kCtWords,
                                                kPerMuxWords, n * ct_coeffs);
  const unsigned sel_blocks =
      static_cast<unsigned>((n * kSelRows * ct_coeffs + kThreads - 1) / kThreads);
  k_noalloc_split<<<sel_blocks, kThreads, 0, st_>>>(P, d_selectors, 2 * kSelRows,
                                                    scratch + kTableWords + 3 * kCtWords,
                                                    kPerMuxWords, n * kSelRows * ct_coeffs);
  const int l = static_cast<int>(params->l_ep);
  k_noalloc_mux<<<dim3(n, 2), kThreads, l * kN * sizeof(uint32_t), st_>>>(
      P, scratch, l, static_cast<int>(params->base_log2));
  k_noalloc_compose<<<blocks, kThreads, 0, st_>>>(P, scratch, d_out, n * ct_coeffs);
  if (cudaGetLastError() != cudaSuccess) return OPIR_ERR_CUDA;
  return OPIR_OK;
}
