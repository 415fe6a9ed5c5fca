// First-dimension scan on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Per residue r and NTT level l the scan is C = A . Q mod q_r with
// A = database rows [other x n0] and Q = query columns [n0 x 2B], all values
// < 2^29 (matrix.cpp:240-350, the reference's level_mat_mat_32). Both operands
// are stored as four byte planes (A = sum_i 2^(8i) A_i, Q = sum_j 2^(8j) Q_j),
// so C = sum_s 2^(8s) S_s with S_s = sum_{i+j=s} A_i . Q_j, s = 0..6. Every
// A_i . Q_j is an exact unsigned-int8 product with int32 accumulation; an S_s
// sums at most four of them, so n0 <= 8192 keeps it below 2^31
// (4 x 8192 x 255 x 255 < 2^31).
//
// One MMA per A plane and K step multiplies A_i by the four Q planes at once
// (they sit next to each other in shared memory and form one B operand of
// N = 4 ntile rows), writing TMEM columns [i ntile, (i + 4) ntile): the
// accumulator of S_s is columns [s ntile, (s + 1) ntile), shared by the MMAs
// of every (i, j) with i + j = s. Each A tile is read from shared memory once
// per K step, and an accumulator set is 7 ntile columns. The first K step of
// a tile initialises every column exactly once: A_0 Q_0..3 (overwrite s 0-3),
// A_3 Q_1..3 (overwrite s 4-6), then A_3 Q_0, A_1 Q_0..3 and A_2 Q_0..3
// accumulate. The epilogue recombines sum_s S_s 2^(8s) mod q in exact 64-bit
// arithmetic (7 terms < 2^31 x 2^29).
//
// Structure: persistent CTAs (one per SM), 10 warps:
//   warp 0      TMA producer: 3-D tiled loads (128B swizzle) of 4 A planes
//               [128 rows x 128 B] and 4 Q planes [ntile x 128 B] per stage
//   warp 1      TMEM owner + MMA issuer (one elected lane)
//   warps 2..9  epilogue, two warps per TMEM lane quadrant (each takes half
//               of the tile's columns): tcgen05.ld of the accumulators, recombination,
//               modular reduction, stores of C
// Two smem stages ring between producer and MMA. With ntile = 16 or 32 two
// accumulator sets (TMEM columns 0 and 256) ring between MMA and epilogue so
// the MMA warp does not wait for the previous tile's epilogue; ntile = 64 (a
// batch of 32 queries in one pass over the database) uses one set. Every
// mbarrier wait is bounded in time; on timeout the kernel records an error
// code, drains its own in-flight copies and MMAs, frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <set>

#include <cstring>
#include <stdexcept>
#include <string>

#include "opir_kernels.h"
#include "opir_scan_tc.h"
#include "opir_tc.cuh"

namespace opir {

namespace {

using namespace tc;

constexpr int kM = 128;          // MMA M / rows per tile
constexpr int kMaxStages = 8;
constexpr int kThreadsTc = 320;
constexpr int kEpilogueThreads = 256;
constexpr size_t kBarrierBytes = 256;  // mbarriers, TMEM slot, abort flag
constexpr uint32_t kTmemCols = 512;

// x mod q with mu = floor((2^64 - 1) / q), by Barrett's 64-bit quotient.
__device__ __forceinline__ uint32_t reduce64_barrett(uint64_t x, uint32_t q, uint64_t mu) {
  const uint64_t qhat = __umul64hi(x, mu);
  uint64_t r = x - qhat * q;
  if (r >= q) r -= q;
  if (r >= q) r -= q;
  return static_cast<uint32_t>(r);
}
// x mod q for any 64-bit x, from one 32-bit high product when mu = floor((2^64
// - 1) / q) = 8 2^32 + mu_lo (the 29-bit residues; the launcher checks),
// so with x = xh 2^32 + xl, x mu / 2^64 = 8 xh + xh mu_lo / 2^32 + xl / 2^29
// + xl mu_lo / 2^64; the estimate drops three fractions below 1 each, so it
// lies within 3 of floor(x mu / 2^64) > x / q - 2 - 1/q, r = x - est q <= 4q
// (< 2^32: 32-bit arithmetic is exact), and three corrections finish.
__device__ __forceinline__ uint32_t reduce64_tc(uint64_t x, uint32_t q, uint64_t mu) {
  const uint32_t xh = static_cast<uint32_t>(x >> 32), xl = static_cast<uint32_t>(x);
  const uint32_t est = (xh << 3) + __umulhi(xh, static_cast<uint32_t>(mu)) + (xl >> 29);
  uint32_t r = xl - est * q;
  r = min(r, r - 2 * q);
  r = min(r, r - q);
  return min(r, r - q);
}

// FAST: every residue's mu is 8 2^32 + mu_lo (reduce64_tc), else Barrett
// (the client's one-residue products mod small_q use the same kernel).
template <int KT, bool FAST>
__global__ void __launch_bounds__(kThreadsTc, 1)
k_scan_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmQ,
          TcScanArgs a) {
  extern __shared__ __align__(1024) uint8_t smraw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smraw) + 1023) &
                                            ~static_cast<uintptr_t>(1023));
  const uint32_t stages = a.stages;
  const uint32_t a_plane = kM * KT;                // 16 or 8 KiB
  const uint32_t q_plane = a.ntile * KT;
  const uint32_t stage_bytes = 4 * a_plane + 4 * q_plane;
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + stages * stage_bytes);
  uint64_t *empty = full + kMaxStages;
  uint64_t *acc_full = empty + kMaxStages;  // [2]
  uint64_t *acc_empty = acc_full + 2;       // [2]
  uint64_t *drain = acc_empty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], kEpilogueThreads);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     sa(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t per_z = a.col_tiles * a.m_tiles;
  const uint32_t n_items = per_z * a.zcount;

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    uint32_t stage = 0, phase = 0, total = 0;  // total: stage loads issued
    bool ok = true;
    for (uint32_t it = blockIdx.x; ok && it < n_items; it += gridDim.x) {
      const uint32_t ct = it % a.col_tiles, mt = (it / a.col_tiles) % a.m_tiles, z = it / per_z;
      for (uint32_t kt = 0; ok && kt < a.k_tiles; ++kt) {
        if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, a.wait_cycles)) { ok = false; break; }
        if (lane == 0) {
          uint8_t *st = sm + stage * stage_bytes;
          mbar_expect_tx(&full[stage], stage_bytes);
          for (int pl = 0; pl < 4; ++pl)
            tma_load_3d(st + pl * a_plane, &tmA, &full[stage], kt * KT, mt * kM, z * 4 + pl);
          for (int pl = 0; pl < 4; ++pl)
            tma_load_3d(st + 4 * a_plane + pl * q_plane, &tmQ, &full[stage], kt * KT,
                        ct * a.ntile, z * 4 + pl);
        }
        __syncwarp();
        ++total;
        if (++stage == stages) { stage = 0; phase ^= 1; }
      }
    }
    if (!ok) {
      if (lane == 0) { *abort_flag = 1; atomicOr(a.err, 1u); }
    }
    // own copies in flight must land before the CTA may exit
    for (uint32_t s = 0; s < stages; ++s) {
      const uint32_t issued = (total + stages - 1 - s) / stages;  // loads into stage s
      if (issued == 0) continue;
      const long long t0 = clock64();
      while (!mbar_try(&full[s], (issued - 1) & 1)) {
        if (clock64() - t0 > kWaitCycles) { if (lane == 0) atomicOr(a.err, 8u); break; }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------- MMA issuer
    const uint32_t nt = a.ntile;
    // A, B: unsigned 8-bit, K-major, dense; D: s32; M = 128; N as given
    auto idesc_n = [](uint32_t n) {
      return (2u << 4) | ((n >> 3) << 17) | (static_cast<uint32_t>(kM >> 4) << 24);
    };
    const uint32_t id4 = idesc_n(4 * nt), id3 = idesc_n(3 * nt), id1 = idesc_n(nt);
    const uint32_t nbufs = 2 * 7 * nt <= 512 ? 2 : 1;
    uint32_t stage = 0, phase = 0, acc_phases = 0, buf = 0;  // bit b: phase of set b
    bool ok = true;
    for (uint32_t it = blockIdx.x; ok && it < n_items; it += gridDim.x) {
      if (!mbar_wait(&acc_empty[buf], ((acc_phases >> buf) & 1) ^ 1, abort_flag, a.wait_cycles)) { ok = false; break; }
      fence_after();
      const uint32_t acc = tmem + buf * 256;  // S_s at columns acc + s nt
      for (uint32_t kt = 0; kt < a.k_tiles; ++kt) {
        if (!mbar_wait(&full[stage], phase, abort_flag, a.wait_cycles)) { ok = false; break; }
        fence_after();
        if (lane == 0) {
          const uint32_t base = sa(sm + stage * stage_bytes);
#pragma unroll
          for (int ks = 0; ks < KT / 32; ++ks) {
            const uint32_t qa = base + 4 * a_plane + ks * 32;  // Q planes 0..3
            const uint64_t db = smem_desc<KT>(qa);
            if (kt == 0 && ks == 0) {
              const uint64_t a0 = smem_desc<KT>(base), a3 = smem_desc<KT>(base + 3 * a_plane);
              mma_u8(acc, a0, db, id4, 0);                                   // S_0..3  = A_0 Q_0..3
              mma_u8(acc + 4 * nt, a3, smem_desc<KT>(qa + q_plane), id3, 0); // S_4..6  = A_3 Q_1..3
              mma_u8(acc + 3 * nt, a3, db, id1, 1);                          // S_3    += A_3 Q_0
#pragma unroll
              for (int i = 1; i < 3; ++i)
                mma_u8(acc + i * nt, smem_desc<KT>(base + i * a_plane), db, id4, 1);
            } else {
#pragma unroll
              for (int i = 0; i < 4; ++i)
                mma_u8(acc + i * nt, smem_desc<KT>(base + i * a_plane + ks * 32), db, id4, 1);
            }
          }
          mma_commit(&empty[stage]);  // frees the stage when these MMAs finish
        }
        __syncwarp();
        if (++stage == stages) { stage = 0; phase ^= 1; }
      }
      if (!ok) break;
      if (lane == 0) mma_commit(&acc_full[buf]);
      __syncwarp();
      acc_phases ^= 1u << buf;
      if (nbufs == 2) buf ^= 1;
    }
    if (!ok && lane == 0) { *abort_flag = 1; atomicOr(a.err, 2u); }
    // all MMAs issued by this thread must finish before TMEM is released
    if (lane == 0) mma_commit(drain);
    __syncwarp();
    const long long t0 = clock64();
    while (!mbar_try(drain, 0)) {
      if (clock64() - t0 > kWaitCycles) { if (lane == 0) atomicOr(a.err, 16u); break; }
    }
  } else {
    // --------------------------------------------------------- epilogue
    const int quad = warp & 3;             // TMEM lane quadrant of this warp
    const uint32_t half = (warp - 2) >> 2;   // which half of the tile's columns
    const int row = quad * 32 + lane;
    uint32_t acc_phases = 0, buf = 0;  // bit b: phase of set b
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
      if (!mbar_wait(&acc_full[buf], (acc_phases >> buf) & 1, abort_flag, a.wait_cycles)) {
        if (lane == 0) { *abort_flag = 1; atomicOr(a.err, 4u); }
        break;
      }
      fence_after();
      const uint32_t ct = it % a.col_tiles, mt = (it / a.col_tiles) % a.m_tiles, z = it / per_z;
      const int res = z >= a.levels_per_res ? 1 : 0;
      const uint32_t q = res ? a.q[1] : a.q[0];
      const uint64_t mu = res ? a.mu[1] : a.mu[0];
      uint32_t w[7];
#pragma unroll
      for (int s2 = 0; s2 < 7; ++s2) w[s2] = res ? a.w[1][s2] : a.w[0][s2];
      const uint32_t m = mt * kM + row;
      // cmat[z][column][row]: a warp's 32 rows of one column are 128
      // contiguous bytes
      uint32_t *dst = a.cmat + static_cast<uint64_t>(z) * a.ncols * a.other + m;
      const uint32_t col0 = ct * a.ntile;
      const uint32_t nt = a.ntile;
      const uint32_t tbase = tmem + buf * 256 + (static_cast<uint32_t>(quad * 32) << 16);
      // this warp's nt / 2 (<= 32) columns are read and reduced into
      // registers, the TMEM set is handed back, then the values are stored
      uint32_t outv[32];
      const uint32_t cbeg = half * (nt / 2), cend = cbeg + nt / 2;  // nt / 2 <= 32
      for (uint32_t h0 = cbeg; h0 < cend; h0 += 32) {
        const bool last = h0 + 32 >= cend;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const uint32_t c0 = h0 + 8 * cc;
          if (c0 >= cend) break;
          uint32_t P[7][8];
#pragma unroll
          for (int s2 = 0; s2 < 7; ++s2) tmem_ld8(tbase + s2 * nt + c0, P[s2]);
          tmem_wait_ld();
          uint64_t acc[8];
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            acc[c] = static_cast<uint64_t>(P[0][c]) * w[0];
#pragma unroll
            for (int s2 = 1; s2 < 7; ++s2) acc[c] += static_cast<uint64_t>(P[s2][c]) * w[s2];
          }
#pragma unroll
          for (int c = 0; c < 8; ++c)
            outv[8 * cc + c] = FAST ? reduce64_tc(acc[c], q, mu) : reduce64_barrett(acc[c], q, mu);
        }
        if (last) {  // the accumulators are in registers: hand the TMEM set back first
          fence_before();
          mbar_arrive(&acc_empty[buf]);
          acc_phases ^= 1u << buf;
          if (2 * 7 * nt <= 512) buf ^= 1;
        }
        if (m < a.other) {
#pragma unroll
          for (int c = 0; c < 32; ++c)
            if (h0 + c < cend && col0 + h0 + c < a.ncols)
              dst[static_cast<uint64_t>(col0 + h0 + c) * a.other] = outv[c];
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static const EncodeTiledFn fn = [] {  // initialised once, thread-safe
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || p == nullptr)
      return static_cast<EncodeTiledFn>(nullptr);
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  if (!fn) throw std::runtime_error("cuTensorMapEncodeTiled unavailable");
  return fn;
}

// Largest dynamic shared memory a block may opt into on sm_100.
constexpr size_t kSmemLimit = 227 * 1024;

// Raises the kernels' dynamic shared memory limit once per device.
void configure_scan_tc() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return;
  for (const void *k : {reinterpret_cast<const void *>(k_scan_tc<128, true>),
                        reinterpret_cast<const void *>(k_scan_tc<64, true>),
                        reinterpret_cast<const void *>(k_scan_tc<128, false>),
                        reinterpret_cast<const void *>(k_scan_tc<64, false>)}) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(kSmemLimit));
    if (e != cudaSuccess)
      throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  }
  done.insert(dev);
}

// Recombination-rate probe: the epilogue arithmetic above (NC shift-class
// sums S_s < 2^31 -> sum_s S_s (2^(8s) mod q) in 64 bits -> reduce64_tc)
// on register-resident sums, 8 outputs per thread per iteration, without the
// TMEM loads and stores: the rate at which an SM finishes one output of an
// int8 product of byte-sliced 29-bit residues when nothing else is in the
// way. The multipliers take one bit of the running result after every
// iteration (NC adds per 8 outputs), so no product can be computed once for
// several iterations; the values are not meaningful and `sink` keeps the
// work alive.
template <int NC>
__global__ void __launch_bounds__(256)
k_recombine_rate(uint32_t *__restrict__ sink, uint32_t iters, uint32_t q, uint64_t mu, uint32_t w0) {
  uint32_t P[NC][8];
  uint32_t w[NC];
#pragma unroll
  for (int s = 0; s < NC; ++s) {
    w[s] = (w0 + 977u * s) % q;
#pragma unroll
    for (int c = 0; c < 8; ++c) P[s][c] = (threadIdx.x * 64 + s * 8 + c + blockIdx.x) & 0x7fffffffu;
  }
  uint32_t acc = 0;
  for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      uint64_t x = static_cast<uint64_t>(P[0][c]) * w[0];
#pragma unroll
      for (int s = 1; s < NC; ++s) x += static_cast<uint64_t>(P[s][c]) * w[s];
      acc ^= reduce64_tc(x, q, mu);
    }
#pragma unroll
    for (int s = 0; s < NC; ++s) w[s] += acc & 1u;  // stays below 2^29 + iters
  }
  sink[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace

// 3-D byte tensor [planes][rows][k] (k innermost, row stride = k_bytes),
// boxes of [1][box_rows][box_k] with box_k-byte swizzle (128 or 64); rows and
// k past the extents read as zero.
void make_plane_map(CUtensorMap *map, const uint8_t *base, uint64_t k_bytes, uint64_t rows,
                    uint64_t planes, uint32_t box_rows, uint32_t box_k) {
  if (k_bytes % 16 != 0) throw std::invalid_argument("plane row stride must be a multiple of 16");
  if (box_k != 128 && box_k != 64) throw std::invalid_argument("box_k must be 128 or 64");
  const cuuint64_t dims[3] = {k_bytes, rows, planes};
  const cuuint64_t strides[2] = {k_bytes, k_bytes * rows};
  const cuuint32_t box[3] = {box_k, box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3,
                                 const_cast<uint8_t *>(base), dims, strides, box, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 box_k == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string(static_cast<int>(r)));
}

size_t scan_tc_smem(uint32_t ntile, uint32_t kt, uint32_t stages) {
  return 1024 + static_cast<size_t>(stages) * (4ull * kM * kt + 4ull * ntile * kt) + kBarrierBytes;
}

uint32_t scan_tc_max_stages(uint32_t ntile, uint32_t kt) {
  const size_t stage = 4ull * kM * kt + 4ull * ntile * kt;
  const size_t n = (kSmemLimit - 1024 - kBarrierBytes) / stage;
  return static_cast<uint32_t>(n < static_cast<size_t>(kMaxStages) ? n : kMaxStages);
}

void launch_scan_tc(const CUtensorMap &mapA, const CUtensorMap &mapQ, const TcScanArgs &args,
                    int sm_count, cudaStream_t st) {
  if ((args.kt != 128 && args.kt != 64) || args.stages < 2 ||
      args.stages > scan_tc_max_stages(args.ntile, args.kt) ||
      (args.ntile != 16 && args.ntile != 32 && args.ntile != 64))
    throw std::invalid_argument("tensor-core scan: unsupported tile configuration");
  const size_t smem = scan_tc_smem(args.ntile, args.kt, args.stages);
  configure_scan_tc();
  const uint64_t items = static_cast<uint64_t>(args.col_tiles) * args.m_tiles * args.zcount;
  const unsigned grid = static_cast<unsigned>(items < static_cast<uint64_t>(sm_count) ? items : sm_count);
  TcScanArgs a = args;  // 0: the default limit (~1 s)
  if (a.wait_cycles <= 0) a.wait_cycles = tc::kWaitCycles;
  const bool fast = (a.mu[0] >> 32) == 8 && (a.mu[1] >> 32) == 8;
  if (a.kt == 128 && fast)
    k_scan_tc<128, true><<<grid, kThreadsTc, smem, st>>>(mapA, mapQ, a);
  else if (a.kt == 128)
    k_scan_tc<128, false><<<grid, kThreadsTc, smem, st>>>(mapA, mapQ, a);
  else if (fast)
    k_scan_tc<64, true><<<grid, kThreadsTc, smem, st>>>(mapA, mapQ, a);
  else
    k_scan_tc<64, false><<<grid, kThreadsTc, smem, st>>>(mapA, mapQ, a);
  note_launches(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("k_scan_tc: ") + cudaGetErrorString(e));
}

uint32_t recombine_rate_blocks(int sms, int classes) {
  int occ = 0;
  const cudaError_t e =
      classes == 5 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_recombine_rate<5>, 256, 0)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_recombine_rate<7>, 256, 0);
  if (e != cudaSuccess || occ < 1) occ = 1;
  return static_cast<uint32_t>(sms) * static_cast<uint32_t>(occ);
}

uint64_t launch_recombine_rate(uint32_t *sink, uint32_t blocks, uint32_t iters, int classes,
                               cudaStream_t st) {
  if (classes != 5 && classes != 7) throw std::invalid_argument("recombine probe: 5 or 7 classes");
  const uint32_t q = 536813569u;  // the first k1_comp residue
  const uint64_t mu = ~0ull / q;
  if (classes == 5)
    k_recombine_rate<5><<<blocks, 256, 0, st>>>(sink, iters, q, mu, 123456789u);
  else
    k_recombine_rate<7><<<blocks, 256, 0, st>>>(sink, iters, q, mu, 123456789u);
  note_launches(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("k_recombine_rate: ") + cudaGetErrorString(e));
  return static_cast<uint64_t>(blocks) * 256 * iters * 8;
}

}  // namespace opir
