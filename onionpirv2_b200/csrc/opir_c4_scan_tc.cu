// First-dimension scan of the two-limb parameter set on the tcgen05 tensor
// cores (sm_100a).
//
// Per limb and NTT level z the scan is C = A . Q mod q_limb with A the
// database rows [other x n0] and Q the query columns [n0 x 2B], values
// < 2^60 (matrix.cpp:36-151, the reference's u64 level_mat_mat). Both
// operands are stored as eight byte planes (A = sum_i 2^(8i) A_i,
// Q = sum_j 2^(8j) Q_j), so C = sum_s 2^(8s) S_s with
// S_s = sum_{i+j=s} A_i . Q_j for s = 0..14. Each A_i . Q_j is an exact
// unsigned-int8 product with int32 accumulation. A class sums at most eight
// of them and the top planes hold 4 bits (60-bit values), so a class is below
// (6 x 255 x 255 + 2 x 255 x 15) n0 < 2^31 for every n0 <= 4096.
//
// One MMA per A plane and K step multiplies A_i by the eight Q planes at once
// (adjacent in shared memory, one B operand of N = 8 ntile rows) into TMEM
// columns [i ntile, (i + 8) ntile): the accumulator of S_s is columns
// [s ntile, (s + 1) ntile). The first K step of a tile initialises each
// column once: A_0 Q_0..7 (overwrite S_0..7), A_7 Q_1..7 (overwrite S_8..14),
// then A_7 Q_0 and A_1..6 Q_0..7 accumulate. The epilogue forms
// lo = sum_{s<8} S_s 2^(8s) and hi = sum_{s>=8} S_s 2^(8(s-8)) exactly and
// returns (lo + (hi mod q) (2^64 mod q)) mod q.
//
// Structure (as the single-modulus tensor-core scan): persistent CTAs, 10
// warps -- TMA producer, TMEM owner + MMA issuer, 8 epilogue warps (two per
// TMEM lane quadrant, each taking half of the tile's columns). K tiles of 64
// bytes with 64-byte swizzle; ntile = 16 (two accumulator sets of 240
// columns) or 32 (one set of 480). Every mbarrier wait is bounded; on timeout
// the kernel records an error bit, drains its own copies and MMAs, frees
// TMEM and returns.
//
// With two column tiles (more than 8 queries) the tiles of one row tile run
// on CTAs b and b ^ 1 and load the same database tile; their producers
// publish the item they start and wait up to ~20 us for the partner, so the
// second load of a tile finds it in L2 instead of drifting apart by more
// than L2 holds. The wait is soft: past its bound the producer goes on (the
// partner may not be resident yet when other kernels share the GPU).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

#include "opir_c4_kernels.h"
#include "opir_tc.cuh"

namespace opir4 {

namespace {

using namespace opir::tc;
using u128 = unsigned __int128;

constexpr int kM = 128;
constexpr int kKT = 64;             // K bytes per stage (64-byte swizzle)
constexpr int kPlanes = 8;
constexpr int kClasses = 15;
constexpr int kMaxStages4 = 4;
constexpr int kThreadsTc = 320;
constexpr int kEpilogueThreads = 256;
constexpr size_t kBarrierBytes = 256;
constexpr uint32_t kTmemCols = 512;
constexpr size_t kSmemLimit = 227 * 1024;
constexpr long long kPairWaitCycles = 40000;  // ~20 us

template <uint64_t Q>
__device__ __forceinline__ uint64_t red128_tc(u128 x) {  // x < 2^126 -> [0, q)
  constexpr uint64_t c = static_cast<uint64_t>((static_cast<u128>(1) << 64) % Q);
  constexpr uint64_t cs = static_cast<uint64_t>((static_cast<u128>(c) << 64) / Q);
  constexpr uint64_t mu = ~0ull / Q;
  const uint64_t h = static_cast<uint64_t>(x >> 64), l = static_cast<uint64_t>(x);
  const uint64_t r1 = h * c - __umul64hi(h, cs) * Q;
  const uint64_t r2 = l - __umul64hi(l, mu) * Q;
  uint64_t r = r1 + r2;
  r = min(r, r - 4 * Q);
  r = min(r, r - 2 * Q);
  return min(r, r - Q);
}

// (lo + (hi mod q) 2^64) mod q for one limb
template <uint64_t Q>
__device__ __forceinline__ uint64_t combine(u128 lo, u128 hi) {
  constexpr uint64_t c64 = static_cast<uint64_t>((static_cast<u128>(1) << 64) % Q);
  const uint64_t h = red128_tc<Q>(hi);
  return red128_tc<Q>(lo + static_cast<u128>(h) * c64);  // < 2^88 + 2^120
}

__global__ void __launch_bounds__(kThreadsTc, 1)
k4_scan_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmQ,
           Tc4Args a) {
  extern __shared__ __align__(1024) uint8_t smraw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smraw) + 1023) &
                                            ~static_cast<uintptr_t>(1023));
  const uint32_t stages = a.stages;
  const uint32_t nt = a.ntile;
  const uint32_t a_plane = kM * kKT;   // 8 KiB
  const uint32_t q_plane = nt * kKT;
  const uint32_t stage_bytes = kPlanes * (a_plane + q_plane);
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + stages * stage_bytes);
  uint64_t *empty = full + kMaxStages4;
  uint64_t *acc_full = empty + kMaxStages4;  // [2]
  uint64_t *acc_empty = acc_full + 2;        // [2]
  uint64_t *drain = acc_empty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t nbufs = 2 * kClasses * nt <= 512 ? 2 : 1;

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
    uint32_t stage = 0, phase = 0, total = 0, started = 0;
    bool ok = true;
    const uint32_t partner = blockIdx.x ^ 1u;
    const bool paired = a.progress != nullptr && a.col_tiles == 2 && partner < gridDim.x;
    for (uint32_t it = blockIdx.x; ok && it < n_items; it += gridDim.x) {
      const uint32_t ct = it % a.col_tiles, mt = (it / a.col_tiles) % a.m_tiles, z = it / per_z;
      ++started;
      if (paired && lane == 0) {
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.progress + blockIdx.x),
                     "r"(started)
                     : "memory");
        const long long t0 = clock64();
        for (;;) {
          uint32_t other;
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                       : "=r"(other)
                       : "l"(a.progress + partner)
                       : "memory");
          if (other >= started || clock64() - t0 > kPairWaitCycles) break;
        }
      }
      __syncwarp();
      for (uint32_t kt = 0; ok && kt < a.k_tiles; ++kt) {
        if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag, a.wait_cycles)) { ok = false; break; }
        if (lane == 0) {
          uint8_t *st = sm + stage * stage_bytes;
          mbar_expect_tx(&full[stage], stage_bytes);
          for (int pl = 0; pl < kPlanes; ++pl)
            tma_load_3d(st + pl * a_plane, &tmA, &full[stage], kt * kKT, mt * kM,
                        z * kPlanes + pl);
          for (int pl = 0; pl < kPlanes; ++pl)
            tma_load_3d(st + kPlanes * a_plane + pl * q_plane, &tmQ, &full[stage], kt * kKT,
                        ct * nt, z * kPlanes + pl);
        }
        __syncwarp();
        ++total;
        if (++stage == stages) { stage = 0; phase ^= 1; }
      }
    }
    if (!ok) {
      if (lane == 0) { *abort_flag = 1; atomicOr(a.err, 1u); }
    }
    for (uint32_t s = 0; s < stages; ++s) {  // own copies must land before exit
      const uint32_t issued = (total + stages - 1 - s) / stages;
      if (issued == 0) continue;
      const long long t0 = clock64();
      while (!mbar_try(&full[s], (issued - 1) & 1)) {
        if (clock64() - t0 > kWaitCycles) { if (lane == 0) atomicOr(a.err, 8u); break; }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------- MMA issuer
    // A, B: unsigned 8-bit, K-major; D: s32; M = 128
    auto idesc_n = [](uint32_t n) {
      return (2u << 4) | ((n >> 3) << 17) | (static_cast<uint32_t>(kM >> 4) << 24);
    };
    const uint32_t id8 = idesc_n(8 * nt), id7 = idesc_n(7 * nt), id1 = idesc_n(nt);
    uint32_t stage = 0, phase = 0, acc_phases = 0, buf = 0;
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
          for (int ks = 0; ks < kKT / 32; ++ks) {
            const uint32_t qa = base + kPlanes * a_plane + ks * 32;  // Q planes 0..7
            const uint64_t db = smem_desc<kKT>(qa);
            if (kt == 0 && ks == 0) {
              const uint64_t a0 = smem_desc<kKT>(base);
              const uint64_t a7 = smem_desc<kKT>(base + 7 * a_plane);
              mma_u8(acc, a0, db, id8, 0);                                     // S_0..7  = A_0 Q_0..7
              mma_u8(acc + 8 * nt, a7, smem_desc<kKT>(qa + q_plane), id7, 0);  // S_8..14 = A_7 Q_1..7
              mma_u8(acc + 7 * nt, a7, db, id1, 1);                            // S_7    += A_7 Q_0
#pragma unroll
              for (int i = 1; i < 7; ++i)
                mma_u8(acc + i * nt, smem_desc<kKT>(base + i * a_plane), db, id8, 1);
            } else {
#pragma unroll
              for (int i = 0; i < kPlanes; ++i)
                mma_u8(acc + i * nt, smem_desc<kKT>(base + i * a_plane + ks * 32), db, id8, 1);
            }
          }
          mma_commit(&empty[stage]);
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
    if (lane == 0) mma_commit(drain);
    __syncwarp();
    const long long t0 = clock64();
    while (!mbar_try(drain, 0)) {
      if (clock64() - t0 > kWaitCycles) { if (lane == 0) atomicOr(a.err, 16u); break; }
    }
  } else {
    // --------------------------------------------------------- epilogue
    const int quad = warp & 3;
    const uint32_t half = (warp - 2) >> 2;
    const int row = quad * 32 + lane;
    uint32_t acc_phases = 0, buf = 0;
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
      if (!mbar_wait(&acc_full[buf], (acc_phases >> buf) & 1, abort_flag, a.wait_cycles)) {
        if (lane == 0) { *abort_flag = 1; atomicOr(a.err, 4u); }
        break;
      }
      fence_after();
      const uint32_t ct = it % a.col_tiles, mt = (it / a.col_tiles) % a.m_tiles, z = it / per_z;
      const bool limb1 = z >= static_cast<uint32_t>(kN);
      const uint32_t m = mt * kM + row;
      // cmat[z][column][row]: a warp's 32 rows of one column are contiguous
      uint64_t *dst = a.cmat + static_cast<uint64_t>(z) * a.ncols * a.other + m;
      const uint32_t col0 = ct * nt;
      const uint32_t tbase = tmem + buf * 256 + (static_cast<uint32_t>(quad * 32) << 16);
      const uint32_t cbeg = half * (nt / 2);  // this warp's nt / 2 (8 or 16) columns
      uint64_t outv[16];
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        const uint32_t c0 = cbeg + 8 * cc;
        if (8 * cc >= static_cast<int>(nt / 2)) break;
        u128 lo[8], hi[8];
        {
          uint32_t P[8][8];
#pragma unroll
          for (int s2 = 0; s2 < 8; ++s2) tmem_ld8(tbase + s2 * nt + c0, P[s2]);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            u128 v = P[7][c];
#pragma unroll
            for (int s2 = 6; s2 >= 0; --s2) v = (v << 8) + P[s2][c];
            lo[c] = v;
          }
        }
        {
          uint32_t P[7][8];
#pragma unroll
          for (int s2 = 0; s2 < 7; ++s2) tmem_ld8(tbase + (8 + s2) * nt + c0, P[s2]);
          tmem_wait_ld();
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            u128 v = P[6][c];
#pragma unroll
            for (int s2 = 5; s2 >= 0; --s2) v = (v << 8) + P[s2][c];
            hi[c] = v;
          }
        }
#pragma unroll
        for (int c = 0; c < 8; ++c)
          outv[8 * cc + c] = limb1 ? combine<kQ1>(lo[c], hi[c]) : combine<kQ0>(lo[c], hi[c]);
      }
      // the accumulators are in registers: hand the TMEM set back first
      fence_before();
      mbar_arrive(&acc_empty[buf]);
      acc_phases ^= 1u << buf;
      if (nbufs == 2) buf ^= 1;
      if (m < a.other) {
#pragma unroll
        for (int c = 0; c < 16; ++c)
          if (c < static_cast<int>(nt / 2) && col0 + cbeg + c < a.ncols)
            dst[static_cast<uint64_t>(col0 + cbeg + c) * a.other] = outv[c];
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

void configure() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return;
  const cudaError_t e = cudaFuncSetAttribute(k4_scan_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kSmemLimit));
  if (e != cudaSuccess)
    throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  done.insert(dev);
}

}  // namespace

size_t scan_tc4_smem(uint32_t ntile, uint32_t stages) {
  return 1024 + static_cast<size_t>(stages) * kPlanes * (kM + ntile) * kKT + kBarrierBytes;
}

uint32_t scan_tc4_max_stages(uint32_t ntile) {
  const size_t stage = static_cast<size_t>(kPlanes) * (kM + ntile) * kKT;
  const size_t n = (kSmemLimit - 1024 - kBarrierBytes) / stage;
  return static_cast<uint32_t>(n < static_cast<size_t>(kMaxStages4) ? n : kMaxStages4);
}

void launch_scan_tc4(const CUtensorMap &mapA, const CUtensorMap &mapQ, const Tc4Args &args,
                     int sm_count, cudaStream_t st) {
  // zcount: 2 x 4096 levels of CONFIG_N4096_K2_MP, or the 2048 levels of the
  // one-limb CONFIG_N2048_K1 (whose prime is limb 0's, kQ0)
  if ((args.ntile != 16 && args.ntile != 32) || args.stages < 2 ||
      args.stages > scan_tc4_max_stages(args.ntile) || (args.zcount != 2u * kN && args.zcount != 2048u))
    throw std::invalid_argument("tensor-core scan of 64-bit limbs: unsupported tile configuration");
  const size_t smem = scan_tc4_smem(args.ntile, args.stages);
  configure();
  const uint64_t items = static_cast<uint64_t>(args.col_tiles) * args.m_tiles * args.zcount;
  const unsigned grid =
      static_cast<unsigned>(items < static_cast<uint64_t>(sm_count) ? items : sm_count);
  if (args.progress != nullptr && grid > 1024)
    throw std::invalid_argument("two-limb tensor-core scan: pairing counters hold 1024 CTAs");
  if (args.progress != nullptr) {
    const cudaError_t me = cudaMemsetAsync(args.progress, 0, grid * sizeof(uint32_t), st);
    if (me != cudaSuccess)
      throw std::runtime_error(std::string("k4_scan_tc progress: ") + cudaGetErrorString(me));
  }
  Tc4Args a = args;  // 0: the default limit (~1 s)
  if (a.wait_cycles <= 0) a.wait_cycles = opir::tc::kWaitCycles;
  k4_scan_tc<<<grid, kThreadsTc, smem, st>>>(mapA, mapQ, a);
  note_launches(1);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("k4_scan_tc: ") + cudaGetErrorString(e));
}

}  // namespace opir4
