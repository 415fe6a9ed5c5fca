// Device helpers for the tcgen05 kernels: mbarriers with bounded waits,
// TMA tile loads, shared-memory matrix descriptors, kind::i8 MMAs and TMEM
// loads, as inline PTX for sm_100a.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace opir {
namespace tc {

constexpr long long kWaitCycles = 1ll << 31;  // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t sa(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sa(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Non-blocking test of a phase (mbarrier.test_wait returns at once, where
// try_wait may suspend the thread for a while before it answers).
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sa(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Limits below this many cycles poll with test_wait, so that a short limit
// is measured in cycles rather than in try_wait's own suspension time.
constexpr long long kPollBelow = 1ll << 20;

// Bounded wait, called by all 32 lanes of a warp together: false on timeout
// (`limit` cycles) or when another role aborted. The answer is the same on
// every lane (a lane whose phase completed still reports false when another
// lane gave up), so the caller's branches and the .sync.aligned tcgen05
// instructions after it never diverge. A completed phase stays complete
// until this warp acts on it, and the abort flag and the clock only move one
// way, so each lane's stop condition never reverts.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, volatile int *abort_flag,
                                          long long limit = kWaitCycles) {
  const long long t0 = clock64();
  const bool poll = limit < kPollBelow;
  bool done = false;
  for (;;) {
    done = done || (poll ? mbar_test(b, parity) : mbar_try(b, parity));
    const bool stop = done || *abort_flag != 0 || clock64() - t0 > limit;
    if (__all_sync(0xffffffffu, stop)) break;
  }
  return __all_sync(0xffffffffu, done);
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(sa(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(sa(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Shared-memory matrix descriptor, K-major, KT-byte swizzle (KT = 128: 128B
// swizzle; KT = 64: 64B swizzle): 8-row groups of KT-byte rows (SBO = 8 KT
// bytes), Blackwell descriptor version 1.
template <int KT>
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1) << 16;                     // LBO (unused when swizzled)
  d |= static_cast<uint64_t>((8 * KT) >> 4) << 32;         // SBO
  d |= static_cast<uint64_t>(1) << 46;                     // version
  d |= static_cast<uint64_t>(KT == 128 ? 2 : 4) << 61;     // SWIZZLE_128B / SWIZZLE_64B
  return d;
}
__device__ __forceinline__ void mma_u8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sa(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(addr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace tc
}  // namespace opir
