// scl_tma.cuh -- bulk asynchronous copies (the TMA unit's cp.async.bulk)
// from global into shared memory, completed on an mbarrier, with bounded
// waits.
//
// A stage kernel stages its line segment (cells plus ghost cells) with one
// bulk copy per component plane issued by one thread: no per-thread load
// instructions, no per-thread address arithmetic, and the copy engine moves
// whole 16-byte granules.  Every copy here reads this GPU's own memory and
// writes the issuing CTA's own shared memory; none uses cluster multicast.
//
// Rules the callers keep (checked on the host before such a kernel is
// chosen, see the launchers): the global source and the shared destination
// start on 16-byte boundaries and every size is a multiple of 16 bytes.
#pragma once
#include <cstdint>

#include "scl_common.cuh"

namespace scl {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised mbarrier visible to the asynchronous proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory before
// later asynchronous-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of bulk-copy traffic on the barrier.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Bulk copy of `bytes` (multiple of 16) from global src to shared dst (both
// 16-byte aligned); its completion is counted on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of bar to complete, for at most limit_ns of device
// time.  Returns false when the limit ran out (the caller raises
// SCL_STATUS_TIMEOUT and stops using the buffer).
constexpr uint64_t MBAR_LIMIT_NS = 1000000000ull;   // 1 s: far above any copy of a few KB

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint64_t limit_ns = MBAR_LIMIT_NS) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

}  // namespace scl
