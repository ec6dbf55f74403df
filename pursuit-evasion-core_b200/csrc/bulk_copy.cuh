// Bulk asynchronous copies (the TMA engine's cp.async.bulk, global ->
// shared, no tensor map, into this CTA only) and the shared-memory
// mbarriers they complete on, as inline PTX for sm_100a.  Used by the
// persistent stage kernels that stream planes into shared-memory rings.
#pragma once

#include <cstdint>

namespace pe {
namespace bulk {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

// Arrive on `bar` once and expect `bytes` of copies to complete on it.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "{\n .reg .b64 state;\n"
      " mbarrier.arrive.expect_tx.shared::cta.b64 state, [%0], %1;\n}" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// One try: returns once the phase of `parity` has completed, or false after
// the hardware's time limit.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bulk copy global -> shared (16-byte aligned, size multiple of 16) that
// signals `bar` with its byte count.
__device__ __forceinline__ void bulk_load(void *dst, const void *src,
                                          uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Orders this thread's earlier shared-memory accesses before its later
// bulk copies into shared memory.
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders this thread's earlier global-memory accesses, including what it
// acquired at a grid-wide barrier (other CTAs' stores), before its later
// bulk copies, which read global memory through the async proxy.
__device__ __forceinline__ void fence_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile(
      "{\n .reg .b64 state;\n"
      " mbarrier.arrive.shared::cta.b64 state, [%0];\n}" ::"r"(smem_u32(bar))
      : "memory");
}

// Bounded wait for one mbarrier phase: at most `limit` tries.  Returns false
// (and ORs 1 into *timeout_flag) when the limit is reached.
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t parity,
                                           unsigned int *timeout_flag, unsigned limit) {
  for (unsigned i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(timeout_flag, 1u);
  return false;
}

}  // namespace bulk
}  // namespace pe
