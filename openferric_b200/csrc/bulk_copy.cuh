// bulk_copy.cuh - 1-D bulk asynchronous copies (global -> shared) completed on
// an mbarrier, for sm_90+ (cp.async.bulk, PTX ISA 8.0), and the mbarrier
// operations of producer/consumer rings in shared memory.  Each copy lands in
// the issuing CTA's own shared memory, and the sources are this GPU's own
// memory.
//
// Every wait is bounded: mbar_wait gives up after `limit_ns` of the global
// timer and returns false, so a caller can record an error and return instead
// of spinning for ever.
#pragma once

#include <cstdint>

namespace of {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async proxy (the bulk copies).
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One plain arrival (release at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// One arrival that also announces `bytes` of transactions for the phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// `bytes` (a multiple of 16) from 16-byte aligned global `src` to 16-byte
// aligned shared `dst`; completion is counted on `bar`.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase of parity `parity` of `bar` to complete; false after
// `limit_ns` nanoseconds without completion.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}

// try_wait with a suspend-time hint: the thread sleeps in the barrier until
// the phase completes or about `hint_ns` pass, instead of polling.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// mbar_wait whose polls suspend the waiting warp in the barrier for up to
// `hint_ns` each: a warp waiting on a slower partner warp then leaves the
// issue slots to the warps doing work instead of spinning.
__device__ __forceinline__ bool mbar_wait_backoff(uint32_t bar, uint32_t parity, uint64_t limit_ns,
                                                  uint32_t hint_ns) {
  if (mbar_try_wait_suspend(bar, parity, hint_ns)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait_suspend(bar, parity, hint_ns)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

}  // namespace of
