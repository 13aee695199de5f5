// bulk.cuh — shared-memory staging with the Tensor Memory Accelerator's bulk
// copies (cp.async.bulk, no tensor map, no multicast) completed on an
// mbarrier, and a bounded wait on that barrier.
//
// A bulk copy wants its global source and shared destination 16-byte
// aligned and its size a multiple of 16 bytes; callers widen a span to those
// boundaries (the device CSR arrays are allocated with 16 bytes of tail
// padding so a widened span never leaves its allocation).
#pragma once

#include <cstdint>

namespace wc {

__device__ inline uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Initialises an mbarrier expecting `count` arrivals per phase, and makes
// the initialisation visible to the asynchronous proxy.
__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of bulk copies to come.
__device__ inline void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// An L2 policy under which the lines a load brings in are the first to be
// evicted: for data streamed once per pass (a CSR's arrays), so that it does
// not push out the vectors that the gathers re-read.
__device__ inline uint64_t l2_evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// An L2 policy under which the lines are kept longest: for the vector the
// gathers of a pull re-read (its values are read once per entry).
__device__ inline uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Global → shared bulk copy of `bytes` (a multiple of 16, both addresses
// 16-byte aligned), completing its bytes on `bar`.
__device__ inline void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// bulk_load under an L2 policy (l2_evict_first_policy for a stream).
__device__ inline void bulk_load_hint(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                      uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
  return done != 0;
}

__device__ inline uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase of `bar` with the given parity to complete, for at
// most about `limit_ns`; false if it did not.
__device__ inline bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 2000000000ull) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t start = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - start > limit_ns) return false;
  }
}

}  // namespace wc
