// Bulk-copy pipeline primitives (sm_90+/sm_100a): mbarrier phases and 1D bulk copies
// (cp.async.bulk, the TMA's untiled form) from global into this CTA's shared memory.
//
// Every wait is bounded in time: a wait that has not completed after its limit (a kernel
// argument, WAIT_NS = 1 s by default) of the global timer returns false, and the caller
// records an error and leaves the pipeline instead of spinning on (a poll of
// mbarrier.try_wait may itself suspend, so a bound on the number of polls would not bound
// the time).  The final drain of a producer, which makes sure none of its own bulk copies
// is still in flight when the CTA exits, always waits up to at least WAIT_NS.
#pragma once

#include <stdint.h>

namespace omb {

constexpr uint64_t WAIT_NS = 1000000000ull;  // 1 s

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
// make initialised barriers visible to the async (bulk-copy) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase with the given parity to complete; false after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint64_t limit_ns = WAIT_NS) {
  if (mbar_test(b, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_test(b, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// Limit of a producer's final drain wait.
__device__ __forceinline__ uint64_t drain_limit(uint64_t limit_ns) { return limit_ns > WAIT_NS ? limit_ns : WAIT_NS; }
// Bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) completing on `b`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}

// Error codes a pipeline kernel records in its error word (first error wins).
enum PipeError : int { PIPE_OK = 0, PIPE_FULL_TIMEOUT = 1, PIPE_EMPTY_TIMEOUT = 2, PIPE_DRAIN_TIMEOUT = 3 };
__device__ __forceinline__ void pipe_fail(int* err, int code) { atomicCAS(err, 0, code); }

}  // namespace omb
