// tcgen05 plumbing shared by the tensor-core kernels (sm_100a): shared-memory
// addresses, MMA completion through an mbarrier with a bounded wait, and the
// fences that order thread-side work against the tensor core's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bbkde {

constexpr long long kTcWaitLimit = 1ll << 26;   // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(mbar)
               : "memory");
}

// Bounded wait for the mbarrier phase `parity` to complete; false on expiry.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
  for (long long i = 0; i < kTcWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace bbkde
