// Device helpers shared by the tensor-core kernels (qk_dense_tc.cu,
// qk_dense_i8.cu): shared-memory addresses, tcgen05 fences, shared-memory
// operand descriptors and the bounded mbarrier wait.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qk {

constexpr long long kTcWaitLimit = 20000000;   // mbarrier polls before giving up

__device__ __forceinline__ uint32_t s_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory descriptor of a K-major operand in the canonical 128-byte-
// swizzle layout (rows of 128 bytes, 8-row groups 1024 bytes apart, atoms
// 1024-byte aligned) whose MMA step starts at byte address a.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t a) {
    uint64_t d = (uint64_t)((a >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;                          // leading byte offset: unused (swizzled K-major)
    d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;   // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                          // 128-byte swizzle
    return d;
}

// Bounded wait for the phase with parity `parity` of bar; 0 if it gave up.
__device__ __forceinline__ uint32_t tc_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done = 0;
    for (long long t = 0; t < kTcWaitLimit && !done; ++t) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(s_u32(bar)), "r"(parity)
            : "memory");
    }
    return done;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s_u32(bar)) : "memory");
}

// Arrive on bar once every tcgen05 operation this thread issued before has
// completed.
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s_u32(bar))
                 : "memory");
}

}  // namespace qk
