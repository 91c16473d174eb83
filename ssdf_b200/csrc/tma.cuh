// tma.cuh -- bulk (non-tensor) TMA copies global -> shared with an mbarrier, and bounded waits.
//
// Only the plain cp.async.bulk form is used: the destination is this CTA's own shared memory and
// the source this GPU's global memory (no multicast, no clusters). Every wait is bounded: after
// kMaxSpin polls it gives up and reports it, so a lost copy can never hang the GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ssdf_b200 {

constexpr unsigned kMaxSpin = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the barrier initialisation visible to the async proxy before the first copy.
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst (shared) <- src (global), `bytes` a multiple of 16, both 16-byte aligned.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Waits for the phase with the given parity to complete; false if it did not within kMaxSpin polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (unsigned it = 0; it < kMaxSpin; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace ssdf_b200
