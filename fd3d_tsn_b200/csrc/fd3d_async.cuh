// fd3d_async.cuh -- mbarrier and bulk-copy primitives (sm_90+ PTX, used on sm_100a).
//
// Every copy here moves data between this GPU's global memory and the issuing CTA's
// shared memory; nothing is multicast.  Waits are bounded: mbar_wait gives up after
// TMA_WAIT_LIMIT polls and the caller records ST_TIMEOUT.
#pragma once
#include <cstdint>
#include "fd3d_common.cuh"

namespace fd3d {

constexpr int TMA_WAIT_LIMIT = 1 << 20;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait on an mbarrier phase; false after TMA_WAIT_LIMIT unsuccessful polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int n = 0; n < TMA_WAIT_LIMIT; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16),
// completion counted on the mbarrier in transaction bytes
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"((uint64_t)src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Programmatic dependent launch: a grid launched with programmatic stream serialization
// waits here until the grid before it has completed and its memory is visible (a no-op
// for a grid launched without it); once every CTA of a grid has passed
// pdl_launch_dependents, the next grid's CTAs may be scheduled and wait in pdl_wait.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace fd3d
