// mbarrier.cuh -- shared-memory mbarriers for bulk copies, with the bounded wait every bulk-copy
// wait of the library uses (the wait gives up after a fixed number of polls instead of hanging).
#pragma once
#include <cstdint>

namespace su2g {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    return done != 0;
}

// Poll until the phase with parity `phase` completes or `limit` polls have failed; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t phase, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

}  // namespace su2g
