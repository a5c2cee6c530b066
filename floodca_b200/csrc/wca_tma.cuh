// TMA row tiles for the pair sweep: PTX wrappers for mbarriers and 2-D
// tensor loads (cp.async.bulk.tensor, no multicast), and the host-side
// tensor maps of a session's padded fields.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

namespace fcab {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init1(uint32_t bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
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

// Waits for the barrier phase of the given parity; false after about 2^31
// cycles (about a second), so a lost transfer ends in an error, not a hang.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
    if (mbar_test(bar, parity))
        return true;
    const long long t0 = clock64();
    while (!mbar_test(bar, parity)) {
        if (clock64() - t0 > (1ll << 31))
            return false;
    }
    return true;
}

// Orders this thread's earlier generic-proxy accesses to shared memory
// before later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 2-D tiled load of box (c0, c1) of `map` into shared memory at dst,
// completing on `bar` (c0 * element size must be a multiple of 16 bytes).
__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                              int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

}  // namespace fcab
