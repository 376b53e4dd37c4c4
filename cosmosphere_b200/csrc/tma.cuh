/*
 * tma.cuh -- bulk asynchronous copies (the TMA unit's 1-D cp.async.bulk) from this GPU's
 * global memory into a warp's shared-memory stage, completed on an mbarrier, and the
 * bounded waits every device-side wait of the library goes through.
 *
 * Only the plain global -> shared form is issued: no cluster multicast, and the source is
 * always this GPU's own memory.  cp.async.bulk needs 16-byte aligned addresses and a size
 * that is a multiple of 16 bytes; the staged records are 32-byte double4s starting at
 * 32-byte boundaries, so every copy meets that.
 *
 * Bounded waits.  A wait polls until its condition holds or a time limit (globaltimer
 * nanoseconds, read every 64 polls) passes; then it gives up, the caller raises a bit in
 * the device error word, and the host reports it.  The limit is a kernel argument taken
 * from the host-side setting (cosmo_x_set_wait_limit; 1 s by default).
 */
#pragma once

#include <cstdint>

#include "common.cuh"

namespace cosmo {

// Host-side limit of every bounded device wait, in nanoseconds.
long long wait_limit_ns();

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Time limit of one wait: over() is true once limitNs has passed since its first call.
struct WaitClock
{
    unsigned long long start = 0;
    unsigned int polls = 0;
    __device__ __forceinline__ bool over(long long limitNs)
    {
        if ((polls++ & 63u) != 0u) return false;
        const unsigned long long t = global_ns();
        if (start == 0) { start = t; return false; }
        return (long long)(t - start) > limitNs;
    }
};

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make the initialised barriers visible to the async proxy (the copy engine).
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Wait for the phase of parity `parity` to complete; false if the limit passed first.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limitNs)
{
    WaitClock clk;
    while (!mbar_try_wait(bar, parity))
        if (clk.over(limitNs)) return false;
    return true;
}

// Bulk copy of `bytes` (a multiple of 16) from global memory at src to shared memory at
// dst (both 16-byte aligned), completing `bytes` of transaction count on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Order this thread's earlier shared-memory reads before later async-proxy writes (a bulk
// copy into the same buffer).
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One warp's staging area: kStages buffers of 32 particle records, one mbarrier each, the
// barriers' phase bits, and a flag set when a wait gave up (the warp then loads directly).
constexpr int kStages = 2;

struct WarpStage
{
    double4 buf[kStages][32];
    uint64_t bar[kStages];
    uint32_t phase;
    uint32_t broken;
};

// What a staged stream needs: the warp's area, the device error word and the wait limit.
struct StageRef
{
    WarpStage* ws;
    int* err;
    long long limitNs;
};

// Set up a warp's staging area (once per kernel, before its first use; all lanes call).
__device__ __forceinline__ void stage_init(WarpStage& ws)
{
    if ((threadIdx.x & 31) == 0)
    {
        for (int b = 0; b < kStages; ++b) mbar_init(&ws.bar[b], 1);
        ws.phase = 0;
        ws.broken = 0;
        fence_mbar_init();
    }
    __syncwarp();
}

} // namespace cosmo
