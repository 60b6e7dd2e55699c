// Thin wrappers over the sm_90+/sm_100 async-copy PTX used by the tiled
// kernels: mbarriers and tensor-map (TMA) tile loads into shared memory.
// Only CTA-local loads from this GPU's global memory are issued (no cluster
// multicast).
#pragma once

#include <cstdint>

namespace potts {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Invalidates an mbarrier (all its phases complete or abandoned) before the
// same shared memory is initialised as an mbarrier again.
__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Orders this thread's global-memory accesses through the generic proxy with
// its later (or, for a writer, other threads' later) async-proxy accesses
// (TMA loads) of the same memory.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait that may suspend the thread for up to `ns` nanoseconds before
// reporting that the phase is still incomplete (fewer polling instructions).
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity, uint32_t ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Waits for phase `parity` of the barrier: at most kWaitTries try_waits that
// each suspend the thread for up to kWaitSleepNs (about 2 s in all).  Gives up
// early when *abort is set by another warp, and sets it when it runs out of
// tries.  Warp-uniform: every lane of the calling warp must call it; all get
// the same answer.
constexpr int kWaitTries = 2000;
constexpr uint32_t kWaitSleepNs = 1000000;

__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, volatile int *abort)
{
    bool done = mbar_try_wait(bar, parity);
    for (int i = 0; i < kWaitTries && !done; ++i) {
        if (*abort) break;
        done = mbar_try_wait_sleep(bar, parity, kWaitSleepNs);
    }
    if (!done) *abort = 1;
    return __all_sync(0xffffffffu, done) != 0;
}

// Bounded wait without the abort flag (used after an abort, for loads in flight).
constexpr int kDrainTries = 200;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int tries)
{
    if (mbar_try_wait(bar, parity)) return true;
    for (int i = 0; i < tries; ++i)
        if (mbar_try_wait_sleep(bar, parity, kWaitSleepNs)) return true;
    return false;
}

// Single-thread form (for the producer lane).
__device__ __forceinline__ bool mbar_wait_thread(uint64_t *bar, uint32_t parity, volatile int *abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    for (int i = 0; i < kWaitTries; ++i) {
        if (*abort) return false;
        if (mbar_try_wait_sleep(bar, parity, kWaitSleepNs)) return true;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const void *tmap, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_addr(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, uint64_t *bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Bulk prefetch of a tensor box into L2 (no shared memory, no barrier): the
// later TMA load of the same box then reads from L2.
__device__ __forceinline__ void tma_prefetch_l2_2d(const void *tmap, int x, int y)
{
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];"
                 ::"l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y)
                 : "memory");
}

__device__ __forceinline__ void tma_prefetch_l2_3d(const void *tmap, int x, int y, int z)
{
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];"
                 ::"l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}

// Acquire a tensor map that generic-proxy writes (host copies) produced.
__device__ __forceinline__ void tma_fence_acquire_desc(const void *tmap)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(tmap))
                 : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const void *tmap)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

}  // namespace potts
