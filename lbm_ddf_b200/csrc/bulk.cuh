// bulk.cuh — thin wrappers over the sm_90+/sm_100a bulk asynchronous copy
// (TMA, untiled) and mbarrier PTX used by the row-staged step.  Every copy
// moves one contiguous row between this GPU's global memory and the issuing
// CTA's own shared memory (no copy fans out to other CTAs of a cluster).
//
// Rules the callers keep: global and shared addresses 16-byte aligned, sizes
// a multiple of 16 bytes; shared memory written by ordinary stores is made
// visible to the bulk store with fence_proxy_async() and a barrier first.
#pragma once

#include <cstdint>

namespace lbm {
namespace bulk {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the initialised barrier visible to the asynchronous proxy
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// one poll of phase `parity`; true once that phase has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// nanoseconds of the GPU's global timer
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: false if the phase did not complete within max_polls polls
// or max_ns nanoseconds (a poll may suspend the thread for a hardware-
// dependent time, so the poll count alone does not bound the time).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_polls, uint64_t max_ns) {
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < max_polls; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 63u && global_ns() - t0 > max_ns) return false;
    }
    return false;
}

// global -> shared, completion counted on `bar` (bytes)
__device__ __forceinline__ void load_row(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// shared -> global, tracked by the issuing thread's bulk group
__device__ __forceinline__ void store_row(void *gmem_dst, const void *smem_src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmem_dst),
                 "r"(smem_addr(smem_src)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void store_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// waits until the committed bulk stores have finished reading shared memory
__device__ __forceinline__ void store_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// orders this thread's ordinary shared-memory stores before later bulk copies
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace bulk
}  // namespace lbm
