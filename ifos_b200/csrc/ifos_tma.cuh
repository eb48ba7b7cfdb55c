// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a.
// Loads only, never with cluster multicast; every wait is bounded.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ifos {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Plain arrive (count 1) on an mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Suspend-time hint (ns) of a barrier poll: a waiting thread sleeps in the
// poll instead of re-issuing it, leaving issue slots to the computing warps.
#ifndef IFOS_WAIT_HINT_NS
#define IFOS_WAIT_HINT_NS 20000
#endif

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(IFOS_WAIT_HINT_NS)
        : "memory");
    return ok != 0;
}

// Non-blocking test of a phase (no suspension).
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// 3-D tiled bulk tensor load into shared memory, completion on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait: gives up after at most 2^16 polls (each may sleep up to the
// suspend hint, so about a second in all), records `code` in *err and returns
// false.  The TMA engine cannot stall indefinitely on in-bounds loads, so the
// limit is only a guard.
// With an explicit `polls` (a caller-set limit) every poll is a
// non-blocking test, so that a short limit runs out in a few instructions.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err, int code,
                                                  long polls = 0) {
    if (polls > 0) {
        for (long it = 0; it < polls; it++)
            if (mbar_test_wait(bar, parity)) return true;
    } else {
        for (long it = 0; it < (1L << 16); it++)
            if (mbar_try_wait(bar, parity)) return true;
    }
    if (err) atomicExch(err, code);
    return false;
}

}  // namespace ifos
