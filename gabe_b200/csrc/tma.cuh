// Bulk (TMA) copies between global and shared memory with mbarrier
// completion, and bounded waits.
//
// cp.async.bulk moves a contiguous run of bytes (16-byte aligned at both
// ends, a multiple of 16 bytes long) from global to shared memory without
// using the issuing threads' registers; one thread issues the copies of a
// tile and every thread waits on the tile's mbarrier, whose transaction
// count the copies decrement as they land.  Only this GPU's own memory is
// ever a source here, and no copy uses cluster multicast.
//
// Waits are bounded: a wait that sees no completion for kWaitNs of GPU
// time gives up, raises ST_TIMEOUT in the caller's status word and returns
// false, so that a kernel whose copies never land ends instead of hanging.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace gabe {
namespace tma {

constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s of GPU time per wait

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async proxy (the copies).
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory
// before later async-proxy (bulk copy) accesses of it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One arrival that also announces `bytes` of copies to come.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

// Global -> shared copy of `bytes` bytes, completing on `bar`.
__device__ __forceinline__ void load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Waits until the barrier's phase with parity `parity` has completed.
// false (and ST_TIMEOUT in *status) if it did not within limit_ns.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, uint32_t parity, unsigned int *status,
                                              unsigned long long limit_ns) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_test(bar, parity)) {
        if (now_ns() - t0 > limit_ns) {
            atomicOr(status, ST_TIMEOUT);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned int *status) {
    return mbar_wait_for(bar, parity, status, kWaitNs);
}

// After a wait gave up: waits (bounded again) for the last fill of each of
// the nb ring barriers, so that no copy is still landing in shared memory
// when the block exits.  fills[b] counts the fills issued into buffer b.
__device__ __forceinline__ void drain(uint64_t *bar, const int *fills, int nb, unsigned int *status) {
    for (int b = 0; b < nb; b++)
        if (fills[b] > 0) mbar_wait(&bar[b], (uint32_t)((fills[b] - 1) & 1), status);
}

}  // namespace tma
}  // namespace gabe
