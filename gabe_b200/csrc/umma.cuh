// Fifth-generation tensor cores (tcgen05) and tiled TMA loads, as inline PTX.
//
// An MMA reads both operands from shared memory through 64-bit matrix
// descriptors and accumulates into tensor memory (TMEM: 128 lanes x 512
// 32-bit columns per SM); one thread issues it, and tcgen05.commit makes an
// mbarrier arrive once every MMA that thread issued so far has completed.
// Operands here are K-major BF16 tiles laid out with the 128-byte swizzle
// that the tiled TMA load writes: rows of 64 elements (128 bytes), the
// 16-byte chunk c of row r stored at chunk c ^ (r % 8), groups of 8 rows
// 1024 bytes apart, every tile 1024-byte aligned.  Loads read this GPU's
// own memory only and none uses cluster multicast.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "tma.cuh"

namespace gabe {
namespace umma {

// Shared-memory descriptor of a K-major, 128-byte-swizzled tile starting at
// shared address `sa` (1024-byte aligned, or advanced from such a start by
// a multiple of 32 bytes within the first row to select a 16-element K
// step): start >> 4 in bits 0-13, leading byte offset 16 B (unused by the
// swizzled K-major form) in bits 16-29, stride byte offset 1024 B between
// 8-row groups in bits 32-45, descriptor version 1 in bits 46-47, layout
// 2 = 128-byte swizzle in bits 61-63.
__device__ __forceinline__ uint64_t desc_k128(uint32_t sa) {
    return (uint64_t)((sa >> 4) & 0x3FFFu) | ((uint64_t)(16 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16 with BF16 A and B (both K-major) and
// an FP32 accumulator: D format in bits 4-5 (1 = F32), A and B formats in
// bits 7-9 and 10-12 (1 = BF16), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[adesc] * B[bdesc]^T, one M x N x 16 step; accumulate = 0
// overwrites D.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The barrier arrives (once) when every MMA this thread issued has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tma::saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Whole-warp TMEM allocation of ncols columns (a power of two >= 32); the
// base address lands in *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tma::saddr(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Whole-warp read of 32 consecutive columns of the warp's 32 TMEM lanes:
// lane i receives row (lane base + i), columns col .. col + 31.  The wait
// is in the same statement, so the values are complete when it returns.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Plain arrival on an mbarrier (no transaction count).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tma::saddr(bar)) : "memory");
}

// Tiled 2-D TMA load of the box at element coordinates (x, y) of the tensor
// map into shared memory, completing on bar.  x (the contiguous dimension)
// must be a multiple of 16 bytes' worth of elements.
__device__ __forceinline__ void load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            tma::saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(tma::saddr(bar))
        : "memory");
}

// Tiled 2-D TMA store of a shared-memory box to element coordinates (x, y)
// of the tensor map (rows past the tensor's extent are not written), as
// one bulk group of the issuing thread; x as for load_2d, y >= 0.
__device__ __forceinline__ void store_2d(const CUtensorMap *map, int x, int y, const void *src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(tma::saddr(src))
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Waits until at most N of this thread's bulk store groups are still
// reading shared memory (their sources may then be overwritten) ...
template <int N>
__device__ __forceinline__ void store_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// ... or until all of them have completed.
__device__ __forceinline__ void store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace umma
}  // namespace gabe
