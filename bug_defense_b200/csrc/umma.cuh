// Fifth-generation tensor-core (tcgen05) helpers: shared-memory matrix descriptors, the f16-kind
// instruction descriptor, TMEM allocation, MMA issue/commit and TMEM loads.
//
// Descriptor encodings follow the PTX ISA's tcgen05 "shared memory descriptor" and "instruction
// descriptor" tables (the same bit layout CUTLASS's cute/arch/mma_sm100_desc.hpp declares):
//   smem descriptor: [0,14) start address >> 4, [16,30) leading byte offset >> 4,
//                    [32,46) stride byte offset >> 4, [46,48) version = 1, [49,52) base offset,
//                    [52] lbo mode, [61,64) layout (0 none, 6 swizzle-32B, 4 swizzle-64B, 2 swizzle-128B)
//   instr descriptor (kind::f16): [4,6) D format (1 = f32), [7,10) A format (1 = bf16),
//                    [10,13) B format (1 = bf16), [15] A major (0 K, 1 MN), [16] B major,
//                    [17,23) N >> 3, [24,29) M >> 4
// Canonical layouts used here (element = bf16, "core matrix" = 8 rows x 16 bytes):
//   K-major, no swizzle:  rows of 16 B (8 K-elements), 8-row groups SBO apart, K chunks LBO apart.
//   MN-major, no swizzle: K-rows of 16 B (8 MN-elements), 8 K-rows per 128-byte core matrix,
//                         K groups LBO apart, 8-element MN blocks SBO apart.
#pragma once

#include <cstdint>

#include "tma.cuh"

namespace bd {

enum UmmaLayout : uint32_t { UMMA_NONE = 0, UMMA_SW128 = 2, UMMA_SW64 = 4, UMMA_SW32 = 6 };

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    d |= (uint64_t)(layout & 7) << 61;
    return d;
}

// kind::f16 instruction descriptor: bf16 x bf16 -> f32, dense.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N, bool a_mn_major, bool b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) | ((b_mn_major ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrive once on the mbarrier when every tcgen05.mma this thread issued so far has completed.
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-collective TMEM allocation of ncols (power of two >= 32); the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 columns of 32-bit words: thread t of the warp receives lane (base lane + t).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Non-tensor bulk copy global -> shared (both 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}


}  // namespace bd
