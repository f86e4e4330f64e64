// Tensor Memory Accelerator (TMA) helpers for the plane-streaming stencils: host-side tensor-map
// encoding for C-order (nx, ny, nz) float grids and device-side mbarrier / bulk-tensor copies.
// Every wait is bounded: after TMA_SPIN_LIMIT polls it raises an error flag instead of hanging.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace bd {

// A waiting thread is suspended for up to TMA_SUSPEND_NS per poll (the hardware wakes it when the
// phase completes), so TMA_SPIN_LIMIT polls bound a wait to about 4 s before it reports a timeout.
constexpr unsigned TMA_SPIN_LIMIT = 1u << 22;
constexpr unsigned TMA_SUSPEND_NS = 1000;

// 3-D tiled map over a float grid: dims (innermost first) {nz, ny, nx}; box {bz, by, bx}.
// Requires nz % 4 == 0 (16-byte row stride) and a 16-byte aligned base; returns false otherwise.
bool make_tmap_3d_f32(CUtensorMap* out, const void* base, int nx, int ny, int nz, int bz, int by, int bx);
// 3-D tiled map over a byte grid whose z rows are `pitch` bytes apart (pitch % 16 == 0, >= nz);
// elements past nz read as 0.
bool make_tmap_3d_u8(CUtensorMap* out, const void* base, int nx, int ny, int nz, int pitch, int bz, int by, int bx);

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Plain arrive (count 1) on an mbarrier; release semantics order this thread's earlier accesses.
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait for the phase with the given parity: at most `limit` polls; false on timeout.
__device__ __forceinline__ bool mbar_wait_limit(unsigned long long* bar, unsigned parity, unsigned limit) {
    const unsigned a = smem_addr(bar);
    for (unsigned it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(TMA_SUSPEND_NS)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The kernels' wait: bounded by TMA_SPIN_LIMIT polls (about 4 s).
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    return mbar_wait_limit(bar, parity, TMA_SPIN_LIMIT);
}

// Orders this thread's earlier generic-proxy shared-memory accesses before later async-proxy
// (TMA) writes to the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 3-D tile load into shared memory; c0 (innermost) must keep c0 * 4 bytes 16-byte aligned.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace bd
