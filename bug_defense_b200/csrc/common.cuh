// Shared helpers for the libbugdef kernels: status/error plumbing, the counter-based
// RNG and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

#include "../../include/bugdef.h"

namespace bd {

// ---- error state (thread-local message of the last failure) ------------------------
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
// Absorbed-weight tallies are 64-bit fixed point: weight * 2^36 per deposit, rounded to nearest.
// Integer sums are exact and independent of the order of the atomic additions (FP32 sums of
// millions of deposits lose the small ones once the voxel total dwarfs them). A photon deposits at
// most its weight (<= 1 plus rare roulette gains), so 2^26 photons per launch keep every voxel sum
// below 2^62.
constexpr float kTallyScale = 68719476736.0f;          // 2^36
constexpr long long kTallyMaxPhotons = 1LL << 26;
// Plume neighbourhood mask: one byte per voxel, z rows padded to a 16-byte pitch.
inline int plume_mask_pitch(int nz) { return (nz + 15) / 16 * 16; }
inline size_t plume_mask_only_bytes(int nx, int ny, int nz) {
    return ((size_t)nx * ny * plume_mask_pitch(nz) + 255) / 256 * 256;
}
// Then the live z groups of the direct plume kernel's columns (x chunk, 16-row y tile): one count
// byte per column, then per column the ascending ids of its 4-voxel z groups that hold void
// (at most (nz + 3) / 4 <= 255 ids; sized for one x plane per chunk).
constexpr int kPlumeZRows = 16;
inline size_t plume_zlist_offset(int nx, int ny, int nz) { return plume_mask_only_bytes(nx, ny, nz); }
inline size_t plume_zlist_bytes(int nx, int ny, int nz) {
    const size_t cols = (size_t)nx * ((ny + kPlumeZRows - 1) / kPlumeZRows);
    return (cols * (1 + (size_t)(nz + 3) / 4) + 255) / 256 * 256;
}
// Then the compact-order state of the direct plume kernel: 16 header words (unit count, chosen
// x planes per unit, unit count per candidate), the live-group bitmaps of every (x plane, y tile)
// (8 words each), then the units (16 bytes: column << 5 | band and the band's 8 group ids), at
// most one per band of every column.
inline size_t plume_units_offset(int nx, int ny, int nz) {
    return plume_zlist_offset(nx, ny, nz) + plume_zlist_bytes(nx, ny, nz);
}
inline size_t plume_unit_capacity(int nx, int ny, int nz) {
    const size_t cols = (size_t)nx * ((ny + kPlumeZRows - 1) / kPlumeZRows);
    return cols * (((size_t)(nz + 3) / 4 + 7) / 8);
}
inline size_t plume_units_bytes(int nx, int ny, int nz) {
    const size_t cols = (size_t)nx * ((ny + kPlumeZRows - 1) / kPlumeZRows);
    return ((16 + cols * 8) * sizeof(unsigned) + plume_unit_capacity(nx, ny, nz) * 16 + 255) / 256 * 256;
}
inline size_t plume_mask_bytes(int nx, int ny, int nz) {
    return plume_units_offset(nx, ny, nz) + plume_units_bytes(nx, ny, nz);
}

// Launch-shape knobs (BD_TUNE_*) and the generation counter bumped by every change.
int tune_value(int knob);
int tune_generation();

#define BD_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return ::bd::cuda_status(_e, #call);     \
    } while (0)

#define BD_CHECK_LAUNCH(what)                                           \
    do {                                                                \
        cudaError_t _e = cudaGetLastError();                            \
        if (_e != cudaSuccess) return ::bd::cuda_status(_e, what);      \
    } while (0)

#define BD_REQUIRE(cond, ...)                                           \
    do {                                                                \
        if (!(cond)) return ::bd::fail(BD_ERR_INVALID_ARG, __VA_ARGS__); \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline int grid_for(int64_t n, int block, int cap = 148 * 32) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

// ---- Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11). Counter-based: the stream of photon p is a pure function of
// (seed, p, draw index), so no RNG state lives in memory. ----------------------------
struct Philox {
    static constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    static constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    __host__ __device__ static inline void round(uint32_t& x0, uint32_t& x1, uint32_t& x2,
                                                 uint32_t& x3, uint32_t k0, uint32_t k1) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(M0, x0), lo0 = M0 * x0;
        uint32_t hi1 = __umulhi(M1, x2), lo1 = M1 * x2;
#else
        uint64_t p0 = (uint64_t)M0 * x0, p1 = (uint64_t)M1 * x2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t y0 = hi1 ^ x1 ^ k0, y2 = hi0 ^ x3 ^ k1;
        x0 = y0; x1 = lo1; x2 = y2; x3 = lo0;
    }
    __host__ __device__ static inline uint4 gen(uint4 c, uint32_t k0, uint32_t k1) {
        uint32_t x0 = c.x, x1 = c.y, x2 = c.z, x3 = c.w;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            round(x0, x1, x2, x3, k0, k1);
            k0 += W0; k1 += W1;
        }
        return make_uint4(x0, x1, x2, x3);
    }
};

// Per-photon stream: counter = (photon lo, photon hi, draw block, 0x42444d43 'BDMC').
struct PhotonRng {
    uint32_t k0, k1, p_lo, p_hi, blk;
    uint32_t r0, r1, r2, r3;
    int left;
    __device__ inline void init(uint64_t seed, uint64_t photon) {
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        p_lo = (uint32_t)photon; p_hi = (uint32_t)(photon >> 32);
        blk = 0; left = 0;
    }
    __device__ inline uint32_t next_u32() {
        if (left == 0) {
            uint4 v = Philox::gen(make_uint4(p_lo, p_hi, blk++, 0x42444d43u), k0, k1);
            r0 = v.x; r1 = v.y; r2 = v.z; r3 = v.w; left = 4;
        }
        uint32_t out = r0;
        r0 = r1; r1 = r2; r2 = r3; --left;
        return out;
    }
    // uniform in [0, 1): 24 significant bits
    __device__ inline float uniform() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
    // uniform in (0, 1): never 0, for logarithms
    __device__ inline float uniform_pos() {
        return ((float)(next_u32() >> 8) + 0.5f) * (1.0f / 16777216.0f);
    }
};

__device__ __forceinline__ size_t vidx(int i, int j, int k, int ny, int nz) {
    return ((size_t)i * ny + j) * nz + k;
}

}  // namespace bd
