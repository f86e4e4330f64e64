// Plume transport in the void domain (plume.py:18-80, metal_ablation_solver.py:193-240): FTCS
// diffusion with upwind drift, zero flux at solid walls (the neighbour value is replaced by the
// centre), Dirichlet 0 on the outer walls, clamped at 0, optional first-order decay.
//
// Kernels (all evaluate the same per-voxel expression, ftcs(), so they are bit-identical):
//   k_plume_resident  default (BD_PLUME_KERNEL_RESIDENT): one persistent CTA per column tile of at
//                     most 15 x 20 keeps its tile of the field in shared memory for every step of a
//                     stage and swaps a one-voxel halo with its four neighbours through L2 per step
//   k_plume_direct_z  (BD_PLUME_KERNEL_DIRECT, and the fallback when the tiles exceed the SMs): one
//                     launch per step, a CTA per 32 (z) x 16 (y) tile column marching x planes over
//                     the column's live z groups
//   k_plume_step      any grid (nz % 4 != 0): one voxel per thread
// Layout: C-order (nx, ny, nz), z fastest; the neighbourhood of every voxel is one mask byte.
#include "common.cuh"
#include "engine.cuh"

#include <algorithm>
#include <cmath>

namespace bd {

constexpr int PM_TZ = 32, PM_TY = 8;  // k_plume_mask / k_plume_step block: 32 z x 8 y

// Plume neighbourhood byte per voxel, rebuilt whenever the void domain changes (epoch end); the
// bytes of one (x, y) column start every mz = plume_mask_pitch(nz) bytes (16-byte rows):
//   bit 6: voxel is void            bit 7: voxel is void and not on an outer wall (FTCS update)
//   bits 0-5: -x +x -y +y -z +z neighbour is void (otherwise its value is replaced by the centre,
//   the zero-flux wall of plume.py:61-71)
#define BD_PM_VOID 0x40u
#define BD_PM_UPDATE 0x80u
__global__ void k_plume_mask(int nx, int ny, int nz, int mz, const uint8_t* __restrict__ F,
                             uint8_t* __restrict__ M, const int* __restrict__ zlimit) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int j = blockIdx.x * PM_TY + threadIdx.y;
    const int i = blockIdx.y;
    if (j >= ny) return;
    const int plane = ny * nz;
    const bool xy_interior = (i > 0 && i < nx - 1 && j > 0 && j < ny - 1);
    const int col = i * plane + j * nz;
    const size_t mcol = ((size_t)i * ny + j) * mz;
    for (int k = threadIdx.x; k < zl; k += PM_TZ) {
        const int idx = col + k;
        uint8_t m = 0;
        if (F[idx] & BD_FLAG_VOID) {
            m = BD_PM_VOID;
            if (xy_interior && k > 0 && k < nz - 1) {
                m |= BD_PM_UPDATE;
                m |= (F[idx - plane] & BD_FLAG_VOID) ? 0x01 : 0;
                m |= (F[idx + plane] & BD_FLAG_VOID) ? 0x02 : 0;
                m |= (F[idx - nz] & BD_FLAG_VOID) ? 0x04 : 0;
                m |= (F[idx + nz] & BD_FLAG_VOID) ? 0x08 : 0;
                m |= (F[idx - 1] & BD_FLAG_VOID) ? 0x10 : 0;
                m |= (F[idx + 1] & BD_FLAG_VOID) ? 0x20 : 0;
            }
        }
        M[mcol + k] = m;
    }
}

struct PlumeConst {
    float dxy_x, dxy_y, dz_z;  // D_xy*idx2, D_xy*idy2, D_z*idz2
    float vz_over_dz, dtp, decay;
};

// Stencil weights of one step: C' = decay * (w0 C + wx (C-x + C+x) + wy (C-y + C+y) + wb C-z + wt C+z),
// the FTCS step of plume.py:46-80 with the upwind drift term folded into wt and w0.
struct PlumeW {
    float w0, wx, wy, wb, wt, decay;
};

__host__ __device__ inline PlumeW plume_weights(const PlumeConst& c) {
    PlumeW k;
    k.wx = c.dtp * c.dxy_x; k.wy = c.dtp * c.dxy_y; k.wb = c.dtp * c.dz_z;
    k.wt = k.wb + c.dtp * c.vz_over_dz;
    k.w0 = 1.0f - 2.0f * (k.wx + k.wy + k.wb) - c.dtp * c.vz_over_dz;
    k.decay = c.decay;
    return k;
}

// One voxel's FTCS update from its neighbours and mask byte, the expression of every plume kernel.
// The rounding of each operation is spelled out so that every kernel (and every inlining context)
// produces the same bits. FAST: the caller has established that, if the voxel is updated, all six
// neighbours are void.
template <bool FAST>
__device__ __forceinline__ float ftcs(float c0, float w, float e, float s, float n, float b, float t, unsigned m,
                                      const PlumeW& k) {
    if (!FAST) {
        w = (m & 0x01) ? w : c0;
        e = (m & 0x02) ? e : c0;
        s = (m & 0x04) ? s : c0;
        n = (m & 0x08) ? n : c0;
        b = (m & 0x10) ? b : c0;
        t = (m & 0x20) ? t : c0;
    }
    float a = __fmul_rn(k.w0, c0);
    a = __fmaf_rn(k.wx, __fadd_rn(w, e), a);
    a = __fmaf_rn(k.wy, __fadd_rn(s, n), a);
    a = __fmaf_rn(k.wb, b, a);
    a = __fmaf_rn(k.wt, t, a);
    const float u = fmaxf(__fmul_rn(a, k.decay), 0.0f);
    return (m & BD_PM_UPDATE) ? u : 0.0f;
}

// true when every voxel of the byte set `m` that is updated has all six neighbours void
__device__ __forceinline__ bool all_interior(unsigned m) {
    const unsigned upd = (m >> 7) & 0x01010101u;
    return (m & (upd * 0x3Fu)) == upd * 0x3Fu;
}

// Four consecutive z voxels (one float4 and their four mask bytes); zb / zt: the voxels below and
// above the group. FAST as in ftcs.
template <bool FAST>
__device__ __forceinline__ float4 ftcs4(float4 c, float4 w, float4 e, float4 s, float4 n, float zb, float zt,
                                       unsigned m, const PlumeW& k) {
    float4 v;
    v.x = ftcs<FAST>(c.x, w.x, e.x, s.x, n.x, zb, c.y, m & 0xffu, k);
    v.y = ftcs<FAST>(c.y, w.y, e.y, s.y, n.y, c.x, c.z, (m >> 8) & 0xffu, k);
    v.z = ftcs<FAST>(c.z, w.z, e.z, s.z, n.z, c.y, c.w, (m >> 16) & 0xffu, k);
    v.w = ftcs<FAST>(c.w, w.w, e.w, s.w, n.w, c.z, zt, m >> 24, k);
    return v;
}

// mask bytes of a 4-voxel group starting at z = k that lie below the void limit zl
__device__ __forceinline__ unsigned zkeep_mask(int zl, int k) {
    const int nk = zl - k;
    return nk >= 4 ? 0xffffffffu : (nk <= 0 ? 0u : (0xffffffffu >> (8 * (4 - nk))));
}

// ---- k_plume_step: any grid ----------------------------------------------------------------
// One FTCS step. CTA (y tile, x plane); a thread owns the voxels k = tx, tx+32, ... < zlim of one
// (x, y) column (zlim = *zlimit when given, every void voxel lies above it, else nz). Non-void voxels
// are written (as 0) only when full_write is set: the engine keeps them 0 in both ping-pong buffers.
__global__ void __launch_bounds__(PM_TZ * PM_TY) k_plume_step(int nx, int ny, int nz, int mz, PlumeConst c,
                                                              const float* __restrict__ C, float* __restrict__ Cn,
                                                              const uint8_t* __restrict__ M,
                                                              const int* __restrict__ zlimit, int full_write) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int j = blockIdx.x * PM_TY + threadIdx.y;
    const int i = blockIdx.y;
    if (j >= ny) return;
    const PlumeW kw = plume_weights(c);
    const int plane = ny * nz;
    const int col = i * plane + j * nz;
    const size_t mcol = ((size_t)i * ny + j) * mz;
    for (int k = threadIdx.x; k < zl; k += PM_TZ) {
        const int idx = col + k;
        const unsigned m = __ldg(&M[mcol + k]);
        if (!(m & BD_PM_UPDATE)) {
            if ((m & BD_PM_VOID) || full_write) Cn[idx] = 0.0f;
            continue;
        }
        // an updated voxel is never on an outer wall: all six neighbours exist
        Cn[idx] = ftcs<false>(__ldg(&C[idx]), __ldg(&C[idx - plane]), __ldg(&C[idx + plane]), __ldg(&C[idx - nz]),
                              __ldg(&C[idx + nz]), __ldg(&C[idx - 1]), __ldg(&C[idx + 1]), m, kw);
    }
}

// ---- k_plume_direct / k_plume_direct_z: one launch per step --------------------------------
// A CTA is one 32 (z) x 16 (y) tile and marches xc x planes; thread = 4 consecutive z voxels of
// one row, a warp 8 such groups x 4 rows (one 128-byte line per row and load). The thread keeps the
// x-1 / x float4 of its row in registers and loads, per plane, the next plane's float4 and the
// centre plane's y neighbours from the (L2-resident) field beside the plane's mask bytes (one
// 32-bit load): one L2 round trip per plane, at the price of loads a tissue plane does not need. The
// z neighbours come from the neighbouring lanes by shuffle (the tile's edge lanes load them).
// Latency is hidden by the many independent CTAs of a step. Warp-uniform paths: no void (nothing to
// do), every updated voxel with six void neighbours (no selects), the general path. Needs nz % 4 == 0
// and 16-byte aligned fields.
constexpr int PL_BZ = 32;
constexpr int PD_BY = 16;  // rows per CTA (8 * PD_BY threads)
static_assert(PD_BY == kPlumeZRows, "z-list columns follow the direct kernel's y tiles");

__global__ void __launch_bounds__(8 * PD_BY) k_plume_direct(const float* __restrict__ C, float* __restrict__ Cn,
                                                            const uint8_t* __restrict__ M, int nx, int ny, int nz,
                                                            int mz, int xc, PlumeConst c,
                                                            const int* __restrict__ zlimit, int full_write) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int k0 = blockIdx.x * PL_BZ;
    const int ib = blockIdx.z * xc, ie = min(nx, ib + xc);
    if (k0 >= zl || ib >= ie) return;  // uniform over the CTA
    const int zg = threadIdx.x & 7;
    const int j = blockIdx.y * PD_BY + (threadIdx.x >> 3), k = k0 + 4 * zg;
    const bool act = zl - k > 0 && j < ny;
    const bool in = j < ny && k < nz;
    const unsigned zkeep = zkeep_mask(zl, k);
    const size_t plane = (size_t)ny * nz;
    const size_t mplane = (size_t)ny * mz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    size_t idx = ((size_t)ib * ny + j) * nz + k;
    const uint8_t* mp = M + ((size_t)ib * ny + j) * mz + k;
    const PlumeW kw = plume_weights(c);
    float4 cw = in && ib > 0 ? __ldg(reinterpret_cast<const float4*>(C + idx - plane)) : z4;
    float4 cc = in ? __ldg(reinterpret_cast<const float4*>(C + idx)) : z4;
    for (int i = ib; i < ie; ++i, idx += plane, mp += mplane) {
        const unsigned mr = act ? (__ldg(reinterpret_cast<const unsigned*>(mp)) & zkeep) : 0u;
        const float4 ce = in && i + 1 < nx ? __ldg(reinterpret_cast<const float4*>(C + idx + plane)) : z4;
        const float4 cs = in && j > 0 ? __ldg(reinterpret_cast<const float4*>(C + idx - nz)) : z4;
        const float4 cn = in && j + 1 < ny ? __ldg(reinterpret_cast<const float4*>(C + idx + nz)) : z4;
        float eb = 0.0f, et = 0.0f;
        if (zg == 0 && in && k > 0) eb = __ldg(C + idx - 1);
        if (zg == 7 && in && k + 4 < nz) et = __ldg(C + idx + 4);
        const unsigned vd = mr & 0x40404040u;
        if (__any_sync(0xffffffffu, act && (vd || full_write))) {
            float zb = __shfl_up_sync(0xffffffffu, cc.w, 1, 8);
            float zt = __shfl_down_sync(0xffffffffu, cc.x, 1, 8);
            if (zg == 0) zb = eb;
            if (zg == 7) zt = et;
            const float4 v = __all_sync(0xffffffffu, all_interior(mr) || !act)
                                 ? ftcs4<true>(cc, cw, ce, cs, cn, zb, zt, mr, kw)
                                 : ftcs4<false>(cc, cw, ce, cs, cn, zb, zt, mr, kw);
            if (act && (vd || full_write)) {
                float* dst = Cn + idx;
                if (full_write || vd == 0x40404040u) {
                    *reinterpret_cast<float4*>(dst) = v;
                } else {
                    if (vd & 0x00000040u) dst[0] = v.x;
                    if (vd & 0x00004000u) dst[1] = v.y;
                    if (vd & 0x00400000u) dst[2] = v.z;
                    if (vd & 0x40000000u) dst[3] = v.w;
                }
            }
        }
        cw = cc;
        cc = ce;
    }
}

// Live z groups of every (x chunk, y tile) column of the direct kernel: a CTA per column (grid
// n_yt x n_chunks), thread g = the 4-voxel z group g; live when any of the column's planes and rows
// holds a void voxel in the group below the void z-limit (the mask bytes at or above it are not
// rebuilt, so they are masked off here). The void domain is fixed within a plume stage, so the
// lists are built once per stage, after the mask.
__global__ void __launch_bounds__(256) k_plume_zlist(const uint8_t* __restrict__ M, int nx, int ny, int nz, int mz,
                                                     int xc, const int* __restrict__ zlimit,
                                                     uint8_t* __restrict__ zlist) {
    __shared__ int wcount[8];
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int G = (nz + 3) / 4;
    const int n_yt = gridDim.x;
    const int n_cols = gridDim.x * gridDim.y;
    const int col = blockIdx.y * n_yt + blockIdx.x;
    const int ib = blockIdx.y * xc, ie = min(nx, ib + xc);
    const int j0 = blockIdx.x * PD_BY, j1 = min(ny, j0 + PD_BY);
    const int g = threadIdx.x;
    bool live = false;
    if (g < G && zl - 4 * g > 0) {
        const unsigned keep = zkeep_mask(zl, 4 * g);
        for (int i = ib; i < ie && !live; ++i)
            for (int j = j0; j < j1; ++j)
                if (__ldg(reinterpret_cast<const unsigned*>(M + ((size_t)i * ny + j) * mz + 4 * g)) & keep &
                    0x40404040u) {
                    live = true;
                    break;
                }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, live);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wcount[w] = __popc(bal);
    __syncthreads();
    int before = 0;
    for (int q = 0; q < w; ++q) before += wcount[q];
    if (live) zlist[n_cols + (size_t)col * G + before + __popc(bal & ((1u << lane) - 1u))] = (uint8_t)g;
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int q = 0; q < 8; ++q) tot += wcount[q];
        zlist[col] = (uint8_t)tot;
    }
}

// As k_plume_direct, but band blockIdx.x of a column takes the column's live groups 8 b .. 8 b + 7
// from its z list instead of 8 consecutive groups, so z tiles that are partly tissue cost only
// their void groups. A lane whose z neighbour group is not held by the neighbouring lane loads that
// neighbour voxel instead of taking it by shuffle. Voxels outside the lists are not void and are
// never written.
__global__ void __launch_bounds__(8 * PD_BY, 9) k_plume_direct_z(const float* __restrict__ C, float* __restrict__ Cn,
                                                                 const uint8_t* __restrict__ M, int nx, int ny,
                                                                 int nz, int mz, int xc, PlumeConst c,
                                                                 const int* __restrict__ zlimit,
                                                                 const uint8_t* __restrict__ zlist) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int G = (nz + 3) / 4;
    const int n_cols = gridDim.y * gridDim.z;
    const int col = blockIdx.z * gridDim.y + blockIdx.y;
    const int cnt = zlist[col];
    const int b0 = blockIdx.x * 8;
    const int ib = blockIdx.z * xc, ie = min(nx, ib + xc);
    if (b0 >= cnt || ib >= ie) return;  // uniform over the CTA
    const int zg = threadIdx.x & 7;
    const int g = b0 + zg < cnt ? (int)zlist[n_cols + (size_t)col * G + b0 + zg] : -2;
    const int gp = __shfl_up_sync(0xffffffffu, g, 1, 8);
    const int gn = __shfl_down_sync(0xffffffffu, g, 1, 8);
    const bool zb_lane = zg > 0 && gp == g - 1;  // the -z neighbour is the previous lane's last voxel
    const bool zt_lane = zg < 7 && gn == g + 1;  // the +z neighbour is the next lane's first voxel
    const int j = blockIdx.y * PD_BY + (threadIdx.x >> 3), k = 4 * max(g, 0);
    const bool act = g >= 0 && zl - k > 0 && j < ny;
    const bool in = g >= 0 && j < ny && k < nz;
    const unsigned zkeep = zkeep_mask(zl, k);
    const size_t plane = (size_t)ny * nz;
    const size_t mplane = (size_t)ny * mz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    size_t idx = ((size_t)ib * ny + j) * nz + k;
    const uint8_t* mp = M + ((size_t)ib * ny + j) * mz + k;
    const PlumeW kw = plume_weights(c);
    float4 cw = in && ib > 0 ? __ldg(reinterpret_cast<const float4*>(C + idx - plane)) : z4;
    float4 cc = in ? __ldg(reinterpret_cast<const float4*>(C + idx)) : z4;
    for (int i = ib; i < ie; ++i, idx += plane, mp += mplane) {
        const unsigned mr = act ? (__ldg(reinterpret_cast<const unsigned*>(mp)) & zkeep) : 0u;
        const float4 ce = in && i + 1 < nx ? __ldg(reinterpret_cast<const float4*>(C + idx + plane)) : z4;
        const float4 cs = in && j > 0 ? __ldg(reinterpret_cast<const float4*>(C + idx - nz)) : z4;
        const float4 cn = in && j + 1 < ny ? __ldg(reinterpret_cast<const float4*>(C + idx + nz)) : z4;
        float eb = 0.0f, et = 0.0f;
        if (!zb_lane && in && k > 0) eb = __ldg(C + idx - 1);
        if (!zt_lane && in && k + 4 < nz) et = __ldg(C + idx + 4);
        const unsigned vd = mr & 0x40404040u;
        if (__any_sync(0xffffffffu, act && vd)) {
            float zb = __shfl_up_sync(0xffffffffu, cc.w, 1, 8);
            float zt = __shfl_down_sync(0xffffffffu, cc.x, 1, 8);
            if (!zb_lane) zb = eb;
            if (!zt_lane) zt = et;
            const float4 v = __all_sync(0xffffffffu, all_interior(mr) || !act)
                                 ? ftcs4<true>(cc, cw, ce, cs, cn, zb, zt, mr, kw)
                                 : ftcs4<false>(cc, cw, ce, cs, cn, zb, zt, mr, kw);
            if (act && vd) {
                float* dst = Cn + idx;
                if (vd == 0x40404040u) {
                    *reinterpret_cast<float4*>(dst) = v;
                } else {
                    if (vd & 0x00000040u) dst[0] = v.x;
                    if (vd & 0x00004000u) dst[1] = v.y;
                    if (vd & 0x00400000u) dst[2] = v.z;
                    if (vd & 0x40000000u) dst[3] = v.w;
                }
            }
        }
        cw = cc;
        cc = ce;
    }
}

// ---- k_plume_resident: a whole stage in one launch ------------------------------------------
// The (x, y) columns are cut into tiles_x x tiles_y tiles of at most RS_TX x RS_TY columns, one CTA
// per tile, all resident at once (cooperative launch, one CTA per SM). A CTA copies its tile of the
// field, with a one-column ring of its neighbours' columns, into shared memory for z < min(zl, RS_Z)
// (zl = void z-limit) and keeps it there for every step of the stage. A step marches the tile's x
// planes; a thread owns RS_PPT (y, 4-voxel z group) positions of a plane and keeps the x-1 / x float4
// of each in registers, reads the x+1 / y+-1 / z+-1 neighbours from shared memory, and, after a CTA
// barrier (every read of the plane done), writes the plane's new values in place. The new values of
// the tile's boundary columns are also stored to the global ping-pong buffer of the next state;
// after the step a release flag tells the four neighbours, each CTA waits (acquire) for its
// neighbours' flags and copies their boundary columns into its ring. Neighbours are therefore never
// more than one step apart, and two global buffers suffice: a buffer is rewritten two steps after it
// was read. Voxels at z >= RS_Z (craters deeper than the shared-memory column) are updated straight
// from and to the global ping-pong buffers by the same CTA in the same plane pass. The final state
// of the tile is written to buffer (n_steps & 1). Every wait is bounded in time: on a timeout the
// CTA raises *err and stops (the stage result is then undefined and the engine reports
// BD_ERR_TIMEOUT).
constexpr int RS_TX = 15, RS_TY = 20, RS_Z = 128, RS_THREADS = 320, RS_PPT = 2;
constexpr int RS_G = RS_Z / 4;  // float4 groups per shared-memory column
static_assert(RS_TY * RS_G <= RS_PPT * RS_THREADS, "every shared-memory position of a plane needs a thread slot");
constexpr size_t RS_C_BYTES = (size_t)(RS_TX + 2) * (RS_TY + 2) * RS_Z * sizeof(float);
constexpr size_t RS_M_BYTES = (size_t)RS_TX * RS_TY * RS_Z;
constexpr size_t RS_SMEM = RS_C_BYTES + RS_M_BYTES + 16;
constexpr long long RS_TIMEOUT_NS = 500000000LL;  // 0.5 s per wait (a step takes microseconds)

struct ResidentArgs {
    float* buf0;          // the field at the start of the stage (the state of even steps)
    float* buf1;          // the other ping-pong buffer (odd steps)
    const uint8_t* M;     // neighbourhood bytes (pitch mz)
    const int* zlimit;    // void z-limit on the device, or nullptr for nz
    unsigned* flags;      // per CTA: steps completed in this launch (zeroed before the launch)
    int* err;
    int nx, ny, nz, mz;
    int tiles_x, tiles_y, n_steps;
    PlumeConst c;
};

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(RS_THREADS, 1) k_plume_resident(ResidentArgs a) {
    extern __shared__ __align__(16) unsigned char rs_smem[];
    float* Cs = reinterpret_cast<float*>(rs_smem);
    float4* Cs4 = reinterpret_cast<float4*>(rs_smem);
    const unsigned* Ms4 = reinterpret_cast<const unsigned*>(rs_smem + RS_C_BYTES);
    unsigned* Ms4w = reinterpret_cast<unsigned*>(rs_smem + RS_C_BYTES);
    volatile int* s_fail = reinterpret_cast<volatile int*>(rs_smem + RS_C_BYTES + RS_M_BYTES);

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int zl = a.zlimit ? min(max(*a.zlimit, 0), nz) : nz;
    if (zl == 0) return;  // no void voxel: nothing to advance (uniform over the grid)
    const int b = blockIdx.x;
    const int bx = b % a.tiles_x, by = b / a.tiles_x;
    const int x0 = bx * nx / a.tiles_x, x1 = (bx + 1) * nx / a.tiles_x;
    const int y0 = by * ny / a.tiles_y, y1 = (by + 1) * ny / a.tiles_y;
    const int tx = x1 - x0, ty = y1 - y0;
    const int zs = min(zl, RS_Z);      // voxels of a column held in shared memory
    const int Gs = (zs + 3) / 4;       // their float4 groups
    const int Gg = (zl + 3) / 4 - Gs;  // groups per column kept in global memory (zl > RS_Z)
    const int row = ty + 2;            // ring rows per plane
    const size_t plane = (size_t)ny * nz;
    const int tid = threadIdx.x;
    const PlumeW kw = plume_weights(a.c);
    auto cidx = [&](int lx, int ly) { return (lx * row + ly) * RS_G; };  // float4 index of a smem column
    auto gidx = [&](int x, int y, int k) { return ((size_t)x * ny + y) * nz + k; };

    // zero the shared field (ring columns outside the grid and z >= zl stay 0), then load the tile
    // and its ring (corners excluded) at the stage's start state, and the tile's mask bytes
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = tid; i < (tx + 2) * row * RS_G; i += RS_THREADS) Cs4[i] = z4;
    if (tid == 0) *s_fail = 0;
    __syncthreads();
    for (int i = tid; i < (tx + 2) * row * Gs; i += RS_THREADS) {
        const int g = i % Gs, col = i / Gs, ly = col % row, lx = col / row;
        const int x = x0 + lx - 1, y = y0 + ly - 1;
        const bool corner = (lx == 0 || lx == tx + 1) && (ly == 0 || ly == ty + 1);
        if (corner || x < 0 || x >= nx || y < 0 || y >= ny) continue;
        Cs4[cidx(lx, ly) + g] = __ldcg(reinterpret_cast<const float4*>(a.buf0 + gidx(x, y, 4 * g)));
    }
    for (int i = tid; i < tx * ty * Gs; i += RS_THREADS) {
        const int g = i % Gs, col = i / Gs, y = col % ty, px = col / ty;
        const unsigned m =
            __ldg(reinterpret_cast<const unsigned*>(a.M + ((size_t)(x0 + px) * ny + y0 + y) * a.mz + 4 * g));
        Ms4w[(px * ty + y) * RS_G + g] = m & zkeep_mask(zl, 4 * g);
    }
    __syncthreads();

    int py[RS_PPT], pg[RS_PPT];
    bool pv[RS_PPT];
#pragma unroll
    for (int q = 0; q < RS_PPT; ++q) {
        const int p = tid + q * RS_THREADS;
        pv[q] = p < ty * Gs;
        py[q] = pv[q] ? p / Gs : 0;
        pg[q] = pv[q] ? p % Gs : 0;
    }
    float4 cw[RS_PPT], cc[RS_PPT];
#pragma unroll
    for (int q = 0; q < RS_PPT; ++q) {
        cw[q] = pv[q] ? Cs4[cidx(0, py[q] + 1) + pg[q]] : z4;
        cc[q] = pv[q] ? Cs4[cidx(1, py[q] + 1) + pg[q]] : z4;
    }

    bool failed = false;
    for (int t = 0; t < a.n_steps; ++t) {
        const float* gcur = (t & 1) ? a.buf1 : a.buf0;
        float* gnxt = (t & 1) ? a.buf0 : a.buf1;
        for (int px = 0; px < tx; ++px) {
            const int lx = px + 1, x = x0 + px;
            float4 v[RS_PPT], ce[RS_PPT];
            unsigned mm[RS_PPT];
            bool fast = true;
#pragma unroll
            for (int q = 0; q < RS_PPT; ++q) {
                mm[q] = pv[q] ? Ms4[(px * ty + py[q]) * RS_G + pg[q]] : 0u;
                fast = fast && (!pv[q] || all_interior(mm[q]));
            }
            fast = __all_sync(0xffffffffu, fast);
#pragma unroll
            for (int q = 0; q < RS_PPT; ++q) {
                v[q] = z4;
                ce[q] = z4;
                if (!pv[q]) continue;
                const int c0 = cidx(lx, py[q] + 1);
                ce[q] = Cs4[cidx(lx + 1, py[q] + 1) + pg[q]];
                const float4 cs = Cs4[cidx(lx, py[q]) + pg[q]];
                const float4 cn = Cs4[cidx(lx, py[q] + 2) + pg[q]];
                const int k = 4 * pg[q];
                const float zb = k > 0 ? Cs[c0 * 4 + k - 1] : 0.0f;
                float zt = 0.0f;
                if (k + 4 < RS_Z) zt = Cs[c0 * 4 + k + 4];
                else if (Gg > 0) zt = __ldcg(gcur + gidx(x, y0 + py[q], RS_Z));
                v[q] = fast ? ftcs4<true>(cc[q], cw[q], ce[q], cs, cn, zb, zt, mm[q], kw)
                            : ftcs4<false>(cc[q], cw[q], ce[q], cs, cn, zb, zt, mm[q], kw);
            }
            // columns deeper than the shared-memory part: from and to the global buffers
            for (int p = tid; p < ty * Gg; p += RS_THREADS) {
                const int y = p / Gg, k = 4 * (Gs + p % Gg), yy = y0 + y;
                const size_t idx = gidx(x, yy, k);
                const unsigned m = __ldg(reinterpret_cast<const unsigned*>(a.M + ((size_t)x * ny + yy) * a.mz + k)) &
                                   zkeep_mask(zl, k);
                const float4 c = __ldcg(reinterpret_cast<const float4*>(gcur + idx));
                const float4 w = x > 0 ? __ldcg(reinterpret_cast<const float4*>(gcur + idx - plane)) : z4;
                const float4 e = x + 1 < nx ? __ldcg(reinterpret_cast<const float4*>(gcur + idx + plane)) : z4;
                const float4 s = yy > 0 ? __ldcg(reinterpret_cast<const float4*>(gcur + idx - nz)) : z4;
                const float4 n = yy + 1 < ny ? __ldcg(reinterpret_cast<const float4*>(gcur + idx + nz)) : z4;
                const float zb = k == RS_Z ? Cs[cidx(lx, y + 1) * 4 + RS_Z - 1] : __ldcg(gcur + idx - 1);
                const float zt = k + 4 < nz ? __ldcg(gcur + idx + 4) : 0.0f;
                *reinterpret_cast<float4*>(gnxt + idx) = ftcs4<false>(c, w, e, s, n, zb, zt, m, kw);
            }
            __syncthreads();  // every read of plane px (and of its neighbours' old values) is done
            const bool xedge = px == 0 || px == tx - 1;
#pragma unroll
            for (int q = 0; q < RS_PPT; ++q) {
                if (!pv[q]) continue;
                Cs4[cidx(lx, py[q] + 1) + pg[q]] = v[q];
                if (xedge || py[q] == 0 || py[q] == ty - 1)
                    *reinterpret_cast<float4*>(gnxt + gidx(x, y0 + py[q], 4 * pg[q])) = v[q];
                cw[q] = cc[q];
                cc[q] = ce[q];
            }
        }
        __syncthreads();  // the step's boundary stores of every thread are issued
        if (tid == 0) {
            __threadfence();
            st_release_gpu(a.flags + b, (unsigned)(t + 1));
        }
        if (t + 1 == a.n_steps) break;
        if (tid < 4) {
            const int nbx = bx + (tid == 0 ? -1 : tid == 1 ? 1 : 0), nby = by + (tid == 2 ? -1 : tid == 3 ? 1 : 0);
            if (nbx >= 0 && nbx < a.tiles_x && nby >= 0 && nby < a.tiles_y) {
                const unsigned* f = a.flags + nby * a.tiles_x + nbx;
                const long long t0 = global_ns();
                while (ld_acquire_gpu(f) < (unsigned)(t + 1)) {
                    if (global_ns() - t0 > RS_TIMEOUT_NS) {
                        *s_fail = 1;
                        atomicExch(a.err, 1);
                        break;
                    }
                }
                __threadfence();
            }
        }
        __syncthreads();
        if (*s_fail) {
            failed = true;
            break;
        }
        // the neighbours' boundary columns at the new state into the ring
        const int nring = (2 * ty + 2 * tx) * Gs;
        for (int i = tid; i < nring; i += RS_THREADS) {
            const int g = i % Gs, r = i / Gs;
            int lx, ly;
            if (r < 2 * ty) {
                lx = (r < ty) ? 0 : tx + 1;
                ly = (r % ty) + 1;
            } else {
                const int r2 = r - 2 * ty;
                ly = (r2 < tx) ? 0 : ty + 1;
                lx = (r2 % tx) + 1;
            }
            const int x = x0 + lx - 1, y = y0 + ly - 1;
            if (x < 0 || x >= nx || y < 0 || y >= ny) continue;
            Cs4[cidx(lx, ly) + g] = __ldcg(reinterpret_cast<const float4*>(gnxt + gidx(x, y, 4 * g)));
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < RS_PPT; ++q) {
            cw[q] = pv[q] ? Cs4[cidx(0, py[q] + 1) + pg[q]] : z4;
            cc[q] = pv[q] ? Cs4[cidx(1, py[q] + 1) + pg[q]] : z4;
        }
    }
    if (failed) return;
    // the tile's final state (z < zs; deeper voxels are already in this buffer)
    float* out = (a.n_steps & 1) ? a.buf1 : a.buf0;
    for (int i = tid; i < tx * ty * Gs; i += RS_THREADS) {
        const int g = i % Gs, col = i / Gs, y = col % ty, px = col / ty;
        *reinterpret_cast<float4*>(out + gidx(x0 + px, y0 + y, 4 * g)) = Cs4[cidx(px + 1, y + 1) + g];
    }
}

struct ResidentPlan {
    bool ok = false;
    int tiles_x = 0, tiles_y = 0, grid = 0;
};

// The resident kernel runs when nz % 4 == 0 and one CTA per tile fits on the GPU at once.
static ResidentPlan resident_plan(int nx, int ny, int nz) {
    ResidentPlan r;
    if (nz % 4 != 0) return r;
    int dev = 0, sms = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return r;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return r;
    r.tiles_x = (nx + RS_TX - 1) / RS_TX;
    r.tiles_y = (ny + RS_TY - 1) / RS_TY;
    r.grid = r.tiles_x * r.tiles_y;
    if (r.grid > sms || r.grid > kPlumeMaxTiles) return r;
    if (cudaFuncSetAttribute(k_plume_resident, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMEM) !=
        cudaSuccess)
        return r;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_plume_resident, RS_THREADS, RS_SMEM) != cudaSuccess ||
        occ < 1)
        return r;
    r.ok = true;
    return r;
}

bool plume_resident_active(const BdPlumeParams* p) {
    return tune_value(BD_TUNE_PLUME_KERNEL) == BD_PLUME_KERNEL_RESIDENT && resident_plan(p->nx, p->ny, p->nz).ok;
}

// per-CTA step flags of the resident kernel, after the z lists in the plume scratch buffer
static unsigned* resident_flags(uint8_t* mask, int nx, int ny, int nz) {
    return reinterpret_cast<unsigned*>(mask + plume_zlist_offset(nx, ny, nz) + plume_zlist_bytes(nx, ny, nz));
}

int plume_policy_steps(const BdPlumeParams* p, int* n_steps, float* dt_step, float* decay_step) {
    const double idx2 = 1.0 / ((double)p->dx * p->dx), idy2 = 1.0 / ((double)p->dy * p->dy);
    const double idz2 = 1.0 / ((double)p->dz * p->dz);
    const double d_rate = (double)p->D_xy * (idx2 + idy2) + (double)p->D_z * idz2;
    const double dt = p->dt;
    const bool decays = p->tau_linger > 0.0f && std::isfinite(p->tau_linger);
    if (p->dt_policy == BD_PLUME_DT_AS_GIVEN) {
        *n_steps = 1; *dt_step = (float)dt;
        *decay_step = decays ? (float)std::exp(-dt / p->tau_linger) : 1.0f;
    } else if (p->dt_policy == BD_PLUME_DT_METAL) {
        // dt_plume = min(dt, 0.45 / (2 d_rate)); decay still uses the substep dt
        float dr = (float)p->D_xy * ((float)idx2 + (float)idy2) + (float)p->D_z * (float)idz2;
        *n_steps = 1;
        *dt_step = dr > 1e-6f ? std::min((float)dt, 0.45f / (2.0f * dr)) : (float)dt;
        *decay_step = decays ? (float)std::exp(-dt / p->tau_linger) : 1.0f;
    } else if (p->dt_policy == BD_PLUME_DT_SUBCYCLE) {
        int n = p->n_sub;
        if (n <= 0) {
            // FTCS with upwind drift keeps every coefficient >= 0 while
            // dt (2 d_rate + vz/dz) <= 1; use 90 % of that limit.
            const double rate = 2.0 * d_rate + std::max(0.0, (double)p->vz) / p->dz;
            n = std::max(1, (int)std::ceil(dt * rate / 0.9 - 1e-9));
        }
        *n_steps = n;
        *dt_step = (float)(dt / n);
        *decay_step = decays ? (float)std::exp(-(dt / n) / p->tau_linger) : 1.0f;
    } else {
        return fail(BD_ERR_INVALID_ARG, "unknown plume dt policy %d", p->dt_policy);
    }
    return BD_OK;
}

// A plume stage: n_substeps x (steps per substep) FTCS steps on the ping-pong pair (Ca, Cb), the
// field in Ca on entry. *in_b = 1 when the result ends in Cb. With full_first (the context API, whose
// non-void voxels may hold anything) the mask covers the whole grid and every voxel is written.
int plume_launch(const BdPlumeParams* p, float* Ca, float* Cb, int n_substeps, const uint8_t* F, int* in_b,
                 cudaStream_t st, const int* zlimit, int full_first, uint8_t* mask, int* err) {
    int steps;
    float dtp, decay;
    int rc = plume_policy_steps(p, &steps, &dtp, &decay);
    if (rc) return rc;
    PlumeConst c;
    c.dxy_x = p->D_xy / (p->dx * p->dx);
    c.dxy_y = p->D_xy / (p->dy * p->dy);
    c.dz_z = p->D_z / (p->dz * p->dz);
    c.vz_over_dz = p->vz > 0.0f ? p->vz / p->dz : 0.0f;
    c.dtp = dtp;
    c.decay = decay;
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int mz = plume_mask_pitch(nz);
    const int* zl = full_first ? nullptr : zlimit;
    k_plume_mask<<<dim3((ny + PM_TY - 1) / PM_TY, nx), dim3(PM_TZ, PM_TY), 0, st>>>(nx, ny, nz, mz, F, mask, zl);
    BD_CHECK_LAUNCH("k_plume_mask");
    const long long total = (long long)steps * n_substeps;
    const int kernel = tune_value(BD_TUNE_PLUME_KERNEL);
    if (kernel == BD_PLUME_KERNEL_RESIDENT && total <= (1LL << 30)) {
        const ResidentPlan plan = resident_plan(nx, ny, nz);
        if (plan.ok) {
            ResidentArgs a;
            a.buf0 = Ca; a.buf1 = Cb;
            a.M = mask; a.zlimit = zl; a.flags = resident_flags(mask, nx, ny, nz); a.err = err;
            a.nx = nx; a.ny = ny; a.nz = nz; a.mz = mz;
            a.tiles_x = plan.tiles_x; a.tiles_y = plan.tiles_y; a.n_steps = (int)total;
            a.c = c;
            BD_CUDA(cudaMemsetAsync(a.flags, 0, sizeof(unsigned) * plan.grid, st));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(plan.grid);
            cfg.blockDim = dim3(RS_THREADS);
            cfg.dynamicSmemBytes = RS_SMEM;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            BD_CUDA(cudaLaunchKernelEx(&cfg, k_plume_resident, a));
            if (in_b) *in_b = (int)(total & 1);
            return BD_OK;
        }
    }
    const bool vec = nz % 4 == 0;  // the direct kernels move float4 groups
    const int xc = tune_value(BD_TUNE_PLUME_XC);
    const dim3 dgrid((nz + PL_BZ - 1) / PL_BZ, (ny + PD_BY - 1) / PD_BY, (nx + xc - 1) / xc);
    // live z groups per direct-kernel column, from this stage's mask
    uint8_t* zlist = nullptr;
    if (vec && !full_first && (nz + 3) / 4 <= 255) {
        zlist = mask + plume_zlist_offset(nx, ny, nz);
        k_plume_zlist<<<dim3((ny + PD_BY - 1) / PD_BY, (nx + xc - 1) / xc), 256, 0, st>>>(mask, nx, ny, nz, mz, xc, zl,
                                                                                          zlist);
        BD_CHECK_LAUNCH("k_plume_zlist");
    }
    for (long long s = 0; s < total; ++s) {
        const float* in = (s & 1) ? Cb : Ca;
        float* out = (s & 1) ? Ca : Cb;
        // the context API writes every voxel in the first two steps (one per ping-pong buffer)
        const int full = (full_first && s < 2) ? 1 : 0;
        if (zlist)
            k_plume_direct_z<<<dgrid, 8 * PD_BY, 0, st>>>(in, out, mask, nx, ny, nz, mz, xc, c, zl, zlist);
        else if (vec)
            k_plume_direct<<<dgrid, 8 * PD_BY, 0, st>>>(in, out, mask, nx, ny, nz, mz, xc, c, zl, full);
        else
            k_plume_step<<<dim3((ny + PM_TY - 1) / PM_TY, nx), dim3(PM_TZ, PM_TY), 0, st>>>(nx, ny, nz, mz, c, in, out,
                                                                                        mask, zl, full);
    }
    BD_CHECK_LAUNCH("k_plume_step");
    if (in_b) *in_b = (int)(total & 1);
    return BD_OK;
}
}  // namespace bd

using namespace bd;

extern "C" int bd_plume_advance(const BdPlumeParams* p, float* Ca, float* Cb, int n_substeps, const uint8_t* F,
                                int* in_b, void* stream) {
    BD_REQUIRE(p != nullptr, "bd_plume_advance: params is NULL");
    BD_REQUIRE(p->nx > 0 && p->ny > 0 && p->nz > 0, "bd_plume_advance: grid dims must be positive");
    BD_REQUIRE(Ca && Cb && F, "bd_plume_advance: NULL field");
    BD_REQUIRE(n_substeps >= 0, "bd_plume_advance: n_substeps must be >= 0");
    BD_REQUIRE((long long)p->nx * p->ny * p->nz < (1LL << 31), "bd_plume_advance: grid exceeds 2^31 voxels");
    if (n_substeps == 0) {
        if (in_b) *in_b = 0;
        return BD_OK;
    }
    cudaStream_t st = as_stream(stream);
    unsigned char* scratch = nullptr;  // plume neighbourhood bytes + a 4-byte error flag
    const size_t flag_off = plume_mask_bytes(p->nx, p->ny, p->nz);
    BD_CUDA(cudaMallocAsync((void**)&scratch, flag_off + 16, st));
    int* err = reinterpret_cast<int*>(scratch + flag_off);
    int rc = BD_OK;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) rc = plume_launch(p, Ca, Cb, n_substeps, F, in_b, st, nullptr, 1, scratch, err);
    int host_err = 0;
    if (e == cudaSuccess && rc == BD_OK) e = cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e2 = cudaFreeAsync(scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, "bd_plume_advance");
    if (e2 != cudaSuccess) return cuda_status(e2, "bd_plume_advance: cudaFreeAsync");
    if (host_err) return fail(BD_ERR_TIMEOUT, "bd_plume_advance: a bounded wait of the resident plume kernel timed out");
    return BD_OK;
}

extern "C" int bd_plume_steps_per_substep(const BdPlumeParams* p, int* n_steps, float* dt_step) {
    BD_REQUIRE(p && n_steps && dt_step, "bd_plume_steps_per_substep: NULL argument");
    float decay;
    return plume_policy_steps(p, n_steps, dt_step, &decay);
}
