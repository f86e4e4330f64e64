// Plume transport in the void domain (plume.py:18-80, metal_ablation_solver.py:193-240): FTCS
// diffusion with upwind drift, zero flux at solid walls (the neighbour value is replaced by the
// centre), Dirichlet 0 on the outer walls, clamped at 0, optional first-order decay.
//
// Kernels (all evaluate the same per-voxel expression, ftcs1 / ftcs4, so they are bit-identical):
//   k_plume_direct_z  default (BD_PLUME_KERNEL_DIRECT): one launch per step, a CTA per 32 (z) x 16 (y)
//                     tile column marching x planes over the column's live z groups
//   k_plume_direct_c  (BD_PLUME_KERNEL_COMPACT): the same per-unit code, one wave of CTAs looping
//                     over a compact list of the live units, x planes per unit chosen per stage
//   k_plume_step      any grid (nz % 4 != 0): one voxel per thread
// Layout: C-order (nx, ny, nz), z fastest; the neighbourhood of every voxel is one mask byte.
#include "common.cuh"
#include "engine.cuh"

#include <algorithm>
#include <atomic>
#include <vector>
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

// Weights of one step. plume.py:46-80 updates a void voxel as
//   C' = decay * (C + dt (D_xy (lap_x + lap_y) + D_z lap_z - v (C - C_{+z}) / dz)),
// with a solid neighbour's value replaced by the centre's (zero flux). Every kernel keeps solid
// voxels at 0, so that replacement is the same as adding the solid neighbour's weight to the centre:
//   C' = decay * (w0eff C + wx (C_-x + C_+x) + wy (C_-y + C_+y) + wb C_-z + wt C_+z),
// w0eff = w0 + the weights of the solid neighbours, one of 64 values picked by the six neighbour
// bits of the voxel's mask byte. The table is built once per stage on the host, in float32, in a
// fixed order, so every kernel applies the same weights.
struct PlumeTab {
    float wx, wy, wb, wt, decay;
    int decays;          // decay != 1 (a factor of exactly 1 is skipped: x * 1 == x)
    float w0eff[64];
};

static PlumeTab make_plume_tab(const PlumeConst& c) {
    PlumeTab t;
    t.wx = c.dtp * c.dxy_x;
    t.wy = c.dtp * c.dxy_y;
    t.wb = c.dtp * c.dz_z;
    const float adv = c.dtp * c.vz_over_dz;
    t.wt = t.wb + adv;
    const float w0 = 1.0f - 2.0f * (t.wx + t.wy + t.wb) - adv;
    for (int b = 0; b < 64; ++b) {
        float e = w0;
        if (!(b & 0x01)) e += t.wx;
        if (!(b & 0x02)) e += t.wx;
        if (!(b & 0x04)) e += t.wy;
        if (!(b & 0x08)) e += t.wy;
        if (!(b & 0x10)) e += t.wb;
        if (!(b & 0x20)) e += t.wt;
        t.w0eff[b] = e;
    }
    t.decay = c.decay;
    t.decays = c.decay != 1.0f;
    return t;
}

// One voxel (the scalar form; the packed form below performs the same operations per component).
__device__ __forceinline__ float ftcs1(float c0, float w, float e, float s, float n, float b, float t, unsigned m,
                                       const PlumeTab& k) {
    float a = __fmul_rn(k.w0eff[m & 0x3Fu], c0);
    a = __fmaf_rn(k.wx, __fadd_rn(w, e), a);
    a = __fmaf_rn(k.wy, __fadd_rn(s, n), a);
    a = __fmaf_rn(k.wb, b, a);
    a = __fmaf_rn(k.wt, t, a);
    if (k.decays) a = __fmul_rn(a, k.decay);
    return (m & BD_PM_UPDATE) ? fmaxf(a, 0.0f) : 0.0f;
}

// Four consecutive z voxels (one float4 and their four mask bytes); zb / zt: the voxels below and
// above the group. Pairs of voxels go through the packed FP32x2 operations of sm_100 (each lane
// rounded as the scalar operation), which halves the arithmetic instructions.
// w0eff: the table of effective centre weights, wherever the caller keeps it (shared memory in
// every step kernel).
__device__ __forceinline__ float4 ftcs4(float4 c, float4 w, float4 e, float4 s, float4 n, float zb, float zt,
                                        unsigned m, const PlumeTab& k, const float* w0eff) {
    const float2 wx = make_float2(k.wx, k.wx), wy = make_float2(k.wy, k.wy);
    const float2 wb = make_float2(k.wb, k.wb), wt = make_float2(k.wt, k.wt);
    // a group whose four voxels have six void neighbours each (the bulk of the domain) needs no lookup
    float2 wa, wc;
    if ((m & 0x3F3F3F3Fu) == 0x3F3F3F3Fu) {
        wa = wc = make_float2(w0eff[0x3F], w0eff[0x3F]);
    } else {
        wa = make_float2(w0eff[m & 0x3Fu], w0eff[(m >> 8) & 0x3Fu]);
        wc = make_float2(w0eff[(m >> 16) & 0x3Fu], w0eff[(m >> 24) & 0x3Fu]);
    }
    float2 a = __fmul2_rn(wa, make_float2(c.x, c.y));
    float2 b = __fmul2_rn(wc, make_float2(c.z, c.w));
    a = __ffma2_rn(wx, __fadd2_rn(make_float2(w.x, w.y), make_float2(e.x, e.y)), a);
    b = __ffma2_rn(wx, __fadd2_rn(make_float2(w.z, w.w), make_float2(e.z, e.w)), b);
    a = __ffma2_rn(wy, __fadd2_rn(make_float2(s.x, s.y), make_float2(n.x, n.y)), a);
    b = __ffma2_rn(wy, __fadd2_rn(make_float2(s.z, s.w), make_float2(n.z, n.w)), b);
    a = __ffma2_rn(wb, make_float2(zb, c.x), a);
    b = __ffma2_rn(wb, make_float2(c.y, c.z), b);
    a = __ffma2_rn(wt, make_float2(c.y, c.z), a);
    b = __ffma2_rn(wt, make_float2(c.w, zt), b);
    if (k.decays) {
        const float2 d = make_float2(k.decay, k.decay);
        a = __fmul2_rn(a, d);
        b = __fmul2_rn(b, d);
    }
    float4 v;
    v.x = (m & 0x00000080u) ? fmaxf(a.x, 0.0f) : 0.0f;
    v.y = (m & 0x00008000u) ? fmaxf(a.y, 0.0f) : 0.0f;
    v.z = (m & 0x00800000u) ? fmaxf(b.x, 0.0f) : 0.0f;
    v.w = (m & 0x80000000u) ? fmaxf(b.y, 0.0f) : 0.0f;
    return v;
}

// mask bytes of a 4-voxel group starting at z = k that lie below the void limit zl
__device__ __forceinline__ unsigned zkeep_mask(int zl, int k) {
    const int nk = zl - k;
    return nk >= 4 ? 0xffffffffu : (nk <= 0 ? 0u : (0xffffffffu >> (8 * (4 - nk))));
}

// Non-void voxels of a field set to 0 (the context API's input may hold anything there): afterwards
// both ping-pong buffers satisfy the invariant every step relies on.
__global__ void k_plume_clear(float* __restrict__ Ca, float* __restrict__ Cb, const uint8_t* __restrict__ M, int nx,
                              int ny, int nz, int mz) {
    const long long n = (long long)nx * ny * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long col = i / nz;
        const int k = (int)(i - col * nz);
        if (!(M[col * mz + k] & BD_PM_VOID)) {
            Ca[i] = 0.0f;
            Cb[i] = 0.0f;
        }
    }
}

// ---- k_plume_step: any grid ----------------------------------------------------------------
// One FTCS step. CTA (y tile, x plane); a thread owns the voxels k = tx, tx+32, ... < zlim of one
// (x, y) column (zlim = *zlimit when given, every void voxel lies above it, else nz); only void
// voxels are written (solid voxels stay 0).
__global__ void __launch_bounds__(PM_TZ * PM_TY) k_plume_step(int nx, int ny, int nz, int mz,
                                                              const __grid_constant__ PlumeTab k,
                                                              const float* __restrict__ C, float* __restrict__ Cn,
                                                              const uint8_t* __restrict__ M,
                                                              const int* __restrict__ zlimit) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int j = blockIdx.x * PM_TY + threadIdx.y;
    const int i = blockIdx.y;
    if (j >= ny) return;
    const int plane = ny * nz;
    const int col = i * plane + j * nz;
    const size_t mcol = ((size_t)i * ny + j) * mz;
    for (int z = threadIdx.x; z < zl; z += PM_TZ) {
        const int idx = col + z;
        const unsigned m = __ldg(&M[mcol + z]);
        if (!(m & BD_PM_VOID)) continue;
        if (!(m & BD_PM_UPDATE)) {
            Cn[idx] = 0.0f;
            continue;
        }
        // an updated voxel is never on an outer wall: all six neighbours exist
        Cn[idx] = ftcs1(__ldg(&C[idx]), __ldg(&C[idx - plane]), __ldg(&C[idx + plane]), __ldg(&C[idx - nz]),
                        __ldg(&C[idx + nz]), __ldg(&C[idx - 1]), __ldg(&C[idx + 1]), m, k);
    }
}

// ---- k_plume_direct / k_plume_direct_z: one launch per step --------------------------------
// A CTA is one 32 (z) x 16 (y) tile and marches xc x planes; thread = 4 consecutive z voxels of
// one row, a warp 8 such groups x 4 rows (one 128-byte line per row and load). The thread keeps the
// x-1 / x float4 of its row in registers and loads, per plane, the next plane's float4 and the
// centre plane's y neighbours from the (L2-resident) field beside the plane's mask bytes (one
// 32-bit load): one L2 round trip per plane, at the price of loads a tissue plane does not need. The
// z neighbours come from the neighbouring lanes by shuffle (the tile's edge lanes load them).
// Latency is hidden by the many independent CTAs of a step. Only void voxels are written. Needs
// nz % 4 == 0 and 16-byte aligned fields.
constexpr int PL_BZ = 32;
constexpr int PD_BY = 16;  // rows per CTA (8 * PD_BY threads)
static_assert(PD_BY == kPlumeZRows, "z-list columns follow the direct kernel's y tiles");

__device__ __forceinline__ void store_void(float* dst, float4 v, unsigned vd) {
    if (vd == 0x40404040u) {
        *reinterpret_cast<float4*>(dst) = v;
    } else {
        if (vd & 0x00000040u) dst[0] = v.x;
        if (vd & 0x00004000u) dst[1] = v.y;
        if (vd & 0x00400000u) dst[2] = v.z;
        if (vd & 0x40000000u) dst[3] = v.w;
    }
}

__global__ void __launch_bounds__(8 * PD_BY) k_plume_direct(const float* __restrict__ C, float* __restrict__ Cn,
                                                            const uint8_t* __restrict__ M, int nx, int ny, int nz,
                                                            int mz, int xc, const __grid_constant__ PlumeTab k,
                                                            const int* __restrict__ zlimit) {
    __shared__ float w0s[64];
    if (threadIdx.x < 64) w0s[threadIdx.x] = k.w0eff[threadIdx.x];
    __syncthreads();
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int k0 = blockIdx.x * PL_BZ;
    const int ib = blockIdx.z * xc, ie = min(nx, ib + xc);
    if (k0 >= zl || ib >= ie) return;  // uniform over the CTA
    const int zg = threadIdx.x & 7;
    const int j = blockIdx.y * PD_BY + (threadIdx.x >> 3), z = k0 + 4 * zg;
    const bool act = zl - z > 0 && j < ny;
    const bool in = j < ny && z < nz;
    const unsigned zkeep = zkeep_mask(zl, z);
    const size_t plane = (size_t)ny * nz;
    const size_t mplane = (size_t)ny * mz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    size_t idx = ((size_t)ib * ny + j) * nz + z;
    const uint8_t* mp = M + ((size_t)ib * ny + j) * mz + z;
    float4 cw = in && ib > 0 ? __ldg(reinterpret_cast<const float4*>(C + idx - plane)) : z4;
    float4 cc = in ? __ldg(reinterpret_cast<const float4*>(C + idx)) : z4;
    for (int i = ib; i < ie; ++i, idx += plane, mp += mplane) {
        const unsigned mr = act ? (__ldg(reinterpret_cast<const unsigned*>(mp)) & zkeep) : 0u;
        const float4 ce = in && i + 1 < nx ? __ldg(reinterpret_cast<const float4*>(C + idx + plane)) : z4;
        const float4 cs = in && j > 0 ? __ldg(reinterpret_cast<const float4*>(C + idx - nz)) : z4;
        const float4 cn = in && j + 1 < ny ? __ldg(reinterpret_cast<const float4*>(C + idx + nz)) : z4;
        float eb = 0.0f, et = 0.0f;
        if (zg == 0 && in && z > 0) eb = __ldg(C + idx - 1);
        if (zg == 7 && in && z + 4 < nz) et = __ldg(C + idx + 4);
        const unsigned vd = mr & 0x40404040u;
        if (__any_sync(0xffffffffu, act && vd)) {
            float zb = __shfl_up_sync(0xffffffffu, cc.w, 1, 8);
            float zt = __shfl_down_sync(0xffffffffu, cc.x, 1, 8);
            if (zg == 0) zb = eb;
            if (zg == 7) zt = et;
            const float4 v = ftcs4(cc, cw, ce, cs, cn, zb, zt, mr, k, w0s);
            if (act && vd) store_void(Cn + idx, v, vd);
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

// One unit of the direct kernel: band `band` of column `col` (y tile yt, x chunk xch of xc planes)
// takes the column's live groups 8 band .. 8 band + 7 from its z list instead of 8 consecutive
// groups, so z tiles that are partly tissue cost only their void groups. A lane whose z neighbour
// group is not held by the neighbouring lane loads that neighbour voxel instead of taking it by
// shuffle. Voxels outside the lists are not void and are never written. Uniform over the CTA.
// g: this lane's z group (-2 when the band has no group for the lane); uniform early exit over the
// CTA when the x chunk is empty.
__device__ __forceinline__ void plume_unit_groups(const float* __restrict__ C, float* __restrict__ Cn,
                                                  const uint8_t* __restrict__ M, int nx, int ny, int nz, int mz,
                                                  int xc, const PlumeTab& k, int zl, int g, int yt, int xch,
                                                  const float* w0s) {
    const int ib = xch * xc, ie = min(nx, ib + xc);
    if (ib >= ie) return;
    const int zg = threadIdx.x & 7;
    const int gp = __shfl_up_sync(0xffffffffu, g, 1, 8);
    const int gn = __shfl_down_sync(0xffffffffu, g, 1, 8);
    const bool zb_lane = zg > 0 && gp == g - 1;  // the -z neighbour is the previous lane's last voxel
    const bool zt_lane = zg < 7 && gn == g + 1;  // the +z neighbour is the next lane's first voxel
    const int j = yt * PD_BY + ((threadIdx.x & 127) >> 3), z = 4 * max(g, 0);
    const bool act = g >= 0 && zl - z > 0 && j < ny;
    const bool in = g >= 0 && j < ny && z < nz;
    const unsigned zkeep = zkeep_mask(zl, z);
    // 32-bit element offsets (grids have < 2^31 voxels); rows past the grid load nothing
    const int plane = ny * nz, mplane = ny * mz;
    const int jj = min(j, ny - 1);
    int off = (ib * ny + jj) * nz + z;
    int moff = (ib * ny + jj) * mz + z;
    const bool ys = in && j > 0, yn = in && j + 1 < ny;
    const bool ebl = !zb_lane && in && z > 0, etl = !zt_lane && in && z + 4 < nz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 cw = in && ib > 0 ? __ldg(reinterpret_cast<const float4*>(C + (off - plane))) : z4;
    float4 cc = in ? __ldg(reinterpret_cast<const float4*>(C + off)) : z4;
    for (int i = ib; i < ie; ++i, off += plane, moff += mplane) {
        const unsigned mr = act ? (__ldg(reinterpret_cast<const unsigned*>(M + moff)) & zkeep) : 0u;
        const float4 ce = in && i + 1 < nx ? __ldg(reinterpret_cast<const float4*>(C + (off + plane))) : z4;
        const float4 cs = ys ? __ldg(reinterpret_cast<const float4*>(C + (off - nz))) : z4;
        const float4 cn = yn ? __ldg(reinterpret_cast<const float4*>(C + (off + nz))) : z4;
        const float eb = ebl ? __ldg(C + (off - 1)) : 0.0f;
        const float et = etl ? __ldg(C + (off + 4)) : 0.0f;
        const unsigned vd = mr & 0x40404040u;
        if (__any_sync(0xffffffffu, act && vd)) {
            float zb = __shfl_up_sync(0xffffffffu, cc.w, 1, 8);
            float zt = __shfl_down_sync(0xffffffffu, cc.x, 1, 8);
            if (!zb_lane) zb = eb;
            if (!zt_lane) zt = et;
            const float4 v = ftcs4(cc, cw, ce, cs, cn, zb, zt, mr, k, w0s);
            if (act && vd) store_void(Cn + off, v, vd);
        }
        cw = cc;
        cc = ce;
    }
}

// The unit (column col, band) with its groups read from the column's z list.
__device__ __forceinline__ void plume_direct_unit(const float* __restrict__ C, float* __restrict__ Cn,
                                                  const uint8_t* __restrict__ M, int nx, int ny, int nz, int mz,
                                                  int xc, const PlumeTab& k, int zl, const uint8_t* __restrict__ zlist,
                                                  int n_cols, int col, int yt, int xch, int band, const float* w0s) {
    const int G = (nz + 3) / 4;
    const int cnt = zlist[col];
    const int b0 = band * 8;
    if (b0 >= cnt) return;  // uniform over the CTA
    const int zg = threadIdx.x & 7;
    const int g = b0 + zg < cnt ? (int)zlist[n_cols + col * G + b0 + zg] : -2;
    plume_unit_groups(C, Cn, M, nx, ny, nz, mz, xc, k, zl, g, yt, xch, w0s);
}

// BD_PLUME_KERNEL_DIRECT: grid (bands, y tiles, x chunks); CTAs past a column's live bands exit at once.
__global__ void __launch_bounds__(8 * PD_BY, 9) k_plume_direct_z(const float* __restrict__ C, float* __restrict__ Cn,
                                                                 const uint8_t* __restrict__ M, int nx, int ny,
                                                                 int nz, int mz, int xc,
                                                                 const __grid_constant__ PlumeTab k,
                                                                 const int* __restrict__ zlimit,
                                                                 const uint8_t* __restrict__ zlist) {
    __shared__ float w0s[64];
    if (threadIdx.x < 64) w0s[threadIdx.x] = k.w0eff[threadIdx.x];
    __syncthreads();
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int col = blockIdx.z * gridDim.y + blockIdx.y;
    plume_direct_unit(C, Cn, M, nx, ny, nz, mz, xc, k, zl, zlist, gridDim.y * gridDim.z, col, blockIdx.y, blockIdx.z,
                      blockIdx.x, w0s);
}

// ---- BD_PLUME_KERNEL_COMPACT: the direct kernel over a compact list of live units ------------
// A step's CTAs are dispatched at a limited rate and the step ends with its last CTA, so the step is
// fastest when the live units about fill one wave of resident CTAs: each CTA then runs exactly one
// unit, and no empty CTA is dispatched between working ones. Once per stage the x planes per unit
// (xc) are chosen on the device: per (x plane, y tile) bitmaps of the live z groups give the unit
// count of every candidate xc, and the smallest xc whose count fits the wave (3 % over allowed)
// wins (fewer planes per unit = a shorter CTA). The z list and the unit list are then built for it
// and the step kernel, one wave of CTAs, loops over the units. Region layout (32-bit words, from
// plume_units_offset): [0] unit count, [1] chosen xc, [4 + c - kPlumeXcMin] unit count for xc = c,
// then the bitmaps (nx x y tiles x kPlumeBitWords), then the units: 16 bytes each, {column << 5 |
// band, 0, the band's 8 z-group ids as bytes (0xFF: none)}.
constexpr int kPlumeXcMin = 2, kPlumeXcMax = 12;
constexpr int kPlumeBitWords = 8;  // 32-group words of a bitmap: 4-voxel groups <= 255
constexpr int kPlumeHdrWords = 16;

// bit g of (x plane i, y tile yt): a voxel of group g below the void z-limit in the tile's rows is void
__global__ void __launch_bounds__(256) k_plume_planebits(const uint8_t* __restrict__ M, int nx, int ny, int nz,
                                                         int mz, const int* __restrict__ zlimit,
                                                         unsigned* __restrict__ bits) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int G = (nz + 3) / 4;
    const int yt = blockIdx.x, i = blockIdx.y, n_yt = gridDim.x;
    const int j0 = yt * PD_BY, j1 = min(ny, j0 + PD_BY);
    const int g = threadIdx.x;
    bool live = false;
    if (g < G && zl - 4 * g > 0) {
        const unsigned keep = zkeep_mask(zl, 4 * g);
        for (int j = j0; j < j1 && !live; ++j)
            live = (__ldg(reinterpret_cast<const unsigned*>(M + ((size_t)i * ny + j) * mz + 4 * g)) & keep &
                    0x40404040u) != 0u;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, live);
    if ((threadIdx.x & 31) == 0) bits[((size_t)i * n_yt + yt) * kPlumeBitWords + (threadIdx.x >> 5)] = bal;
}

// live units (bands of 8 live groups) for candidate xc = kPlumeXcMin + blockIdx.x
__global__ void __launch_bounds__(1024) k_plume_unit_counts(const unsigned* __restrict__ bits, int nx, int n_yt,
                                                            int G, unsigned* __restrict__ hdr) {
    __shared__ int tot;
    if (threadIdx.x == 0) tot = 0;
    __syncthreads();
    const int c = kPlumeXcMin + blockIdx.x;
    const int n_xch = (nx + c - 1) / c;
    const int W = (G + 31) / 32;
    int mine = 0;
    for (int p = threadIdx.x; p < n_xch * n_yt; p += blockDim.x) {
        const int xch = p / n_yt, yt = p - xch * n_yt;
        const int ib = xch * c, ie = min(nx, ib + c);
        int live = 0;
        for (int w = 0; w < W; ++w) {
            unsigned o = 0u;
            for (int i = ib; i < ie; ++i) o |= __ldg(&bits[((size_t)i * n_yt + yt) * kPlumeBitWords + w]);
            live += __popc(o);
        }
        mine += (live + 7) / 8;
    }
    atomicAdd(&tot, mine);
    __syncthreads();
    if (threadIdx.x == 0) hdr[4 + blockIdx.x] = (unsigned)tot;
}

// the smallest candidate xc whose unit count fits slot_cap (else the largest)
__global__ void k_plume_pick_xc(unsigned* __restrict__ hdr, int slot_cap) {
    if (threadIdx.x != 0) return;
    int pick = kPlumeXcMax;
    for (int c = kPlumeXcMin; c <= kPlumeXcMax; ++c)
        if ((int)hdr[4 + c - kPlumeXcMin] <= slot_cap) {
            pick = c;
            break;
        }
    hdr[1] = (unsigned)pick;
}

// z lists of the chosen xc's columns from the bitmaps (the layout of k_plume_zlist's lists); grid
// (y tiles, x chunks of the smallest candidate), chunks past the chosen xc's exit
__global__ void __launch_bounds__(256) k_plume_zlist_bits(const unsigned* __restrict__ bits, int nx, int nz,
                                                          const unsigned* __restrict__ hdr,
                                                          uint8_t* __restrict__ zlist) {
    __shared__ int wcount[8];
    const int c = (int)hdr[1];
    const int n_xch = (nx + c - 1) / c;
    const int yt = blockIdx.x, xch = blockIdx.y, n_yt = gridDim.x;
    if (xch >= n_xch) return;  // uniform over the CTA
    const int G = (nz + 3) / 4;
    const int n_cols = n_yt * n_xch;
    const int col = xch * n_yt + yt;
    const int ib = xch * c, ie = min(nx, ib + c);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned o = 0u;
    if (32 * w < G)
        for (int i = ib; i < ie; ++i) o |= __ldg(&bits[((size_t)i * n_yt + yt) * kPlumeBitWords + w]);
    const int g = threadIdx.x;
    const bool live = g < G && ((o >> lane) & 1u);
    const unsigned bal = __ballot_sync(0xffffffffu, live);
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

// the unit list of the chosen xc's columns, in column order: one CTA, a block-wide exclusive scan
// of the bands per column
__global__ void __launch_bounds__(1024) k_plume_units(const uint8_t* __restrict__ zlist, int nx, int n_yt, int G,
                                                      unsigned* __restrict__ hdr, uint4* __restrict__ units) {
    __shared__ int part[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int c = (int)hdr[1];
    const int n_cols = n_yt * ((nx + c - 1) / c);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c0 = 0; c0 < n_cols; c0 += 1024) {
        const int col = c0 + threadIdx.x;
        const int nb = col < n_cols ? (zlist[col] + 7) / 8 : 0;
        int v = nb;  // inclusive scan within the warp
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) part[w] = v;
        __syncthreads();
        if (w == 0) {
            int x = part[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            part[lane] = x;
        }
        __syncthreads();
        const int excl = base + (w > 0 ? part[w - 1] : 0) + v - nb;
        for (int b = 0; b < nb; ++b) {
            // the band's group ids, one byte per lane (0xFF: no group), so that a step's CTA learns
            // its unit with one 16-byte load
            const uint8_t* gl = zlist + n_cols + (size_t)col * G + 8 * b;
            const int n_in = min(8, (int)zlist[col] - 8 * b);
            unsigned lo = 0u, hi = 0u;
            for (int q = 0; q < 8; ++q) {
                const unsigned gq = q < n_in ? (unsigned)gl[q] : 0xFFu;
                if (q < 4) lo |= gq << (8 * q);
                else hi |= gq << (8 * (q - 4));
            }
            units[excl + b] = make_uint4(((unsigned)col << 5) | (unsigned)b, 0u, lo, hi);
        }
        __syncthreads();
        if (threadIdx.x == 1023) base = excl + nb;
        __syncthreads();
    }
    if (threadIdx.x == 0) hdr[0] = (unsigned)base;
}

// One step over the unit list: a wave of CTAs, each running kPlumeUnitsPerCta units at a time, one per
// 128-thread group (the groups share no barrier): group g of CTA b runs units 3b + g, 3b + g + 3 grid,
// ... A step's wave is then dispatched as a third as many CTAs with the same resident threads per SM.
constexpr int kPlumeUnitsPerCta = 3;
__global__ void __launch_bounds__(8 * PD_BY * kPlumeUnitsPerCta, 3) k_plume_direct_c(const float* __restrict__ C, float* __restrict__ Cn,
                                                                 const uint8_t* __restrict__ M, int nx, int ny,
                                                                 int nz, int mz, const __grid_constant__ PlumeTab k,
                                                                 const int* __restrict__ zlimit,
                                                                 const unsigned* __restrict__ hdr,
                                                                 const uint4* __restrict__ units, int n_yt,
                                                                 int unit_cap) {
    // the CTA's first unit record is loaded beside the header (not after the unit count is known):
    // one L2 round trip before the field loads; a record past the count is never used
    const int grp = threadIdx.x >> 7;  // this thread's unit slot within the CTA
    const int u0 = (int)blockIdx.x * kPlumeUnitsPerCta + grp;
    const uint4 r0 = __ldg(&units[min(u0, unit_cap - 1)]);
    const int nu = (int)__ldg(&hdr[0]);
    const int xc = (int)__ldg(&hdr[1]);
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    __shared__ float w0s[64];
    if (threadIdx.x < 64) w0s[threadIdx.x] = k.w0eff[threadIdx.x];
    __syncthreads();
    const int zg = threadIdx.x & 7;
    for (int u = u0; u < nu; u += gridDim.x * kPlumeUnitsPerCta) {
        // column << 5 | band, then the band's 8 group ids
        const uint4 r = u == u0 ? r0 : __ldg(&units[u]);
        const int col = (int)(r.x >> 5);
        const int xch = col / n_yt;
        const unsigned gb = ((zg < 4 ? r.z : r.w) >> (8 * (zg & 3))) & 0xFFu;
        plume_unit_groups(C, Cn, M, nx, ny, nz, mz, xc, k, zl, gb == 0xFFu ? -2 : (int)gb, col - xch * n_yt, xch,
                          w0s);
    }
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

// One wave of the compact step kernel on the current device: resident CTAs per SM x SMs (cached).
static int compact_slots() {
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
    const int d = dev < 64 ? dev : 63;
    int v = cache[d].load();
    if (v > 0) return v;
    int nsm = 0, per = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_plume_direct_c, 8 * PD_BY * kPlumeUnitsPerCta, 0);
    v = std::max(1, nsm) * std::max(1, per) * kPlumeUnitsPerCta;  // units of one wave
    cache[d].store(v);
    return v;
}

// A plume stage: n_substeps x (steps per substep) FTCS steps on the ping-pong pair (Ca, Cb), the
// field in Ca on entry. *in_b = 1 when the result ends in Cb. With full_first (the context API, whose
// non-void voxels may hold anything) the mask covers the whole grid and the non-void voxels of both
// buffers are set to 0 first (every step keeps them 0).
int plume_launch(const BdPlumeParams* p, float* Ca, float* Cb, int n_substeps, const uint8_t* F, int* in_b,
                 cudaStream_t st, const int* zlimit, int full_first, uint8_t* mask) {
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
    const PlumeTab tab = make_plume_tab(c);
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int mz = plume_mask_pitch(nz);
    BD_REQUIRE((long long)nx * ny * mz < (1LL << 31), "plume: grid %dx%dx%d exceeds 2^31 mask bytes", nx, ny, nz);
    const int* zl = full_first ? nullptr : zlimit;
    k_plume_mask<<<dim3((ny + PM_TY - 1) / PM_TY, nx), dim3(PM_TZ, PM_TY), 0, st>>>(nx, ny, nz, mz, F, mask, zl);
    BD_CHECK_LAUNCH("k_plume_mask");
    if (full_first) {
        k_plume_clear<<<grid_for((int64_t)nx * ny * nz, 256), 256, 0, st>>>(Ca, Cb, mask, nx, ny, nz, mz);
        BD_CHECK_LAUNCH("k_plume_clear");
    }
    const long long total = (long long)steps * n_substeps;
    const int kernel = tune_value(BD_TUNE_PLUME_KERNEL);
    const bool vec = nz % 4 == 0;  // the direct kernels move float4 groups
    if (kernel == BD_PLUME_KERNEL_COMPACT && vec && (nz + 3) / 4 <= 255) {
        const int n_yt = (ny + PD_BY - 1) / PD_BY;
        unsigned* hdr = reinterpret_cast<unsigned*>(mask + plume_units_offset(nx, ny, nz));
        unsigned* bits = hdr + kPlumeHdrWords;
        uint4* units = reinterpret_cast<uint4*>(bits + (size_t)nx * n_yt * kPlumeBitWords);
        const int unit_cap = (int)plume_unit_capacity(nx, ny, nz);
        uint8_t* zlist = mask + plume_zlist_offset(nx, ny, nz);
        const int slots = compact_slots();
        k_plume_planebits<<<dim3(n_yt, nx), 256, 0, st>>>(mask, nx, ny, nz, mz, zl, bits);
        k_plume_unit_counts<<<kPlumeXcMax - kPlumeXcMin + 1, 1024, 0, st>>>(bits, nx, n_yt, (nz + 3) / 4, hdr);
        k_plume_pick_xc<<<1, 32, 0, st>>>(hdr, slots + slots * 3 / 100);
        k_plume_zlist_bits<<<dim3(n_yt, (nx + kPlumeXcMin - 1) / kPlumeXcMin), 256, 0, st>>>(bits, nx, nz, hdr, zlist);
        k_plume_units<<<1, 1024, 0, st>>>(zlist, nx, n_yt, (nz + 3) / 4, hdr, units);
        BD_CHECK_LAUNCH("k_plume_units");
        for (long long s = 0; s < total; ++s) {
            const float* in = (s & 1) ? Cb : Ca;
            float* out = (s & 1) ? Ca : Cb;
            k_plume_direct_c<<<slots / kPlumeUnitsPerCta, 8 * PD_BY * kPlumeUnitsPerCta, 0, st>>>(
                in, out, mask, nx, ny, nz, mz, tab, zl, hdr, units, n_yt, unit_cap);
        }
        BD_CHECK_LAUNCH("k_plume_direct_c");
        if (in_b) *in_b = (int)(total & 1);
        return BD_OK;
    }
    const int xc = tune_value(BD_TUNE_PLUME_XC);
    const dim3 dgrid((nz + PL_BZ - 1) / PL_BZ, (ny + PD_BY - 1) / PD_BY, (nx + xc - 1) / xc);
    // live z groups per direct-kernel column, from this stage's mask
    uint8_t* zlist = nullptr;
    if (vec && (nz + 3) / 4 <= 255) {
        zlist = mask + plume_zlist_offset(nx, ny, nz);
        k_plume_zlist<<<dim3((ny + PD_BY - 1) / PD_BY, (nx + xc - 1) / xc), 256, 0, st>>>(mask, nx, ny, nz, mz, xc, zl,
                                                                                          zlist);
        BD_CHECK_LAUNCH("k_plume_zlist");
    }
    for (long long s = 0; s < total; ++s) {
        const float* in = (s & 1) ? Cb : Ca;
        float* out = (s & 1) ? Ca : Cb;
        if (zlist)
            k_plume_direct_z<<<dgrid, 8 * PD_BY, 0, st>>>(in, out, mask, nx, ny, nz, mz, xc, tab, zl, zlist);
        else if (vec)
            k_plume_direct<<<dgrid, 8 * PD_BY, 0, st>>>(in, out, mask, nx, ny, nz, mz, xc, tab, zl);
        else
            k_plume_step<<<dim3((ny + PM_TY - 1) / PM_TY, nx), dim3(PM_TZ, PM_TY), 0, st>>>(nx, ny, nz, mz, tab, in, out,
                                                                                        mask, zl);
    }
    BD_CHECK_LAUNCH("k_plume_step");
    if (in_b) *in_b = (int)(total & 1);
    return BD_OK;
}

// ---- batched stages: several instances' plume steps in one launch per step ------------------
// The instances may differ in diffusivity, so each carries its own weights and step count. They
// are ranked by step count (rank 0 steps longest); a unit of rank r is (r << 27) | (column << 5) |
// band, and the unit list is in (rank, column) order, so the units of step s are a prefix of it:
// those of the ranks that still step. The header holds the unit count [0] and, at [16 + r], the
// units of ranks 0..r; the units follow at word 64.
struct PlumeInstDev {
    float* Ca;
    float* Cb;
    const uint8_t* mask;
    const int* zlimit;
    long long steps;  // FTCS steps of the stage (steps per substep x substeps)
    PlumeTab tab;
};
constexpr int kBatchHdrWords = 64;

__global__ void __launch_bounds__(1024) k_plume_batch_units(const PlumeInstDev* __restrict__ insts, int n,
                                                            int n_cols, size_t zoff, unsigned* __restrict__ hdr) {
    __shared__ int part[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    unsigned* units = hdr + kBatchHdrWords;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int total = n * n_cols;
    for (int c0 = 0; c0 < total; c0 += 1024) {
        const int q = c0 + threadIdx.x;
        int nb = 0, r = 0, col = 0;
        if (q < total) {
            r = q / n_cols;
            col = q - r * n_cols;
            nb = (insts[r].mask[zoff + col] + 7) / 8;
        }
        int v = nb;  // inclusive scan within the warp
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) part[w] = v;
        __syncthreads();
        if (w == 0) {
            int x = part[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            part[lane] = x;
        }
        __syncthreads();
        const int excl = base + (w > 0 ? part[w - 1] : 0) + v - nb;
        for (int b = 0; b < nb; ++b) units[excl + b] = ((unsigned)r << 27) | ((unsigned)col << 5) | (unsigned)b;
        if (q < total && col == n_cols - 1) hdr[16 + r] = (unsigned)(excl + nb);  // units of ranks 0..r
        __syncthreads();
        if (threadIdx.x == 1023) base = excl + nb;
        __syncthreads();
    }
    if (threadIdx.x == 0) hdr[0] = (unsigned)base;
}

// step s of every instance that still steps: a wave of CTAs looping over a prefix of the units. At
// the start every CTA copies each instance's buffers, void z-limit and weights into shared memory,
// so a unit costs the same dependent loads as one of the compact kernel.
constexpr int kBatchMax = 32;
__global__ void __launch_bounds__(8 * PD_BY, 8) k_plume_direct_b(const PlumeInstDev* __restrict__ insts, int n,
                                                                 long long s, int nx, int ny, int nz, int mz, int xc,
                                                                 size_t zoff, const unsigned* __restrict__ hdr,
                                                                 int n_yt) {
    __shared__ float w0s[kBatchMax][64];
    __shared__ float sc[kBatchMax][6];  // wx, wy, wb, wt, decay, decays
    __shared__ const float* cin[kBatchMax];
    __shared__ float* cout[kBatchMax];
    __shared__ const uint8_t* msk[kBatchMax];
    __shared__ int zls[kBatchMax];
    __shared__ int nu_s;
    const int odd = (int)(s & 1);
    for (int q = threadIdx.x; q < n * 64; q += blockDim.x) w0s[q >> 6][q & 63] = insts[q >> 6].tab.w0eff[q & 63];
    if (threadIdx.x < n) {
        const PlumeInstDev& in = insts[threadIdx.x];
        float* t = sc[threadIdx.x];
        t[0] = in.tab.wx;
        t[1] = in.tab.wy;
        t[2] = in.tab.wb;
        t[3] = in.tab.wt;
        t[4] = in.tab.decay;
        t[5] = in.tab.decays ? 1.0f : 0.0f;
        cin[threadIdx.x] = odd ? in.Cb : in.Ca;
        cout[threadIdx.x] = odd ? in.Ca : in.Cb;
        msk[threadIdx.x] = in.mask;
        zls[threadIdx.x] = in.zlimit ? min(max(*in.zlimit, 0), nz) : nz;
    }
    if (threadIdx.x == 0) {
        int r = 0;
        while (r < n && insts[r].steps > s) ++r;
        nu_s = r > 0 ? (int)hdr[16 + r - 1] : 0;
    }
    __syncthreads();
    const int nu = nu_s;
    const unsigned* units = hdr + kBatchHdrWords;
    const int n_cols = n_yt * ((nx + xc - 1) / xc);
    for (int u = blockIdx.x; u < nu; u += gridDim.x) {
        const unsigned v = __ldg(&units[u]);
        const int ri = (int)(v >> 27);
        PlumeTab kt;
        kt.wx = sc[ri][0];
        kt.wy = sc[ri][1];
        kt.wb = sc[ri][2];
        kt.wt = sc[ri][3];
        kt.decay = sc[ri][4];
        kt.decays = sc[ri][5] != 0.0f;
        const int col = (int)((v >> 5) & 0x3FFFFFu);
        const int xch = col / n_yt;
        const uint8_t* M = msk[ri];
        plume_direct_unit(cin[ri], cout[ri], M, nx, ny, nz, mz, xc, kt, zls[ri], M + zoff, n_cols, col,
                          col - xch * n_yt, xch, (int)(v & 31u), w0s[ri]);
    }
}

size_t plume_batch_desc_bytes(int n) { return sizeof(PlumeInstDev) * (size_t)n; }

size_t plume_batch_units_words(int n, int nx, int ny, int nz) {
    const size_t cols = (size_t)nx * ((ny + PD_BY - 1) / PD_BY);
    const size_t bands = ((size_t)(nz + 3) / 4 + 7) / 8;
    return kBatchHdrWords + (size_t)n * cols * bands;
}

static int batch_steps(const PlumeInstHost& q, long long* total, PlumeTab* tab) {
    int steps;
    float dtp, decay;
    int rc = plume_policy_steps(q.params, &steps, &dtp, &decay);
    if (rc) return rc;
    const BdPlumeParams* p = q.params;
    PlumeConst c;
    c.dxy_x = p->D_xy / (p->dx * p->dx);
    c.dxy_y = p->D_xy / (p->dy * p->dy);
    c.dz_z = p->D_z / (p->dz * p->dz);
    c.vz_over_dz = p->vz > 0.0f ? p->vz / p->dz : 0.0f;
    c.dtp = dtp;
    c.decay = decay;
    if (tab) *tab = make_plume_tab(c);
    *total = (long long)steps * q.n_substeps;
    return BD_OK;
}

int plume_batch_prepare(int n, const PlumeInstHost* insts, void* dev, int* order, long long* max_steps) {
    BD_REQUIRE(n >= 1 && n <= kBatchMax, "plume batch: 1..%d instances, got %d", kBatchMax, n);
    std::vector<long long> total(n);
    std::vector<PlumeTab> tabs(n);
    for (int i = 0; i < n; ++i) {
        int rc = batch_steps(insts[i], &total[i], &tabs[i]);
        if (rc) return rc;
        order[i] = i;
    }
    std::stable_sort(order, order + n, [&](int a, int b) { return total[a] > total[b]; });
    std::vector<PlumeInstDev> h(n);
    for (int r = 0; r < n; ++r) {
        const PlumeInstHost& q = insts[order[r]];
        h[r].Ca = q.Ca;
        h[r].Cb = q.Cb;
        h[r].mask = q.mask;
        h[r].zlimit = q.zlimit;
        h[r].steps = total[order[r]];
        h[r].tab = tabs[order[r]];
    }
    *max_steps = total[order[0]];
    BD_CUDA(cudaMemcpy(dev, h.data(), sizeof(PlumeInstDev) * n, cudaMemcpyHostToDevice));
    return BD_OK;
}

int plume_batch_launch(int n, const PlumeInstHost* insts, const int* order, const void* dev, long long max_steps,
                       unsigned* units, cudaStream_t st) {
    const BdPlumeParams* p = insts[0].params;
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int mz = plume_mask_pitch(nz);
    BD_REQUIRE((long long)nx * ny * mz < (1LL << 31), "plume batch: grid exceeds 2^31 mask bytes");
    const int xc = tune_value(BD_TUNE_PLUME_XC);
    const int n_yt = (ny + PD_BY - 1) / PD_BY, n_xch = (nx + xc - 1) / xc;
    const size_t zoff = plume_zlist_offset(nx, ny, nz);
    for (int i = 0; i < n; ++i) {
        const PlumeInstHost& q = insts[i];
        k_plume_mask<<<dim3((ny + PM_TY - 1) / PM_TY, nx), dim3(PM_TZ, PM_TY), 0, st>>>(nx, ny, nz, mz, q.flags, q.mask,
                                                                                       q.zlimit);
        k_plume_zlist<<<dim3(n_yt, n_xch), 256, 0, st>>>(q.mask, nx, ny, nz, mz, xc, q.zlimit, q.mask + zoff);
    }
    BD_CHECK_LAUNCH("k_plume_zlist");
    const PlumeInstDev* d = static_cast<const PlumeInstDev*>(dev);
    k_plume_batch_units<<<1, 1024, 0, st>>>(d, n, n_yt * n_xch, zoff, units);
    BD_CHECK_LAUNCH("k_plume_batch_units");
    static std::atomic<int> per_sm{0};  // resident CTAs per SM of the batched step kernel
    if (per_sm.load() == 0) {
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_plume_direct_b, 8 * PD_BY, 0);
        per_sm.store(std::max(1, v));
    }
    int dev_id = 0, nsm = 0;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id);
    const int slots = std::max(1, nsm) * per_sm.load();
    for (long long s = 0; s < max_steps; ++s)
        k_plume_direct_b<<<slots, 8 * PD_BY, 0, st>>>(d, n, s, nx, ny, nz, mz, xc, zoff, units, n_yt);
    BD_CHECK_LAUNCH("k_plume_direct_b");
    // an instance whose step count is odd ends in its Cb buffer
    const long long nv = (long long)nx * ny * nz;
    for (int i = 0; i < n; ++i) {
        long long total = 0;
        int rc = batch_steps(insts[i], &total, nullptr);
        if (rc) return rc;
        if (total & 1)
            BD_CUDA(cudaMemcpyAsync(insts[i].Ca, insts[i].Cb, sizeof(float) * nv, cudaMemcpyDeviceToDevice, st));
    }
    (void)order;
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
    unsigned char* scratch = nullptr;  // plume neighbourhood bytes, z lists and unit lists
    BD_CUDA(cudaMallocAsync((void**)&scratch, plume_mask_bytes(p->nx, p->ny, p->nz), st));
    const int rc = plume_launch(p, Ca, Cb, n_substeps, F, in_b, st, nullptr, 1, scratch);
    cudaError_t e2 = cudaFreeAsync(scratch, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, "bd_plume_advance");
    if (e2 != cudaSuccess) return cuda_status(e2, "bd_plume_advance: cudaFreeAsync");
    return BD_OK;
}

extern "C" int bd_plume_steps_per_substep(const BdPlumeParams* p, int* n_steps, float* dt_step) {
    BD_REQUIRE(p && n_steps && dt_step, "bd_plume_steps_per_substep: NULL argument");
    float decay;
    return plume_policy_steps(p, n_steps, dt_step, &decay);
}
