// Explicit 7-point bioheat stencil, fused ablation substep and plume transport.
//
// Thermal update (voxel_thermal_3d.py:30-112, voxel_thermal_metal.py:56-134):
//   T' = T + dt (sum_faces k_face (T_nb - T) / d^2 + Q) / rho_cp,
//   k_face = 2 k_c k_n / (k_c + k_n + 1e-12); x/y faces insulated; z faces convective
//   (series half-cell + h_eff, or the Metal fused kernel's -h_eff (T - T_amb)/dz).
// Fused substep (metal_ablation_solver.py:71-191; CPU twin coupled_ablation.py:515-531):
//   + latent-heat plateau (voxel_thermal_3d.py:115-143), Arrhenius damage
//   (coupled_ablation.py:33-40) and first-order char kinetics (coupled_ablation.py:43-58),
//   all pointwise on the trial temperature, so one pass per substep does everything.
// Plume (plume.py:18-80, metal_ablation_solver.py:193-240): FTCS diffusion + upwind drift
//   in the void domain, Neumann at solid walls, Dirichlet 0 on the outer walls.
//
// Layout: z fastest. A CTA owns a 32 (z) x 8 (y) column tile and marches along x (the
// slowest axis), rotating the x-1 / x / x+1 values of T and k through registers, so each
// T and k value is fetched from DRAM once per substep; y/z neighbours come from L1.
#include "common.cuh"
#include "tma.cuh"

#include <algorithm>
#include <cmath>

namespace bd {

constexpr int TZ = 32, TY = 8;

struct Geo {
    int nx, ny, nz, ni;
    float idx2, idy2, idz2, dz, h_eff, t_amb, dt;
};

// Harmonic face conductance 2 k_c k_n / (k_c + k_n + 1e-12). The quotient uses the fast
// reciprocal path (<= 2 ulp): six precise IEEE divisions per voxel made the stencil
// instruction-bound, while the parity bar on T is 1e-4 relative.
__device__ __forceinline__ float kface(float a, float b) { return __fdividef(2.0f * a * b, a + b + 1e-12f); }

template <int BC>
__device__ __forceinline__ float zwall_flux(float Tc, float kc, const Geo& g) {
    if (BC == BD_BC_SERIES) {
        // voxel_thermal_3d.py:97,105
        return g.h_eff > 0.0f
                   ? (g.t_amb - Tc) / (g.dz * (0.5f * g.dz / fmaxf(kc, 1e-30f) + 1.0f / fmaxf(g.h_eff, 1e-30f)))
                   : 0.0f;
    } else {
        // metal_ablation_solver.py:141,150
        return -g.h_eff * (Tc - g.t_amb) / g.dz;
    }
}

struct AblConst {
    float t_abl, t_void, q_scale;
    float arr_A, arr_EaR, char_A, char_EaR;
    int zero_src_in_ablated, is_active;
};

// MODE 0: thermal only. MODE 1: fused ablation substep.
// Each thread marches NI x-planes of one (y, z) column; T and k of plane i+2 are prefetched
// while plane i is computed so two DRAM round trips are in flight per thread.
template <int MODE, int BC, bool ARR, bool CHAR>
__global__ void __launch_bounds__(TZ * TY) k_substep(Geo g, AblConst c, const float* __restrict__ T,
                                                     float* __restrict__ Tn, const float* __restrict__ src,
                                                     const float* __restrict__ K, const float* __restrict__ R,
                                                     const uint8_t* __restrict__ F, float* __restrict__ H,
                                                     float* __restrict__ Om, float* __restrict__ Chi) {
    const int k = blockIdx.x * TZ + threadIdx.x;
    const int j = blockIdx.y * TY + threadIdx.y;
    if (k >= g.nz || j >= g.ny) return;
    const int i0 = blockIdx.z * g.ni;
    const int i1 = min(i0 + g.ni, g.nx);
    const int plane = g.ny * g.nz;
    const int base = j * g.nz + k;

    int idx = i0 * plane + base;
    float Tm = 0.0f, km = 0.0f, Tp = 0.0f, kp = 0.0f;
    float Tc = __ldg(&T[idx]), kc = __ldg(&K[idx]);
    if (i0 > 0) { Tm = __ldg(&T[idx - plane]); km = __ldg(&K[idx - plane]); }
    if (i0 + 1 < g.nx) { Tp = __ldg(&T[idx + plane]); kp = __ldg(&K[idx + plane]); }

    for (int i = i0; i < i1; ++i, idx += plane) {
        // prefetch plane i+2 (the x+1 neighbour of the next iteration)
        float Tq = 0.0f, kq = 0.0f;
        if (i + 2 < g.nx && i + 1 < i1) { Tq = __ldg(&T[idx + 2 * plane]); kq = __ldg(&K[idx + 2 * plane]); }
        const float rho = __ldg(&R[idx]);
        uint8_t f = 0;
        if (MODE == 1) f = __ldg(&F[idx]);
        float q = 0.0f;
        if (c.is_active) q = __ldg(&src[idx]);

        const bool has_e = (i + 1 < g.nx);
        float fw = (i > 0) ? kface(kc, km) * (Tm - Tc) * g.idx2 : 0.0f;
        float fe = has_e ? kface(kc, kp) * (Tp - Tc) * g.idx2 : 0.0f;
        float fs = 0.0f, fn = 0.0f, ft, fb;
        if (j > 0)        fs = kface(kc, __ldg(&K[idx - g.nz])) * (__ldg(&T[idx - g.nz]) - Tc) * g.idy2;
        if (j + 1 < g.ny) fn = kface(kc, __ldg(&K[idx + g.nz])) * (__ldg(&T[idx + g.nz]) - Tc) * g.idy2;
        if (k > 0)        ft = kface(kc, __ldg(&K[idx - 1])) * (__ldg(&T[idx - 1]) - Tc) * g.idz2;
        else              ft = zwall_flux<BC>(Tc, kc, g);
        if (k + 1 < g.nz) fb = kface(kc, __ldg(&K[idx + 1])) * (__ldg(&T[idx + 1]) - Tc) * g.idz2;
        else              fb = zwall_flux<BC>(Tc, kc, g);
        const float div = fw + fe + fs + fn + ft + fb;

        const float cap = fmaxf(rho, 1e-12f);
        q *= c.q_scale;
        if (MODE == 1 && c.zero_src_in_ablated && (f & BD_FLAG_ABLATED)) q = 0.0f;
        float Tt = Tc + __fdividef(g.dt * (div + q), cap);

        if (MODE == 1) {
            const bool abl = (f & BD_FLAG_ABLATED) != 0;
            const bool dry = (f & BD_FLAG_DRY) != 0;
            if (abl) {
                if (Tt > c.t_void) Tt = c.t_void;
            } else if (!dry) {
                float h = H[idx];
                if (Tt > c.t_abl) {
                    h += (Tt - c.t_abl) * rho;
                    Tt = c.t_abl;
                    H[idx] = h;
                } else if (h > 0.0f) {
                    float rel = fminf(h, (c.t_abl - Tt) * rho);
                    H[idx] = h - rel;
                    Tt = Tt + rel / rho;
                }
            }
            if (ARR && !abl) Om[idx] += g.dt * c.arr_A * expf(-c.arr_EaR / (Tt + 273.15f));
            if (CHAR && dry && !abl) {
                float rate = c.char_A * expf(-c.char_EaR / (Tt + 273.15f));
                float x = Chi[idx];
                Chi[idx] = 1.0f - (1.0f - x) * expf(-rate * g.dt);
            }
        }
        Tn[idx] = Tt;
        Tm = Tc; km = kc; Tc = Tp; kc = kp; Tp = Tq; kp = kq;
    }
}

// TMA-staged fused substep: same arithmetic as k_substep, but a CTA owns a 32 (z) x 16 (y) tile
// and marches a chunk of x planes; T and k tiles of each plane (1-voxel y halo, 4-voxel z halo)
// stream through a 4-stage shared-memory ring filled by the TMA engine, and the per-voxel fields of
// the next plane (rho_cp, source, flags, H) are fetched into registers one plane ahead.
constexpr int ST_BZ = 32, ST_BY = 16, ST_PZ = ST_BZ + 8, ST_PY = ST_BY + 2, ST_STAGES = 4;
constexpr unsigned ST_TILE_BYTES = ST_PZ * ST_PY * sizeof(float);
constexpr int ST_STRIDE = ((ST_PZ * ST_PY * (int)sizeof(float) + 127) / 128) * 128 / (int)sizeof(float);
static_assert(ST_STRIDE * sizeof(float) % 128 == 0, "stage stride must keep 128-byte alignment");

template <int MODE, int BC, bool ARR, bool CHAR>
__global__ void __launch_bounds__(TZ * TY) k_substep_tma(const __grid_constant__ CUtensorMap t_map,
                                                         const __grid_constant__ CUtensorMap k_map, Geo g,
                                                         AblConst c, float* __restrict__ Tn,
                                                         const float* __restrict__ src, const float* __restrict__ R,
                                                         const uint8_t* __restrict__ F, float* __restrict__ H,
                                                         float* __restrict__ Om, float* __restrict__ Chi,
                                                         int xc, int* __restrict__ err) {
    __shared__ __align__(128) float ringT[ST_STAGES][ST_STRIDE];
    __shared__ __align__(128) float ringK[ST_STAGES][ST_STRIDE];
    __shared__ __align__(8) unsigned long long bar[ST_STAGES];
    const int k0 = blockIdx.x * ST_BZ;
    const int j0 = blockIdx.y * ST_BY;
    const int ib = blockIdx.z * xc;
    const int ie = min(g.nx, ib + xc);
    if (ib >= ie) return;
    const int tid = threadIdx.y * TZ + threadIdx.x;
    if (tid == 0) {
        for (int q = 0; q < ST_STAGES; ++q) mbar_init(&bar[q], 1);
        mbar_init_fence();
    }
    __syncthreads();
    const int nplanes = ie - ib + 2;
    if (tid == 0) {
        for (int q = 0; q < ST_STAGES && q < nplanes; ++q) {
            mbar_expect_tx(&bar[q], 2 * ST_TILE_BYTES);
            tma_load_3d(ringT[q], &t_map, k0 - 4, j0 - 1, ib - 1 + q, &bar[q]);
            tma_load_3d(ringK[q], &k_map, k0 - 4, j0 - 1, ib - 1 + q, &bar[q]);
        }
    }
    const int plane = g.ny * g.nz;
    const int k = k0 + threadIdx.x;
    const int jr[2] = {j0 + (int)threadIdx.y, j0 + (int)threadIdx.y + TY};
    const bool rowok[2] = {k < g.nz && jr[0] < g.ny, k < g.nz && jr[1] < g.ny};
    float rho_n[2] = {0.f, 0.f}, q_n[2] = {0.f, 0.f}, h_n[2] = {0.f, 0.f};
    uint8_t f_n[2] = {0, 0};
#pragma unroll
    for (int r = 0; r < 2; ++r)
        if (rowok[r]) {
            const int idx = ib * plane + jr[r] * g.nz + k;
            rho_n[r] = __ldg(&R[idx]);
            if (c.is_active) q_n[r] = __ldg(&src[idx]);
            if (MODE == 1) { f_n[r] = __ldg(&F[idx]); h_n[r] = H[idx]; }
        }
    bool ok = mbar_wait(&bar[0], 0);
    ok = mbar_wait(&bar[1], 0) && ok;
    for (int i = ib; i < ie; ++i) {
        const int q = i - ib + 1;
        float rho_c[2], q_c[2], h_c[2];
        uint8_t f_c[2];
#pragma unroll
        for (int r = 0; r < 2; ++r) { rho_c[r] = rho_n[r]; q_c[r] = q_n[r]; h_c[r] = h_n[r]; f_c[r] = f_n[r]; }
        if (i + 1 < ie) {
#pragma unroll
            for (int r = 0; r < 2; ++r)
                if (rowok[r]) {
                    const int idx = (i + 1) * plane + jr[r] * g.nz + k;
                    rho_n[r] = __ldg(&R[idx]);
                    if (c.is_active) q_n[r] = __ldg(&src[idx]);
                    if (MODE == 1) { f_n[r] = __ldg(&F[idx]); h_n[r] = H[idx]; }
                }
        }
        ok = mbar_wait(&bar[(q + 1) % ST_STAGES], ((q + 1) / ST_STAGES) & 1) && ok;
        const float* Tm = ringT[(q - 1) % ST_STAGES];
        const float* Tc_ = ringT[q % ST_STAGES];
        const float* Tp = ringT[(q + 1) % ST_STAGES];
        const float* Km = ringK[(q - 1) % ST_STAGES];
        const float* Kc = ringK[q % ST_STAGES];
        const float* Kp = ringK[(q + 1) % ST_STAGES];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            if (!rowok[r]) continue;
            const int j = jr[r];
            const int jy = j - j0;
            const int idx = i * plane + j * g.nz + k;
            const int t = (jy + 1) * ST_PZ + threadIdx.x + 4;
            const float Tc = Tc_[t], kc = Kc[t];
            const float fw = (i > 0) ? kface(kc, Km[t]) * (Tm[t] - Tc) * g.idx2 : 0.0f;
            const float fe = (i + 1 < g.nx) ? kface(kc, Kp[t]) * (Tp[t] - Tc) * g.idx2 : 0.0f;
            const float fs = (j > 0) ? kface(kc, Kc[t - ST_PZ]) * (Tc_[t - ST_PZ] - Tc) * g.idy2 : 0.0f;
            const float fn = (j + 1 < g.ny) ? kface(kc, Kc[t + ST_PZ]) * (Tc_[t + ST_PZ] - Tc) * g.idy2 : 0.0f;
            const float ft = (k > 0) ? kface(kc, Kc[t - 1]) * (Tc_[t - 1] - Tc) * g.idz2 : zwall_flux<BC>(Tc, kc, g);
            const float fb = (k + 1 < g.nz) ? kface(kc, Kc[t + 1]) * (Tc_[t + 1] - Tc) * g.idz2
                                            : zwall_flux<BC>(Tc, kc, g);
            const float div = fw + fe + fs + fn + ft + fb;
            const float rho = rho_c[r];
            const float cap = fmaxf(rho, 1e-12f);
            const uint8_t f = f_c[r];
            float qv = q_c[r] * c.q_scale;
            if (MODE == 1 && c.zero_src_in_ablated && (f & BD_FLAG_ABLATED)) qv = 0.0f;
            if (!c.is_active) qv = 0.0f;
            float Tt = Tc + __fdividef(g.dt * (div + qv), cap);
            if (MODE == 1) {
                const bool abl = (f & BD_FLAG_ABLATED) != 0;
                const bool dry = (f & BD_FLAG_DRY) != 0;
                if (abl) {
                    if (Tt > c.t_void) Tt = c.t_void;
                } else if (!dry) {
                    const float h = h_c[r];
                    if (Tt > c.t_abl) {
                        H[idx] = h + (Tt - c.t_abl) * rho;
                        Tt = c.t_abl;
                    } else if (h > 0.0f) {
                        const float rel = fminf(h, (c.t_abl - Tt) * rho);
                        H[idx] = h - rel;
                        Tt = Tt + rel / rho;
                    }
                }
                if (ARR && !abl) Om[idx] += g.dt * c.arr_A * expf(-c.arr_EaR / (Tt + 273.15f));
                if (CHAR && dry && !abl) {
                    const float rate = c.char_A * expf(-c.char_EaR / (Tt + 273.15f));
                    const float x = Chi[idx];
                    Chi[idx] = 1.0f - (1.0f - x) * expf(-rate * g.dt);
                }
            }
            Tn[idx] = Tt;
        }
        __syncthreads();  // every thread is done with plane i-1's stage
        if (tid == 0 && q + 3 < nplanes) {
            const int s = (q + 3) % ST_STAGES;
            fence_proxy_async_smem();
            mbar_expect_tx(&bar[s], 2 * ST_TILE_BYTES);
            tma_load_3d(ringT[s], &t_map, k0 - 4, j0 - 1, i + 3, &bar[s]);
            tma_load_3d(ringK[s], &k_map, k0 - 4, j0 - 1, i + 3, &bar[s]);
        }
    }
    if (!ok) {
        atomicExch(err, 1);
        for (int q = 0; q < ST_STAGES; ++q) {
            const int last = nplanes - 1 - ((nplanes - 1 - q) % ST_STAGES + ST_STAGES) % ST_STAGES;
            if (last >= 0) mbar_wait(&bar[q], (last / ST_STAGES) & 1);
        }
    }
}

struct PlumeConst {
    float dxy_x, dxy_y, dz_z;  // D_xy*idx2, D_xy*idy2, D_z*idz2
    float vz_over_dz, dtp, decay;
};

// Plume neighbourhood byte per voxel, rebuilt whenever the void domain changes (epoch end); the
// bytes of one (x, y) column start every mz = plume_mask_pitch(nz) bytes (16-byte rows for TMA):
//   bit 6: voxel is void            bit 7: voxel is void and not on an outer wall (FTCS update)
//   bits 0-5: -x +x -y +y -z +z neighbour is void (otherwise its value is replaced by the centre,
//   the zero-flux wall of plume.py:61-71)
#define BD_PM_VOID 0x40u
#define BD_PM_UPDATE 0x80u
__global__ void k_plume_mask(int nx, int ny, int nz, int mz, const uint8_t* __restrict__ F,
                             uint8_t* __restrict__ M, const int* __restrict__ zlimit) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int j = blockIdx.x * TY + threadIdx.y;
    const int i = blockIdx.y;
    if (j >= ny) return;
    const int plane = ny * nz;
    const bool xy_interior = (i > 0 && i < nx - 1 && j > 0 && j < ny - 1);
    const int col = i * plane + j * nz;
    const size_t mcol = ((size_t)i * ny + j) * mz;
    for (int k = threadIdx.x; k < zl; k += TZ) {
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

// One FTCS plume step (plume.py:46-80). CTA (y tile, x plane); a thread owns the voxels
// k = tx, tx+32, ... < zlim of one (x, y) column, zlim = *zlimit when given (every void voxel
// lies above it) else nz. The neighbourhood comes from the mask byte; the six neighbour values
// are loaded unconditionally and selected, so no load depends on another. Non-void voxels are
// written (as 0) only when full_write is set: the engine keeps them 0 in both ping-pong
// buffers, so a step touches only the void domain plus one mask byte per voxel.
__global__ void __launch_bounds__(TZ * TY) k_plume_step(int nx, int ny, int nz, int mz, PlumeConst c,
                                                        const float* __restrict__ C, float* __restrict__ Cn,
                                                        const uint8_t* __restrict__ M,
                                                        const int* __restrict__ zlimit, int full_write) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int j = blockIdx.x * TY + threadIdx.y;
    const int i = blockIdx.y;
    if (j >= ny) return;
    const int plane = ny * nz;
    const int col = i * plane + j * nz;
    const size_t mcol = ((size_t)i * ny + j) * mz;
    for (int k = threadIdx.x; k < zl; k += TZ) {
        const int idx = col + k;
        const uint8_t m = __ldg(&M[mcol + k]);
        if (!(m & BD_PM_UPDATE)) {
            if ((m & BD_PM_VOID) || full_write) Cn[idx] = 0.0f;
            continue;
        }
        const float c0 = __ldg(&C[idx]);
        const float cw = __ldg(&C[idx - plane]), ce = __ldg(&C[idx + plane]);
        const float cs = __ldg(&C[idx - nz]), cn = __ldg(&C[idx + nz]);
        const float cb = __ldg(&C[idx - 1]), ct = __ldg(&C[idx + 1]);
        const float w = (m & 0x01) ? cw : c0;
        const float e = (m & 0x02) ? ce : c0;
        const float sx = (m & 0x04) ? cs : c0;
        const float nn = (m & 0x08) ? cn : c0;
        const float b = (m & 0x10) ? cb : c0;
        const float t = (m & 0x20) ? ct : c0;
        const float diff = c.dxy_x * (w - 2.0f * c0 + e) + c.dxy_y * (sx - 2.0f * c0 + nn) +
                           c.dz_z * (b - 2.0f * c0 + t);
        const float adv = -c.vz_over_dz * (c0 - t);
        const float v = (c0 + c.dtp * (diff + adv)) * c.decay;
        Cn[idx] = fmaxf(v, 0.0f);
    }
}

// TMA-staged plume step: a CTA owns a 32 (z) x 16 (y) column tile and marches a chunk of x
// planes. Each plane's tile with a one-voxel y halo and a four-voxel z halo (40 x 18 floats, the
// z start kept 16-byte aligned) is copied into a 6-stage shared-memory ring by the TMA engine,
// four planes ahead of the one being computed, so every neighbour read comes from shared memory.
// A thread owns 4 y rows of one z lane (128 threads per CTA) and one thread waits on the copies:
// branches, barriers and barrier polls (a narrow pipe on sm_100) are paid once per plane for four
// voxels per thread instead of two.
constexpr int PL_BZ = 32, PL_BY = 16, PL_PZ = PL_BZ + 8, PL_PY = PL_BY + 2, PL_STAGES = 6;
constexpr int PL_TY = 4, PL_RY = PL_BY / PL_TY;
constexpr unsigned PL_TILE_BYTES = PL_PZ * PL_PY * sizeof(float);
// each stage starts on a 128-byte boundary (TMA shared-memory destination alignment)
constexpr int PL_STRIDE = ((PL_PZ * PL_PY * (int)sizeof(float) + 127) / 128) * 128 / (int)sizeof(float);
static_assert(PL_STRIDE * sizeof(float) % 128 == 0, "stage stride must keep 128-byte alignment");
static_assert(PL_STRIDE >= PL_PZ * PL_PY, "stage too small");

__global__ void __launch_bounds__(TZ * PL_TY) k_plume_step_tma(const __grid_constant__ CUtensorMap in_map,
                                                               float* __restrict__ Cn, const uint8_t* __restrict__ M,
                                                               int nx, int ny, int nz, int mz, int xc, PlumeConst c,
                                                               const int* __restrict__ zlimit, int full_write,
                                                               int* __restrict__ err) {
    __shared__ __align__(128) float ring[PL_STAGES][PL_STRIDE];
    __shared__ __align__(8) unsigned long long bar[PL_STAGES];
    __shared__ int s_fail;
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int k0 = blockIdx.x * PL_BZ;
    const int j0 = blockIdx.y * PL_BY;
    const int ib = blockIdx.z * xc;
    const int ie = min(nx, ib + xc);
    if (k0 >= zl || ib >= ie) return;  // uniform over the CTA
    const int tid = threadIdx.y * TZ + threadIdx.x;
    const int nplanes = ie - ib + 2;  // planes ib-1 .. ie; load index q = plane - (ib - 1)
    if (tid == 0) {
        for (int q = 0; q < PL_STAGES; ++q) mbar_init(&bar[q], 1);
        mbar_init_fence();
        s_fail = 0;
        // loads 0 .. PL_STAGES-2 now; load q + PL_STAGES - 2 is issued at iteration q
        for (int q = 0; q < PL_STAGES - 1 && q < nplanes; ++q) {
            mbar_expect_tx(&bar[q], PL_TILE_BYTES);
            tma_load_3d(ring[q], &in_map, k0 - 4, j0 - 1, ib - 1 + q, &bar[q]);
        }
        if (!mbar_wait(&bar[0], 0) || !mbar_wait(&bar[1], 0)) s_fail = 1;
    }
    // Folded FTCS weights: C' = decay * (w0 c0 + wx (cw+ce) + wy (cs+cn) + wb cb + wt ct),
    // the same update as plume.py:73-79 with the products distributed.
    const float wx = c.dtp * c.dxy_x, wy = c.dtp * c.dxy_y, wb = c.dtp * c.dz_z;
    const float wt = wb + c.dtp * c.vz_over_dz;
    const float w0 = 1.0f - 2.0f * (wx + wy + wb) - c.dtp * c.vz_over_dz;
    const int plane = ny * nz;
    const int k = k0 + threadIdx.x;
    const bool kin = k < zl;
    bool act[PL_RY];
    uint8_t m[PL_RY];
#pragma unroll
    for (int r = 0; r < PL_RY; ++r) {
        const int j = j0 + threadIdx.y + r * PL_TY;
        act[r] = kin && j < ny;
        m[r] = act[r] ? __ldg(&M[((size_t)ib * ny + j) * mz + k]) : 0;   // next plane's bytes fetched a plane ahead
    }
    for (int i = ib; i < ie; ++i) {
        const int q = i - ib + 1;
        uint8_t nm[PL_RY];
#pragma unroll
        for (int r = 0; r < PL_RY; ++r)
            nm[r] = (act[r] && i + 1 < ie) ? __ldg(&M[((size_t)(i + 1) * ny + j0 + threadIdx.y + r * PL_TY) * mz + k])
                                           : 0;
        if (tid == 0 && !s_fail && !mbar_wait(&bar[(q + 1) % PL_STAGES], ((q + 1) / PL_STAGES) & 1)) s_fail = 1;
        __syncthreads();  // load q+1 landed (seen by thread 0); every thread is done with plane i-2's stage
        if (tid == 0 && q + PL_STAGES - 2 < nplanes) {
            const int sl = (q + PL_STAGES - 2) % PL_STAGES;
            fence_proxy_async_smem();
            mbar_expect_tx(&bar[sl], PL_TILE_BYTES);
            tma_load_3d(ring[sl], &in_map, k0 - 4, j0 - 1, ib - 1 + q + PL_STAGES - 2, &bar[sl]);
        }
        const float* tm = ring[(q - 1) % PL_STAGES];
        const float* tc = ring[q % PL_STAGES];
        const float* tp = ring[(q + 1) % PL_STAGES];
#pragma unroll
        for (int r = 0; r < PL_RY; ++r) {
            // branch-free: every lane evaluates the stencil (its tile indices are always inside the
            // shared-memory stage), the mask byte selects neighbours and the result, and a single
            // predicated store writes void voxels only
            const uint8_t mr = m[r];
            const int jy = threadIdx.y + r * PL_TY;
            const int t = (jy + 1) * PL_PZ + threadIdx.x + 4;
            const float c0 = tc[t];
            const float w = (mr & 0x01) ? tm[t] : c0;
            const float e = (mr & 0x02) ? tp[t] : c0;
            const float sx = (mr & 0x04) ? tc[t - PL_PZ] : c0;
            const float nn = (mr & 0x08) ? tc[t + PL_PZ] : c0;
            const float b = (mr & 0x10) ? tc[t - 1] : c0;
            const float tt = (mr & 0x20) ? tc[t + 1] : c0;
            float v = fmaxf((w0 * c0 + wx * (w + e) + wy * (sx + nn) + wb * b + wt * tt) * c.decay, 0.0f);
            v = (mr & BD_PM_UPDATE) ? v : 0.0f;
            if (act[r] && ((mr & BD_PM_VOID) || full_write)) Cn[i * plane + (j0 + jy) * nz + k] = v;
            m[r] = nm[r];
        }
    }
    __syncthreads();
    if (tid == 0 && s_fail) {
        atomicExch(err, 1);
        // drain: every copy issued gets a bounded chance to land before the CTA exits
        const int last = min(nplanes, nplanes - 2 + PL_STAGES - 1);
        for (int q = max(0, last - PL_STAGES); q < last; ++q) mbar_wait(&bar[q % PL_STAGES], (q / PL_STAGES) & 1);
    }
}

// Persistent x-marching plume step. A tile is 32 (z) x 32 (y) voxels and a CTA has 8 consumer
// warps, one per 4-voxel z group; lane l of a warp owns row l of the tile, so a thread holds one
// float4 (4 consecutive z voxels) and a warp's 32 rows share their z range: whether its voxels
// are tissue, bulk void or void next to a wall is (almost always) uniform over the warp. Three
// warp-uniform paths follow: no void voxel (nothing to do), every updated voxel with all six
// neighbours void (the FTCS expression with no neighbour selects; outer-wall voxels, void but not
// updated, take 0), and the general path with the zero-flux neighbour selects. All three evaluate the same expression per voxel, so the result
// is bit-identical to the scalar kernel. A thread marches its row along x keeping the x-1 / x /
// x+1 float4 in registers; the y and z neighbours and the mask bytes come from the centre plane.
// The work is the columns (z tile, y tile) above the void limit times their nx planes, laid end
// to end and cut into gridDim.x equal runs (one or two column segments per CTA, the x halo paid
// once per segment). A producer warp streams each segment's planes ib-1 .. ie, PB planes per
// copy (the concentration planes with a 1-voxel y and 4 / 8-voxel z halo, 44 floats wide so that
// the 32 rows a warp reads fall in distinct banks, plus the planes' 32 x 32 mask bytes, on one
// mbarrier) through a PX_STAGES ring; consumer warps wait on a stage's full barrier and release
// it on its empty barrier once its last plane has been a centre. An mbarrier round trip costs a
// few hundred cycles, comparable to the arithmetic of one 32 x 32 plane, hence several planes
// per stage. Needs nz % 4 == 0. A store writes the whole float4 when all four voxels are void
// (or full_write), else only the void ones.
constexpr int PX_STAGES = 4;  // power of two
constexpr int PX_NW = 8, PX_THREADS = 32 * (PX_NW + 1);
constexpr int PX_PZ = 44, PX_BY = 32, PX_PY = PX_BY + 2;
constexpr unsigned PX_PLANE = PX_PZ * PX_PY * sizeof(float);  // one concentration plane of a stage
constexpr unsigned PX_MPLANE = PL_BZ * PX_BY;                  // one mask plane
static_assert(PX_PZ % 4 == 0 && PX_PZ >= PL_BZ + 5, "z box must hold the tile, both z neighbours, 16-byte rows");
static_assert(PX_PLANE % 16 == 0 && PX_MPLANE % 16 == 0, "planes must keep 16-byte alignment");
template <int PB>
struct PlumeXM {
    static constexpr unsigned C_BYTES = PB * PX_PLANE;
    static constexpr unsigned M_OFF = (C_BYTES + 127) / 128 * 128;
    static constexpr unsigned M_BYTES = PB * PX_MPLANE;
    static constexpr unsigned STAGE = (M_OFF + M_BYTES + 127) / 128 * 128;
    static constexpr unsigned SMEM = PX_STAGES * STAGE;  // dynamic shared memory per CTA
};

// A CTA's run of planes [s0, s1) over the columns laid end to end (column = z tile fastest, then
// y tile; nx planes each), walked as segments (k0, j0, ib, ie) that each stay in one column.
struct PlumeRun {
    int n_kt, by, nx;  // z tiles, y stride of the tiles, x planes per column
    long long s0, s1;
    // compacted sequence (k_plume_xm): column c contributes only its planes x0[c] .. x0[c] + len - 1
    // that hold void voxels, at positions pre[c] .. pre[c+1] - 1; nullptr: every column, nx planes
    const int* pre = nullptr;
    const int* x0 = nullptr;
    int n_cols = 0;
    __device__ __forceinline__ int4 segment(long long pos) const {
        if (pre == nullptr) {
            const int col = (int)(pos / nx), ib = (int)(pos - (long long)col * nx);
            const int ie = (int)min((long long)nx, ib + (s1 - pos));
            return make_int4((col % n_kt) * PL_BZ, (col / n_kt) * by, ib, ie);
        }
        int lo = 0, hi = n_cols - 1;  // the last column starting at or before pos (skips empty ones)
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pre[mid] <= pos) lo = mid; else hi = mid - 1;
        }
        const int ib = x0[lo] + (int)(pos - pre[lo]);
        const int ie = (int)min((long long)(x0[lo] + pre[lo + 1] - pre[lo]), ib + (s1 - pos));
        return make_int4((lo % n_kt) * PL_BZ, (lo / n_kt) * by, ib, ie);
    }
};

// Void x-extent of every (z tile, y tile) column of k_plume_xm, from this stage's mask (voxels at
// or below the void limit are not void). ext = xmin | xmax | prefix, see plume_mask_bytes.
__global__ void k_plume_extent_init(int* __restrict__ ext) {
    for (int i = threadIdx.x; i < kPlumeMaxCols; i += blockDim.x) {
        ext[i] = INT_MAX;
        ext[kPlumeMaxCols + i] = -1;
    }
}

// block (x, y tile): which z tiles of the plane tile hold a void voxel
__global__ void __launch_bounds__(256) k_plume_extent(const uint8_t* __restrict__ M, int nx, int ny, int nz, int mz,
                                                      const int* __restrict__ zlimit, int* __restrict__ ext) {
    __shared__ unsigned long long s_bits;
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int n_kt = (zl + PL_BZ - 1) / PL_BZ;
    const int x = blockIdx.x, jt = blockIdx.y;
    if (threadIdx.x == 0) s_bits = 0ull;
    __syncthreads();
    unsigned long long bits = 0ull;
    for (int i = threadIdx.x; i < PX_BY * zl; i += blockDim.x) {
        const int r = i / zl, z = i - r * zl, j = jt * PX_BY + r;
        if (j < ny && (M[((size_t)x * ny + j) * mz + z] & BD_PM_VOID)) bits |= 1ull << (z / PL_BZ);
    }
    if (bits) atomicOr(&s_bits, bits);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int kt = 0; kt < n_kt; ++kt)
            if (s_bits & (1ull << kt)) {
                atomicMin(&ext[jt * n_kt + kt], x);
                atomicMax(&ext[kPlumeMaxCols + jt * n_kt + kt], x);
            }
    }
}

// one CTA: column lengths -> exclusive prefix (prefix[n_cols] = all planes); empty columns get x0 = 0
__global__ void __launch_bounds__(1024) k_plume_runs(int* __restrict__ ext, int ny, int nz,
                                                     const int* __restrict__ zlimit) {
    __shared__ int wsum[32];
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int n_cols = ((zl + PL_BZ - 1) / PL_BZ) * ((ny + PX_BY - 1) / PX_BY);
    const int c = threadIdx.x, lane = c & 31, warp = c >> 5;
    int len = 0;
    if (c < n_cols) {
        const int lo = ext[c], hi = ext[kPlumeMaxCols + c];
        len = hi >= lo ? hi - lo + 1 : 0;
        if (len == 0) ext[c] = 0;
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    const int before = (warp > 0 ? wsum[warp - 1] : 0) + incl - len;
    int* pre = ext + 2 * kPlumeMaxCols;
    if (c < n_cols) pre[c] = before;
    if (c == n_cols - 1) pre[n_cols] = before + len;
    if (n_cols == 0 && c == 0) pre[0] = 0;
}

// Every lane waits for the copy of load q; the vote keeps a timeout warp-uniform.
__device__ __forceinline__ bool px_wait(unsigned long long* full, int q, volatile int* fail) {
    const bool good = !*fail && mbar_wait(&full[q & (PX_STAGES - 1)], (q / PX_STAGES) & 1);
    if (__all_sync(0xffffffffu, good)) return true;
    *fail = 1;
    return false;
}

// Every lane is done reading stage q: release it (one arrival per consumer warp).
__device__ __forceinline__ void px_release(unsigned long long* empty, int q, int lane) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[q & (PX_STAGES - 1)]);
}

struct PlumeW {
    float w0, wx, wy, wb, wt, decay;
};

// One voxel's FTCS update from its neighbours and mask byte (the expression of every plume kernel);
// FAST: the caller has established that if the voxel is updated all six neighbours are void.
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
    const float u = fmaxf((k.w0 * c0 + k.wx * (w + e) + k.wy * (s + n) + k.wb * b + k.wt * t) * k.decay, 0.0f);
    return (m & BD_PM_UPDATE) ? u : 0.0f;
}

// true when every voxel of the byte set `m` that is updated has all six neighbours void
__device__ __forceinline__ bool all_interior(unsigned m) {
    const unsigned upd = (m >> 7) & 0x01010101u;
    return (m & (upd * 0x3Fu)) == upd * 0x3Fu;
}

// Direct plume step: no staging, no barriers. A CTA is one 32 (z) x 16 (y) tile and marches xc x
// planes; thread = 4 consecutive z voxels of one row, a warp 8 such groups x 4 rows (one 128-byte
// line per row and load). The thread keeps the x-1 / x float4 of its row in registers and loads,
// per plane, the next plane's float4 and the centre plane's y neighbours from the (L2-resident)
// field beside the plane's mask bytes (one 32-bit load), whether or not the warp then has void to
// update: one L2 round trip per plane instead of a mask round trip followed by a data round trip,
// at the price of loads a tissue plane does not need (L2 bandwidth has the headroom). The z
// neighbours come from the neighbouring lanes by shuffle (the tile's edge lanes load them). Latency
// is hidden by the many independent CTAs of a step instead of a copy pipeline. Warp-uniform paths
// as in k_plume_xm; the same per-voxel expression (bit-identical). Needs nz % 4 == 0 and 16-byte
// aligned fields. Measured on the full coupled run: 16-row tiles beat 32 and 64 rows (more CTAs
// to hide latency with); loading the data only after a warp's vote found void was 4 % slower, and
// 8 z voxels per thread on 64 x 16 tiles (twice the loads in flight, 6-8 CTAs per SM) 5-15 %.
constexpr int PD_BY = 16;  // rows per CTA (8 * PD_BY threads)
__global__ void __launch_bounds__(8 * PD_BY) k_plume_direct(const float* __restrict__ C, float* __restrict__ Cn,
                                                      const uint8_t* __restrict__ M, int nx, int ny, int nz, int mz,
                                                      int xc, PlumeConst c, const int* __restrict__ zlimit,
                                                      int full_write) {
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int k0 = blockIdx.x * PL_BZ;
    const int ib = blockIdx.z * xc, ie = min(nx, ib + xc);
    if (k0 >= zl || ib >= ie) return;  // uniform over the CTA
    const int zg = threadIdx.x & 7;
    const int j = blockIdx.y * PD_BY + (threadIdx.x >> 3), k = k0 + 4 * zg;
    const int nk = zl - k;
    const bool act = nk > 0 && j < ny;
    const bool in = j < ny && k < nz;
    const unsigned zkeep = nk >= 4 ? 0xffffffffu : (nk <= 0 ? 0u : (0xffffffffu >> (8 * (4 - nk))));
    const size_t plane = (size_t)ny * nz;
    const size_t mplane = (size_t)ny * mz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    size_t idx = ((size_t)ib * ny + j) * nz + k;
    const uint8_t* mp = M + ((size_t)ib * ny + j) * mz + k;
    PlumeW kw;
    kw.wx = c.dtp * c.dxy_x; kw.wy = c.dtp * c.dxy_y; kw.wb = c.dtp * c.dz_z;
    kw.wt = kw.wb + c.dtp * c.vz_over_dz;
    kw.w0 = 1.0f - 2.0f * (kw.wx + kw.wy + kw.wb) - c.dtp * c.vz_over_dz;
    kw.decay = c.decay;
    // planes i-1 / i of the row
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
            float v[4];
            if (__all_sync(0xffffffffu, all_interior(mr) || !act)) {
                v[0] = ftcs<true>(cc.x, cw.x, ce.x, cs.x, cn.x, zb, cc.y, mr & 0xffu, kw);
                v[1] = ftcs<true>(cc.y, cw.y, ce.y, cs.y, cn.y, cc.x, cc.z, (mr >> 8) & 0xffu, kw);
                v[2] = ftcs<true>(cc.z, cw.z, ce.z, cs.z, cn.z, cc.y, cc.w, (mr >> 16) & 0xffu, kw);
                v[3] = ftcs<true>(cc.w, cw.w, ce.w, cs.w, cn.w, cc.z, zt, mr >> 24, kw);
            } else {
                v[0] = ftcs<false>(cc.x, cw.x, ce.x, cs.x, cn.x, zb, cc.y, mr & 0xffu, kw);
                v[1] = ftcs<false>(cc.y, cw.y, ce.y, cs.y, cn.y, cc.x, cc.z, (mr >> 8) & 0xffu, kw);
                v[2] = ftcs<false>(cc.z, cw.z, ce.z, cs.z, cn.z, cc.y, cc.w, (mr >> 16) & 0xffu, kw);
                v[3] = ftcs<false>(cc.w, cw.w, ce.w, cs.w, cn.w, cc.z, zt, mr >> 24, kw);
            }
            if (act && (vd || full_write)) {
                float* dst = Cn + idx;
                if (full_write || vd == 0x40404040u) {
                    *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (vd & (0x40u << (8 * e))) dst[e] = v[e];
                }
            }
        }
        cw = cc;
        cc = ce;
    }
}

static_assert(PD_BY == kPlumeZRows, "z-list columns follow the direct kernel's y tiles");

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
    const int nk = zl - 4 * g;
    bool live = false;
    if (g < G && nk > 0) {
        const unsigned keep = nk >= 4 ? 0xffffffffu : (0xffffffffu >> (8 * (4 - nk)));
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

// Direct plume step over the live z groups only (steps after the first two of a stage): as
// k_plume_direct, but band blockIdx.x of a column takes the column's live groups 8 b .. 8 b + 7
// from its z list instead of 8 consecutive groups, so z tiles that are partly tissue cost only
// their void groups. A lane whose z neighbour group is not held by the neighbouring lane loads
// that neighbour voxel instead of taking it by shuffle. Same per-voxel expression (bit-identical);
// voxels outside the lists are not void and are written by no step after the first two.
__global__ void __launch_bounds__(8 * PD_BY, 9) k_plume_direct_z(const float* __restrict__ C, float* __restrict__ Cn,
                                                        const uint8_t* __restrict__ M, int nx, int ny, int nz,
                                                        int mz, int xc, PlumeConst c, const int* __restrict__ zlimit,
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
    const int nk = zl - k;
    const bool act = g >= 0 && nk > 0 && j < ny;
    const bool in = g >= 0 && j < ny && k < nz;
    const unsigned zkeep = nk >= 4 ? 0xffffffffu : (nk <= 0 ? 0u : (0xffffffffu >> (8 * (4 - nk))));
    const size_t plane = (size_t)ny * nz;
    const size_t mplane = (size_t)ny * mz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    size_t idx = ((size_t)ib * ny + j) * nz + k;
    const uint8_t* mp = M + ((size_t)ib * ny + j) * mz + k;
    PlumeW kw;
    kw.wx = c.dtp * c.dxy_x; kw.wy = c.dtp * c.dxy_y; kw.wb = c.dtp * c.dz_z;
    kw.wt = kw.wb + c.dtp * c.vz_over_dz;
    kw.w0 = 1.0f - 2.0f * (kw.wx + kw.wy + kw.wb) - c.dtp * c.vz_over_dz;
    kw.decay = c.decay;
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
            float v[4];
            if (__all_sync(0xffffffffu, all_interior(mr) || !act)) {
                v[0] = ftcs<true>(cc.x, cw.x, ce.x, cs.x, cn.x, zb, cc.y, mr & 0xffu, kw);
                v[1] = ftcs<true>(cc.y, cw.y, ce.y, cs.y, cn.y, cc.x, cc.z, (mr >> 8) & 0xffu, kw);
                v[2] = ftcs<true>(cc.z, cw.z, ce.z, cs.z, cn.z, cc.y, cc.w, (mr >> 16) & 0xffu, kw);
                v[3] = ftcs<true>(cc.w, cw.w, ce.w, cs.w, cn.w, cc.z, zt, mr >> 24, kw);
            } else {
                v[0] = ftcs<false>(cc.x, cw.x, ce.x, cs.x, cn.x, zb, cc.y, mr & 0xffu, kw);
                v[1] = ftcs<false>(cc.y, cw.y, ce.y, cs.y, cn.y, cc.x, cc.z, (mr >> 8) & 0xffu, kw);
                v[2] = ftcs<false>(cc.z, cw.z, ce.z, cs.z, cn.z, cc.y, cc.w, (mr >> 16) & 0xffu, kw);
                v[3] = ftcs<false>(cc.w, cw.w, ce.w, cs.w, cn.w, cc.z, zt, mr >> 24, kw);
            }
            if (act && vd) {
                float* dst = Cn + idx;
                if (vd == 0x40404040u) {
                    *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (vd & (0x40u << (8 * e))) dst[e] = v[e];
                }
            }
        }
        cw = cc;
        cc = ce;
    }
}

template <int PB>
__global__ void __launch_bounds__(PX_THREADS, 1) k_plume_xm(const __grid_constant__ CUtensorMap c_map,
                                                         const __grid_constant__ CUtensorMap m_map,
                                                         float* __restrict__ Cn, int nx, int ny, int nz, PlumeConst c,
                                                         const int* __restrict__ zlimit,
                                                         const int* __restrict__ ext, int full_write,
                                                         int* __restrict__ err) {
    using X = PlumeXM<PB>;
    extern __shared__ __align__(128) unsigned char ring[];
    __shared__ __align__(8) unsigned long long full[PX_STAGES], empty[PX_STAGES];
    __shared__ volatile int s_fail;
    __shared__ int s_x0[kPlumeMaxCols], s_pre[kPlumeMaxCols + 1];
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int n_kt = (zl + PL_BZ - 1) / PL_BZ;
    const int n_cols = n_kt * ((ny + PX_BY - 1) / PX_BY);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    long long total = (long long)n_cols * nx;
    PlumeRun run{n_kt, PX_BY, nx, 0, 0};
    if (ext) {
        // only the planes of each column that hold void voxels (k_plume_extent / k_plume_runs)
        for (int i = tid; i <= n_cols; i += blockDim.x) {
            s_pre[i] = ext[2 * kPlumeMaxCols + i];
            if (i < n_cols) s_x0[i] = ext[i];
        }
        __syncthreads();
        total = s_pre[n_cols];
        run.pre = s_pre;
        run.x0 = s_x0;
        run.n_cols = n_cols;
    }
    run.s0 = total * blockIdx.x / gridDim.x;
    run.s1 = total * (blockIdx.x + 1) / gridDim.x;
    if (run.s0 >= run.s1) return;  // uniform over the CTA
    if (tid == 0) {
        for (int q = 0; q < PX_STAGES; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], PX_NW);
        }
        mbar_init_fence();
        s_fail = 0;
    }
    __syncthreads();
    int issued = 0;  // producer: loads issued
    if (warp == PX_NW) {
        // ---- producer warp (one lane): planes ib-1 .. ie of each segment, PB per load ----
        if (lane == 0) {
            for (long long pos = run.s0; pos < run.s1 && !s_fail;) {
                const int4 t = run.segment(pos);
                pos += t.w - t.z;
                const int nb = (t.w - t.z + 2 + PB - 1) / PB;
                for (int b = 0; b < nb; ++b) {
                    const int sl = issued & (PX_STAGES - 1);
                    if (issued >= PX_STAGES && !mbar_wait(&empty[sl], ((issued / PX_STAGES) - 1) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(&full[sl], X::C_BYTES + X::M_BYTES);
                    unsigned char* st = ring + sl * X::STAGE;
                    tma_load_3d(st, &c_map, t.x - 4, t.y - 1, t.z - 1 + PB * b, &full[sl]);
                    tma_load_3d(st + X::M_OFF, &m_map, t.x, t.y, t.z - 1 + PB * b, &full[sl]);
                    ++issued;
                }
            }
        }
    } else {
        // ---- consumer warps: warp = z group, lane = tile row ----
        PlumeW kw;
        kw.wx = c.dtp * c.dxy_x; kw.wy = c.dtp * c.dxy_y; kw.wb = c.dtp * c.dz_z;
        kw.wt = kw.wb + c.dtp * c.vz_over_dz;
        kw.w0 = 1.0f - 2.0f * (kw.wx + kw.wy + kw.wb) - c.dtp * c.vz_over_dz;
        kw.decay = c.decay;
        const int plane = ny * nz;
        const int t0 = (lane + 1) * PX_PZ + 4 + 4 * warp;  // this thread's float4 in a plane (16-byte aligned)
        const int mo = X::M_OFF + lane * PL_BZ + 4 * warp;  // its four mask bytes in mask plane 0
        int L = 0;                                          // load index of the segment's first load
        bool ok = true;
        for (long long pos = run.s0; pos < run.s1 && ok;) {
            const int4 t = run.segment(pos);
            const int k0 = t.x, j0 = t.y, ib = t.z, ie = t.w;
            pos += ie - ib;
            const int np = ie - ib + 2, nb = (np + PB - 1) / PB;  // planes ib-1 .. ie in nb loads
            const int k = k0 + 4 * warp;
            // bytes of voxels at or below zl are cleared: the mask is only rebuilt above zl
            const int nk = zl - k;
            const unsigned zkeep = nk >= 4 ? 0xffffffffu : (nk <= 0 ? 0u : (0xffffffffu >> (8 * (4 - nk))));
            const bool act = nk > 0 && j0 + lane < ny;
            float* dst = Cn + (size_t)ib * plane + (size_t)(j0 + lane) * nz + k;
            int waited = 0, released = 0;  // loads of this segment waited for / released
            // segment plane q lives in load q / PB, plane q % PB of that stage
#define BD_PX_PLANE(q) (ring + ((L + (q) / PB) & (PX_STAGES - 1)) * X::STAGE + ((q) % PB) * PX_PLANE)
#define BD_PX_NEED(q)                                                         \
    while (ok && waited <= (q) / PB) {                                        \
        if (!px_wait(full, L + waited, &s_fail)) ok = false;                  \
        ++waited;                                                             \
    }
            BD_PX_NEED(1)
            if (!ok) break;
            float4 cw = *reinterpret_cast<const float4*>(BD_PX_PLANE(0) + 4 * t0);
            float4 cc = *reinterpret_cast<const float4*>(BD_PX_PLANE(1) + 4 * t0);
            if (PB == 1) { px_release(empty, L, lane); released = 1; }
            for (int q = 1; q < np - 1; ++q, dst += plane) {  // q: centre plane (x = ib - 1 + q)
                BD_PX_NEED(q + 1)
                if (!ok) break;
                const unsigned char* sc = BD_PX_PLANE(q);
                const float* tc = reinterpret_cast<const float*>(sc);
                const float4 ce = *reinterpret_cast<const float4*>(BD_PX_PLANE(q + 1) + 4 * t0);
                const unsigned mr =
                    *reinterpret_cast<const unsigned*>(ring + ((L + q / PB) & (PX_STAGES - 1)) * X::STAGE + mo +
                                                       (q % PB) * PX_MPLANE) & zkeep;
                const unsigned vd = mr & 0x40404040u;  // void bit of each of the four voxels
                // every voxel that is updated has all six neighbours void (outer-wall and tissue voxels,
                // not updated, take 0 as on the general path)
                const bool bulk = all_interior(mr);
                if (__any_sync(0xffffffffu, act && (vd || full_write))) {
                    const float4 cs = *reinterpret_cast<const float4*>(tc + t0 - PX_PZ);
                    const float4 cn = *reinterpret_cast<const float4*>(tc + t0 + PX_PZ);
                    const float zb = tc[t0 - 1], zt = tc[t0 + 4];
                    float v[4];
                    if (__all_sync(0xffffffffu, bulk || !act)) {
                        v[0] = ftcs<true>(cc.x, cw.x, ce.x, cs.x, cn.x, zb, cc.y, mr & 0xffu, kw);
                        v[1] = ftcs<true>(cc.y, cw.y, ce.y, cs.y, cn.y, cc.x, cc.z, (mr >> 8) & 0xffu, kw);
                        v[2] = ftcs<true>(cc.z, cw.z, ce.z, cs.z, cn.z, cc.y, cc.w, (mr >> 16) & 0xffu, kw);
                        v[3] = ftcs<true>(cc.w, cw.w, ce.w, cs.w, cn.w, cc.z, zt, mr >> 24, kw);
                    } else {
                        v[0] = ftcs<false>(cc.x, cw.x, ce.x, cs.x, cn.x, zb, cc.y, mr & 0xffu, kw);
                        v[1] = ftcs<false>(cc.y, cw.y, ce.y, cs.y, cn.y, cc.x, cc.z, (mr >> 8) & 0xffu, kw);
                        v[2] = ftcs<false>(cc.z, cw.z, ce.z, cs.z, cn.z, cc.y, cc.w, (mr >> 16) & 0xffu, kw);
                        v[3] = ftcs<false>(cc.w, cw.w, ce.w, cs.w, cn.w, cc.z, zt, mr >> 24, kw);
                    }
                    if (act && (vd || full_write)) {
                        if (full_write || vd == 0x40404040u) {
                            *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; ++e)
                                if (vd & (0x40u << (8 * e))) dst[e] = v[e];
                        }
                    }
                }
                // plane q was the last plane of its load: every plane of that load has been read
                if ((q + 1) % PB == 0) {
                    px_release(empty, L + released, lane);
                    ++released;
                }
                cw = cc;
                cc = ce;
            }
            if (!ok) break;
            for (; released < nb; ++released) px_release(empty, L + released, lane);
            L += nb;
#undef BD_PX_PLANE
#undef BD_PX_NEED
        }
    }
    __syncthreads();
    if (tid == PX_NW * 32 && s_fail) {
        atomicExch(err, 1);
        // drain: the copies still in flight get a bounded chance to land before the CTA exits
        for (int q = max(0, issued - PX_STAGES); q < issued; ++q)
            mbar_wait(&full[q & (PX_STAGES - 1)], (q / PX_STAGES) & 1);
    }
}

// Two FTCS steps per pass (temporal blocking), otherwise the x-marching kernel's structure: the
// plane stream, ring protocol, warp = 4-voxel z group and lane = row. Lane l holds row y = j0 - 1 + l;
// each thread computes the first step on the 6 voxels z = k-1 .. k+4 of its row (its 4 plus both z
// neighbours), the second step on its 4, taking the first step's y neighbours from lanes l +- 1 by
// shuffle. Lanes 0 and 31 carry the first step's y halo, so a tile outputs 30 rows (j0 .. j0+29) and
// a segment streams planes ib-2 .. ie+1. Per time step this halves the planes streamed, the ring
// round trips, the global stores and the launches; the first step's values never leave registers.
// Each voxel's update is the single-step expression (bit-identical to one-step kernels). The mask
// tile is 64 bytes wide (z k0-16 .. k0+47) so the neighbours' bytes at k0-1 and k0+32 are present.
// With full_write the result buffer alone would be fully written, so the context API's first two
// steps run on the one-step kernel.
constexpr int PT_BY = 30, PT_MZ = 64;
constexpr unsigned PT_MPLANE = PT_MZ * PX_BY;
template <int PB>
struct PlumeTB {
    static constexpr unsigned C_BYTES = PB * PX_PLANE;
    static constexpr unsigned M_OFF = (C_BYTES + 127) / 128 * 128;
    static constexpr unsigned M_BYTES = PB * PT_MPLANE;
    static constexpr unsigned STAGE = (M_OFF + M_BYTES + 127) / 128 * 128;
    static constexpr unsigned SMEM = PX_STAGES * STAGE;
};

template <int PB>
__global__ void __launch_bounds__(PX_THREADS, 1) k_plume_tb(const __grid_constant__ CUtensorMap c_map,
                                                         const __grid_constant__ CUtensorMap m_map,
                                                         float* __restrict__ Cn, int nx, int ny, int nz, PlumeConst c,
                                                         const int* __restrict__ zlimit, int* __restrict__ err) {
    using X = PlumeTB<PB>;
    extern __shared__ __align__(128) unsigned char ring[];
    __shared__ __align__(8) unsigned long long full[PX_STAGES], empty[PX_STAGES];
    __shared__ volatile int s_fail;
    const int zl = zlimit ? min(max(*zlimit, 0), nz) : nz;
    const int n_kt = (zl + PL_BZ - 1) / PL_BZ;
    const long long total = (long long)n_kt * ((ny + PT_BY - 1) / PT_BY) * nx;
    const PlumeRun run{n_kt, PT_BY, nx, total * blockIdx.x / gridDim.x, total * (blockIdx.x + 1) / gridDim.x};
    if (run.s0 >= run.s1) return;  // uniform over the CTA
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int q = 0; q < PX_STAGES; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], PX_NW);
        }
        mbar_init_fence();
        s_fail = 0;
    }
    __syncthreads();
    int issued = 0;
    if (warp == PX_NW) {
        // ---- producer warp (one lane): planes ib-2 .. ie+1 of each segment, PB per load ----
        if (lane == 0) {
            for (long long pos = run.s0; pos < run.s1 && !s_fail;) {
                const int4 t = run.segment(pos);
                pos += t.w - t.z;
                const int nb = (t.w - t.z + 4 + PB - 1) / PB;
                for (int b = 0; b < nb; ++b) {
                    const int sl = issued & (PX_STAGES - 1);
                    if (issued >= PX_STAGES && !mbar_wait(&empty[sl], ((issued / PX_STAGES) - 1) & 1)) {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(&full[sl], X::C_BYTES + X::M_BYTES);
                    unsigned char* st = ring + sl * X::STAGE;
                    tma_load_3d(st, &c_map, t.x - 4, t.y - 2, t.z - 2 + PB * b, &full[sl]);
                    tma_load_3d(st + X::M_OFF, &m_map, t.x - 16, t.y - 1, t.z - 2 + PB * b, &full[sl]);
                    ++issued;
                }
            }
        }
    } else {
        // ---- consumer warps: warp = z group, lane = row y = j0 - 1 + lane ----
        PlumeW kw;
        kw.wx = c.dtp * c.dxy_x; kw.wy = c.dtp * c.dxy_y; kw.wb = c.dtp * c.dz_z;
        kw.wt = kw.wb + c.dtp * c.vz_over_dz;
        kw.w0 = 1.0f - 2.0f * (kw.wx + kw.wy + kw.wb) - c.dtp * c.vz_over_dz;
        kw.decay = c.decay;
        const int plane = ny * nz;
        const int t0 = (lane + 1) * PX_PZ + 4 + 4 * warp;          // own row, z = k (16-byte aligned)
        const int mo = X::M_OFF + lane * PT_MZ + 16 + 4 * warp;    // own mask bytes, z = k
        int L = 0;
        bool ok = true;
        for (long long pos = run.s0; pos < run.s1 && ok;) {
            const int4 t = run.segment(pos);
            const int k0 = t.x, j0 = t.y, ib = t.z, ie = t.w;
            pos += ie - ib;
            const int np = ie - ib + 4, nb = (np + PB - 1) / PB;  // planes ib-2 .. ie+1 in nb loads
            const int k = k0 + 4 * warp;
            // mask bytes of z = k-1 .. k+4 that lie at or below zl are cleared (not rebuilt there)
            const int nk = zl - k;
            const unsigned zkeep = nk >= 4 ? 0xffffffffu : (nk <= 0 ? 0u : (0xffffffffu >> (8 * (4 - nk))));
            const bool lo_ok = k >= 1 && k - 1 < zl, hi_ok = k + 4 < zl;
            const bool store = lane >= 1 && lane <= PT_BY && j0 - 1 + lane < ny && nk > 0;
            float* dst = Cn + (size_t)ib * plane + (size_t)(j0 - 1 + lane) * nz + k;
            int waited = 0, released = 0;
#define BD_PT_PLANE(q) (ring + ((L + (q) / PB) & (PX_STAGES - 1)) * X::STAGE + ((q) % PB) * PX_PLANE)
#define BD_PT_MASK(q) (ring + ((L + (q) / PB) & (PX_STAGES - 1)) * X::STAGE + mo + ((q) % PB) * PT_MPLANE)
            // C0 of planes q-2, q-1 and C1 of planes q-3, q-2 (x-rotation), z = k-1 .. k+4
            float a0[6], a1[6], b0[6], b1[6];
            unsigned mprev = 0;  // mask bytes z = k .. k+3 of the plane C2 is computed on
#pragma unroll
            for (int e = 0; e < 6; ++e) a0[e] = a1[e] = b0[e] = b1[e] = 0.0f;
            for (int q = 0; q < np; ++q) {
                while (ok && waited <= q / PB) {
                    if (!px_wait(full, L + waited, &s_fail)) ok = false;
                    ++waited;
                }
                if (!ok) break;
                float a2[6];
                {
                    const float* tq = reinterpret_cast<const float*>(BD_PT_PLANE(q));
                    const float4 v = *reinterpret_cast<const float4*>(tq + t0);
                    a2[0] = tq[t0 - 1]; a2[1] = v.x; a2[2] = v.y; a2[3] = v.z; a2[4] = v.w; a2[5] = tq[t0 + 4];
                }
                float b2[6];
#pragma unroll
                for (int e = 0; e < 6; ++e) b2[e] = 0.0f;
                unsigned mcur = 0;
                if (q >= 2) {
                    // ---- first step on plane q-1 (centre), z = k-1 .. k+4 ----
                    const unsigned char* mq = BD_PT_MASK(q - 1);
                    mcur = *reinterpret_cast<const unsigned*>(mq) & zkeep;
                    const unsigned mlo = lo_ok ? mq[-1] : 0u, mhi = hi_ok ? mq[4] : 0u;
                    const bool live = __any_sync(0xffffffffu, ((mcur | mlo | mhi) & 0x40404040u) != 0);
                    if (live) {
                        const float* tc = reinterpret_cast<const float*>(BD_PT_PLANE(q - 1));
                        const float4 sv = *reinterpret_cast<const float4*>(tc + t0 - PX_PZ);
                        const float4 nv = *reinterpret_cast<const float4*>(tc + t0 + PX_PZ);
                        const float s6[6] = {tc[t0 - PX_PZ - 1], sv.x, sv.y, sv.z, sv.w, tc[t0 - PX_PZ + 4]};
                        const float n6[6] = {tc[t0 + PX_PZ - 1], nv.x, nv.y, nv.z, nv.w, tc[t0 + PX_PZ + 4]};
                        const float zm = tc[t0 - 2], zp = tc[t0 + 5];
                        const unsigned m6[6] = {mlo, mcur & 0xffu, (mcur >> 8) & 0xffu, (mcur >> 16) & 0xffu,
                                                mcur >> 24, mhi};
                        const bool fast = all_interior(mcur) && all_interior(mlo) && all_interior(mhi);
                        if (__all_sync(0xffffffffu, fast)) {
#pragma unroll
                            for (int e = 0; e < 6; ++e)
                                b2[e] = ftcs<true>(a1[e], a0[e], a2[e], s6[e], n6[e], e > 0 ? a1[e - 1] : zm,
                                                   e < 5 ? a1[e + 1] : zp, m6[e], kw);
                        } else {
#pragma unroll
                            for (int e = 0; e < 6; ++e)
                                b2[e] = ftcs<false>(a1[e], a0[e], a2[e], s6[e], n6[e], e > 0 ? a1[e - 1] : zm,
                                                    e < 5 ? a1[e + 1] : zp, m6[e], kw);
                        }
                    }
                }
                // the smem of plane q-1 has been read for the last time: release its load when it was
                // the load's last plane
                if (q >= 1 && q % PB == 0) {
                    px_release(empty, L + released, lane);
                    ++released;
                }
                if (q >= 4) {
                    // ---- second step on plane q-2 = x ib-4+q, z = k .. k+3, from C1 of planes q-3 .. q-1 ----
                    float sy[4], ny4[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        sy[e] = __shfl_up_sync(0xffffffffu, b1[e + 1], 1);
                        ny4[e] = __shfl_down_sync(0xffffffffu, b1[e + 1], 1);
                    }
                    const unsigned vd = mprev & 0x40404040u;
                    if (__any_sync(0xffffffffu, store && vd != 0)) {
                        float v[4];
                        if (__all_sync(0xffffffffu, !store || all_interior(mprev))) {
#pragma unroll
                            for (int e = 0; e < 4; ++e)
                                v[e] = ftcs<true>(b1[e + 1], b0[e + 1], b2[e + 1], sy[e], ny4[e], b1[e], b1[e + 2],
                                                  (mprev >> (8 * e)) & 0xffu, kw);
                        } else {
#pragma unroll
                            for (int e = 0; e < 4; ++e)
                                v[e] = ftcs<false>(b1[e + 1], b0[e + 1], b2[e + 1], sy[e], ny4[e], b1[e], b1[e + 2],
                                                   (mprev >> (8 * e)) & 0xffu, kw);
                        }
                        if (store && vd) {
                            if (vd == 0x40404040u) {
                                *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
                            } else {
#pragma unroll
                                for (int e = 0; e < 4; ++e)
                                    if (vd & (0x40u << (8 * e))) dst[e] = v[e];
                            }
                        }
                    }
                    dst += plane;
                }
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    a0[e] = a1[e]; a1[e] = a2[e];
                    b0[e] = b1[e]; b1[e] = b2[e];
                }
                mprev = mcur;
            }
            if (!ok) break;
            for (; released < nb; ++released) px_release(empty, L + released, lane);
            L += nb;
#undef BD_PT_PLANE
#undef BD_PT_MASK
        }
    }
    __syncthreads();
    if (tid == PX_NW * 32 && s_fail) {
        atomicExch(err, 1);
        for (int q = max(0, issued - PX_STAGES); q < issued; ++q)
            mbar_wait(&full[q & (PX_STAGES - 1)], (q / PX_STAGES) & 1);
    }
}

__global__ void k_pack_flags(const uint8_t* __restrict__ abl, const uint8_t* __restrict__ dry,
                             const uint8_t* __restrict__ vd, long long n, uint8_t* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        uint8_t a = abl[i] ? 1 : 0, d = dry[i] ? 1 : 0;
        uint8_t v = vd ? (vd[i] ? 1 : 0) : a;
        out[i] = (uint8_t)(a * BD_FLAG_ABLATED | d * BD_FLAG_DRY | v * BD_FLAG_VOID);
    }
}

static dim3 tile_grid(int nx, int ny, int nz, int ni) {
    return dim3((nz + TZ - 1) / TZ, (ny + TY - 1) / TY, (nx + ni - 1) / ni);
}

static int pick_ni(int nx, int ny, int nz) {
    // short marches (~8 planes) and several waves of 256-thread CTAs: enough independent
    // DRAM round trips in flight to cover latency without a long serial chain per thread
    long long cols = (long long)((nz + TZ - 1) / TZ) * ((ny + TY - 1) / TY);
    long long want = 148LL * 6 * 4;
    long long chunks = std::max(1LL, want / std::max(1LL, cols));
    int ni = (int)std::max(4LL, ((long long)nx + chunks - 1) / chunks);
#ifndef BD_STENCIL_NI
#define BD_STENCIL_NI 8
#endif
    ni = std::min(ni, BD_STENCIL_NI);
    return std::min(ni, std::max(nx, 1));
}

static Geo make_geo(int nx, int ny, int nz, float dx, float dy, float dz, float dt, float h, float tamb) {
    Geo g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.ni = pick_ni(nx, ny, nz);
    g.idx2 = 1.0f / (dx * dx); g.idy2 = 1.0f / (dy * dy); g.idz2 = 1.0f / (dz * dz);
    g.dz = dz; g.h_eff = h; g.t_amb = tamb; g.dt = dt;
    return g;
}

template <int MODE, int BC, bool ARR, bool CHAR>
static void launch_substeps(const Geo& g, const AblConst& c, float* Ta, float* Tb, int n, const float* src,
                            const float* K, const float* R, const uint8_t* F, float* H, float* Om, float* Chi,
                            cudaStream_t st, int* err) {
    CUtensorMap ma, mb, mk;
#ifdef BD_NO_TMA
    err = nullptr;
#endif
    const bool tma = err != nullptr && make_tmap_3d_f32(&ma, Ta, g.nx, g.ny, g.nz, ST_PZ, ST_PY, 1) &&
                     make_tmap_3d_f32(&mb, Tb, g.nx, g.ny, g.nz, ST_PZ, ST_PY, 1) &&
                     make_tmap_3d_f32(&mk, K, g.nx, g.ny, g.nz, ST_PZ, ST_PY, 1);
    if (tma) {
        const int xc = tune_value(BD_TUNE_STENCIL_XC);
        const dim3 grid((g.nz + ST_BZ - 1) / ST_BZ, (g.ny + ST_BY - 1) / ST_BY, (g.nx + xc - 1) / xc);
        for (int s = 0; s < n; ++s) {
            float* out = (s & 1) ? Ta : Tb;
            k_substep_tma<MODE, BC, ARR, CHAR><<<grid, dim3(TZ, TY), 0, st>>>((s & 1) ? mb : ma, mk, g, c, out, src,
                                                                             R, F, H, Om, Chi, xc, err);
        }
        return;
    }
    dim3 grid = tile_grid(g.nx, g.ny, g.nz, g.ni), block(TZ, TY);
    for (int s = 0; s < n; ++s) {
        const float* in = (s & 1) ? Tb : Ta;
        float* out = (s & 1) ? Ta : Tb;
        k_substep<MODE, BC, ARR, CHAR><<<grid, block, 0, st>>>(g, c, in, out, src, K, R, F, H, Om, Chi);
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

// Runs `launch(err)` with a 4-byte device error flag, then synchronises the stream and turns a
// raised flag (a bounded TMA wait that timed out) into BD_ERR_TIMEOUT.
template <typename F>
static int with_error_flag(cudaStream_t st, const char* what, F launch) {
    int* err = nullptr;
    BD_CUDA(cudaMallocAsync((void**)&err, sizeof(int), st));
    int rc = BD_OK;
    int host_err = 0;
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) rc = launch(err);
    if (e == cudaSuccess && rc == BD_OK) e = cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e2 = cudaFreeAsync(err, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, what);
    if (e2 != cudaSuccess) return cuda_status(e2, what);
    if (host_err) return fail(BD_ERR_TIMEOUT, "%s: a bounded TMA wait timed out", what);
    return BD_OK;
}

}  // namespace bd

using namespace bd;

extern "C" int bd_thermal_advance(const BdThermalParams* p, float* Ta, float* Tb, int n, const float* src,
                                  const float* K, const float* R, void* stream) {
    BD_REQUIRE(p != nullptr, "bd_thermal_advance: params is NULL");
    BD_REQUIRE(p->nx > 0 && p->ny > 0 && p->nz > 0, "bd_thermal_advance: grid dims must be positive");
    BD_REQUIRE(Ta && Tb && K && R, "bd_thermal_advance: NULL field");
    BD_REQUIRE(!p->is_active || src != nullptr, "bd_thermal_advance: active source needs src");
    BD_REQUIRE(p->bc_mode == BD_BC_SERIES || p->bc_mode == BD_BC_METAL, "bd_thermal_advance: bad bc_mode");
    BD_REQUIRE(n >= 0, "bd_thermal_advance: n_substeps must be >= 0");
    BD_REQUIRE((long long)p->nx * p->ny * p->nz < (1LL << 31), "bd_thermal_advance: grid exceeds 2^31 voxels");
    if (n == 0) return BD_OK;
    Geo g = make_geo(p->nx, p->ny, p->nz, p->dx, p->dy, p->dz, p->dt, p->h_eff, p->t_ambient);
    AblConst c{};
    c.q_scale = p->q_scale;
    c.is_active = p->is_active;
    cudaStream_t st = as_stream(stream);
    return with_error_flag(st, "bd_thermal_advance", [&](int* err) -> int {
        if (p->bc_mode == BD_BC_SERIES)
            launch_substeps<0, BD_BC_SERIES, false, false>(g, c, Ta, Tb, n, src, K, R, nullptr, nullptr, nullptr,
                                                           nullptr, st, err);
        else
            launch_substeps<0, BD_BC_METAL, false, false>(g, c, Ta, Tb, n, src, K, R, nullptr, nullptr, nullptr,
                                                          nullptr, st, err);
        BD_CHECK_LAUNCH("k_substep<thermal>");
        return BD_OK;
    });
}

namespace bd {
int ablation_launch(const BdAblationParams* p, float* Ta, float* Tb, int n, float* H, float* Om, float* Chi,
                    const uint8_t* F, const float* src, const float* K, const float* R, cudaStream_t st, int* err) {
    Geo g = make_geo(p->nx, p->ny, p->nz, p->dx, p->dy, p->dz, p->dt, p->h_eff, p->t_ambient);
    AblConst c;
    c.t_abl = p->t_abl; c.t_void = p->t_void; c.q_scale = p->q_scale;
    c.arr_A = p->arr_A; c.arr_EaR = p->arr_Ea_over_R; c.char_A = p->char_A; c.char_EaR = p->char_Ea_over_R;
    c.zero_src_in_ablated = p->zero_src_in_ablated; c.is_active = p->is_active;
    const bool arr = p->has_arrhenius != 0, chr = p->has_char != 0;
#define BD_ABL_CASE(BCV, A_, C_)                                                                 \
    if (p->bc_mode == BCV && arr == A_ && chr == C_) {                                           \
        launch_substeps<1, BCV, A_, C_>(g, c, Ta, Tb, n, src, K, R, F, H, Om, Chi, st, err);     \
        BD_CHECK_LAUNCH("k_substep<ablation>");                                                  \
        return BD_OK;                                                                            \
    }
    BD_ABL_CASE(BD_BC_SERIES, false, false)
    BD_ABL_CASE(BD_BC_SERIES, false, true)
    BD_ABL_CASE(BD_BC_SERIES, true, false)
    BD_ABL_CASE(BD_BC_SERIES, true, true)
    BD_ABL_CASE(BD_BC_METAL, false, false)
    BD_ABL_CASE(BD_BC_METAL, false, true)
    BD_ABL_CASE(BD_BC_METAL, true, false)
    BD_ABL_CASE(BD_BC_METAL, true, true)
#undef BD_ABL_CASE
    return fail(BD_ERR_INVALID_ARG, "bd_ablation_advance: bad bc_mode %d", p->bc_mode);
}

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
    const dim3 grid((p->ny + TY - 1) / TY, p->nx);
    const int mz = plume_mask_pitch(p->nz);
    // with full_first the whole grid is masked (the context API's first steps write every voxel)
    k_plume_mask<<<grid, dim3(TZ, TY), 0, st>>>(p->nx, p->ny, p->nz, mz, F, mask, full_first ? nullptr : zlimit);
    BD_CHECK_LAUNCH("k_plume_mask");
    CUtensorMap map_a, map_b, map_m;
#ifdef BD_NO_TMA
    err = nullptr;
#endif
    // plume kernel: 0 = scalar TMA kernel, 1 / 2 = persistent x-marching kernel, 2 / 4 planes per copy,
    // 3 = two steps per launch (k_plume_tb, 2 planes per copy; single steps on kernel 1),
    // 4 = direct: k_plume_direct_z over each column's live z groups, k_plume_direct for the first
    //     two (full-write) steps and for nz > 1020
    // (64 registers x 288 threads: at most 3 CTAs per SM; 4 at 56 registers measured slower)
    const int kernel = tune_value(BD_TUNE_PLUME_KERNEL);
    const int shape = kernel >= 3 ? 1 : kernel;  // the one-step kernel (kernel 4 launches its own)
    const int pb = shape == 1 ? 2 : 4;
    const int py = shape == 0 ? PL_PY : PX_PY;
    const int pz = shape == 0 ? PL_PZ : PX_PZ;
    const int bx = shape == 0 ? 1 : pb;
    const bool tma = err != nullptr && make_tmap_3d_f32(&map_a, Ca, p->nx, p->ny, p->nz, pz, py, bx) &&
                     make_tmap_3d_f32(&map_b, Cb, p->nx, p->ny, p->nz, pz, py, bx) &&
                     (shape == 0 || make_tmap_3d_u8(&map_m, mask, p->nx, p->ny, p->nz, mz, PL_BZ, PX_BY, pb));
    CUtensorMap map_m2;
    const bool two = tma && kernel == 3 && make_tmap_3d_u8(&map_m2, mask, p->nx, p->ny, p->nz, mz, PT_MZ, PX_BY, 2);
    const int xc = tune_value(BD_TUNE_PLUME_XC);
    const dim3 tgrid((p->nz + PL_BZ - 1) / PL_BZ, (p->ny + PL_BY - 1) / PL_BY, (p->nx + xc - 1) / xc);
    // persistent kernels: xc CTAs per SM (capped by occupancy), at most one per plane tile of the grid
    int xm_grid = 0, tb_grid = 0;
    int* xm_ext = nullptr;
    unsigned xm_smem = shape == 1 ? PlumeXM<2>::SMEM : PlumeXM<4>::SMEM;
    if (tma && shape > 0 && kernel < 4) {
        int dev = 0, sms = 0, occ = 0;
        BD_CUDA(cudaGetDevice(&dev));
        BD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (shape == 1) {
            BD_CUDA(cudaFuncSetAttribute(k_plume_xm<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, xm_smem));
            BD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_plume_xm<2>, PX_THREADS, xm_smem));
        } else {
            BD_CUDA(cudaFuncSetAttribute(k_plume_xm<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, xm_smem));
            BD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_plume_xm<4>, PX_THREADS, xm_smem));
        }
        const long long planes =
            (long long)((p->nz + PL_BZ - 1) / PL_BZ) * ((p->ny + PX_BY - 1) / PX_BY) * p->nx;
        xm_grid = (int)std::max(1LL, std::min(planes, (long long)std::max(std::min(occ, xc), 1) * sms));
        // the void x-extent of every column, from this stage's mask: the persistent kernel walks
        // only planes that hold void voxels (the void domain is fixed within the stage)
        const int n_ktmax = (p->nz + PL_BZ - 1) / PL_BZ, n_jt = (p->ny + PX_BY - 1) / PX_BY;
        if (n_ktmax <= 64 && n_ktmax * n_jt <= kPlumeMaxCols) {
            xm_ext = reinterpret_cast<int*>(mask + plume_mask_only_bytes(p->nx, p->ny, p->nz));
            k_plume_extent_init<<<1, 1024, 0, st>>>(xm_ext);
            k_plume_extent<<<dim3(p->nx, n_jt), 256, 0, st>>>(mask, p->nx, p->ny, p->nz, mz,
                                                              full_first ? nullptr : zlimit, xm_ext);
            k_plume_runs<<<1, 1024, 0, st>>>(xm_ext, p->ny, p->nz, full_first ? nullptr : zlimit);
            BD_CHECK_LAUNCH("k_plume_runs");
        }
        if (two) {
            int occ2 = 0;
            BD_CUDA(cudaFuncSetAttribute(k_plume_tb<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         PlumeTB<2>::SMEM));
            BD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_plume_tb<2>, PX_THREADS, PlumeTB<2>::SMEM));
            const long long planes2 =
                (long long)((p->nz + PL_BZ - 1) / PL_BZ) * ((p->ny + PT_BY - 1) / PT_BY) * p->nx;
            tb_grid = (int)std::max(1LL, std::min(planes2, (long long)std::max(std::min(occ2, xc), 1) * sms));
        }
    }
    // live z groups per direct-kernel column, from this stage's mask (steps after the first two)
    uint8_t* zlist = nullptr;
    if (tma && kernel == 4 && (p->nz + 3) / 4 <= 255) {
        zlist = mask + plume_zlist_offset(p->nx, p->ny, p->nz);
        k_plume_zlist<<<dim3((p->ny + PD_BY - 1) / PD_BY, (p->nx + xc - 1) / xc), 256, 0, st>>>(
            mask, p->nx, p->ny, p->nz, mz, xc, full_first ? nullptr : zlimit, zlist);
        BD_CHECK_LAUNCH("k_plume_zlist");
    }
    const long long total = (long long)steps * n_substeps;
    long long launches = 0;  // each launch moves the field to the other buffer
    for (long long s = 0; s < total;) {
        const bool odd = launches & 1;
        const float* in = odd ? Cb : Ca;
        float* out = odd ? Ca : Cb;
        const int full = (full_first && s < 2) ? 1 : 0;
        const CUtensorMap& map = odd ? map_b : map_a;
        const int* zl = full ? nullptr : zlimit;
        ++launches;
        if (kernel == 4 && tma && zlist && !full) {
            ++s;
            k_plume_direct_z<<<dim3((p->nz + PL_BZ - 1) / PL_BZ, (p->ny + PD_BY - 1) / PD_BY, (p->nx + xc - 1) / xc),
                               8 * PD_BY, 0, st>>>(in, out, mask, p->nx, p->ny, p->nz, mz, xc, c, zl, zlist);
            continue;
        }
        if (kernel == 4 && tma) {
            ++s;
            k_plume_direct<<<dim3((p->nz + PL_BZ - 1) / PL_BZ, (p->ny + PD_BY - 1) / PD_BY, (p->nx + xc - 1) / xc),
                             8 * PD_BY, 0, st>>>(in, out, mask, p->nx, p->ny, p->nz, mz, xc, c, zl, full);
            continue;
        }
        if (two && !full && total - s >= 2) {
            k_plume_tb<2><<<tb_grid, PX_THREADS, PlumeTB<2>::SMEM, st>>>(map, map_m2, out, p->nx, p->ny, p->nz, c, zl,
                                                                       err);
            s += 2;
            continue;
        }
        ++s;
        if (tma && shape == 1)
            k_plume_xm<2><<<xm_grid, PX_THREADS, xm_smem, st>>>(map, map_m, out, p->nx, p->ny, p->nz, c, zl,
                                                                full ? nullptr : xm_ext, full, err);
        else if (tma && shape == 2)
            k_plume_xm<4><<<xm_grid, PX_THREADS, xm_smem, st>>>(map, map_m, out, p->nx, p->ny, p->nz, c, zl,
                                                                full ? nullptr : xm_ext, full, err);
        else if (tma)
            k_plume_step_tma<<<tgrid, dim3(TZ, PL_TY), 0, st>>>(map, out, mask, p->nx, p->ny, p->nz, mz, xc, c, zl,
                                                             full, err);
        else
            k_plume_step<<<grid, dim3(TZ, TY), 0, st>>>(p->nx, p->ny, p->nz, mz, c, in, out, mask,
                                                        full ? nullptr : zlimit, full);
    }
    BD_CHECK_LAUNCH("k_plume_step");
    if (in_b) *in_b = (int)(launches & 1);
    return BD_OK;
}
}  // namespace bd

extern "C" int bd_ablation_advance(const BdAblationParams* p, float* Ta, float* Tb, int n, float* H, float* Om,
                                   float* Chi, const uint8_t* F, const float* src, const float* K, const float* R,
                                   void* stream) {
    BD_REQUIRE(p != nullptr, "bd_ablation_advance: params is NULL");
    BD_REQUIRE(p->nx > 0 && p->ny > 0 && p->nz > 0, "bd_ablation_advance: grid dims must be positive");
    BD_REQUIRE(Ta && Tb && H && F && K && R, "bd_ablation_advance: NULL field");
    BD_REQUIRE(!p->is_active || src != nullptr, "bd_ablation_advance: active source needs src");
    BD_REQUIRE(!p->has_arrhenius || Om != nullptr, "bd_ablation_advance: Arrhenius needs Omega");
    BD_REQUIRE(!p->has_char || Chi != nullptr, "bd_ablation_advance: char kinetics need chi");
    BD_REQUIRE(n >= 0, "bd_ablation_advance: n_substeps must be >= 0");
    BD_REQUIRE((long long)p->nx * p->ny * p->nz < (1LL << 31), "bd_ablation_advance: grid exceeds 2^31 voxels");
    if (n == 0) return BD_OK;
    cudaStream_t st = as_stream(stream);
    return with_error_flag(st, "bd_ablation_advance", [&](int* err) -> int {
        return ablation_launch(p, Ta, Tb, n, H, Om, Chi, F, src, K, R, st, err);
    });
}

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
    // the context API may hold arbitrary values in non-void voxels: the first two steps write
    // every voxel (one per ping-pong buffer), later steps touch the void domain only
    if (e == cudaSuccess) rc = plume_launch(p, Ca, Cb, n_substeps, F, in_b, st, nullptr, 1, scratch, err);
    int host_err = 0;
    if (e == cudaSuccess && rc == BD_OK) e = cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e2 = cudaFreeAsync(scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, "bd_plume_advance");
    if (e2 != cudaSuccess) return cuda_status(e2, "bd_plume_advance: cudaFreeAsync");
    if (host_err) return fail(BD_ERR_TIMEOUT, "bd_plume_advance: a TMA wait timed out");
    return BD_OK;
}

extern "C" int bd_plume_steps_per_substep(const BdPlumeParams* p, int* n_steps, float* dt_step) {
    BD_REQUIRE(p && n_steps && dt_step, "bd_plume_steps_per_substep: NULL argument");
    float decay;
    return plume_policy_steps(p, n_steps, dt_step, &decay);
}

extern "C" int bd_pack_flags(const uint8_t* abl, const uint8_t* dry, const uint8_t* vd, int64_t n, uint8_t* out,
                             void* stream) {
    BD_REQUIRE(abl && dry && out, "bd_pack_flags: NULL mask");
    if (n <= 0) return BD_OK;
    k_pack_flags<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(abl, dry, vd, n, out);
    BD_CHECK_LAUNCH("k_pack_flags");
    return BD_OK;
}
