// Explicit 7-point bioheat stencil and the fused ablation substep (the plume is in plume.cu).
//
// Thermal update (voxel_thermal_3d.py:30-112, voxel_thermal_metal.py:56-134):
//   T' = T + dt (sum_faces k_face (T_nb - T) / d^2 + Q) / rho_cp,
//   k_face = 2 k_c k_n / (k_c + k_n + 1e-12); x/y faces insulated; z faces convective
//   (series half-cell + h_eff, or the Metal fused kernel's -h_eff (T - T_amb)/dz).
// Fused substep (metal_ablation_solver.py:71-191; CPU twin coupled_ablation.py:515-531):
//   + latent-heat plateau (voxel_thermal_3d.py:115-143), Arrhenius damage
//   (coupled_ablation.py:33-40) and first-order char kinetics (coupled_ablation.py:43-58),
//   all pointwise on the trial temperature, so one pass per substep does everything.
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

// Unused dynamic shared memory that lets at most `cap` substep CTAs share an SM (0: no cap). The
// plume stage runs beside the substeps; capping them leaves the plume's CTAs room on every SM (16 KB
// of shared memory per SM stay free for them). The kernel's limit is raised once per instantiation.
static size_t substep_pad_bytes(int cap, const void* kernel) {
    if (cap <= 0) return 0;
    int dev = 0, per_sm = 0, per_block = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return 0;
    const long long reserve = 1024;                  // per-CTA shared memory the system keeps
    long long pad = ((long long)per_sm - 16384) / cap - (long long)fa.sharedSizeBytes - reserve;
    pad = std::max(0LL, std::min(pad, (long long)per_block - (long long)fa.sharedSizeBytes));
    if (pad > 48 * 1024 && fa.maxDynamicSharedSizeBytes < pad)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pad);
    return (size_t)pad;
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
        const size_t pad = substep_pad_bytes(tune_value(BD_TUNE_STENCIL_CAP), (const void*)k_substep_tma<MODE, BC, ARR, CHAR>);
        for (int s = 0; s < n; ++s) {
            float* out = (s & 1) ? Ta : Tb;
            k_substep_tma<MODE, BC, ARR, CHAR><<<grid, dim3(TZ, TY), pad, st>>>((s & 1) ? mb : ma, mk, g, c, out, src,
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

extern "C" int bd_pack_flags(const uint8_t* abl, const uint8_t* dry, const uint8_t* vd, int64_t n, uint8_t* out,
                             void* stream) {
    BD_REQUIRE(abl && dry && out, "bd_pack_flags: NULL mask");
    if (n <= 0) return BD_OK;
    k_pack_flags<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(abl, dry, vd, n, out);
    BD_CHECK_LAUNCH("k_pack_flags");
    return BD_OK;
}
