// Epoch-end geometry update: phase / property interpolation, voxel removal, air-gap breach,
// plume injection + extinction saturation and the packed MC properties of the next epoch.
//
// Reference (all host numba/numpy in the reference, even in GPU mode):
//   _update_phase_properties_numba      simulation/coupled_ablation.py:77-180
//   _update_single_stage_ablation_numba simulation/coupled_ablation.py:61-74
//   _remove (+ air-gap breach)          simulation/coupled_ablation.py:628-660
//   compute_void_mask                   simulation/coupled_ablation.py:619-626
//   MultispectralPlumeField.inject      simulation/plume.py:292-331 (point injection)
//   sync_extinction                     simulation/plume.py:352-366
//   plume-augmented MC properties       simulation/coupled_ablation.py:445-452
//   diagnostics                         simulation/coupled_ablation.py:594-617
//
// Three launches per epoch because the reference has two grid-wide dependencies:
//   k_phase_remove   per voxel: T_peak, phase update, removal; counts n_new
//   k_gap_breach     per column: breach through the air gap when n_new > 0, gap_open flag
//   k_void_plume     per voxel: void bit, plume inject / saturate, MC props, diagnostics
#include "common.cuh"
#include "engine.cuh"

namespace bd {

__device__ __forceinline__ float gv(const GridRef& r, size_t i) { return r.ptr ? r.ptr[i] : r.value; }

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) r += sh[q];
    return r;  // valid on thread 0
}

// ---- 1. phase update + removal ----------------------------------------------------------
__global__ void __launch_bounds__(256) k_phase_remove(PhaseArgs a, long long nv) {
    __shared__ unsigned long long sh[8];
    unsigned long long mine = 0;
    const float t_now = a.dyn->t_now;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        const float T = a.T[i];
        if (a.T_peak) a.T_peak[i] = fmaxf(a.T_peak[i], T);
        uint8_t f = a.flags[i];
        f &= (uint8_t)~BD_FLAG_NEWLY;
        bool rem = false;
        if (!(f & BD_FLAG_ABLATED)) {
            if (a.single_stage) {
                // coupled_ablation.py:61-74
                rem = (a.H[i] >= a.h_lat[i]) && (T >= a.t_abl);
            } else {
                bool dry = (f & BD_FLAG_DRY) != 0;
                float h = a.H[i];
                const float hl_raw = a.h_lat[i];
                const float hl = fmaxf(hl_raw, 1e-30f);
                const float dmua = gv(a.ds_mu_a, i), dk = gv(a.ds_k, i), drho = gv(a.ds_rho, i);
                if (!dry && h > 0.0f) {
                    const float frac = fminf(fmaxf(h / hl, 0.0f), 1.0f);
                    const float wa = a.wet_mu_a[i], wk = a.wet_k[i], wr = a.wet_rho[i];
                    a.mu_a[i] = wa + (dmua - wa) * frac;
                    a.k[i] = wk + (dk - wk) * frac;
                    a.rho[i] = wr + (drho - wr) * frac;
                    if (h >= hl_raw) {
                        dry = true;
                        f |= BD_FLAG_DRY;
                        a.H[i] = 0.0f;
                        a.mu_a[i] = dmua;
                        a.mu_s[i] = gv(a.ds_mu_s, i);
                        a.g[i] = gv(a.ds_g, i);
                        a.n[i] = gv(a.ds_n, i);
                        a.k[i] = dk;
                        a.rho[i] = drho;
                    }
                }
                if (dry) {
                    if (a.has_cs) {
                        const float c = a.chi ? a.chi[i] : 0.0f;
                        if (a.has_cs_mu_a) a.mu_a[i] = dmua + c * (gv(a.cs_mu_a, i) - dmua);
                        if (a.has_cs_mu_s) {
                            const float dms = gv(a.ds_mu_s, i);
                            a.mu_s[i] = dms + c * (gv(a.cs_mu_s, i) - dms);
                        }
                        if (a.has_cs_k) a.k[i] = dk + c * (gv(a.cs_k, i) - dk);
                        float r = a.has_cs_rho ? drho + c * (gv(a.cs_rho, i) - drho) : a.rho[i];
                        const float mn = a.k[i] / a.alpha_max;
                        if (r < mn) r = mn;
                        a.rho[i] = r;
                        rem = (T >= gv(a.cs_t_rem, i)) || (c >= a.cs_chi_rem);
                    } else {
                        rem = T >= gv(a.ds_t_rem, i);
                    }
                }
            }
        }
        if (a.to_remove) a.to_remove[i] = rem ? 1 : 0;
        if (rem && a.apply_removal) {
            // _remove (coupled_ablation.py:632-643)
            f = (uint8_t)((f | BD_FLAG_ABLATED | BD_FLAG_NEWLY) & ~BD_FLAG_DRY);
            if (a.chi) a.chi[i] = 0.0f;
            if (a.ablation_time) a.ablation_time[i] = t_now;
            a.mu_a[i] = 0.0f; a.mu_s[i] = 0.0f; a.g[i] = 0.0f; a.n[i] = 1.0f;
            a.k[i] = a.k_void;
            a.rho[i] = a.rho_void;
            a.T[i] = a.t_void;
            a.H[i] = 0.0f;
            ++mine;
        }
        a.flags[i] = f;
    }
    unsigned long long s = block_sum(mine, sh);
    if (threadIdx.x == 0 && s) atomicAdd(&a.dyn->n_new, s);
}

// ---- 2. air-gap breach (coupled_ablation.py:645-654) and gap_open (:619-626) ----------
__global__ void k_gap_breach(PhaseArgs a) {
    const int ncol = a.nx * a.ny;
    const int k0 = a.gap_k0, k1 = a.gap_k1;
    const bool removed = a.dyn->n_new > 0;
    const float t_now = a.dyn->t_now;
    unsigned any = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += gridDim.x * blockDim.x) {
        const size_t base = (size_t)c * a.nz;
        if (!(a.flags[base + k0 - 1] & BD_FLAG_ABLATED)) continue;
        any = 1;
        if (removed && !(a.flags[base + k0] & BD_FLAG_ABLATED)) {
            for (int k = k0; k < k1; ++k) {
                a.flags[base + k] |= BD_FLAG_ABLATED;
                if (a.ablation_time) a.ablation_time[base + k] = t_now;
            }
        }
    }
    if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(&a.dyn->gap_open, 1u);
}

// ---- 3. void mask, plume inject/sync, packed MC properties, diagnostics ---------------
__global__ void __launch_bounds__(256) k_void_plume(PhaseArgs a, long long nv) {
    __shared__ double shd[8];
    const bool gap_open = a.gap_k0 > 0 && a.dyn->gap_open != 0;
    const bool inject = !a.props_only && a.dyn->n_new > 0;
    const int mid_col = (a.nx / 2) * a.ny + a.ny / 2;
    double tau_sum = 0.0, abl_sum = 0.0, abl_cnt = 0.0;
    float peak = 0.0f;
    int kmax = -1;
    unsigned long long n_void = 0;
    // (column, z) of voxel i, stepped with the grid stride instead of two 64-bit divisions per voxel
    const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int sk = (int)(stride % a.nz);
    const long long sc = stride / a.nz;
    long long col = i0 / a.nz;
    int k = (int)(i0 - col * a.nz);
    for (long long i = i0; i < nv; i += stride, col += sc, k += sk) {
        if (k >= a.nz) {
            k -= a.nz;
            ++col;
        }
        uint8_t f = a.flags[i];
        const bool ablated = (f & BD_FLAG_ABLATED) != 0;
        const bool vd = ablated || (gap_open && k >= a.gap_k0 && k < a.gap_k1);
        f = vd ? (uint8_t)(f | BD_FLAG_VOID) : (uint8_t)(f & ~BD_FLAG_VOID);
        a.flags[i] = f;
        if (vd) {
            kmax = max(kmax, k);
            ++n_void;
        }
        float mu_ext = 0.0f;
        if (a.has_plume) {
            float raw = a.plume[i];
            if (inject && (f & BD_FLAG_NEWLY)) raw = raw + a.delta_mu;   // plume.py:329
            if (!vd) raw = 0.0f;                                           // plume.py:330-331, :357-358
            a.plume[i] = raw;
            if (vd) mu_ext = a.mu_max > 0.0f ? a.mu_max * tanhf(raw / a.mu_max) : raw;  // :359-363
            a.mu_ext[i] = mu_ext;
            const float mua_p = mu_ext * a.ratio_a;
            peak = fmaxf(peak, mua_p);
            if (col == mid_col) tau_sum += (double)mua_p;
            if (ablated) { abl_sum += (double)mua_p; abl_cnt += 1.0; }
        } else if (ablated) {
            abl_cnt += 1.0;
        }
        if (a.props) {
            float ma = a.mu_a[i], ms = a.mu_s[i], gg = a.g[i];
            if (a.has_plume) {
                ma = ma + mu_ext * a.ratio_a;
                ms = ms + mu_ext * a.ratio_s;
                if (mu_ext > 0.001f && ablated) gg = a.g_plume;
            }
            const float mt = ma + ms;
            reinterpret_cast<float4*>(a.props)[i] = make_float4(mt, mt > 0.0f ? ma / mt : 0.0f, gg, a.n[i]);
        }
    }
    __shared__ unsigned long long shu[8];
    const unsigned long long nvb = block_sum(n_void, shu);
    double s0 = block_sum(tau_sum, shd);
    double s1 = block_sum(abl_sum, shd);
    double s2 = block_sum(abl_cnt, shd);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) peak = fmaxf(peak, __shfl_xor_sync(0xffffffffu, peak, o));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    if ((threadIdx.x & 31) == 0 && kmax >= 0) atomicMax(&a.dyn->void_zlimit, kmax + 1);
    if (a.props_only) return;              // the epoch's diagnostics are already complete
    __shared__ float shp[8];
    if ((threadIdx.x & 31) == 0) shp[threadIdx.x >> 5] = peak;
    __syncthreads();
    if (threadIdx.x == 0) {
        float pm = 0.0f;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) pm = fmaxf(pm, shp[q]);
        if (s0 != 0.0) atomicAdd(&a.dyn->plume_tau_sum, s0);
        if (s1 != 0.0) atomicAdd(&a.dyn->plume_abl_sum, s1);
        if (s2 != 0.0) atomicAdd(&a.dyn->n_ablated, s2);
        if (nvb) atomicAdd(&a.dyn->n_void, nvb);
        // non-negative floats order like their bit patterns
        if (pm > 0.0f) atomicMax(&a.dyn->plume_peak_bits, __float_as_uint(pm));
    }
}

int phase_launch(const PhaseArgs& args, int mode, cudaStream_t st) {
    PhaseArgs a = args;
    a.props_only = mode == BD_PHASE_PROPS ? 1 : 0;
    const long long nv = (long long)a.nx * a.ny * a.nz;
    const int blocks = grid_for(nv, 256, 148 * 16);
    if (mode == BD_PHASE_PROPS) {
        k_void_plume<<<blocks, 256, 0, st>>>(a, nv);
        BD_CHECK_LAUNCH("k_void_plume");
        return BD_OK;
    }
    if (mode == BD_PHASE_FULL) {
        k_phase_remove<<<blocks, 256, 0, st>>>(a, nv);
        BD_CHECK_LAUNCH("k_phase_remove");
    }
    if (a.gap_k0 > 0) {
        k_gap_breach<<<grid_for((long long)a.nx * a.ny, 128, 148 * 8), 128, 0, st>>>(a);
        BD_CHECK_LAUNCH("k_gap_breach");
    }
    k_void_plume<<<blocks, 256, 0, st>>>(a, nv);
    BD_CHECK_LAUNCH("k_void_plume");
    return BD_OK;
}

}  // namespace bd
