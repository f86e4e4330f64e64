// Voxel Monte Carlo photon transport (hop-drop-spin with optical-depth voxel marching).
//
// Algorithm follows the reference CPU tracer simulation/voxel_mc_3d.py:123-337
// (_trace_one_photon) and its Metal twin simulation/voxel_mc_metal.py:173-332:
//   launch (Gaussian / top-hat / Kim disks, oblique footprint stretch u1/cos(theta))
//   -> deterministic entrance Fresnel split + Snell refraction
//   -> loop: tau = -ln(xi) consumed voxel by voxel; collision absorbs w*mu_a/mu_t,
//      Russian roulette at w < 1e-4 (survive 1/10 with w*10), Henyey-Greenstein scatter;
//      face crossings do Fresnel/TIR or Snell at index steps, exits tally R_diff / T / lateral.
//
// B200 design:
//   * one persistent grid, photons handed out by a global atomic queue; every lane advances its
//     photon by one event per loop iteration and takes a new photon as soon as its own ends, so
//     warps stay full while the per-photon event counts differ by orders of magnitude;
//   * Philox-4x32-10 counter-based RNG keyed on (seed, photon index): no RNG state in memory
//     and a photon's path does not depend on which thread traced it;
//   * optical properties packed as one float4 {mu_t, mu_a/mu_t, g, n} per voxel read through
//     the read-only (L1/texture) path: one 16-byte load per event;
//   * absorbed weight and track length tallied with fire-and-forget FP32 reductions;
//   * FP64 ledger: per-thread FP64 registers for the per-event channels, per-block shared
//     accumulators for per-photon channels, one partial per block reduced in a fixed order.
#include "common.cuh"

#include <stdlib.h>

#include <algorithm>
#include <atomic>
#include <mutex>

namespace bd {

struct McDev {
    int nx, ny, nz, launch_axis;
    float dx, dy, dz, lx, ly, lz;
    float ux0, uy0, uz0, cos_ph, sin_ph, cos_th_safe;
    float xc, yc, zc, sigma, radius;
    int profile;
    float n_amb, rmax2;
    int options;
    long long n_photons, offset, max_events;
    unsigned long long seed;
    float eq_eps;     // Fresnel index-equality guard
    float step_eps;   // internal index-step threshold
    float entry_eps;  // entrance refraction threshold
};

__device__ __forceinline__ float fresnel_unpol(float n1, float n2, float cos_i, float eq_eps) {
    // voxel_mc_3d.py:33-48 / voxel_mc_metal.py:70-83
    if (fabsf(n1 - n2) < eq_eps) return 0.0f;
    cos_i = fminf(1.0f, fabsf(cos_i));
    if (cos_i > 0.999999f) {
        float r = (n1 - n2) / (n1 + n2);
        return r * r;
    }
    float q = n1 / n2;
    float sin_t2 = q * q * (1.0f - cos_i * cos_i);
    if (sin_t2 >= 1.0f) return 1.0f;
    float cos_t = sqrtf(1.0f - sin_t2);
    float a = n1 * cos_i, b = n2 * cos_t, c = n1 * cos_t, d = n2 * cos_i;
    float rs = (a - b) / (a + b);
    float rp = (c - d) / (c + d);
    return 0.5f * (rs * rs + rp * rp);
}

// Snell refraction across an axis-aligned face (voxel_mc_3d.py:51-69)
__device__ __forceinline__ void refract_axis(float& ux, float& uy, float& uz, int axis, float eta) {
    if (axis == 0) {
        float s = ux > 0.0f ? 1.0f : -1.0f;
        uy *= eta; uz *= eta;
        ux = s * sqrtf(fmaxf(0.0f, 1.0f - uy * uy - uz * uz));
    } else if (axis == 1) {
        float s = uy > 0.0f ? 1.0f : -1.0f;
        ux *= eta; uz *= eta;
        uy = s * sqrtf(fmaxf(0.0f, 1.0f - ux * ux - uz * uz));
    } else {
        float s = uz > 0.0f ? 1.0f : -1.0f;
        ux *= eta; uy *= eta;
        uz = s * sqrtf(fmaxf(0.0f, 1.0f - ux * ux - uy * uy));
    }
}

// Henyey-Greenstein deflection + uniform azimuth (voxel_mc_3d.py:229-262)
__device__ __forceinline__ void scatter_hg(float& ux, float& uy, float& uz, float g, PhotonRng& rng) {
    float xi = rng.uniform();
    float cost;
    if (fabsf(g) < 1e-4f) {
        cost = 2.0f * xi - 1.0f;
    } else {
        float t = (1.0f - g * g) / (1.0f - g + 2.0f * g * xi);
        cost = (1.0f + g * g - t * t) / (2.0f * g);
        cost = fminf(1.0f, fmaxf(-1.0f, cost));
    }
    float sint = sqrtf(fmaxf(0.0f, 1.0f - cost * cost));
    float sinp, cosp;
    sincospif(2.0f * rng.uniform(), &sinp, &cosp);
    float nx, ny, nz;
    if (fabsf(uz) > 0.99999f) {
        float sz = uz > 0.0f ? 1.0f : -1.0f;
        nx = sint * cosp;
        ny = sint * sinp;
        nz = cost * sz;
    } else {
        float den = sqrtf(fmaxf(1.0f - uz * uz, 1e-12f));
        float f = sint / den;
        nx = f * (ux * uz * cosp - uy * sinp) + ux * cost;
        ny = f * (uy * uz * cosp + ux * sinp) + uy * cost;
        nz = -sint * cosp * den + uz * cost;
    }
    float nn = nx * nx + ny * ny + nz * nz;
    if (nn > 1e-24f) {
        float r = rsqrtf(nn);
        nx *= r; ny *= r; nz *= r;
    }
    ux = nx; uy = ny; uz = nz;
}

// Transverse launch offsets (voxel_mc_3d.py:101-120)
__device__ __forceinline__ void beam_offsets(const McDev& P, PhotonRng& rng, float& u1, float& u2) {
    if (P.profile == BD_BEAM_TOPHAT) {
        float r = P.radius * sqrtf(rng.uniform());
        float s, c;
        sincospif(2.0f * rng.uniform(), &s, &c);
        u1 = r * c; u2 = r * s;
        return;
    }
    if (P.profile == BD_BEAM_KIM_EXP_DISK || P.profile == BD_BEAM_KIM_GAUSS_DISK) {
        float rn = 0.0f;
        // rejection sampling; acceptance >= e^-2, so 256 tries all fail with p < 1e-16
        for (int t = 0; t < 256; ++t) {
            rn = sqrtf(rng.uniform());
            float acc = (P.profile == BD_BEAM_KIM_EXP_DISK) ? expf(-2.0f * rn) : expf(-2.0f * rn * rn);
            if (rng.uniform() < acc) break;
        }
        float s, c;
        sincospif(2.0f * rng.uniform(), &s, &c);
        u1 = P.radius * rn * c; u2 = P.radius * rn * s;
        return;
    }
    // Gaussian: Box-Muller pair with per-axis sigma
    float a = rng.uniform_pos();
    float b = rng.uniform();
    float r = sqrtf(-2.0f * logf(a)) * P.sigma;
    float s, c;
    sincospif(2.0f * b, &s, &c);
    u1 = r * c; u2 = r * s;
}

// Per-thread FP64 accumulator for the per-collision channel (absorbed weight); the rare
// channels (exits, roulette, truncation, absorption in void) go straight to the block's
// partial row with FP64 atomics, so no block-wide barrier is needed anywhere in the kernel.
struct ThreadLedger {
    double absorbed;
    unsigned collisions, crossings, reflections;
};

// The photon a lane is tracing. The kernel advances every lane by one event per loop iteration,
// and a lane whose photon has ended takes the next photon from the queue in the same loop, so the
// lanes of a warp are not held back until the warp's longest photon ends (event counts per photon
// differ by orders of magnitude). A photon's random stream and arithmetic do not depend on the
// lane that traces it or on when it is traced.
struct PhotonState {
    PhotonRng rng;
    float x, y, z, ux, uy, uz, iux, iuy, iuz, tau, w;
    float4 pr;
    int ix, iy, iz, idx;
    long long ev;
};

// Launch: transverse offsets, footprint test, entrance Fresnel split and refraction, first
// optical depth. Returns false when the photon never enters the grid (booked here).
template <int DEPTH>  // 2: launch along +z at z=0 ; 0: launch along +x at x=0
__device__ __forceinline__ bool photon_launch(const McDev& P, long long pid, const float4* __restrict__ props,
                                              double* __restrict__ latz, double* sl, PhotonState& s) {
    s.rng.init(P.seed, (unsigned long long)(P.offset + pid));
    float u1, u2;
    beam_offsets(P, s.rng, u1, u2);
    const float stretch = u1 / P.cos_th_safe;
    if (DEPTH == 2) {
        s.x = P.xc + stretch * P.cos_ph - u2 * P.sin_ph;
        s.y = P.yc + stretch * P.sin_ph + u2 * P.cos_ph;
        s.z = 0.0f;
        bool out = s.x < 0.0f || s.x >= P.lx || s.y < 0.0f || s.y >= P.ly;
        if (!out && P.rmax2 > 0.0f) {
            float a = s.x - P.xc, b = s.y - P.yc;
            out = a * a + b * b >= P.rmax2;
        }
        if (out) {
            atomicAdd(&sl[BD_LEDGER_LATERAL], 1.0);
            if (latz) atomicAdd(&latz[0], 1.0);
            return false;
        }
        s.ix = min((int)(s.x / P.dx), P.nx - 1);
        s.iy = min((int)(s.y / P.dy), P.ny - 1);
        s.iz = 0;
    } else {
        s.x = 0.0f;
        s.y = P.yc + stretch * P.cos_ph - u2 * P.sin_ph;
        s.z = P.zc + stretch * P.sin_ph + u2 * P.cos_ph;
        bool out = s.y < 0.0f || s.y >= P.ly || s.z < 0.0f || s.z >= P.lz;
        if (!out && P.rmax2 > 0.0f) {
            float a = s.y - P.yc, b = s.z - P.zc;
            out = a * a + b * b >= P.rmax2;
        }
        if (out) {
            atomicAdd(&sl[BD_LEDGER_LATERAL], 1.0);
            if (latz) atomicAdd(&latz[0], 1.0);
            return false;
        }
        s.ix = 0;
        s.iy = min((int)(s.y / P.dy), P.ny - 1);
        s.iz = min((int)(s.z / P.dz), P.nz - 1);
    }
    s.ux = P.ux0; s.uy = P.uy0; s.uz = P.uz0;
    s.idx = s.ix * (P.ny * P.nz) + s.iy * P.nz + s.iz;

    // entrance face: deterministic specular split + refraction (voxel_mc_3d.py:183-192)
    s.pr = __ldg(&props[s.idx]);
    {
        float n_in = s.pr.w;
        float cos_in = (DEPTH == 2) ? s.uz : s.ux;
        float r = fresnel_unpol(P.n_amb, n_in, cos_in, P.eq_eps);
        s.w = 1.0f - r;
        // the ledger books what the FP32 weight actually lost, so it closes exactly
        atomicAdd(&sl[BD_LEDGER_SPECULAR], 1.0 - (double)s.w);
        if (s.w <= 0.0f) return false;
        if (fabsf(n_in - P.n_amb) > P.entry_eps) refract_axis(s.ux, s.uy, s.uz, DEPTH, P.n_amb / n_in);
    }
    s.iux = fabsf(s.ux) > 1e-15f ? 1.0f / s.ux : 0.0f;
    s.iuy = fabsf(s.uy) > 1e-15f ? 1.0f / s.uy : 0.0f;
    s.iuz = fabsf(s.uz) > 1e-15f ? 1.0f / s.uz : 0.0f;
    s.tau = -__logf(fmaxf(s.rng.uniform(), 1e-12f));
    s.ev = 0;
    return true;
}

// One event of the hop-drop-spin loop (voxel_mc_3d.py:194-337): a collision inside the voxel or a
// crossing of its exit face. Returns false when the photon has ended (its weight booked).
template <int DEPTH>
__device__ __forceinline__ bool photon_event(const McDev& P, const float4* __restrict__ props,
                                             const uint8_t* __restrict__ flags, float* __restrict__ A,
                                             unsigned long long* __restrict__ A64, float* __restrict__ L,
                                             double* __restrict__ latz, double* sl, ThreadLedger& tl,
                                             PhotonState& s, bool metal, bool tally_l) {
    const float dx = P.dx, dy = P.dy, dz = P.dz;
    // exact ray/box distance to the exit face (voxel_mc_3d.py:72-98)
    float sx = s.ux > 1e-15f ? ((float)(s.ix + 1) * dx - s.x) * s.iux
                             : (s.ux < -1e-15f ? ((float)s.ix * dx - s.x) * s.iux : 1e30f);
    float sy = s.uy > 1e-15f ? ((float)(s.iy + 1) * dy - s.y) * s.iuy
                             : (s.uy < -1e-15f ? ((float)s.iy * dy - s.y) * s.iuy : 1e30f);
    float sz = s.uz > 1e-15f ? ((float)(s.iz + 1) * dz - s.z) * s.iuz
                             : (s.uz < -1e-15f ? ((float)s.iz * dz - s.z) * s.iuz : 1e30f);
    int axis;
    float s_exit;
    if (sx <= sy && sx <= sz) { axis = 0; s_exit = fmaxf(sx, 0.0f); }
    else if (sy <= sz)        { axis = 1; s_exit = fmaxf(sy, 0.0f); }
    else                      { axis = 2; s_exit = fmaxf(sz, 0.0f); }
    const float mu_t = s.pr.x;

    if (mu_t > 1e-12f && mu_t * s_exit >= s.tau) {
        // ---- interaction inside the voxel ----
        ++tl.collisions;
        float st = s.tau / mu_t;
        if (tally_l) atomicAdd(&L[s.idx], s.w * st);
        s.x += st * s.ux; s.y += st * s.uy; s.z += st * s.uz;
        if (P.rmax2 > 0.0f) {
            float a = (DEPTH == 2) ? s.x - P.xc : s.y - P.yc;
            float b = (DEPTH == 2) ? s.y - P.yc : s.z - P.zc;
            if (a * a + b * b >= P.rmax2) {
                atomicAdd(&sl[BD_LEDGER_LATERAL], (double)s.w);
                if (latz) atomicAdd(&latz[DEPTH == 2 ? s.iz : s.ix], (double)s.w);
                return false;
            }
        }
        {
            const float dw = s.w * s.pr.y;
            const float w_new = s.w - dw;
            if (A64) atomicAdd(&A64[s.idx], __float2ull_rn(dw * kTallyScale));
            else atomicAdd(&A[s.idx], dw);
            const double lost = (double)s.w - (double)w_new;  // exact: both are FP32 values
            if (flags != nullptr && (__ldg(&flags[s.idx]) & BD_FLAG_ABLATED)) atomicAdd(&sl[BD_LEDGER_ABSORBED_VOID], lost);
            else tl.absorbed += lost;
            s.w = w_new;
        }
        if (s.w < 1e-4f) {
            if (s.rng.uniform() < 0.1f) {
                const float w10 = s.w * 10.0f;
                atomicAdd(&sl[BD_LEDGER_ROULETTE_GAIN], (double)w10 - (double)s.w);
                s.w = w10;
            } else {
                atomicAdd(&sl[BD_LEDGER_ROULETTE_LOSS], (double)s.w);
                return false;
            }
        }
        scatter_hg(s.ux, s.uy, s.uz, s.pr.z, s.rng);
        s.iux = fabsf(s.ux) > 1e-15f ? 1.0f / s.ux : 0.0f;
        s.iuy = fabsf(s.uy) > 1e-15f ? 1.0f / s.uy : 0.0f;
        s.iuz = fabsf(s.uz) > 1e-15f ? 1.0f / s.uz : 0.0f;
        s.tau = -__logf(fmaxf(s.rng.uniform(), 1e-12f));
        return true;
    }

    // ---- traverse the chord and land exactly on the exit face ----
    ++tl.crossings;
    s.tau -= mu_t * s_exit;
    if (tally_l) atomicAdd(&L[s.idx], s.w * s_exit);
    s.x += s_exit * s.ux; s.y += s_exit * s.uy; s.z += s_exit * s.uz;
    int jx = s.ix, jy = s.iy, jz = s.iz;
    if (axis == 0)      { int sd = s.ux > 0.0f ? 1 : -1; jx += sd; s.x = sd > 0 ? (float)(s.ix + 1) * dx : (float)s.ix * dx; }
    else if (axis == 1) { int sd = s.uy > 0.0f ? 1 : -1; jy += sd; s.y = sd > 0 ? (float)(s.iy + 1) * dy : (float)s.iy * dy; }
    else                { int sd = s.uz > 0.0f ? 1 : -1; jz += sd; s.z = sd > 0 ? (float)(s.iz + 1) * dz : (float)s.iz * dz; }

    if (axis == DEPTH) {
        const int jd = (DEPTH == 2) ? jz : jx;
        const int nd = (DEPTH == 2) ? P.nz : P.nx;
        if (jd < 0) {
            // leaving through the entrance face: Fresnel / TIR against ambient
            float cos_out = (DEPTH == 2) ? s.uz : s.ux;
            float r = fresnel_unpol(s.pr.w, P.n_amb, cos_out, P.eq_eps);
            if (r > 0.0f && s.rng.uniform() < r) {
                ++tl.reflections;
                if (DEPTH == 2) { s.uz = -s.uz; s.iuz = -s.iuz; } else { s.ux = -s.ux; s.iux = -s.iux; }
                return true;
            }
            atomicAdd(&sl[BD_LEDGER_DIFFUSE], (double)s.w);
            return false;
        }
        if (jd >= nd) {
            atomicAdd(&sl[BD_LEDGER_TRANSMITTED], (double)s.w);
            return false;
        }
    } else if (jx < 0 || jx >= P.nx || jy < 0 || jy >= P.ny || jz < 0 || jz >= P.nz) {
        atomicAdd(&sl[BD_LEDGER_LATERAL], (double)s.w);
        if (latz) atomicAdd(&latz[DEPTH == 2 ? s.iz : s.ix], (double)s.w);
        return false;
    }
    if (!metal && P.rmax2 > 0.0f) {
        float a = (DEPTH == 2) ? s.x - P.xc : s.y - P.yc;
        float b = (DEPTH == 2) ? s.y - P.yc : s.z - P.zc;
        if (a * a + b * b >= P.rmax2) {
            atomicAdd(&sl[BD_LEDGER_LATERAL], (double)s.w);
            if (latz) atomicAdd(&latz[DEPTH == 2 ? s.iz : s.ix], (double)s.w);
            return false;
        }
    }
    const int jidx = jx * (P.ny * P.nz) + jy * P.nz + jz;
    float4 pn = __ldg(&props[jidx]);
    float n1 = s.pr.w, n2 = pn.w;
    if (fabsf(n1 - n2) > P.step_eps) {
        float cos_face = axis == 0 ? s.ux : (axis == 1 ? s.uy : s.uz);
        float r = fresnel_unpol(n1, n2, cos_face, P.eq_eps);
        if ((!metal || r > 0.0f) && s.rng.uniform() < r) {
            ++tl.reflections;
            if (axis == 0) { s.ux = -s.ux; s.iux = -s.iux; }
            else if (axis == 1) { s.uy = -s.uy; s.iuy = -s.iuy; }
            else { s.uz = -s.uz; s.iuz = -s.iuz; }
            return true;
        }
        refract_axis(s.ux, s.uy, s.uz, axis, n1 / n2);
        s.iux = fabsf(s.ux) > 1e-15f ? 1.0f / s.ux : 0.0f;
        s.iuy = fabsf(s.uy) > 1e-15f ? 1.0f / s.uy : 0.0f;
        s.iuz = fabsf(s.uz) > 1e-15f ? 1.0f / s.uz : 0.0f;
    }
    s.ix = jx; s.iy = jy; s.iz = jz;
    s.idx = jidx;
    s.pr = pn;
    return true;
}

#ifndef BD_MC_MIN_BLOCKS
#define BD_MC_MIN_BLOCKS 8
#endif
template <int DEPTH>
__global__ void __launch_bounds__(128, BD_MC_MIN_BLOCKS) k_mc_trace(McDev P, const float4* __restrict__ props,
                                                     const uint8_t* __restrict__ flags, float* __restrict__ A,
                                                     unsigned long long* __restrict__ A64,
                                                     float* __restrict__ L, double* __restrict__ latz,
                                                     unsigned long long* __restrict__ queue,
                                                     double* __restrict__ partials,
                                                     const long long* __restrict__ offset_dev) {
    // a photon-stream offset kept in device memory lets a captured graph advance it per replay
    if (offset_dev != nullptr) P.offset += *offset_dev;
    double* sl = partials + (size_t)blockIdx.x * BD_LEDGER_LEN;  // zeroed before the launch
    ThreadLedger tl;
    tl.absorbed = 0.0;
    tl.collisions = tl.crossings = tl.reflections = 0u;
    const bool metal = (P.options & BD_MC_METAL_SEMANTICS) != 0;
    const bool tally_l = (P.options & BD_MC_TALLY_FLUENCE) != 0 && L != nullptr;

    const unsigned long long N = (unsigned long long)P.n_photons;
    PhotonState s;
    bool live = false;
    for (;;) {
        if (!live) {
            const unsigned long long p = atomicAdd(queue, 1ull);
            if (p >= N) break;
            live = photon_launch<DEPTH>(P, (long long)p, props, latz, sl, s);
            if (!live) continue;
        }
        if (s.ev >= P.max_events) {
            // event cap reached: the remaining weight is accounted, not lost
            atomicAdd(&sl[BD_LEDGER_TRUNCATED], (double)s.w);
            live = false;
            continue;
        }
        ++s.ev;
        live = photon_event<DEPTH>(P, props, flags, A, A64, L, latz, sl, tl, s, metal, tally_l);
    }
    // warp reduction of the per-thread channels, one FP64 atomic per warp and channel
    double v0 = tl.absorbed;
    unsigned c0 = tl.collisions, c1 = tl.crossings, c2 = tl.reflections;
    __syncwarp();  // every lane reaches here (no early return): reconverge for the shuffles
    const unsigned mask = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(mask, v0, o);
        c0 += __shfl_xor_sync(mask, c0, o);
        c1 += __shfl_xor_sync(mask, c1, o);
        c2 += __shfl_xor_sync(mask, c2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sl[BD_LEDGER_ABSORBED], v0);
        atomicAdd(&sl[BD_LEDGER_COLLISIONS], (double)c0);
        atomicAdd(&sl[BD_LEDGER_CROSSINGS], (double)c1);
        atomicAdd(&sl[BD_LEDGER_REFLECTIONS], (double)c2);
    }
}

// Fixed-order reduction of the per-block partials (deterministic for a given grid).
__global__ void k_ledger_reduce(const double* __restrict__ partials, int nblocks, double launched,
                                double* __restrict__ ledger) {
    int ch = threadIdx.x;
    if (ch >= BD_LEDGER_LEN) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partials[(size_t)b * BD_LEDGER_LEN + ch];
    if (ch == BD_LEDGER_LAUNCHED) s = launched;
    ledger[ch] = s;
}

__global__ void k_pack_props(const float* __restrict__ mu_a, const float* __restrict__ mu_s,
                             const float* __restrict__ g, const float* __restrict__ n,
                             const float* __restrict__ mu_ext, const uint8_t* __restrict__ flags,
                             float ra, float rs, float g_plume, long long nv, float4* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv;
         i += (long long)gridDim.x * blockDim.x) {
        float a = mu_a[i], s = mu_s[i], gg = g[i], nn = n[i];
        if (mu_ext != nullptr) {
            float e = mu_ext[i];
            a = a + e * ra;
            s = s + e * rs;
            if (e > 0.001f && (flags[i] & BD_FLAG_ABLATED)) gg = g_plume;
        }
        float mt = a + s;
        float ratio = mt > 0.0f ? a / mt : 0.0f;
        out[i] = make_float4(mt, ratio, gg, nn);
    }
}

// A[i] += fixed-point tally[i] in weight units; the tally is left zeroed for the next launch.
__global__ void k_tally_finalize(unsigned long long* __restrict__ t64, float* __restrict__ A, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long v = t64[i];
        if (v != 0ull) {
            A[i] += (float)((double)v * (1.0 / (double)kTallyScale));
            t64[i] = 0ull;
        }
    }
}

__global__ void k_fold(float* __restrict__ src, double* __restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float v = src[i];
        if (v != 0.0f) {
            dst[i] += (double)v;
            src[i] = 0.0f;
        }
    }
}

}  // namespace bd

// ------------------------------------------------------------------------------------
struct BdMcContext {
    unsigned long long* queue = nullptr;
    double* partials = nullptr;
    unsigned long long* tally64 = nullptr;   // fixed-point absorbed tally, grown to the largest grid
    long long tally_cap = 0;
    int partial_blocks = 0;
    int device = -1;
    int sm_count = 148;
};

using namespace bd;

extern "C" int bd_mc_create(BdMcContext** out) {
    BD_REQUIRE(out != nullptr, "bd_mc_create: out is NULL");
    BdMcContext* c = new BdMcContext();
    BD_CUDA(cudaGetDevice(&c->device));
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    // 16 resident 128-thread blocks per SM is the occupancy ceiling of k_mc_trace
    c->partial_blocks = c->sm_count * 16;
    cudaError_t e = cudaMalloc(&c->queue, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&c->partials, sizeof(double) * BD_LEDGER_LEN * c->partial_blocks);
    if (e != cudaSuccess) {
        cudaFree(c->queue);
        delete c;
        return cuda_status(e, "bd_mc_create: cudaMalloc");
    }
    *out = c;
    return BD_OK;
}

extern "C" int bd_mc_destroy(BdMcContext* c) {
    if (!c) return BD_OK;
    cudaFree(c->queue);
    cudaFree(c->partials);
    cudaFree(c->tally64);
    delete c;
    return BD_OK;
}

namespace bd {
int mc_validate(const BdMcParams* p) {
    BD_REQUIRE(p != nullptr, "bd_mc_trace: params is NULL");
    BD_REQUIRE(p->nx > 0 && p->ny > 0 && p->nz > 0, "bd_mc_trace: grid dims must be positive");
    BD_REQUIRE(p->dx > 0 && p->dy > 0 && p->dz > 0, "bd_mc_trace: voxel size must be positive");
    BD_REQUIRE(p->launch_axis == 0 || p->launch_axis == 1, "bd_mc_trace: launch_axis must be 0 (z) or 1 (x)");
    BD_REQUIRE(p->beam_profile >= 0 && p->beam_profile <= 3, "bd_mc_trace: unknown beam profile %d", p->beam_profile);
    BD_REQUIRE(p->n_photons >= 0, "bd_mc_trace: n_photons must be >= 0");
    BD_REQUIRE(p->max_events > 0, "bd_mc_trace: max_events must be > 0");
    BD_REQUIRE(p->cos_th_safe > 0.0f, "bd_mc_trace: cos_th_safe must be > 0");
    return BD_OK;
}

McDev mc_dev_params(const BdMcParams* p) {
    McDev d;
    d.nx = p->nx; d.ny = p->ny; d.nz = p->nz; d.launch_axis = p->launch_axis;
    d.dx = p->dx; d.dy = p->dy; d.dz = p->dz; d.lx = p->lx; d.ly = p->ly; d.lz = p->lz;
    d.ux0 = p->init_ux; d.uy0 = p->init_uy; d.uz0 = p->init_uz;
    d.cos_ph = p->cos_ph; d.sin_ph = p->sin_ph; d.cos_th_safe = p->cos_th_safe;
    d.xc = p->x_center; d.yc = p->y_center; d.zc = p->z_center;
    d.sigma = p->sigma_axis; d.radius = p->beam_radius; d.profile = p->beam_profile;
    d.n_amb = p->n_ambient; d.rmax2 = p->r_max_sq; d.options = p->options;
    d.n_photons = p->n_photons; d.offset = p->photon_offset; d.max_events = p->max_events;
    d.seed = p->seed;
    const bool metal = (p->options & BD_MC_METAL_SEMANTICS) != 0;
    d.eq_eps = metal ? 1e-6f : 1e-9f;
    d.step_eps = metal ? 1e-4f : 1e-9f;
    d.entry_eps = metal ? 1e-6f : 1e-9f;
    return d;
}

// Launch with caller-provided scratch (queue counter + per-block partials).
int mc_launch(const BdMcParams* p, const float* props, const uint8_t* flags, float* A, float* L,
              double* latz, double* ledger, unsigned long long* queue, double* partials, int max_blocks,
              int sm_count, cudaStream_t st, const long long* offset_dev, unsigned long long* tally64) {
    McDev d = mc_dev_params(p);
    // resident 128-thread CTAs per SM of each kernel variant: computed once, shared by host threads
    static std::atomic<int> per_sm[2] = {{0}, {0}};
    const int ax = p->launch_axis == 0 ? 0 : 1;
    int occ = per_sm[ax].load(std::memory_order_relaxed);
    if (occ == 0) {
        int nb = 0;
        if (ax == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_mc_trace<2>, 128, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_mc_trace<0>, 128, 0);
        occ = std::max(1, std::min(nb, 16));
        cudaGetLastError();
        per_sm[ax].store(occ, std::memory_order_relaxed);
    }
    const int want = tune_value(BD_TUNE_MC_BLOCKS_PER_SM);
    const int use_sm = want > 0 ? std::min(want, occ) : occ;
    int blocks = (int)std::min<long long>((p->n_photons + 127) / 128, (long long)sm_count * use_sm);
    blocks = std::max(1, std::min(blocks, max_blocks));
    BD_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st));
    BD_CUDA(cudaMemsetAsync(partials, 0, sizeof(double) * BD_LEDGER_LEN * blocks, st));
    const float4* pr = reinterpret_cast<const float4*>(props);
    if (p->launch_axis == 0)
        k_mc_trace<2><<<blocks, 128, 0, st>>>(d, pr, flags, A, tally64, L, latz, queue, partials, offset_dev);
    else
        k_mc_trace<0><<<blocks, 128, 0, st>>>(d, pr, flags, A, tally64, L, latz, queue, partials, offset_dev);
    BD_CHECK_LAUNCH("k_mc_trace");
    if (tally64) {
        const long long nv = (long long)p->nx * p->ny * p->nz;
        k_tally_finalize<<<grid_for(nv, 256), 256, 0, st>>>(tally64, A, nv);
        BD_CHECK_LAUNCH("k_tally_finalize");
    }
    k_ledger_reduce<<<1, 32, 0, st>>>(partials, blocks, (double)p->n_photons, ledger);
    BD_CHECK_LAUNCH("k_ledger_reduce");
    return BD_OK;
}
}  // namespace bd

extern "C" int bd_mc_trace(BdMcContext* c, const BdMcParams* p, const float* props, const uint8_t* flags,
                           float* A, float* L, double* lat_depth, double* ledger, void* stream) {
    BD_REQUIRE(c != nullptr, "bd_mc_trace: context is NULL");
    int rc = mc_validate(p);
    if (rc) return rc;
    BD_REQUIRE(props != nullptr && A != nullptr && ledger != nullptr, "bd_mc_trace: props, A and ledger are required");
    BD_REQUIRE(!(p->options & BD_MC_TALLY_FLUENCE) || L != nullptr, "bd_mc_trace: BD_MC_TALLY_FLUENCE needs L");
    BD_REQUIRE(p->n_photons <= kTallyMaxPhotons,
               "bd_mc_trace: at most %lld photons per launch (fixed-point tally range); split into batches",
               (long long)kTallyMaxPhotons);
    const long long nv = (long long)p->nx * p->ny * p->nz;
    if (nv > c->tally_cap) {
        cudaFree(c->tally64);
        c->tally64 = nullptr;
        c->tally_cap = 0;
        BD_CUDA(cudaMalloc(&c->tally64, sizeof(unsigned long long) * nv));
        BD_CUDA(cudaMemset(c->tally64, 0, sizeof(unsigned long long) * nv));
        c->tally_cap = nv;
    }
    return mc_launch(p, props, flags, A, L, lat_depth, ledger, c->queue, c->partials, c->partial_blocks,
                     c->sm_count, as_stream(stream), nullptr, c->tally64);
}

extern "C" int bd_mc_pack_props(const float* mu_a, const float* mu_s, const float* g, const float* n,
                                const float* mu_ext, const uint8_t* flags, float ra, float rs, float g_plume,
                                int64_t nv, float* out, void* stream) {
    BD_REQUIRE(mu_a && mu_s && g && n && out, "bd_mc_pack_props: NULL property pointer");
    BD_REQUIRE(nv >= 0, "bd_mc_pack_props: negative size");
    BD_REQUIRE(mu_ext == nullptr || flags != nullptr, "bd_mc_pack_props: plume extinction needs flags");
    if (nv == 0) return BD_OK;
    k_pack_props<<<grid_for(nv, 256), 256, 0, as_stream(stream)>>>(mu_a, mu_s, g, n, mu_ext, flags, ra, rs,
                                                                    g_plume, nv, reinterpret_cast<float4*>(out));
    BD_CHECK_LAUNCH("k_pack_props");
    return BD_OK;
}

extern "C" int bd_fold_f32_to_f64(float* src, double* dst, int64_t n, void* stream) {
    BD_REQUIRE(src && dst, "bd_fold_f32_to_f64: NULL pointer");
    if (n <= 0) return BD_OK;
    k_fold<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(src, dst, n);
    BD_CHECK_LAUNCH("k_fold");
    return BD_OK;
}

// ------------------------------------------------------------------------------------
// Allocation-free variant of bd_mc_trace.
//
// Some callers cannot call cudaMalloc once they are running: a control loop that must keep a
// fixed latency per laser pulse (the allocator may synchronise the device or block on the
// driver), or a host framework that owns all device memory through its own pool and does not
// allow side allocations. bd_mc_trace_noalloc needs no allocation at all: its scratch (the
// photon-queue counter and one FP64 ledger row per block) is a file-scope device array of fixed
// size, which every GPU that loads this library holds until the process exits.
namespace bd {
constexpr int MC_NOALLOC_MAX_BLOCKS = 2048;
constexpr size_t MC_NOALLOC_QUEUE_BYTES = 256;
static __device__ __align__(256) unsigned char g_mc_noalloc_scratch[MC_NOALLOC_QUEUE_BYTES +
                                                                    sizeof(double) * BD_LEDGER_LEN *
                                                                        MC_NOALLOC_MAX_BLOCKS];
constexpr int MC_NOALLOC_MAX_DEVICES = 64;
static void* g_mc_noalloc_ptr[MC_NOALLOC_MAX_DEVICES] = {nullptr};
static int g_mc_noalloc_sms[MC_NOALLOC_MAX_DEVICES] = {0};
static std::mutex g_mc_noalloc_mu;
}  // namespace bd

extern "C" int bd_mc_trace_noalloc(const BdMcParams* p, const float* props, const uint8_t* flags, float* A,
                                   float* L, double* lat_depth, double* ledger, void* stream) {
    int rc = mc_validate(p);
    if (rc) return rc;
    BD_REQUIRE(props != nullptr && A != nullptr && ledger != nullptr,
               "bd_mc_trace_noalloc: props, A and ledger are required");
    BD_REQUIRE(!(p->options & BD_MC_TALLY_FLUENCE) || L != nullptr, "bd_mc_trace_noalloc: BD_MC_TALLY_FLUENCE needs L");
    int dev = 0;
    BD_CUDA(cudaGetDevice(&dev));
    BD_REQUIRE(dev >= 0 && dev < MC_NOALLOC_MAX_DEVICES, "bd_mc_trace_noalloc: device ordinal %d >= %d", dev,
               MC_NOALLOC_MAX_DEVICES);
    void* base = nullptr;
    int sms = 0;
    {
        // set-up once per device, with that device current: the array's name is only a host-side
        // stand-in, the kernel must be given the device address of this device's copy. The address
        // is cached for the life of the device's primary context: do not use this entry point across
        // a cudaDeviceReset of that device.
        std::lock_guard<std::mutex> lock(g_mc_noalloc_mu);
        if (g_mc_noalloc_ptr[dev] == nullptr) {
            void* ptr = nullptr;
            BD_CUDA(cudaGetSymbolAddress(&ptr, g_mc_noalloc_scratch));
            int n = 0;
            BD_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
            g_mc_noalloc_ptr[dev] = ptr;
            g_mc_noalloc_sms[dev] = n;
        }
        base = g_mc_noalloc_ptr[dev];
        sms = g_mc_noalloc_sms[dev];
    }
    // the kernel is persistent (a photon queue), so any photon count runs on at most
    // MC_NOALLOC_MAX_BLOCKS blocks: mc_launch caps the grid at the static ledger rows
    unsigned long long* queue = static_cast<unsigned long long*>(base);
    double* partials = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + MC_NOALLOC_QUEUE_BYTES);
    // mc_launch zeroes the queue counter and the ledger rows it uses before the kernel runs
    return mc_launch(p, props, flags, A, L, lat_depth, ledger, queue, partials, MC_NOALLOC_MAX_BLOCKS, sms,
                     as_stream(stream), nullptr, nullptr);
}
