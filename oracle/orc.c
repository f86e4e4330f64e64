/*
 * ORACLE -- test infrastructure only. A plain-C, FP64 restatement of the reference CPU
 * (numba) kernels of yudovsky/bug-defense, used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py as the parity reference and the timed CPU port.
 * Nothing in the product (bug_defense_b200/) links, imports or calls this file.
 *
 * Pinning: tests/golden/ holds fixtures produced by running the reference itself
 * (tests/golden/make_golden.py imports simulation/* from the reference tree): the
 * deterministic kernels are compared to FP64 round-off, the Monte Carlo statistically
 * (the reference CPU MC uses numba's unseeded np.random, voxel_mc_3d.py:111-120,194).
 *
 * Every function cites the reference lines it restates.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IDX(i, j, k) (((size_t)(i) * (size_t)ny + (size_t)(j)) * (size_t)nz + (size_t)(k))

/* ---------------------------------------------------------------------------------------
 * Philox-4x32-10 (Salmon et al., SC'11) -- the same counter-based generator and per-photon
 * counter layout as the GPU kernel, so oracle and GPU photons draw identical uniforms.
 * ------------------------------------------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * x0, p1 = (uint64_t)0xCD9E8D57u * x2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t y0 = hi1 ^ x1 ^ k0, y2 = hi0 ^ x3 ^ k1;
        x0 = y0; x1 = lo1; x2 = y2; x3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

typedef struct {
    uint32_t key[2], p_lo, p_hi, blk, buf[4];
    int left, pos;
} Rng;

static void rng_init(Rng* r, uint64_t seed, uint64_t photon) {
    r->key[0] = (uint32_t)seed; r->key[1] = (uint32_t)(seed >> 32);
    r->p_lo = (uint32_t)photon; r->p_hi = (uint32_t)(photon >> 32);
    r->blk = 0; r->left = 0; r->pos = 0;
}
static uint32_t rng_u32(Rng* r) {
    if (r->left == 0) {
        uint32_t c[4] = {r->p_lo, r->p_hi, r->blk++, 0x42444d43u};
        orc_philox4x32_10(c, r->key, r->buf);
        r->left = 4; r->pos = 0;
    }
    r->left--;
    return r->buf[r->pos++];
}
static double rng_uniform(Rng* r) { return (double)(rng_u32(r) >> 8) * (1.0 / 16777216.0); }
static double rng_uniform_pos(Rng* r) { return ((double)(rng_u32(r) >> 8) + 0.5) * (1.0 / 16777216.0); }

/* ---------------------------------------------------------------------------------------
 * Bioheat stencil: simulation/voxel_thermal_3d.py:30-112 (bc_mode 0) and the Metal fused
 * kernel's z-wall flux, simulation/metal_ablation_solver.py:141,150 (bc_mode 1).
 * ------------------------------------------------------------------------------------- */
void orc_thermal_step(const double* T, double* Tn, const double* Q, const double* kg, const double* rho,
                      int nx, int ny, int nz, double dx, double dy, double dz, double dt, double h_eff,
                      double t_amb, int is_active, int bc_mode) {
    const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), idz2 = 1.0 / (dz * dz);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t c = IDX(i, j, k);
                double Tc = T[c], kc = kg[c], cap = rho[c];
                double fw = 0, fe = 0, fs = 0, fn = 0, ft, fb, kn;
                if (i > 0) { kn = kg[IDX(i - 1, j, k)]; fw = 2 * kc * kn / (kc + kn + 1e-12) * (T[IDX(i - 1, j, k)] - Tc) * idx2; }
                if (i < nx - 1) { kn = kg[IDX(i + 1, j, k)]; fe = 2 * kc * kn / (kc + kn + 1e-12) * (T[IDX(i + 1, j, k)] - Tc) * idx2; }
                if (j > 0) { kn = kg[IDX(i, j - 1, k)]; fs = 2 * kc * kn / (kc + kn + 1e-12) * (T[IDX(i, j - 1, k)] - Tc) * idy2; }
                if (j < ny - 1) { kn = kg[IDX(i, j + 1, k)]; fn = 2 * kc * kn / (kc + kn + 1e-12) * (T[IDX(i, j + 1, k)] - Tc) * idy2; }
                double wall;
                if (bc_mode == 0)
                    wall = h_eff > 0.0 ? (t_amb - Tc) / (dz * (0.5 * dz / fmax(kc, 1e-30) + 1.0 / fmax(h_eff, 1e-30))) : 0.0;
                else
                    wall = -h_eff * (Tc - t_amb) / dz;
                if (k > 0) { kn = kg[IDX(i, j, k - 1)]; ft = 2 * kc * kn / (kc + kn + 1e-12) * (T[IDX(i, j, k - 1)] - Tc) * idz2; }
                else ft = wall;
                if (k < nz - 1) { kn = kg[IDX(i, j, k + 1)]; fb = 2 * kc * kn / (kc + kn + 1e-12) * (T[IDX(i, j, k + 1)] - Tc) * idz2; }
                else fb = wall;
                double div = fw + fe + fs + fn + ft + fb;
                double src = is_active ? Q[c] : 0.0;
                Tn[c] = Tc + dt * (div + src) / cap;
            }
}

/* Latent-heat plateau: simulation/voxel_thermal_3d.py:115-143 */
void orc_plateau(double* T, double* H, const double* rho, const uint8_t* ablated, double t_abl, int64_t n,
                 const uint8_t* dry, double t_void) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double t = T[c];
        if (ablated[c]) {
            if (t > t_void) T[c] = t_void;
        } else if (dry[c]) {
            continue;
        } else if (t > t_abl) {
            H[c] += (t - t_abl) * rho[c];
            T[c] = t_abl;
        } else if (H[c] > 0.0) {
            double cap = rho[c];
            double rel = fmin(H[c], (t_abl - t) * cap);
            H[c] -= rel;
            T[c] = t + rel / cap;
        }
    }
}

/* Arrhenius damage integral: simulation/coupled_ablation.py:33-40 */
void orc_arrhenius(const double* T, double* Om, const uint8_t* ablated, double A, double EaR, double dt, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c)
        if (!ablated[c]) Om[c] += dt * A * exp(-EaR / (T[c] + 273.15));
}

/* First-order char kinetics: simulation/coupled_ablation.py:43-58 */
void orc_char(const double* T, double* chi, const uint8_t* dry, const uint8_t* ablated, double A, double EaR,
              double dt, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c)
        if (dry[c] && !ablated[c]) {
            double rate = A * exp(-EaR / (T[c] + 273.15));
            chi[c] = 1.0 - (1.0 - chi[c]) * exp(-rate * dt);
        }
}

/* Plume FTCS step: simulation/plume.py:18-80 (computed in FP64; the reference field is FP32). */
void orc_plume_step(const double* C, double* Cn, const uint8_t* vd, int nx, int ny, int nz, double dx, double dy,
                    double dz, double dt, double D_xy, double D_z, double vz, double decay) {
    const double idx2 = 1.0 / (dx * dx), idy2 = 1.0 / (dy * dy), idz2 = 1.0 / (dz * dz);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t c = IDX(i, j, k);
                if (!vd[c] || i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || k == 0 || k == nz - 1) {
                    Cn[c] = 0.0;
                    continue;
                }
                double cc = C[c];
                double cw = vd[IDX(i - 1, j, k)] ? C[IDX(i - 1, j, k)] : cc;
                double ce = vd[IDX(i + 1, j, k)] ? C[IDX(i + 1, j, k)] : cc;
                double cs = vd[IDX(i, j - 1, k)] ? C[IDX(i, j - 1, k)] : cc;
                double cn = vd[IDX(i, j + 1, k)] ? C[IDX(i, j + 1, k)] : cc;
                double cb = vd[IDX(i, j, k - 1)] ? C[IDX(i, j, k - 1)] : cc;
                double ct = vd[IDX(i, j, k + 1)] ? C[IDX(i, j, k + 1)] : cc;
                double diff = D_xy * ((cw - 2.0 * cc + ce) * idx2 + (cs - 2.0 * cc + cn) * idy2) +
                              D_z * ((cb - 2.0 * cc + ct) * idz2);
                double adv = vz > 0.0 ? -vz * (cc - ct) / dz : 0.0;
                double v = (cc + dt * (diff + adv)) * decay;
                Cn[c] = v > 0.0 ? v : 0.0;
            }
}

/* ---------------------------------------------------------------------------------------
 * Epoch-end phase / property update: simulation/coupled_ablation.py:77-180.
 * Each dry-state / char-state parameter is a pointer plus a length (1 = scalar, n = per voxel),
 * like the reference's size-1 / size-N arrays.
 * ------------------------------------------------------------------------------------- */
typedef struct { const double* p; int64_t len; } OrcArr;
static inline double av(OrcArr a, int64_t i) { return a.len == 1 ? a.p[0] : a.p[i]; }

void orc_phase_update(double* H, const double* h_lat, const double* T, const double* chi, uint8_t* dry,
                      const uint8_t* ablated, double* mu_a, double* mu_s, double* g, double* n, double* kg,
                      double* rho, const double* wet_mu_a, const double* wet_k, const double* wet_rho,
                      const OrcArr* ds /* mu_a mu_s g n k rho t_rem */, int has_cs, int has_cs_mu_a,
                      const OrcArr* cs /* mu_a mu_s k rho t_rem */, double cs_chi_rem, int has_cs_mu_s,
                      int has_cs_k, int has_cs_rho, double alpha_max, uint8_t* to_remove, int64_t N) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        if (ablated[i]) { to_remove[i] = 0; continue; }
        int is_dry = dry[i] != 0;
        double h = H[i];
        double hl = fmax(h_lat[i], 1e-30);
        if (!is_dry && h > 0.0) {
            double frac = fmin(fmax(h / hl, 0.0), 1.0);
            double dmua = av(ds[0], i), dk = av(ds[4], i), drho = av(ds[5], i);
            mu_a[i] = wet_mu_a[i] + (dmua - wet_mu_a[i]) * frac;
            kg[i] = wet_k[i] + (dk - wet_k[i]) * frac;
            rho[i] = wet_rho[i] + (drho - wet_rho[i]) * frac;
            if (h >= h_lat[i]) {
                is_dry = 1; dry[i] = 1; H[i] = 0.0;
                mu_a[i] = dmua; mu_s[i] = av(ds[1], i); g[i] = av(ds[2], i); n[i] = av(ds[3], i);
                kg[i] = dk; rho[i] = drho;
            }
        }
        if (is_dry) {
            double dmua = av(ds[0], i), dk = av(ds[4], i), drho = av(ds[5], i);
            if (has_cs) {
                double c = chi[i];
                if (has_cs_mu_a) mu_a[i] = dmua + c * (av(cs[0], i) - dmua);
                if (has_cs_mu_s) { double dms = av(ds[1], i); mu_s[i] = dms + c * (av(cs[1], i) - dms); }
                if (has_cs_k) kg[i] = dk + c * (av(cs[2], i) - dk);
                double r = has_cs_rho ? drho + c * (av(cs[3], i) - drho) : rho[i];
                double mn = kg[i] / alpha_max;
                if (r < mn) r = mn;
                rho[i] = r;
                to_remove[i] = (T[i] >= av(cs[4], i)) || (c >= cs_chi_rem);
            } else {
                to_remove[i] = T[i] >= av(ds[6], i);
            }
        } else {
            to_remove[i] = 0;
        }
    }
}

/* ---------------------------------------------------------------------------------------
 * Voxel Monte Carlo: simulation/voxel_mc_3d.py:33-422 in FP64 (CPU semantics by default;
 * metal != 0 applies the Metal deltas of simulation/voxel_mc_metal.py:220,246-252,318).
 * ------------------------------------------------------------------------------------- */
typedef struct {
    int nx, ny, nz, launch_axis, beam_profile, metal;
    double dx, dy, dz, lx, ly, lz;
    double ux0, uy0, uz0, cos_ph, sin_ph, cos_th_safe;
    double xc, yc, zc, sigma, radius, n_amb, rmax2;
    int64_t n_photons, offset, max_events;
    uint64_t seed;
} OrcMcParams;

static double fresnel(double n1, double n2, double cos_i, double eq) {
    if (fabs(n1 - n2) < eq) return 0.0;
    cos_i = fmin(1.0, fabs(cos_i));
    if (cos_i > 0.999999) { double r = (n1 - n2) / (n1 + n2); return r * r; }
    double sin_t2 = (n1 / n2) * (n1 / n2) * (1.0 - cos_i * cos_i);
    if (sin_t2 >= 1.0) return 1.0;
    double cos_t = sqrt(1.0 - sin_t2);
    double rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
    double rp = (n1 * cos_t - n2 * cos_i) / (n1 * cos_t + n2 * cos_i);
    return 0.5 * (rs * rs + rp * rp);
}

static inline void refract3(double* ux, double* uy, double* uz, int axis, double eta) {
    if (axis == 0) {
        double sg = *ux > 0.0 ? 1.0 : -1.0;
        *uy *= eta; *uz *= eta;
        *ux = sg * sqrt(fmax(0.0, 1.0 - *uy * *uy - *uz * *uz));
    } else if (axis == 1) {
        double sg = *uy > 0.0 ? 1.0 : -1.0;
        *ux *= eta; *uz *= eta;
        *uy = sg * sqrt(fmax(0.0, 1.0 - *ux * *ux - *uz * *uz));
    } else {
        double sg = *uz > 0.0 ? 1.0 : -1.0;
        *ux *= eta; *uy *= eta;
        *uz = sg * sqrt(fmax(0.0, 1.0 - *ux * *ux - *uy * *uy));
    }
}

enum { L_SPEC = 1, L_DIFF, L_TRANS, L_LAT, L_ABS, L_ABSV, L_GAIN, L_LOSS, L_TRUNC, L_COL, L_CROSS, L_REFL };

/* One photon packet, voxel_mc_3d.py:123-337 (scalar state, as the reference). */
static void trace_one(const OrcMcParams* P, int64_t pid, const double* mua, const double* mus, const double* gg,
                      const double* nn, double* A, double* L, double* latz, double* led) {
    const int nx = P->nx, ny = P->ny, nz = P->nz;
    const int zl = P->launch_axis == 0;  /* 1: depth axis z; 0: depth axis x */
    const double eq = P->metal ? 1e-6 : 1e-9, step_eps = P->metal ? 1e-4 : 1e-9, entry_eps = P->metal ? 1e-6 : 1e-9;
    const double dx = P->dx, dy = P->dy, dz = P->dz;
    Rng rng;
    rng_init(&rng, P->seed, (uint64_t)(P->offset + pid));
    double u1, u2;
    if (P->beam_profile == 1) {
        double r = P->radius * sqrt(rng_uniform(&rng));
        double a = 2.0 * M_PI * rng_uniform(&rng);
        u1 = r * cos(a); u2 = r * sin(a);
    } else if (P->beam_profile == 2 || P->beam_profile == 3) {
        double rn = 0.0;
        for (int t = 0; t < 256; ++t) {
            rn = sqrt(rng_uniform(&rng));
            double acc = P->beam_profile == 2 ? exp(-2.0 * rn) : exp(-2.0 * rn * rn);
            if (rng_uniform(&rng) < acc) break;
        }
        double a = 2.0 * M_PI * rng_uniform(&rng);
        u1 = P->radius * rn * cos(a); u2 = P->radius * rn * sin(a);
    } else {
        double a = rng_uniform_pos(&rng), b = rng_uniform(&rng);
        double r = sqrt(-2.0 * log(a)) * P->sigma;
        u1 = r * cos(2.0 * M_PI * b); u2 = r * sin(2.0 * M_PI * b);
    }
    double x, y, z, ux = P->ux0, uy = P->uy0, uz = P->uz0;
    int ix, iy, iz;
    const double st = u1 / P->cos_th_safe;
    if (zl) {
        x = P->xc + st * P->cos_ph - u2 * P->sin_ph;
        y = P->yc + st * P->sin_ph + u2 * P->cos_ph;
        z = 0.0;
        int out = x < 0 || x >= P->lx || y < 0 || y >= P->ly;
        if (!out && P->rmax2 > 0) out = (x - P->xc) * (x - P->xc) + (y - P->yc) * (y - P->yc) >= P->rmax2;
        if (out) { led[L_LAT] += 1.0; latz[0] += 1.0; return; }
        ix = (int)(x / dx); if (ix > nx - 1) ix = nx - 1;
        iy = (int)(y / dy); if (iy > ny - 1) iy = ny - 1;
        iz = 0;
    } else {
        x = 0.0;
        y = P->yc + st * P->cos_ph - u2 * P->sin_ph;
        z = P->zc + st * P->sin_ph + u2 * P->cos_ph;
        int out = y < 0 || y >= P->ly || z < 0 || z >= P->lz;
        if (!out && P->rmax2 > 0) out = (y - P->yc) * (y - P->yc) + (z - P->zc) * (z - P->zc) >= P->rmax2;
        if (out) { led[L_LAT] += 1.0; latz[0] += 1.0; return; }
        ix = 0;
        iy = (int)(y / dy); if (iy > ny - 1) iy = ny - 1;
        iz = (int)(z / dz); if (iz > nz - 1) iz = nz - 1;
    }
    size_t c = IDX(ix, iy, iz);
    double n_in = nn[c];
    double r0 = fresnel(P->n_amb, n_in, zl ? uz : ux, eq);
    led[L_SPEC] += r0;
    double w = 1.0 - r0;
    if (w <= 0.0) return;
    if (fabs(n_in - P->n_amb) > entry_eps) refract3(&ux, &uy, &uz, zl ? 2 : 0, P->n_amb / n_in);
    double tau = -log(fmax(rng_uniform(&rng), 1e-12));
    /* per-photon counters kept in registers, booked once when the photon ends */
    double n_col = 0.0, n_cross = 0.0, n_refl = 0.0, absorbed = 0.0;
    for (int64_t ev = 0; ev < P->max_events; ++ev) {
        c = IDX(ix, iy, iz);
        const double ma = mua[c], mt = ma + mus[c];
        double sx, sy, sz;
        if (ux > 1e-15) sx = ((ix + 1) * dx - x) / ux; else if (ux < -1e-15) sx = (ix * dx - x) / ux; else sx = 1e30;
        if (uy > 1e-15) sy = ((iy + 1) * dy - y) / uy; else if (uy < -1e-15) sy = (iy * dy - y) / uy; else sy = 1e30;
        if (uz > 1e-15) sz = ((iz + 1) * dz - z) / uz; else if (uz < -1e-15) sz = (iz * dz - z) / uz; else sz = 1e30;
        int ax;
        double se;
        if (sx <= sy && sx <= sz) { ax = 0; se = sx; }
        else if (sy <= sz) { ax = 1; se = sy; }
        else { ax = 2; se = sz; }
        if (se < 0.0) se = 0.0;
        if (mt > 1e-12 && mt * se >= tau) {
            n_col += 1.0;
            const double sc = tau / mt;
            if (L) L[c] += w * sc;
            x += sc * ux; y += sc * uy; z += sc * uz;
            if (P->rmax2 > 0) {
                double p1 = zl ? x - P->xc : y - P->yc, p2 = zl ? y - P->yc : z - P->zc;
                if (p1 * p1 + p2 * p2 >= P->rmax2) { led[L_LAT] += w; latz[zl ? iz : ix] += w; goto done; }
            }
            const double dw = w * (ma / mt);
            w -= dw;
            A[c] += dw;
            absorbed += dw;
            if (w < 1e-4) {
                if (rng_uniform(&rng) < 0.1) { led[L_GAIN] += 9.0 * w; w *= 10.0; }
                else { led[L_LOSS] += w; goto done; }
            }
            const double g = gg[c], xi = rng_uniform(&rng);
            double ct;
            if (fabs(g) < 1e-4) ct = 2.0 * xi - 1.0;
            else {
                double t = (1.0 - g * g) / (1.0 - g + 2.0 * g * xi);
                ct = (1.0 + g * g - t * t) / (2.0 * g);
                ct = fmax(-1.0, fmin(1.0, ct));
            }
            const double sth = sqrt(fmax(0.0, 1.0 - ct * ct));
            const double psi = 2.0 * M_PI * rng_uniform(&rng), cp = cos(psi), sp = sin(psi);
            double nux, nuy, nuz;
            if (fabs(uz) > 0.99999) {
                double sgz = uz > 0 ? 1.0 : -1.0;
                nux = sth * cp; nuy = sth * sp; nuz = ct * sgz;
            } else {
                double den = sqrt(fmax(1.0 - uz * uz, 1e-12));
                nux = sth * (ux * uz * cp - uy * sp) / den + ux * ct;
                nuy = sth * (uy * uz * cp + ux * sp) / den + uy * ct;
                nuz = -sth * cp * den + uz * ct;
            }
            double nm = sqrt(nux * nux + nuy * nuy + nuz * nuz);
            if (nm > 1e-12) { nux /= nm; nuy /= nm; nuz /= nm; }
            ux = nux; uy = nuy; uz = nuz;
            tau = -log(fmax(rng_uniform(&rng), 1e-12));
            continue;
        }
        n_cross += 1.0;
        tau -= mt * se;
        if (L) L[c] += w * se;
        x += se * ux; y += se * uy; z += se * uz;
        int jx = ix, jy = iy, jz = iz;
        double cos_face;
        if (ax == 0) { int sd = ux > 0 ? 1 : -1; jx += sd; x = sd > 0 ? (ix + 1) * dx : ix * dx; cos_face = ux; }
        else if (ax == 1) { int sd = uy > 0 ? 1 : -1; jy += sd; y = sd > 0 ? (iy + 1) * dy : iy * dy; cos_face = uy; }
        else { int sd = uz > 0 ? 1 : -1; jz += sd; z = sd > 0 ? (iz + 1) * dz : iz * dz; cos_face = uz; }
        const int depth_ax = zl ? 2 : 0;
        if (ax == depth_ax) {
            const int jd = zl ? jz : jx, ndp = zl ? nz : nx;
            if (jd < 0) {
                double r = fresnel(nn[c], P->n_amb, zl ? uz : ux, eq);
                if (r > 0.0 && rng_uniform(&rng) < r) {
                    if (zl) uz = -uz; else ux = -ux;
                    n_refl += 1.0;
                    continue;
                }
                led[L_DIFF] += w;
                goto done;
            }
            if (jd >= ndp) { led[L_TRANS] += w; goto done; }
        } else if (jx < 0 || jx >= nx || jy < 0 || jy >= ny || jz < 0 || jz >= nz) {
            led[L_LAT] += w; latz[zl ? iz : ix] += w;
            goto done;
        }
        if (!P->metal && P->rmax2 > 0) {
            double p1 = zl ? x - P->xc : y - P->yc, p2 = zl ? y - P->yc : z - P->zc;
            if (p1 * p1 + p2 * p2 >= P->rmax2) { led[L_LAT] += w; latz[zl ? iz : ix] += w; goto done; }
        }
        const size_t cj = IDX(jx, jy, jz);
        const double n1 = nn[c], n2 = nn[cj];
        if (fabs(n1 - n2) > step_eps) {
            double r = fresnel(n1, n2, cos_face, eq);
            if ((!P->metal || r > 0.0) && rng_uniform(&rng) < r) {
                if (ax == 0) ux = -ux; else if (ax == 1) uy = -uy; else uz = -uz;
                n_refl += 1.0;
                continue;
            }
            refract3(&ux, &uy, &uz, ax, n1 / n2);
        }
        ix = jx; iy = jy; iz = jz;
    }
    led[L_TRUNC] += w;
done:
    led[L_COL] += n_col;
    led[L_CROSS] += n_cross;
    led[L_REFL] += n_refl;
    led[L_ABS] += absorbed;
}

/* Parallel driver: photons split into n_chunks batches with private FP64 tallies, reduced at
 * the end (the scheme of voxel_mc_3d.py:340-422 / :621-625). A, L (L may be NULL), latz and
 * ledger[16] are ADDED to. */
void orc_mc_trace(const OrcMcParams* P, const double* mua, const double* mus, const double* gg, const double* nn,
                  double* A, double* L, double* latz, double* ledger, int n_chunks) {
    const size_t nv = (size_t)P->nx * P->ny * P->nz;
    const int n_depth = P->launch_axis == 0 ? P->nz : P->nx;
    if (n_chunks < 1) n_chunks = 1;
    double* As = (double*)calloc((size_t)n_chunks * nv, sizeof(double));
    double* Ls = L ? (double*)calloc((size_t)n_chunks * nv, sizeof(double)) : NULL;
    double* Zs = (double*)calloc((size_t)n_chunks * n_depth, sizeof(double));
    double* Gs = (double*)calloc((size_t)n_chunks * 16, sizeof(double));
#pragma omp parallel for schedule(dynamic, 1)
    for (int ch = 0; ch < n_chunks; ++ch) {
        int64_t p0 = (int64_t)(((__int128)ch * P->n_photons) / n_chunks);
        int64_t p1 = (int64_t)(((__int128)(ch + 1) * P->n_photons) / n_chunks);
        for (int64_t p = p0; p < p1; ++p)
            trace_one(P, p, mua, mus, gg, nn, As + (size_t)ch * nv, Ls ? Ls + (size_t)ch * nv : NULL,
                      Zs + (size_t)ch * n_depth, Gs + (size_t)ch * 16);
    }
    for (int ch = 0; ch < n_chunks; ++ch) {
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < (int64_t)nv; ++v) {
            A[v] += As[(size_t)ch * nv + v];
            if (L) L[v] += Ls[(size_t)ch * nv + v];
        }
        for (int d = 0; d < n_depth; ++d) latz[d] += Zs[(size_t)ch * n_depth + d];
        for (int q = 0; q < 16; ++q) ledger[q] += Gs[(size_t)ch * 16 + q];
    }
    ledger[0] += (double)P->n_photons;
    free(As); free(Ls); free(Zs); free(Gs);
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
