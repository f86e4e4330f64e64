"""Precision and energy-balance checks at full size (256^3 voxels at 15 um, 128^3 thermal block).

Monte Carlo: homogeneous and two-layer slabs with properties drawn from mu_a 0.1-10/mm, mu_s
10-100/mm, g 0.7-0.95, n 1.33-1.56 (ambient n = 1), normal and 22 deg pencil beams. The FP32 GPU
transport (FP64 ledger) is compared with the FP64 oracle on the same geometry: reflected, transmitted
and absorbed fractions within 3 combined standard errors, and the per-voxel relative L2 distance
of the absorbed maps no larger than their Monte Carlo noise (estimated from independent halves),
i.e. no FP32 bias visible above the noise. The GPU run uses up to 1e8 photons (fewer for draws
whose photons take thousands of steps, keeping the run to seconds); the oracle a CPU-budgeted count.
The FP32 error itself is isolated by a same-seed comparison: the GPU traces the oracle's first half
on the same Philox photon streams, so the two maps differ only where FP32 rounding changed a
discrete decision of a photon (a boundary, a roulette draw, a Fresnel split); that distance is
reported per case and must stay below the distance between two independent maps of that size.

Thermal: a 128^3 homogeneous block with an instantaneous Gaussian heat deposit, 10,000 substeps of
50 us, against the analytic infinite-medium solution
    T(r, t) = T0 + A (s0^2 / s^2)^(3/2) exp(-r^2 / (2 s^2)),  s^2 = s0^2 + 2 alpha t,
and against the FP64 oracle stencil (same discretisation): FP32 temperatures within 1e-4 of the
temperature scale after all 10,000 steps (the rounding of 10,000 FP32 updates accumulates; the
relative L2 of the temperature rise is reported).
"""
import json
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 256
DX = 0.015


def _draw_layer(rng):
    return dict(mu_a=float(rng.uniform(0.1, 10.0)), mu_s=float(rng.uniform(10.0, 100.0)),
                g=float(rng.uniform(0.7, 0.95)), n=float(rng.uniform(1.33, 1.56)))


def _slab(seed, two_layer):
    rng = np.random.default_rng(seed)
    top = _draw_layer(rng)
    props = {k: np.full((N, N, N), v) for k, v in top.items()}
    info = dict(top=top)
    if two_layer:
        bot = _draw_layer(rng)
        k0 = int(rng.integers(20, 80))                  # interface depth 0.3-1.2 mm
        for k, v in bot.items():
            props[k][:, :, k0:] = v
        info.update(bottom=bot, interface_voxel=k0)
    return props, info


def _rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


CASES = [("homogeneous", False, 0.0, 101), ("homogeneous", False, 22.0, 102),
         ("two_layer", True, 0.0, 103), ("two_layer", True, 22.0, 104)]


@pytest.mark.parametrize("name,two_layer,theta,seed", CASES, ids=[f"{c[0]}_{int(c[2])}deg" for c in CASES])
def test_slab_absorbed_map_matches_fp64_oracle(gpu, orc, name, two_layer, theta, seed):
    props, info = _slab(seed, two_layer)
    L = N * DX
    kw = dict(Lx=L, Ly=L, Lz=L, Nx=N, Ny=N, Nz=N, custom_3d_props=props, spot_dia=1e-3, theta_inc_deg=theta)
    pilot = gpu.run_voxel_mc3d(n_photons=200_000, base_seed=seed, **kw)
    steps = pilot["photon_steps"] / 200_000
    n_gpu = int(min(1e8, 4e10 / steps)) // 2 * 2
    t0 = time.perf_counter()
    orc.run_voxel_mc3d(n_photons=2000, seed=seed + 7, n_chunks=orc.max_threads(), tally_fluence=False, **kw)
    cpu_rate = 2000 / max(time.perf_counter() - t0, 1e-3)
    n_cpu = int(np.clip(cpu_rate * 20.0, 20_000, 2_000_000)) // 2 * 2
    g1 = gpu.run_voxel_mc3d(n_photons=n_gpu // 2, base_seed=seed + 1, **kw)
    g2 = gpu.run_voxel_mc3d(n_photons=n_gpu // 2, base_seed=seed + 2, **kw)
    c1 = orc.run_voxel_mc3d(n_photons=n_cpu // 2, seed=seed + 3, n_chunks=orc.max_threads(), tally_fluence=False, **kw)
    c2 = orc.run_voxel_mc3d(n_photons=n_cpu // 2, seed=seed + 4, n_chunks=orc.max_threads(), tally_fluence=False, **kw)
    A_g = 0.5 * (g1["A_3d"] + g2["A_3d"])
    A_c = 0.5 * (c1["A_3d"] + c2["A_3d"])
    noise_g = np.linalg.norm((g1["A_3d"] - g2["A_3d"]).ravel()) / (2 * np.linalg.norm(A_g.ravel()))
    noise_c = np.linalg.norm((c1["A_3d"] - c2["A_3d"]).ravel()) / (2 * np.linalg.norm(A_c.ravel()))
    rel = _rel_l2(A_g, A_c)
    expect = float(np.hypot(noise_g, noise_c))
    # the same photon streams as the oracle's first half: FP32 vs FP64 arithmetic only
    g3 = gpu.run_voxel_mc3d(n_photons=n_cpu // 2, base_seed=seed + 3, **kw)
    same = _rel_l2(g3["A_3d"], c1["A_3d"])
    indep = _rel_l2(c2["A_3d"], c1["A_3d"])
    report = dict(case=name, theta=theta, layers=info, gpu_photons=n_gpu, cpu_photons=n_cpu,
                  steps_per_photon=steps, rel_l2_gpu_vs_fp64=rel, noise_gpu=float(noise_g), noise_cpu=float(noise_c),
                  rel_l2_same_streams=same, rel_l2_independent=indep,
                  same_streams_fraction_diff={k: g3["spectro_raw"][k] - c1["spectro_raw"][k]
                                              for k in ("R_diff", "Transmission", "Absorption", "Lateral_loss")},
                  ledger_closure_gpu=[g1["ledger_closure"], g2["ledger_closure"]])
    for key in ("R_diff", "Transmission", "Absorption", "Lateral_loss"):
        fg = 0.5 * (g1["spectro_raw"][key] + g2["spectro_raw"][key])
        fc = 0.5 * (c1["spectro_raw"][key] + c2["spectro_raw"][key])
        var = max(fc * (1 - fc), 1e-12)
        se = np.sqrt(var / n_cpu + var / n_gpu)
        report[key] = [fg, fc]
        assert abs(fg - fc) <= 3.0 * se + 1e-6, (key, fg, fc, se)
    print("PRECISION " + json.dumps(report))
    # R_spec is a deterministic Fresnel split: FP32 vs FP64 rounding only
    assert abs(g1["spectro_raw"]["R_spec"] - c1["spectro_raw"]["R_spec"]) < 1e-6
    for g in (g1, g2):
        assert abs(g["ledger_closure"] - 1.0) < 1e-9
        assert abs(g["energy_closure"] - 1.0) < 0.01
    # the maps differ by Monte Carlo noise only: no FP32 bias above it
    assert rel <= 1.25 * expect + 1e-3, (rel, expect)
    # on the same streams the FP32 error is below the noise of an independent map of that size
    assert same < indep, (same, indep)


def test_thermal_gaussian_deposit_matches_analytic_and_fp64(gpu, orc):
    from bug_defense_b200 import thermal
    n, dx, steps, dt = 128, DX, 10_000, 5e-5
    k, rho_cp = 0.2e-3, 4.0e-3                       # W/(mm K), J/(mm^3 K): alpha = 0.05 mm^2/s
    alpha = k / rho_cp
    s0, amp, t_base = 8 * dx, 40.0, 25.0
    c = (np.arange(n) + 0.5) * dx - n * dx / 2
    r2 = c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2
    T0 = t_base + amp * np.exp(-r2 / (2 * s0 * s0))
    K = np.full((n, n, n), k); R = np.full((n, n, n), rho_cp); Q = np.zeros((n, n, n))
    T_gpu = thermal.run_thermal3d_substeps_gpu(T0, Q, K, R, n, n, n, dx, dx, dx, dt, steps, h_eff=0.0,
                                               t_ambient=t_base, is_active=0)
    s2 = s0 * s0 + 2 * alpha * steps * dt
    T_an = t_base + amp * (s0 * s0 / s2) ** 1.5 * np.exp(-r2 / (2 * s2))
    rel_an = _rel_l2(T_gpu - t_base, T_an - t_base)
    # FP64 oracle with the same discretisation
    Ta, Tb = T0.copy(), np.empty_like(T0)
    for _ in range(steps):
        orc.thermal3d_step_explicit(Ta, Tb, Q, K, R, n, n, n, dx, dx, dx, dt, 0.0, t_base, 0)
        Ta, Tb = Tb, Ta
    rel_fp64 = _rel_l2(T_gpu - t_base, Ta - t_base)
    max_fp64 = float(np.abs(T_gpu - Ta).max() / np.abs(Ta).max())
    energy = float((T_gpu - t_base).sum() / (T0 - t_base).sum())
    print("PRECISION " + json.dumps(dict(case="thermal_gaussian_128", steps=steps, rel_l2_vs_analytic=rel_an,
                                         rel_l2_rise_vs_fp64=rel_fp64, max_rel_vs_fp64=max_fp64, heat_ratio=energy)))
    assert max_fp64 < 1e-4
    assert rel_fp64 < 2e-3
    assert rel_an < 5e-3
    assert abs(energy - 1.0) < 1e-4          # insulated faces: the deposit is conserved
