"""The benchmarked configuration against the FP64 oracle, epoch by epoch.

Workload: workloads.full_coupled_run(seed=0), the 200x200x192 grid the benchmark times, with the
engine's default plume_dt_policy='subcycle' (34 FTCS plume steps of dt/34 per 50 us substep at
D = 22.9 mm^2/s). The MC is replaced by a fixed synthetic absorbed map (a Gaussian column that
decays with depth through the dorsal cuticle, with a weaker deposit in the fat body), so both
engines see the same source and the comparison is deterministic; it ablates the cuticle within a
few epochs, breaches the air gap and boils the fat below it.

Each epoch starts the oracle (oracle/engine.py, the reference step_epoch of
simulation/coupled_ablation.py:440-617 in FP64) from the GPU engine's state before the epoch and
compares the states after it, so a threshold decision that flips in FP32 cannot cascade:
  * ablated and dry masks exactly, except voxels whose oracle state before the phase update lies
    within 0.01 K of t_remove, 1e-5 of chi_remove or 1e-4 relative of h_lat;
  * T <= 1e-4 relative, T_peak <= 1e-4 relative, H_acc <= 1e-4 of h_lat, chi <= 1e-5 + 1e-4 rel.,
    optical and thermal properties <= 1e-4 relative, on voxels whose masks agree;
  * the plume raw field and its saturated extinction <= 1e-4 of the field maximum, away from
    flipped voxels; per-epoch removal counts within the flips; plume transmission <= 1e-4 rel.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_ON, N_OFF = 4, 2


def gpu_state(eng) -> dict:
    """The GPU engine's evolving state as float64 / bool host arrays (OracleEngine.load_state keys)."""
    st = dict(T=eng.T, H_acc=eng.H_acc, chi=eng.chi, dry=eng.dry, ablated=eng.ablated, k_grid=eng.k_grid,
              rho_cp_grid=eng.rho_cp_grid, T_peak=eng.T_peak, ablation_time=eng.ablation_time, t=eng.t,
              epoch=eng.epoch)
    for key in ("mu_a", "mu_s", "g", "n"):
        st[key] = eng.optical[key]
    if eng._wet is not None:
        st["wet_mu_a"], st["wet_k"], st["wet_rho_cp"] = (w.double().cpu().numpy() for w in eng._wet)
    if eng.plume is not None:
        st["plume_raw"] = eng.plume.raw.double().cpu().numpy()
        st["plume_mu_ext"] = eng.plume.mu_ext.double().cpu().numpy()
    return st


def fixed_source(geo, a0=2.0e-4, mu_cut=8.0, fat_frac=0.3, mu_fat=2.0) -> np.ndarray:
    """Absorbed fraction per voxel: Gaussian across the beam (sigma = spot / 4), exp(-mu_cut z) through
    the cuticle below the top air, fat_frac * exp(-mu_fat z) from the top of the fat body down."""
    nx, ny, nz = geo["shape"]
    dx = geo["Lx"] / nx
    x = (np.arange(nx) + 0.5) * dx - geo["Lx"] / 2
    y = (np.arange(ny) + 0.5) * dx - geo["Ly"] / 2
    sig = geo["spot_dia"] / 4
    lat = np.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / (2 * sig * sig))
    names = geo["layer_names"]
    prof = np.zeros(nz)
    k_cut = names.index("exocuticle")
    k_fat = names.index("fat")
    for k, nm in enumerate(names):
        if "cuticle" in nm and k < k_fat:
            prof[k] = np.exp(-mu_cut * (k - k_cut) * dx)
        elif k >= k_fat and nm != "below":
            prof[k] = fat_frac * np.exp(-mu_fat * (k - k_fat) * dx)
    return a0 * lat[:, :, None] * prof[None, None, :]


def near_threshold(cap, orc) -> np.ndarray:
    """Voxels whose removal / drying decision is within the FP32 tolerance of its threshold."""
    t_rem = float(orc._cs["t_remove"]) if orc._cs is not None else float(np.max(orc._ds["t_remove"]))
    near = np.abs(cap["T"] - t_rem) <= 0.01
    near |= np.abs(cap["chi"] - orc._cs_chi) <= 1e-5
    near |= (~cap["dry"]) & (np.abs(cap["H_acc"] - orc.h_lat) <= 1e-4 * np.abs(orc.h_lat))
    return near


def compare_epoch(st_g, orc, cap, dg, do, label):
    """Post-epoch GPU state st_g against the oracle engine `orc` after the same epoch."""
    near = near_threshold(cap, orc)
    flip_abl = st_g["ablated"] != orc.ablated
    flip_dry = st_g["dry"] != orc.dry
    bad = (flip_abl | flip_dry) & ~near
    assert not np.any(bad), (label, int(flip_abl.sum()), int(flip_dry.sum()), int(bad.sum()))
    flips = flip_abl | flip_dry
    same = ~flips
    # away from the flipped voxels (their plume injection and removal differ)
    away = same.copy()
    if flips.any():
        from scipy.ndimage import binary_dilation
        away &= ~binary_dilation(flips, iterations=1)

    def rel(a, b, mask):
        return float(np.max(np.abs(a[mask] - b[mask]) / np.maximum(np.abs(b[mask]), 1e-30))) if mask.any() else 0.0

    assert rel(st_g["T"], orc.T, same) <= 1e-4, (label, rel(st_g["T"], orc.T, same))
    assert rel(st_g["T_peak"], orc.T_peak, same) <= 1e-4, label
    dH = np.abs(st_g["H_acc"] - orc.H_acc)[same]
    assert np.all(dH <= 1e-4 * np.abs(orc.h_lat[same]) + 1e-9), (label, float(dH.max()))
    dchi = np.abs(st_g["chi"] - orc.chi)[same]
    assert np.all(dchi <= 1e-5 + 1e-4 * np.abs(orc.chi[same])), (label, float(dchi.max()))
    for key in ("mu_a", "mu_s", "g", "n"):
        assert rel(st_g[key], orc.optical[key], same & (orc.optical[key] != 0)) <= 1e-4, (label, key)
    assert rel(st_g["k_grid"], orc.k_grid, same) <= 1e-4, label
    assert rel(st_g["rho_cp_grid"], orc.rho_cp_grid, same) <= 1e-4, label
    pm = max(float(np.max(orc.plume["raw"])), 1e-12)
    assert np.max(np.abs(st_g["plume_raw"] - orc.plume["raw"])[away]) <= 1e-4 * pm, label
    em = max(float(np.max(orc.plume["mu_ext"])), 1e-12)
    assert np.max(np.abs(st_g["plume_mu_ext"] - orc.plume["mu_ext"])[away]) <= 1e-4 * em, label
    assert abs(dg["n_new"] - do["n_new"]) <= int(flip_abl.sum()), (label, dg["n_new"], do["n_new"])
    assert dg["plume_transmission"] == pytest.approx(do["plume_transmission"], rel=1e-4, abs=1e-7), label
    return int(flips.sum())


def run_epochs(eng, orc, A, powers, label):
    """Step both engines epoch by epoch, the oracle from the GPU state; returns the last GPU state,
    the total removals and flipped voxels, and whether the air gap joined the void domain."""
    k0 = eng.air_gap_range[0] if eng.air_gap_range else None
    total_new, total_flips, breached = 0, 0, False
    st_pre = gpu_state(eng)
    for ep, power in enumerate(powers):
        eng.power = power
        dg = eng.step_epoch(absorbed_map=A if power > 0 else None)
        st_post = gpu_state(eng)
        orc.load_state(st_pre)
        orc.power = power
        cap = {}
        do = orc.step_epoch(absorbed_map=A if power > 0 else None, capture=cap)
        total_flips += compare_epoch(st_post, orc, cap, dg, do, f"{label} epoch {ep + 1}")
        total_new += dg["n_new"]
        if k0:
            breached |= bool(st_post["ablated"][:, :, k0 - 1].any())
        st_pre = st_post
    return st_pre, total_new, total_flips, breached


def test_full_resolution_subcycle_epochs_match_oracle(gpu):
    from oracle.engine import OracleEngine
    import oracle
    from bug_defense_b200 import workloads
    from bug_defense_b200.ablation import plume_steps_per_substep
    geo = workloads.full_coupled_run(seed=0)
    kw = workloads.engine_kwargs(geo)
    eng = gpu.CoupledAblationEngine(**kw)
    assert eng.plume_dt_policy == "subcycle" and eng.shape == (200, 200, 192)
    n_sub, _ = plume_steps_per_substep(eng._desc.plume)
    assert n_sub == 34
    oracle.set_threads(oracle.max_threads())
    orc = OracleEngine(**kw, plume_dt_policy="subcycle")
    st, total_new, total_flips, breached = run_epochs(eng, orc, fixed_source(geo), [40.0] * N_ON + [0.0] * N_OFF,
                                                      "bench config")
    # the run exercised removal, the air-gap breach and boiling
    assert total_new > 1000 and breached
    assert np.any((st["H_acc"] > 0) & ~st["dry"])
    assert total_flips <= 1e-4 * st["T"].size


@pytest.mark.parametrize("extra", [dict(plume_dt_policy="metal"), dict(bc="metal", plume_dt_policy="subcycle"),
                                   dict(plume_dt_policy="as_given")], ids=["plume-metal", "bc-metal", "plume-as_given"])
def test_semantic_switches_match_oracle(gpu, extra):
    """The Metal plume time-step clamp, the Metal z-wall flux and the CPU plume step as given, each
    against the oracle with the same switch, epoch by epoch from the GPU state (48x48x144 grid).
    The step as given is the reference CPU FTCS, stable only while 6 D dt / dx^2 <= 1: that case
    uses D = 0.5 mm^2/s (0.67 at 15 um and 50 us); the workload's D (10-50 mm^2/s) diverges on both
    sides, which is why the engine sub-cycles by default."""
    from oracle.engine import OracleEngine
    from bug_defense_b200 import workloads
    geo = workloads.full_coupled_run(seed=3, nx=48, ny=48, nz=128, n_plume_air=16)
    kw = workloads.engine_kwargs(geo)
    if extra.get("plume_dt_policy") == "as_given":
        kw["plume_closure"] = dict(kw["plume_closure"], D_xy=0.5, D_z=0.5)
    eng = gpu.CoupledAblationEngine(**kw, **extra)
    orc = OracleEngine(**kw, **extra)
    st, total_new, _, _ = run_epochs(eng, orc, fixed_source(geo), [40.0, 40.0, 0.0], str(extra))
    assert total_new > 0


@pytest.mark.parametrize("semantics", ["cpu", "metal"])
def test_single_epoch_stack_matches_oracle_on_same_photon_streams(gpu, semantics):
    """The CPU-runnable single epoch (64x64x128, 20k photons at 22 deg, then 20 x 50 us substeps, no
    ablation or plume) through CoupledAblationEngine and through the oracle engine, which traces the
    same Philox photon streams (epoch e, photon p -> stream (seed, (e << 32) + p)) in FP64. The two
    tallies differ only where FP32 rounding changes a discrete decision of one photon, so R/A/T, the
    absorbed-power map and the temperature after the substeps are compared together."""
    from oracle.engine import OracleEngine
    from bug_defense_b200 import workloads
    geo = workloads.single_epoch_stack(seed=0)
    kw = workloads.single_epoch_kwargs(geo)
    eng = gpu.CoupledAblationEngine(**kw, semantics=semantics)
    orc = OracleEngine(**kw, mc_stream="engine", semantics=semantics)
    dg = eng.step_epoch()
    orc.step_epoch()
    led = dg["ledger"]
    N = float(kw["n_photons"])
    assert led[0] == N and abs((led[1:7].sum() + led[8] + led[9] - led[7]) / N - 1.0) < 1e-9
    o = orc.last_mc["spectro_raw"]
    g = dict(R_spec=led[1] / N, R_diff=led[2] / N, Transmission=led[3] / N, Lateral_loss=led[4] / N,
             Absorption=(led[5] + led[6]) / N)
    for key, v in g.items():
        assert abs(v - o[key]) <= 2e-3, (key, v, o[key])
    Qg, Qo = eng.Q, orc.Q
    l2 = float(np.linalg.norm(Qg - Qo) / np.linalg.norm(Qo))
    dT_g, dT_o = eng.T - 25.0, orc.T - 25.0
    lt = float(np.linalg.norm(dT_g - dT_o) / np.linalg.norm(dT_o))
    print(f"SAME_STREAMS semantics={semantics} rel_l2_Q={l2:.4g} rel_l2_dT={lt:.4g}")
    assert l2 <= 0.05, l2          # two independent 20k-photon maps differ by ~0.5 in this norm
    assert lt <= 0.05, lt
    assert np.max(dT_o) > 1.0
