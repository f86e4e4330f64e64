"""Device-side per-epoch recording (bd_engine_record + Recorder) equals what the production runner
computes from full host copies of the engine state after every epoch
(run_highres_knowledge_suite.py:271-318): xz slices of T, Q, phase and plume absorption, the
centreline along a tilted beam line, the crater depth below the surface, band peak temperatures, the
plume transmission, the perforation and core-boil times and the record's depth axis."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_recorder_matches_host_side_recording(gpu, tmp_path):
    from bug_defense_b200 import workloads
    from bug_defense_b200.coupled import CoupledAblationEngine
    from bug_defense_b200.phase import compute_phase_map
    from bug_defense_b200.record import Recorder
    geo = workloads.full_coupled_run(seed=3, nx=32, ny=32, nz=128, n_plume_air=16)
    kw = workloads.engine_kwargs(geo)
    kw.update(n_photons=40_000, power=80.0)
    eng = CoupledAblationEngine(**kw)
    k_surf = geo["n_air_top"]
    g0, g1 = geo["air_gap_range"]
    bands = ((k_surf, g0), (k_surf + 52, k_surf + 69), (k_surf + 100, k_surf + 110))
    y, ix = eng.Ny // 2, eng.Nx // 2
    # a tilted beam line as the production runner samples its centreline (x index per slice)
    line = np.clip(np.round((0.2 + 0.4 * np.arange(eng.Nz) * eng.dz) / eng.dx).astype(int), 0, eng.Nx - 1)
    rec = Recorder(eng, k_surface=k_surf, bands=bands, ring=4, beam_ix=line)
    gap = np.zeros(eng.shape, bool)
    gap[:, :, g0:g1] = True
    host = []
    for ep in range(10):
        eng.power = 80.0 if ep < 6 else 0.0
        eng._enqueue(0)
        rec.record()
        d = eng._diag(None)                           # the runner's synchronising path, for comparison
        T, Q, abl = eng.T, eng.Q, eng.ablated
        ph = compute_phase_map(T, eng.chi, eng.dry, abl, eng.H_acc, is_air_gap=gap)
        sl = abl[:, y, k_surf:]
        depth = (np.where(sl)[1].max() + 1) * eng.dz if sl.any() else 0.0
        host.append(dict(T=T[:, y, :], Q=Q[:, y, :], phase=ph[:, y, :], plume=eng.plume.mu_a_plume[:, y, :],
                         depth=depth, trans=d["plume_transmission"], time=d["time_s"],
                         peaks=[T[:, y, k0:k1].max() for k0, k1 in bands],
                         line_T=T[line, y, np.arange(eng.Nz)], line_ph=ph[line, y, np.arange(eng.Nz)],
                         perf=bool(abl[:, y, g0 - 1].any()), boil=T[:, y, bands[1][0]:bands[1][1]].max() >= 99.5))
    a = rec.finish()
    assert a["xz_T"].shape == (10, eng.Nx, eng.Nz)
    for ep, h in enumerate(host):
        np.testing.assert_array_equal(a["xz_T"][ep], h["T"].astype(np.float32))
        np.testing.assert_allclose(a["xz_Q"][ep], h["Q"], rtol=1e-6, atol=1e-12)
        np.testing.assert_array_equal(a["xz_phase"][ep], h["phase"])
        np.testing.assert_allclose(a["xz_plume"][ep], h["plume"], rtol=1e-6, atol=1e-9)
        assert a["crater_depths_mm"][ep] == pytest.approx(h["depth"], abs=1e-9)
        assert a["plume_trans"][ep] == pytest.approx(h["trans"], rel=1e-6)
        assert a["times"][ep] == pytest.approx(h["time"], abs=1e-12)
        for key, pk in zip(("peak_T_dorsal", "peak_T_core", "peak_T_ventral"), h["peaks"]):
            assert a[key][ep] == pytest.approx(pk, rel=1e-6)
        np.testing.assert_array_equal(a["centerline_T"][ep], h["line_T"].astype(np.float32))
        np.testing.assert_array_equal(a["centerline_phase"][ep], h["line_ph"])
    assert a["crater_depths_mm"].max() > 0          # 80 W on a 32x32 stack ablates in a few epochs
    # the runner's event times (run_highres_knowledge_suite.py:313-318): first epoch with an ablated
    # voxel just above the air gap in the mid-y slice, first with the core band at 99.5 C
    full = rec.record_arrays(a)
    perf = [h["time"] for h in host if h["perf"]]
    boil = [h["time"] for h in host if h["boil"]]
    assert full["t_perforation_s"] == (pytest.approx(perf[0], abs=1e-12) if perf else None)
    assert full["t_core_boil_s"] == (pytest.approx(boil[0], abs=1e-12) if boil else None)
    np.testing.assert_allclose(full["grid_z"], np.linspace(-k_surf * eng.dz, (eng.Nz - k_surf) * eng.dz, eng.Nz))
    rec2 = Recorder(eng, k_surface=k_surf, bands=bands)
    eng._enqueue(0)
    rec2.record()
    rec2.save_npz(tmp_path / "run.npz", wavelength_nm=532.0, power_w=80.0)
    z = np.load(tmp_path / "run.npz", allow_pickle=True)   # None event times are stored as objects, as the runner does
    for key in ("times", "xz_T", "xz_Q", "xz_phase", "xz_plume", "centerline_phase", "crater_depths_mm", "NZ",
                "t_perforation_s", "t_core_boil_s", "grid_z", "wavelength_nm", "power_w"):
        assert key in z.files


def test_runner_writes_the_suite_record(gpu, tmp_path):
    """The production run (runner.run_highres: the runner's geometry, beam and bands) for its first
    30 epochs: the record carries every key of run_highres_knowledge_suite.py:335-367 and the suite's
    KPIs come out of it (compute_suite_metrics.analyze_npz over a 20 ms pulse)."""
    from bug_defense_b200 import runner
    out = tmp_path / "matrix_532nm_80w.npz"
    rec = runner.run_highres(532.0, 80.0, out, n_epochs=30, log=None)
    z = np.load(out, allow_pickle=True)
    keys = {"times", "grid_x", "grid_y", "grid_z", "centerline_T", "centerline_Q", "centerline_phase", "xz_T", "xz_Q",
            "xz_phase", "xz_plume", "plume_trans", "peak_T_dorsal", "peak_T_core", "peak_T_ventral",
            "crater_depths_mm", "t_perforation_s", "t_core_boil_s", "wavelength_nm", "power_w", "theta_inc_deg",
            "phi_inc_deg", "x_dorsal_centered", "x_ventral_centered", "dorsal_cuticle_um", "air_gap_end_um",
            "ventral_shell_um", "NX", "NY", "NZ", "DX", "DY", "DZ", "dt_epoch"}
    assert keys <= set(z.files)
    assert z["xz_T"].shape == (30, runner.NX, runner.NZ) and z["grid_z"][0] == pytest.approx(-runner.L_AIR_TOP)
    assert z["grid_z"][-1] == pytest.approx(runner.L_BEETLE)
    assert float(z["peak_T_dorsal"].max()) > runner.T_AMBIENT + 50      # 80 W heats the dorsal shell
    m = runner.suite_metrics(str(out), pulse_duration_s=0.02)
    assert m["wavelength_nm"] == 532 and m["power_w"] == 80.0 and m["final_depth_um"] >= 0.0
    assert m["R_pct"] == runner.SPECTRO_MAP[532]["R"]
