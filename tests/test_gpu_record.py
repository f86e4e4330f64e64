"""Device-side per-epoch recording (bd_engine_record + Recorder) equals what the production runner
computes from full host copies of the engine state after every epoch
(run_highres_knowledge_suite.py:271-306): xz slices of T, Q, phase and plume absorption, the crater
depth below the surface, band peak temperatures and the plume transmission."""
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
    rec = Recorder(eng, k_surface=k_surf, bands=bands, ring=4)
    y, ix = eng.Ny // 2, eng.Nx // 2
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
                         peaks=[T[:, y, k0:k1].max() for k0, k1 in bands]))
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
        np.testing.assert_array_equal(a["centerline_T"][ep], h["T"][ix].astype(np.float32))
    assert a["crater_depths_mm"].max() > 0          # 80 W on a 32x32 stack ablates in a few epochs
    rec2 = Recorder(eng, k_surface=k_surf, bands=bands)
    eng._enqueue(0)
    rec2.record()
    rec2.save_npz(tmp_path / "run.npz", wavelength_nm=532.0, power_w=80.0)
    z = np.load(tmp_path / "run.npz")
    for key in ("times", "xz_T", "xz_Q", "xz_phase", "xz_plume", "centerline_phase", "crater_depths_mm", "NZ"):
        assert key in z.files
