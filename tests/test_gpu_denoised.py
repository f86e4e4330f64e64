"""The denoised coupled run (denoised.DenoisedCoupledRun: 15k photons + U-Net) on a small stack: laser
epochs take their source from a 15k-photon map through the trained network, spot checks compare it
with the plain map, and a threshold below the observed distance falls back to plain MC for good."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine(gpu, seed=3):
    from bug_defense_b200 import workloads
    geo = workloads.full_coupled_run(seed=seed, nx=48, ny=48, nz=128, n_plume_air=16)
    kw = workloads.engine_kwargs(geo)
    kw.update(n_photons=150_000, power=40.0)
    return gpu.CoupledAblationEngine(**kw)


def test_denoised_epochs_heat_like_plain_mc_and_check_themselves(gpu):
    from bug_defense_b200.denoised import DenoisedCoupledRun
    eng, ref = _engine(gpu), _engine(gpu)
    run = DenoisedCoupledRun(eng, check_every=2, threshold=10.0)
    for _ in range(6):
        d = run.step_epoch()
        ref.step_epoch()
    assert d["denoised"] and len(d["spot_checks"]) == 3
    rels = [r for _, r, _ in d["spot_checks"]]
    assert all(np.isfinite(r) and 0.0 < r < 1.0 for r in rels), rels
    assert all(b == 10.0 for _, _, b in d["spot_checks"])
    # the same heating as with plain 150k-photon MC to within the maps' noise
    rise, rise_ref = eng.T - 25.0, ref.T - 25.0
    assert rise.max() > 10.0
    assert np.linalg.norm(rise - rise_ref) / np.linalg.norm(rise_ref) < 0.2
    eng.power = 0.0
    d = run.step_epoch()                        # laser off: the engine's own epoch, no MC
    assert len(d["spot_checks"]) == 3


def test_spot_check_above_threshold_falls_back_to_plain_mc(gpu):
    from bug_defense_b200.denoised import DenoisedCoupledRun
    eng = _engine(gpu)
    run = DenoisedCoupledRun(eng, check_every=1, threshold=1e-6)
    d = run.step_epoch()
    assert not d["denoised"] and len(d["spot_checks"]) == 1
    n = run.laser_epochs
    d = run.step_epoch()                        # plain MC from now on: no further denoised epochs
    assert run.laser_epochs == n and len(d["spot_checks"]) == 1
    assert d["ledger"][0] == eng.n_photons      # the engine's own MC ran


def test_equal_error_bound_comes_from_the_plain_maps_noise(gpu):
    """Without a fixed threshold the bound is sqrt(2) x the plain map's relative noise, estimated from
    its two independent halves (~0.1-0.3 for 150k photons on this stack)."""
    from bug_defense_b200.denoised import DenoisedCoupledRun
    eng = _engine(gpu)
    run = DenoisedCoupledRun(eng, check_every=1)
    d = run.step_epoch()
    (_, rel, bound), = d["spot_checks"]
    assert 0.05 < bound / 2 ** 0.5 < 0.5 and np.isfinite(rel)
    assert d["denoised"] == (rel <= bound)
