"""The production runner's geometry and the suite's KPIs against the reference (fixture
tests/golden/runner.npz, made by tests/golden/make_runner_golden.py from
knowledge/beetle/scripts/run_highres_knowledge_suite.py and compute_suite_metrics.py)."""
import json

import numpy as np
import pytest

from bug_defense_b200 import runner


@pytest.fixture(scope="module")
def gold(golden):
    return golden("runner.npz")


@pytest.mark.parametrize("wl", [532, 1470])
def test_build_beetle_model_matches_reference(gold, wl):
    col = runner.slice_columns(wl)
    for key in ("mu_a", "mu_s", "g", "n"):
        np.testing.assert_array_equal(col[key], gold[f"wl{wl}_{key}"])
        np.testing.assert_array_equal(col[key], gold[f"wl{wl}_ds_{key}"])
    for ours, ref in (("k", "k_grid"), ("rho_cp", "rho_cp_grid"), ("h_lat", "h_lat_grid"), ("dry", "dry_mask"),
                      ("ablated", "initial_ablated")):
        np.testing.assert_array_equal(col[ours], gold[f"wl{wl}_{ref}"])
    geo = runner.build_beetle_model(wl)
    assert geo["optical"]["mu_a"].shape == (runner.NX, runner.NY, runner.NZ)
    np.testing.assert_array_equal(geo["optical"]["mu_a"][17, 123], col["mu_a"])
    assert geo["dry_state"]["t_remove"] == runner.T_ABL_CUTICLE


def test_beam_constants_match_reference(gold):
    b = json.loads(str(gold["beam"]))
    assert list(runner.BEAM_CENTER) == pytest.approx(b["beam_center"], abs=1e-15)
    assert runner.THETA_INC_DEG == pytest.approx(b["theta"], abs=1e-12)
    assert runner.NZ == b["nz"] and runner.NZ_AIR_TOP == b["nz_air"]
    ix = runner.beam_columns()
    ref = np.clip(np.round((b["x_top"] + b["tan_theta"] * (np.arange(b["nz"]) * runner.DZ)) / runner.DX).astype(int),
                  0, runner.NX - 1)
    np.testing.assert_array_equal(ix, ref)


@pytest.mark.parametrize("seed", [0, 1])
def test_suite_metrics_match_reference(gold, seed):
    kp = json.loads(str(gold["kpis"]))[seed]
    rec = {k[len(f"rec{seed}_"):]: gold[k] for k in gold.files if k.startswith(f"rec{seed}_")}
    got = runner.suite_metrics(rec)
    for key, v in kp.items():
        if v is None or isinstance(v, str):
            assert got[key] == v, key
        else:
            assert got[key] == pytest.approx(v, rel=1e-12, abs=1e-12), key
