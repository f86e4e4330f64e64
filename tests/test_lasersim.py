"""LaserSim driver host logic against the reference (fixture tests/golden/lasersim_model.npz, made by
tests/golden/make_lasersim_golden.py from simulation/beetle_sim.py and simulation/tissue_stack.py with
the tissue-optics package switched off): the default layer table, per-layer optics, the voxelised
model's per-slice columns and slice ranges, and the region bookkeeping."""
import json

import numpy as np
import pytest

from bug_defense_b200 import lasersim as ls


@pytest.fixture(scope="module")
def gold(golden):
    return golden("lasersim_model.npz")


def test_default_layers_match_reference(gold):
    assert ls.default_setup()["layers"] == json.loads(str(gold["layers_json"]))


def test_layer_optics_match_reference_fallback(gold):
    layers = json.loads(str(gold["layers_json"]))
    for a, wl in enumerate(gold["wavelengths"]):
        for b, lay in enumerate(layers):
            e = ls.fallback_layer_optics(lay, float(wl))
            got = [e["mu_a"], e["mu_s"], e["mu_s_prime"], e["g"], e["n"], e["penetration_depth_mm"]]
            np.testing.assert_array_equal(got, gold["eval"][a, b])
    assert ls.evaluate_layers(layers, 532.0) == json.loads(str(gold["evaluate_layers_532"]))


@pytest.mark.parametrize("voxel", [30, 20])
def test_build_model_matches_reference(gold, voxel):
    layers = json.loads(str(gold["layers_json"]))
    geo = ls.build_model(layers, 532.0, float(voxel))
    tag = f"v{voxel}"
    assert tuple(geo["shape"]) == tuple(gold[f"{tag}_shape"]) and geo["nz_air"] == int(gold[f"{tag}_nz_air"])
    for key in ("mu_a", "mu_s", "g", "n"):
        np.testing.assert_array_equal(geo["optical"][key][0, 0, :], gold[f"{tag}_{key}"])
        assert np.all(geo["optical"][key] == geo["optical"][key][:1, :1, :])
    for key in ("k_grid", "rho_cp_grid", "h_lat_grid"):
        np.testing.assert_array_equal(geo[key][0, 0, :], gold[f"{tag}_{key}"])
    np.testing.assert_array_equal(geo["dry_mask"][0, 0, :], gold[f"{tag}_dry"])
    np.testing.assert_array_equal(geo["is_air"][0, 0, :], gold[f"{tag}_is_air"])
    np.testing.assert_array_equal(geo["initial_ablated"][0, 0, :], gold[f"{tag}_ablated"])
    assert [list(r) for r in geo["ranges"]] == json.loads(str(gold[f"{tag}_ranges"]))
    reg = json.loads(str(gold[f"{tag}_regions"]))
    got = ls.layer_regions(geo["ranges"], geo["nz_air"])
    assert json.loads(json.dumps(got)) == reg
