"""Golden fixture for the LaserSim model builder, made by running the REFERENCE in this container.

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_lasersim_golden.py [/path/to/reference]

Records, with the reference's tissue-optics package switched off (tissue_stack.HAS_TISSUE_OPTICS =
False, the branch bug_defense_b200.lasersim.fallback_layer_optics restates): eval_single_layer of
every default layer at five wavelengths, and beetle_sim.build_model's per-slice property columns,
slice ranges and _regions for the default layers at the preview (30 um) and standard (20 um)
voxel sizes. Tests never import the reference at run time.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
REF = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
sys.path.insert(0, str(REF))

import simulation.tissue_stack as ts  # noqa: E402
import simulation.beetle_sim as bs  # noqa: E402

ts.HAS_TISSUE_OPTICS = False
WAVELENGTHS = (450.0, 532.0, 808.0, 1064.0, 1940.0)
layers = bs.default_setup()["layers"]
out = {"layers_json": json.dumps(layers), "wavelengths": np.array(WAVELENGTHS)}
ev = np.zeros((len(WAVELENGTHS), len(layers), 6))
for a, wl in enumerate(WAVELENGTHS):
    for b, lay in enumerate(layers):
        e = ts.eval_single_layer(lay, wl)
        ev[a, b] = [e["mu_a"], e["mu_s"], e["mu_s_prime"], e["g"], e["n"], e["penetration_depth_mm"]]
out["eval"] = ev
out["evaluate_layers_532"] = json.dumps(bs.evaluate_layers(layers, 532.0))
for voxel in (30.0, 20.0):
    geo = bs.build_model(layers, 532.0, voxel)
    tag = f"v{int(voxel)}"
    out[f"{tag}_shape"] = np.array(geo["shape"])
    out[f"{tag}_nz_air"] = geo["nz_air"]
    for key in ("mu_a", "mu_s", "g", "n"):
        out[f"{tag}_{key}"] = geo["optical"][key][0, 0, :]
    for key in ("k_grid", "rho_cp_grid", "h_lat_grid"):
        out[f"{tag}_{key}"] = geo[key][0, 0, :]
    out[f"{tag}_dry"] = geo["dry_mask"][0, 0, :]
    out[f"{tag}_is_air"] = geo["is_air"][0, 0, :]
    out[f"{tag}_ablated"] = geo["initial_ablated"][0, 0, :]
    out[f"{tag}_ranges"] = json.dumps([list(r) for r in geo["ranges"]])
    out[f"{tag}_regions"] = json.dumps(bs._regions(geo["ranges"], geo["nz_air"]))
np.savez_compressed(OUT / "lasersim_model.npz", **out)
print("wrote", OUT / "lasersim_model.npz")
