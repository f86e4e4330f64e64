"""Generate tests/golden/runner.npz by running the REFERENCE production runner's model builder and the
suite's KPI extraction.

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_runner_golden.py [/path/to/reference]

  * build_beetle_model(wl) of knowledge/beetle/scripts/run_highres_knowledge_suite.py:126-185 at 532 and
    1470 nm (tissue-optics package absent, so simulation/tissue_stack.py uses its built-in rule): every
    grid is constant in x and y, so one (x, y) column of each is stored, with the beam constants.
    The runner module is executed with its plotting and animation imports stubbed and its output
    directories not created (it would write into the reference tree).
  * analyze_npz of knowledge/beetle/scripts/compute_suite_metrics.py:29-135 on two synthetic run records
    (a coarse 80 x 92 grid over the runner's depth range, 210 epochs, a crater with boiling rims, a
    warm core and ventral plate), stored with the KPIs the reference computes from them.
"""
from __future__ import annotations

import json
import os
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
REF = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
sys.path.insert(0, str(REF))
sys.path.insert(0, str(REF / "knowledge" / "beetle" / "scripts"))


def load_runner():
    for name in ("matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    stub = types.ModuleType("knowledge.beetle.scripts.render_native_highres_animation")
    stub.render_native_animation = lambda *a, **k: None
    sys.modules["knowledge.beetle.scripts.render_native_highres_animation"] = stub
    path = REF / "knowledge" / "beetle" / "scripts" / "run_highres_knowledge_suite.py"
    mod = types.ModuleType("run_highres_knowledge_suite")
    mod.__file__ = str(path)
    real = os.makedirs
    os.makedirs = lambda *a, **k: None
    try:
        exec(compile(path.read_text(), str(path), "exec"), mod.__dict__)
    finally:
        os.makedirs = real
    return mod


def synthetic_record(seed):
    rng = np.random.default_rng(seed)
    nx, nz, ne = 80, 92, 210
    dx, dz = 3.0 / nx, 2.76 / nz
    grid_x = np.linspace(0, 3.0, nx)
    grid_z = np.linspace(-0.315, 2.445, nz)
    times = (np.arange(ne) + 1) * 1e-3
    depth_end = rng.uniform(0.3, 1.2)
    depths = depth_end * np.minimum(1.0, times / 0.2) ** 0.7
    xz_T = np.zeros((ne, nx, nz), np.float32)
    xz_phase = np.zeros((ne, nx, nz), np.uint8)
    xc = (np.arange(nx) + 0.5) * dx - 1.5
    zc = grid_z
    for e in (199, 209):
        r = rng.uniform(0.15, 0.35)
        crater = (np.abs(xc)[:, None] < r * np.sqrt(np.clip(1 - zc[None, :] / max(depths[e], 1e-3), 0, 1))) & \
                 (zc[None, :] >= 0) & (zc[None, :] <= depths[e])
        T = 20 + 300 * np.exp(-(xc[:, None] / 0.4) ** 2 - (np.clip(zc[None, :], 0, None) / 0.9) ** 2)
        T += rng.normal(0, 2.0, T.shape)
        ph = np.where(T >= 99.5, 2, 0).astype(np.uint8)
        ph[crater] = 3
        ph[:, zc < 0] = 3
        ph[:, (zc >= 0.165) & (zc <= 0.465)] = 3
        xz_T[e], xz_phase[e] = T, ph
    return dict(times=times, grid_x=grid_x, grid_y=np.linspace(0, 3.0, nx), grid_z=grid_z, xz_T=xz_T,
                xz_phase=xz_phase, crater_depths_mm=depths, DX=dx, DZ=dz, wavelength_nm=[532.0, 1470.0][seed % 2],
                power_w=[40.0, 80.0][seed % 2])


def main():
    run = load_runner()
    out = {}
    for wl in (532, 1470):
        geo = run.build_beetle_model(wl)
        for key in ("mu_a", "mu_s", "g", "n"):
            assert np.all(geo["optical"][key] == geo["optical"][key][:1, :1, :])
            out[f"wl{wl}_{key}"] = geo["optical"][key][0, 0, :]
            out[f"wl{wl}_ds_{key}"] = geo["dry_state"][key][0, 0, :]
        for key in ("k_grid", "rho_cp_grid", "h_lat_grid", "dry_mask", "initial_ablated"):
            out[f"wl{wl}_{key}"] = geo[key][0, 0, :]
    out["beam"] = json.dumps(dict(beam_center=list(run.BEAM_CENTER), theta=run.THETA_INC_DEG, tan_theta=run.TAN_THETA,
                                  x_top=run.X_TOP_PHYS, nz=run.NZ, nz_air=run.NZ_AIR_TOP))
    import compute_suite_metrics as csm
    import tempfile
    kpis = []
    for seed in (0, 1):
        rec = synthetic_record(seed)
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, f"matrix_{seed}.npz")
            np.savez(p, **rec)
            k = csm.analyze_npz(p)
        k.pop("path")
        kpis.append(k)
        for key, v in rec.items():
            out[f"rec{seed}_{key}"] = np.asarray(v)
    out["kpis"] = json.dumps(kpis)
    np.savez_compressed(OUT / "runner.npz", **out)
    print("wrote runner.npz", json.dumps(kpis)[:400])


if __name__ == "__main__":
    main()
