"""The production high-resolution run: geometry, the 1000-epoch schedule, the per-run npz record and
the suite's KPI extraction, on the device engine.

Restates knowledge/beetle/scripts/run_highres_knowledge_suite.py (constants :57-118, the model builder
build_beetle_model :126-185, the run loop :187-329, the record :330-367) and
knowledge/beetle/scripts/compute_suite_metrics.py (analyze_npz :29-135). The per-epoch series come from
the device recorder (record.Recorder) instead of full host copies of the engine state after every
epoch; t_perforation_s and t_core_boil_s are derived from the recorded xz phase slice and the core-band
peak temperature exactly as the runner tests them per epoch.

    python -m bug_defense_b200.runner --wavelength 532 --power 40 --out run.npz
"""
from __future__ import annotations

import math
import time

import numpy as np

from .lasersim import fallback_layer_optics

# ---- the published run (run_highres_knowledge_suite.py:57-118): 15 um isotropic voxels, 200 x 200 x
# 184 grid, 21 slices of ambient air above a 163-slice body, a beam tilted so it enters the dorsal
# surface at x = -0.5 mm and would leave the ventral plate at x = +0.5 mm ----
DX = DY = DZ = 0.015
LX = LY = 3.0
NX, NY = 200, 200
NZ_AIR_TOP, NZ_BEETLE = 21, 163
NZ = NZ_AIR_TOP + NZ_BEETLE
L_AIR_TOP, L_BEETLE = NZ_AIR_TOP * DZ, NZ_BEETLE * DZ
LZ = NZ * DZ
X_DORSAL, X_VENTRAL = 1.0, 2.0                        # mm, entry / exit x of the beam axis
TAN_THETA = (X_VENTRAL - X_DORSAL) / (LZ - L_AIR_TOP)
THETA_INC_DEG = math.degrees(math.atan(TAN_THETA))
PHI_INC_DEG = 0.0
X_TOP = X_DORSAL - L_AIR_TOP * TAN_THETA               # beam axis at the grid's top face
BEAM_CENTER = (X_TOP, LY / 2.0)
SPOT_DIA = 0.50
T_EXPOSURE, T_PULSE, DT_EPOCH, DT_SUB = 1.0, 0.2, 0.001, 1.0 / 20000.0
N_PHOTONS = 150_000
T_AMBIENT, T_BOIL, T_ABL_CUTICLE, H_EFF = 20.0, 100.0, 350.0, 15.0e-6
H_LAT_WATER = 2.26                                      # J/mm^3 of a boiling layer
PLUME_CLOSURE = {'model': 'diffusion', 'D_xy': 1.0, 'D_z': 2.0, 'v_drift': 0.0, 'tau_linger_s': float('inf'),
                 'blast_expansion': False}
WAVELENGTHS = (320, 450, 532, 1064, 1470, 1940, 10600)
POWERS = (20.0, 40.0, 80.0)
# the runner's char kinetics (run_multispectral_matrix.py:69-78)
CHAR_STATE = {'A': 1.0e7, 'Ea': 65000.0, 'mu_a': 15.0, 'mu_s': 20.0, 'k': 0.35e-3, 'rho_cp': 2.0e-3,
              't_remove': T_ABL_CUTICLE, 'chi_remove': 0.95}

# The thirteen-layer tissue table whose optics the runner evaluates (simulation/tissue_stack.py:24-42):
# name, thickness (um), composition by volume fraction. Only the composition enters the optics here.
BASE_LAYERS = [
    {'name': 'epicuticle_wax', 'thickness_um': 2.0, 'composition': {'lipid': 0.85, 'protein': 0.15}},
    {'name': 'exocuticle_sclerotised', 'thickness_um': 60.0,
     'composition': {'chitin': 0.403, 'protein': 0.33, 'water': 0.18, 'melanin': 0.075, 'ommochrome': 0.012}},
    {'name': 'endocuticle', 'thickness_um': 100.0, 'composition': {'water': 0.42, 'chitin': 0.33, 'protein': 0.25}},
    {'name': 'subelytral_air_gap', 'thickness_um': 300.0, 'composition': {'air': 1.0}},
    {'name': 'epidermis', 'thickness_um': 20.0, 'composition': {'water': 0.70, 'protein': 0.22, 'lipid': 0.08}},
    {'name': 'fat_body', 'thickness_um': 300.0, 'composition': {'lipid': 0.50, 'water': 0.38, 'protein': 0.12}},
    {'name': 'hemolymph', 'thickness_um': 250.0, 'composition': {'water': 0.93, 'protein': 0.07}},
    {'name': 'muscle', 'thickness_um': 1581.0, 'composition': {'water': 0.76, 'protein': 0.21, 'lipid': 0.03}},
    {'name': 'fat_body', 'thickness_um': 300.0, 'composition': {'lipid': 0.50, 'water': 0.38, 'protein': 0.12}},
    {'name': 'epidermis', 'thickness_um': 20.0, 'composition': {'water': 0.70, 'protein': 0.22, 'lipid': 0.08}},
    {'name': 'endocuticle', 'thickness_um': 40.0, 'composition': {'water': 0.42, 'chitin': 0.33, 'protein': 0.25}},
    {'name': 'exocuticle_sclerotised', 'thickness_um': 25.0,
     'composition': {'chitin': 0.43, 'protein': 0.352, 'water': 0.18, 'melanin': 0.03, 'ommochrome': 0.008}},
    {'name': 'epicuticle_wax', 'thickness_um': 2.0, 'composition': {'lipid': 0.85, 'protein': 0.15}},
]

# The voxelised body (run_highres_knowledge_suite.py:146-158): slab [k0, k1) below the dorsal surface
# -> (BASE_LAYERS row whose optics it takes, k W/(mm K), rho_cp J/(mm^3 K), h_lat J/mm^3, starts dry).
# Rows 9 and 12 of BASE_LAYERS (ventral epidermis, ventral wax) are not voxelised.
BODY_SLABS = (
    ((0, 1), 0, 0.22e-3, 1.98e-3, 0.0, True),               # epicuticle wax
    ((1, 5), 1, 0.28e-3, 2.40e-3, 0.0, True),               # dorsal exocuticle
    ((5, 11), 2, 0.35e-3, 2.50e-3, 0.0, True),              # dorsal endocuticle (dorsal shell: 11 slices)
    ((11, 31), 3, 0.026e-3, 1.206e-6, 1e12, False),         # subelytral air gap
    ((31, 32), 4, 0.48e-3, 3.50e-3, H_LAT_WATER, False),    # epidermis
    ((32, 52), 5, 0.32e-3, 2.80e-3, H_LAT_WATER, False),    # fat body
    ((52, 69), 6, 0.58e-3, 3.89e-3, H_LAT_WATER, False),    # hemolymph
    ((69, 137), 7, 0.50e-3, 3.65e-3, H_LAT_WATER, False),   # muscle
    ((137, 157), 8, 0.32e-3, 2.80e-3, H_LAT_WATER, False),  # ventral fat
    ((157, 160), 10, 0.35e-3, 2.50e-3, 0.0, True),          # ventral endocuticle
    ((160, 163), 11, 0.28e-3, 2.40e-3, 0.0, True),          # ventral exocuticle + wax
)
AIR_GAP = (NZ_AIR_TOP + 11, NZ_AIR_TOP + 31)             # grid slices of the air gap
# depth bands of the recorded peak temperatures (run_highres_knowledge_suite.py:300-306)
BANDS = ((NZ_AIR_TOP, AIR_GAP[0]), (NZ_AIR_TOP + 52, NZ_AIR_TOP + 69), (NZ_AIR_TOP + 157, NZ_AIR_TOP + 163))
# fixed metadata of the record (run_highres_knowledge_suite.py:358-363)
RECORD_META = dict(x_dorsal_centered=-0.500, x_ventral_centered=+0.500, dorsal_cuticle_um=165.0,
                   air_gap_end_um=465.0, ventral_shell_um=2355.0)


def slice_columns(wl_nm: float, eval_layer=fallback_layer_optics) -> dict:
    """Per-slice property columns (length NZ) of the body at wavelength wl_nm: optics from the
    layer evaluator (default: the reference's rule without the tissue-optics package), thermal
    values from BODY_SLABS; the ambient air above the body starts ablated."""
    ev = [eval_layer(lay, float(wl_nm)) for lay in BASE_LAYERS]
    col = dict(mu_a=np.zeros(NZ), mu_s=np.zeros(NZ), g=np.zeros(NZ), n=np.ones(NZ), k=np.full(NZ, 0.026e-3),
               rho_cp=np.full(NZ, 1.206e-6), h_lat=np.full(NZ, 1e12), dry=np.zeros(NZ, bool),
               ablated=np.arange(NZ) < NZ_AIR_TOP)
    for (k0, k1), row, k, rho_cp, h_lat, dry in BODY_SLABS:
        z = slice(NZ_AIR_TOP + k0, NZ_AIR_TOP + k1)
        for key in ('mu_a', 'mu_s', 'g', 'n'):
            col[key][z] = float(ev[row][key])
        col['k'][z], col['rho_cp'][z], col['h_lat'][z], col['dry'][z] = k, rho_cp, h_lat, dry
    return col


def build_beetle_model(wl_nm: float, eval_layer=fallback_layer_optics, device=None) -> dict:
    """The runner's geometry (build_beetle_model, run_highres_knowledge_suite.py:126-185): full
    (NX, NY, NZ) grids, float64 numpy arrays, or float64 torch tensors expanded on `device` (no host
    grids). Keys as the reference: optical, k_grid, rho_cp_grid, h_lat_grid, dry_mask,
    initial_ablated, dry_state."""
    col = slice_columns(wl_nm, eval_layer)
    shape = (NX, NY, NZ)
    if device is None:
        grid = lambda c: np.broadcast_to(c, shape).copy()
    else:
        import torch
        dev = torch.device(device)
        grid = lambda c: torch.as_tensor(c, device=dev).expand(shape).contiguous()
    optical = {key: grid(col[key]) for key in ('mu_a', 'mu_s', 'g', 'n')}
    k, rho_cp = grid(col['k']), grid(col['rho_cp'])
    dry_state = {key: grid(col[key]) for key in ('mu_a', 'mu_s', 'g', 'n')}
    dry_state.update(k=grid(col['k']), rho_cp=grid(col['rho_cp']), t_remove=T_ABL_CUTICLE)
    return dict(optical=optical, k_grid=k, rho_cp_grid=rho_cp, h_lat_grid=grid(col['h_lat']),
                dry_mask=grid(col['dry']), initial_ablated=grid(col['ablated']), dry_state=dry_state)


def engine_kwargs(geo: dict, wl_nm: float, power_w: float) -> dict:
    """The runner's CoupledAblationEngine arguments (run_highres_knowledge_suite.py:202-229)."""
    return dict(optical_props=geo['optical'], k_grid=geo['k_grid'], rho_cp_grid=geo['rho_cp_grid'],
                h_lat_grid=geo['h_lat_grid'], Lx=LX, Ly=LY, Lz=LZ, power=power_w, spot_dia=SPOT_DIA, t_abl=T_BOIL,
                t_ambient=T_AMBIENT, dt_epoch=DT_EPOCH, dt_sub=DT_SUB, n_photons=N_PHOTONS, h_eff=H_EFF,
                beam_center=BEAM_CENTER, beam_profile='gaussian', theta_inc_deg=THETA_INC_DEG,
                phi_inc_deg=PHI_INC_DEG, dry_state=geo['dry_state'], char_state=CHAR_STATE,
                plume_closure=PLUME_CLOSURE, initial_dry_mask=geo['dry_mask'],
                initial_ablated_mask=geo['initial_ablated'], air_gap_range=AIR_GAP, wavelength_nm=wl_nm)


def beam_columns(nx=NX, nz=NZ, dx=DX, dz=DZ, x_top=X_TOP, tan_theta=TAN_THETA) -> np.ndarray:
    """x index of the beam axis in every slice (the runner's centreline sampling line, :239)."""
    return np.clip(np.round((x_top + tan_theta * (np.arange(nz) * dz)) / dx).astype(int), 0, nx - 1)


def run_highres(wl_nm: float, power_w: float, out_file=None, n_epochs: int | None = None, device=None,
                log=print) -> dict:
    """One run of the suite: the engine on the runner's geometry, the laser on for the first 200 ms of
    1 s, every epoch recorded on the device; writes the runner's npz (when out_file is given) and
    returns its arrays."""
    import torch
    from .coupled import CoupledAblationEngine
    from .record import Recorder
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    geo = build_beetle_model(wl_nm, device=dev)
    eng = CoupledAblationEngine(**engine_kwargs(geo, wl_nm, power_w), device=dev)
    n = int(round(T_EXPOSURE / DT_EPOCH)) if n_epochs is None else int(n_epochs)
    rec = Recorder(eng, k_surface=NZ_AIR_TOP, bands=BANDS, beam_ix=beam_columns(), ring=32)
    t0 = time.time()
    for ep in range(n):
        eng.power = power_w if ep * DT_EPOCH < T_PULSE else 0.0
        eng._enqueue(0)
        rec.record()
        if log and (ep % 100 == 0 or ep == n - 1):
            log(f"{wl_nm:.0f} nm {power_w:.0f} W: epoch {ep + 1}/{n} ({time.time() - t0:.1f} s)")
    meta = dict(wavelength_nm=wl_nm, power_w=power_w, theta_inc_deg=THETA_INC_DEG, phi_inc_deg=PHI_INC_DEG,
                **RECORD_META)
    out = rec.record_arrays(gap_k0=AIR_GAP[0], **meta)
    if out_file is not None:
        np.savez_compressed(out_file, **out)
    return out


# ---- KPIs of a run record (compute_suite_metrics.py) -------------------------------------------
# Spectrophotometric split of the intact 13-layer stack per wavelength, percent (compute_suite_metrics.py:
# 18-26): the suite reports these table values beside each run's KPIs.
SPECTRO_MAP = {
    320: {'R': 6.23, 'A': 92.96, 'T': 0.00, 'Lat': 0.81},
    450: {'R': 13.54, 'A': 77.92, 'T': 0.13, 'Lat': 8.41},
    532: {'R': 19.61, 'A': 61.33, 'T': 0.60, 'Lat': 18.46},
    1064: {'R': 23.68, 'A': 11.51, 'T': 4.58, 'Lat': 60.23},
    1470: {'R': 9.63, 'A': 86.86, 'T': 0.11, 'Lat': 3.40},
    1940: {'R': 5.00, 'A': 94.86, 'T': 0.00, 'Lat': 0.13},
    10600: {'R': 4.28, 'A': 95.72, 'T': 0.00, 'Lat': 0.00},
}


def _disc_volumes(ph, in_tissue, dx, dz):
    """Ablated and boiling volumes (mm^3): each slice's ablated / ablated+boiling voxel counts along x
    taken as the diameter of a disc one slice thick (the suite's axisymmetric estimate)."""
    n_abl = (ph == 3).sum(axis=0)[in_tissue]
    n_boil = (ph == 2).sum(axis=0)[in_tissue]
    r_abl = n_abl * dx / 2.0
    r_tot = (n_abl + n_boil) * dx / 2.0
    return float(np.sum(np.pi * r_abl ** 2 * dz)), float(np.sum(np.pi * np.maximum(r_tot ** 2 - r_abl ** 2, 0.0) * dz))


def suite_metrics(record, pulse_duration_s: float = 0.200, path: str = "") -> dict:
    """The KPIs of compute_suite_metrics.analyze_npz for a run record (an npz path or a dict of its
    arrays): final / mean crater depth over the pulse, penetration speed, mean hole diameter, the
    spectral split of the wavelength, core and ventral temperatures (mean without void, max) and
    ablated / boiling volumes, all at the last epoch of the pulse."""
    d = np.load(record) if isinstance(record, (str, bytes)) or hasattr(record, "__fspath__") else record
    gx = np.asarray(d['grid_x'])
    x = gx - gx[-1] / 2.0
    z_um = np.asarray(d['grid_z']) * 1000.0
    depths = np.asarray(d['crater_depths_mm']) * 1000.0
    dx = float(d['DX']) if 'DX' in d else 0.015
    dz = float(d['DZ']) if 'DZ' in d else 0.015
    n = len(np.asarray(d['times']))
    i_end = min(int(round(pulse_duration_s * 1000.0)) - 1, n - 1)
    final_um = float(depths[i_end])
    ph = np.asarray(d['xz_phase'])[i_end]
    T = np.asarray(d['xz_T'])[i_end]
    shell_gap = (z_um >= 165.0) & (z_um <= 465.0)          # the air gap between 165 and 465 um
    solid = (z_um >= 0) & (z_um <= final_um) & ~shell_gap
    widths = (ph == 3).sum(axis=0)[solid]
    widths = widths[widths > 0] * dx
    centre = np.abs(x) <= 0.30

    def region(z0, z1):
        m = np.outer(centre, (z_um >= z0) & (z_um <= z1))
        valid = m & (ph != 3)
        return (float(T[valid].mean()) if valid.any() else 20.0), (float(T[m].max()) if m.any() else 20.0)

    core_avg, core_max = region(780.0, 1035.0)
    ven_avg, ven_max = region(2355.0, 2445.0)
    v_abl, v_boil = _disc_volumes(ph, (z_um >= 0) & ~shell_gap, dx, dz)
    wl = int(round(float(d['wavelength_nm']))) if 'wavelength_nm' in d else None
    power = float(d['power_w']) if 'power_w' in d else None
    dual = 'laser_states' in d or 'dual' in str(path)
    if 'laser_states' in d and wl is None:
        sp = {'R': 0.0, 'A': 0.0, 'T': 0.0}
    else:
        sp = SPECTRO_MAP.get(wl, {'R': 4.0, 'A': 95.0, 'T': 0.0})
    return {
        'path': str(path) if path else (str(record) if isinstance(record, str) else ""),
        'wavelength_nm': wl, 'power_w': power,
        'final_depth_um': final_um, 'avg_depth_um': float(np.mean(depths[:i_end + 1])),
        'speed_mm_s': float(final_um / 1000.0 / pulse_duration_s),
        'avg_hole_dia_mm': float(widths.mean()) if widths.size else 0.0,
        'R_pct': sp.get('R', 0.0), 'A_pct': sp.get('A', 0.0), 'T_pct': sp.get('T', 0.0),
        'core_avg_T': core_avg, 'core_max_T': core_max, 'ven_avg_T': ven_avg, 'ven_max_T': ven_max,
        'v_abl_mm3': v_abl, 'v_boil_mm3': v_boil,
        'energy_used_j': 4.60 if dual else (float(power * pulse_duration_s) if power is not None else 8.00),
    }


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="one high-resolution run of the suite on the GPU")
    ap.add_argument("--wavelength", type=float, default=532.0)
    ap.add_argument("--power", type=float, default=40.0)
    ap.add_argument("--epochs", type=int, default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    rec = run_highres(a.wavelength, a.power, a.out, n_epochs=a.epochs)
    print(json.dumps(suite_metrics(rec, path=a.out or "")))


if __name__ == "__main__":
    main()
