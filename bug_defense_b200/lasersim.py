"""LaserSim driver on the device engine: the reference's interactive generator
(simulation/beetle_sim.py:201-313, streamed by server.py:55-80 as /api/run) and its model builder
(beetle_sim.py:133-180), same arguments and the same 'setup' / 'frame' / 'done' events.

Differences, all on the host side of the engine:
* the x-z mid-plane slices and the crater depth of a frame come from the engine's device-side
  record (bd_engine_record) instead of full 3-D host copies of T, Q, chi, ... per frame;
* the per-layer optics come from `eval_layer(layer, wavelength_nm)`. The reference evaluates them
  with simulation.tissue_stack.eval_single_layer, which needs its insect_tissue_optics package;
  pass that function to reproduce its properties exactly. The default, `fallback_layer_optics`,
  restates eval_single_layer's own branch for when that package is absent (tissue_stack.py:
  90-196: power-law baseline + melanin + water absorption, Rayleigh/Mie reduced scattering,
  constant g, water-weighted index), including its rounding of the returned values;
* the frame energies use the engine's FP64 photon ledger of each laser epoch.
"""
from __future__ import annotations

import base64
import math
import time

import numpy as np

from .coupled import K_AIR, RHO_CP_AIR, CoupledAblationEngine
from .phase import CHAR_STATE
from .record import Recorder
from . import _lib

LX = LY = 3.0                  # mm lateral domain
AIR_TOP_UM = 315.0             # ambient air above the dorsal surface
T_AMBIENT = 20.0
T_BOIL = 100.0
T_ABL_CUTICLE = 350.0
H_EFF = 15.0e-6                # W/(mm^2 K) surface loss
DT_EPOCH = 0.001               # 1 ms optical/thermal coupling step
DT_SUB = 5.0e-5                # 50 us thermal substep
H_LAT_WATER = 2.26             # J/mm^3 latent heat held by a boiling ('boils') layer

PLUME_CLOSURE = {
    'model': 'diffusion', 'D_xy': 1.0, 'D_z': 2.0, 'v_drift': 0.0, 'tau_linger_s': float('inf'),
    'blast_expansion': False, 'blast_sigma_xy_mm': 0.080, 'blast_sigma_z_mm': 0.090, 'blast_z_bias_mm': 0.0,
}

# voxel size [um] and photons per epoch of each resolution preset
RESOLUTIONS = {
    'preview': {'voxel_um': 30.0, 'photons': 50_000, 'label': 'Preview (30 um voxels)'},
    'standard': {'voxel_um': 20.0, 'photons': 100_000, 'label': 'Standard (20 um voxels)'},
    'full': {'voxel_um': 15.0, 'photons': 150_000, 'label': 'Full (15 um voxels, as published)'},
}

# The published layered body (dorsal shield, subelytral air gap, viscera, ventral shield) with its
# thermal constants: k [W/(mm K)], rho_cp [J/(mm^3 K)]; 'boils' layers hold at 100 C while water
# boils off, 'dry' layers are cuticle that chars and ablates at 350 C (beetle_sim.py:60-100).
def _layer(name, label, um, comp, k, rho_cp, kind):
    return {'name': name, 'label': label, 'thickness_um': um, 'composition': comp, 'k': k, 'rho_cp': rho_cp,
            'kind': kind}


_EXO = {'chitin': 0.403, 'protein': 0.33, 'water': 0.18, 'melanin': 0.075, 'ommochrome': 0.012}
_ENDO = {'water': 0.42, 'chitin': 0.33, 'protein': 0.25}
_FAT = {'lipid': 0.50, 'water': 0.38, 'protein': 0.12}
DEFAULT_LAYERS = [
    _layer('epicuticle_wax', 'Epicuticle wax', 15.0, {'lipid': 0.85, 'protein': 0.15}, 0.22e-3, 1.98e-3, 'dry'),
    _layer('exocuticle_sclerotised', 'Dorsal exocuticle', 60.0, _EXO, 0.28e-3, 2.40e-3, 'dry'),
    _layer('endocuticle', 'Dorsal endocuticle', 90.0, _ENDO, 0.35e-3, 2.50e-3, 'dry'),
    _layer('subelytral_air_gap', 'Subelytral air gap', 300.0, {'air': 1.0}, K_AIR, RHO_CP_AIR, 'air'),
    _layer('epidermis', 'Epidermis', 15.0, {'water': 0.70, 'protein': 0.22, 'lipid': 0.08}, 0.48e-3, 3.50e-3, 'boils'),
    _layer('fat_body', 'Fat body', 300.0, _FAT, 0.32e-3, 2.80e-3, 'boils'),
    _layer('hemolymph', 'Hemolymph', 255.0, {'water': 0.93, 'protein': 0.07}, 0.58e-3, 3.89e-3, 'boils'),
    _layer('muscle', 'Muscle', 1020.0, {'water': 0.76, 'protein': 0.21, 'lipid': 0.03}, 0.50e-3, 3.65e-3, 'boils'),
    _layer('fat_body', 'Ventral fat body', 300.0, _FAT, 0.32e-3, 2.80e-3, 'boils'),
    _layer('endocuticle', 'Ventral endocuticle', 45.0, _ENDO, 0.35e-3, 2.50e-3, 'dry'),
    _layer('exocuticle_sclerotised', 'Ventral exocuticle + wax', 45.0,
           {'chitin': 0.43, 'protein': 0.352, 'water': 0.18, 'melanin': 0.03, 'ommochrome': 0.008}, 0.28e-3, 2.40e-3,
           'dry'),
]
DEFAULT_LASER = {
    'wavelength_nm': 532.0, 'power_w': 40.0, 'spot_dia_mm': 0.5,
    'theta_deg': float(math.degrees(math.atan(1.0 / 2.445))),   # 22.2 deg: crosses the body mid-plane
    'pulse_ms': 200.0, 'duration_ms': 1000.0, 'plume': True, 'resolution': 'full',
}


def default_setup():
    """The editable defaults the UI starts from (beetle_sim.py:103-108)."""
    return {'layers': [dict(l, composition=dict(l['composition'])) for l in DEFAULT_LAYERS],
            'laser': dict(DEFAULT_LASER), 'resolutions': {k: v['label'] for k, v in RESOLUTIONS.items()}}


# components eval_single_layer accepts (others are dropped before normalising the composition)
_COMPONENTS = ('water', 'chitin', 'protein', 'lipid', 'melanin', 'ommochrome', 'plant_pigment', 'hemocyanin',
               'aragonite', 'conchiolin', 'mucin', 'hemoglobin', 'air')
_ALIASES = {'matrix': 'chitin', 'chlorophyll': 'plant_pigment', 'conchiolin_matrix': 'conchiolin',
            'calcite': 'aragonite', 'blood': 'protein', 'oxyhemoglobin': 'protein'}


def _norm_composition(raw: dict) -> dict:
    comp = {}
    for k, v in raw.items():
        k = _ALIASES.get(k, k)
        if k in _COMPONENTS:
            comp[k] = comp.get(k, 0.0) + max(0.0, float(v))
    tot = sum(comp.values())
    return {k: v / tot for k, v in comp.items()} if tot > 0 else {'water': 1.0}


def fallback_layer_optics(layer: dict, wavelength_nm: float) -> dict:
    """mu_a, mu_s [1/mm], g, n of one layer by eval_single_layer's rule without the tissue-optics
    package (tissue_stack.py:130-172), rounded as it rounds them (:180-186)."""
    name = layer.get('name', 'custom_layer')
    comp = _norm_composition(layer.get('composition', {'water': 0.70, 'protein': 0.30}))
    a_prime = float(layer.get('a_prime', 40.0))
    f_ray = float(layer.get('f_rayleigh', 0.20))
    b_mie = float(layer.get('b_mie', 1.1))
    g500 = float(layer.get('g500', 0.90))
    if comp.get('air', 0.0) >= 0.99 or name == 'subelytral_air_gap' or 'air' in name:
        mu_a = mu_s = mu_sp = g = 0.0
        n = 1.00029
    else:
        wl = float(wavelength_nm)
        mu_a = (0.1812 * (wl / 450.0) ** (-3.0) + comp.get('melanin', 0.0) * 51.5 * (wl / 500.0) ** (-3.48)
                + comp.get('water', 0.0) * 0.00092)
        mu_sp = max(1e-4, a_prime * 0.1 * (f_ray * (wl / 500.0) ** (-4.0) + (1.0 - f_ray) * (wl / 500.0) ** (-b_mie)))
        g = min(0.99, g500)
        mu_s = mu_sp / max(1.0 - g, 0.01)
        w = comp.get('water', 0.0)
        n = 1.33 * w + 1.55 * (1.0 - w)
    if mu_a > 1e-5 and mu_sp > 1e-5:
        delta = 1.0 / math.sqrt(3.0 * mu_a * (mu_a + mu_sp))   # diffusion penetration depth [mm]
    elif mu_a > 1e-5:
        delta = 1.0 / mu_a
    else:
        delta = 999.0
    return {'mu_a': round(mu_a, 4), 'mu_s': round(mu_s, 3), 'mu_s_prime': round(mu_sp, 3), 'g': round(g, 3),
            'n': round(n, 3), 'penetration_depth_mm': round(delta, 3)}


def evaluate_layers(layers, wavelength_nm, eval_layer=fallback_layer_optics):
    """Optics of each layer at the wavelength with its depth range [um] (beetle_sim.py:111-122)."""
    out = []
    z = 0.0
    for lay in layers:
        e = eval_layer(lay, float(wavelength_nm))
        th = float(lay['thickness_um'])
        out.append({'mu_a': e['mu_a'], 'mu_s': e['mu_s'], 'mu_s_prime': e['mu_s_prime'], 'g': e['g'], 'n': e['n'],
                    'penetration_depth_mm': e['penetration_depth_mm'], 'z_start_um': round(z, 1),
                    'z_end_um': round(z + th, 1)})
        z += th
    return out


def build_model(layers, wavelength_nm, voxel_um, eval_layer=fallback_layer_optics):
    """Voxelise the layer stack (beetle_sim.py:133-180): arrays and per-layer slice ranges."""
    d = voxel_um / 1000.0
    nx = ny = int(round(LX / d))
    nz_air = int(round(AIR_TOP_UM / voxel_um))
    slices = [max(1, int(round(float(l['thickness_um']) / voxel_um))) for l in layers]
    nz = nz_air + sum(slices)
    shape = (nx, ny, nz)
    # per-slice property columns, broadcast over (x, y) at the end
    col = {k: np.full(nz, v, dtype=np.float64) for k, v in (('mu_a', 0.0), ('mu_s', 0.0), ('g', 0.0), ('n', 1.0),
                                                           ('k', K_AIR), ('rho_cp', RHO_CP_AIR), ('h_lat', 1e12))}
    dry_col = np.zeros(nz, bool)
    air_col = np.zeros(nz, bool)
    air_col[:nz_air] = True
    ranges = []
    k0 = nz_air
    for lay, ns in zip(layers, slices):
        k1 = k0 + ns
        ev = eval_layer(lay, float(wavelength_nm))
        kind = lay.get('kind', 'boils')
        for key in ('mu_a', 'mu_s', 'g', 'n'):
            col[key][k0:k1] = ev[key]
        col['k'][k0:k1] = float(lay['k'])
        col['rho_cp'][k0:k1] = float(lay['rho_cp'])
        col['h_lat'][k0:k1] = {'boils': H_LAT_WATER, 'dry': 0.0, 'air': 1e12}[kind]
        dry_col[k0:k1] = kind == 'dry'
        air_col[k0:k1] = kind == 'air'
        ranges.append((k0, k1, kind, lay.get('name', '')))
        k0 = k1
    full = lambda c: np.broadcast_to(c, shape).copy()
    optical = {k: full(col[k]) for k in ('mu_a', 'mu_s', 'g', 'n')}
    ablated0 = np.zeros(shape, bool)
    ablated0[:, :, :nz_air] = True
    return {
        'shape': shape, 'nz_air': nz_air, 'dz': d, 'ranges': ranges, 'is_air': full(air_col),
        'optical': optical, 'k_grid': full(col['k']), 'rho_cp_grid': full(col['rho_cp']),
        'h_lat_grid': full(col['h_lat']), 'dry_mask': full(dry_col), 'initial_ablated': ablated0,
        'dry_state': {**{k: v.copy() for k, v in optical.items()}, 'k': full(col['k']),
                      'rho_cp': full(col['rho_cp']), 't_remove': T_ABL_CUTICLE},
    }


def layer_regions(ranges, nz_air):
    """Slice bands the frames summarise (the bookkeeping of beetle_sim.py:183-198): the first air layer
    (the air gap), the core (the hemolymph layer, else the middle one of the boiling soft layers,
    else the middle layer), the ventral shell (every slice below the last boiling layer, or the last
    layer when a boiling layer is last) and the dorsal surface slice. `ranges` holds
    (k0, k1, kind, name) per layer, top to bottom."""
    span = lambda r: (r[0], r[1])
    gap = next((span(r) for r in ranges if r[2] == 'air'), None)
    boiling = [i for i, r in enumerate(ranges) if r[2] == 'boils']
    first_of = {}
    for i, r in enumerate(ranges):
        first_of.setdefault(r[3], i)
    if 'hemolymph' in first_of:
        core = first_of['hemolymph']
    elif boiling:
        core = boiling[len(boiling) // 2]
    else:
        core = len(ranges) // 2
    last = len(ranges) - 1
    ventral = (ranges[boiling[-1]][1], ranges[last][1]) if boiling and boiling[-1] < last else span(ranges[last])
    return {'air_gap': gap, 'core': span(ranges[core]), 'ventral': ventral, 'surface': nz_air}


def b64_slice(arr, dtype) -> str:
    """A 2-D slice as base64 of its C-ordered bytes in `dtype` (the frame payload the UI decodes)."""
    return base64.b64encode(memoryview(np.require(arr, dtype=dtype, requirements='C'))).decode('ascii')


def decimation(n: int, cap: int = 120) -> int:
    """Sampling step along an axis of n voxels that keeps at most `cap` samples in a frame."""
    return max(1, -(-n // cap))


def aim_beam(theta_deg: float, body_mm: float, air_mm: float):
    """Beam centre on the grid's top face for which the incident axis, tilted by theta in x, passes
    the lateral centre half-way down the body (below `air_mm` of air above the dorsal surface)."""
    return LX / 2.0 - math.tan(math.radians(theta_deg)) * (air_mm + 0.5 * body_mm), LY / 2.0


def _setup_payload(geo, reg, xs, zs_um, voxel_um, photons, laser_echo):
    """The 'setup' event of beetle_sim.run: sampled axes, grid, reference lines and layer table."""
    d, nz_air = geo['dz'], geo['nz_air']
    depth_um = lambda k: round((k - nz_air) * d * 1000.0, 1)
    gap = reg['air_gap']
    nx, ny, nz = geo['shape']
    return {
        'nx': len(xs), 'nz': len(zs_um),
        'x_mm': [round(v, 4) for v in xs], 'z_um': [round(v, 2) for v in zs_um],
        'grid': f'{nx}x{ny}x{nz}', 'voxel_um': voxel_um, 'photons': photons,
        'lines_um': {'surface': 0.0, 'air_gap_start': depth_um(gap[0]) if gap else None,
                     'air_gap_end': depth_um(gap[1]) if gap else None, 'ventral_shell': depth_um(reg['ventral'][0])},
        'layers': [{'name': r[3], 'kind': r[2], 'z_start_um': depth_um(r[0]), 'z_end_um': depth_um(r[1])}
                   for r in geo['ranges']],
        'laser': laser_echo,
    }


def run(layers, laser, frame_ms_active=2.0, frame_ms_cooling=10.0, eval_layer=fallback_layer_optics, device=None):
    """Generator of events: one 'setup', then 'frame' events, then 'done' (beetle_sim.py:201-313)."""
    res = RESOLUTIONS.get(laser.get('resolution', 'full'), RESOLUTIONS['full'])
    voxel_um = res['voxel_um']
    wl = float(laser['wavelength_nm'])
    power = float(laser['power_w'])
    spot = float(laser['spot_dia_mm'])
    theta = float(laser['theta_deg'])
    pulse_s = float(laser['pulse_ms']) / 1000.0
    total_s = float(laser['duration_ms']) / 1000.0
    photons = int(laser.get('photons') or res['photons'])
    plume_on = bool(laser.get('plume', True))

    geo = build_model(layers, wl, voxel_um, eval_layer)
    nx, ny, nz = geo['shape']
    d = geo['dz']
    nz_air = geo['nz_air']
    l_body = (nz - nz_air) * d
    reg = layer_regions(geo['ranges'], nz_air)
    beam_center = aim_beam(theta, l_body, nz_air * d)

    engine = CoupledAblationEngine(
        optical_props=geo['optical'], k_grid=geo['k_grid'], rho_cp_grid=geo['rho_cp_grid'],
        h_lat_grid=geo['h_lat_grid'], Lx=LX, Ly=LY, Lz=nz * d, power=power, spot_dia=spot, t_abl=T_BOIL,
        t_ambient=T_AMBIENT, dt_epoch=DT_EPOCH, dt_sub=DT_SUB, n_photons=photons, h_eff=H_EFF,
        beam_center=beam_center, beam_profile='gaussian', theta_inc_deg=theta, phi_inc_deg=0.0,
        dry_state=geo['dry_state'], char_state=CHAR_STATE, plume_closure=PLUME_CLOSURE if plume_on else None,
        initial_dry_mask=geo['dry_mask'], initial_ablated_mask=geo['initial_ablated'],
        air_gap_range=reg['air_gap'], wavelength_nm=wl, device=device)

    mid_y = ny // 2
    sx, sz = decimation(nx), decimation(nz)
    grid_x = (np.arange(nx) + 0.5) * d - LX / 2.0
    grid_z = ((np.arange(nz) + 0.5) - nz_air) * d * 1000.0      # um, 0 = dorsal surface
    tissue = ~geo['is_air'][::sx, mid_y, ::sz]
    n_tissue = max(1, int(np.sum(tissue)))
    c0, c1 = reg['core']
    v0, v1 = reg['ventral']
    rec = Recorder(engine, y=mid_y, k_surface=nz_air, bands=((nz_air, nz_air), (c0, c1), (v0, v1)), ring=1)
    echo = {'wavelength_nm': wl, 'power_w': power, 'spot_dia_mm': spot, 'theta_deg': theta,
            'pulse_ms': pulse_s * 1000.0, 'duration_ms': total_s * 1000.0, 'plume': plume_on}
    yield {'event': 'setup', 'data': _setup_payload(geo, reg, grid_x[::sx], grid_z[::sz], voxel_um, photons, echo)}

    n_epochs = int(round(total_s / DT_EPOCH))
    e_inc = e_abs = e_refl = e_trans = 0.0
    last_frame_t = -1e9
    t0 = time.time()
    for ep in range(n_epochs):
        on = ep * DT_EPOCH < pulse_s
        engine.power = power if on else 0.0
        engine._enqueue(0)
        t_ms = (ep + 1) * DT_EPOCH * 1000.0
        if on:
            info = engine._diag(None)
            led = info['ledger']
            launched = max(float(led[_lib.LEDGER_LAUNCHED]), 1.0)
            e = power * DT_EPOCH
            e_inc += e
            e_abs += e * float(info['absorbed_frac'])
            e_refl += e * float(led[_lib.LEDGER_SPECULAR] + led[_lib.LEDGER_DIFFUSE]) / launched
            e_trans += e * float(led[_lib.LEDGER_TRANSMITTED]) / launched
            t_ms = engine.t * 1000.0
        step_ms = frame_ms_active if on else frame_ms_cooling
        if t_ms - last_frame_t + 1e-6 < step_ms and ep != n_epochs - 1:
            continue
        last_frame_t = t_ms
        rec.record()
        rec.finish()                      # one slot: waits for this frame's record only
        row = rec.rows.pop(rec.n - 1)
        T, Q, plume, phase = row['T'], row['Q'], row['plume'], row['phase']
        t_ms = row['time_s'] * 1000.0
        # the core and ventral bands are tissue: phase 3 there means ablated
        core = T[:, c0:c1][phase[:, c0:c1] != 3]
        ven = T[:, v0:v1][phase[:, v0:v1] != 3]
        ph_s = phase[::sx, ::sz]
        elapsed = time.time() - t0
        yield {'event': 'frame', 'data': {
            't_ms': round(t_ms, 2), 'laser_on': bool(on), 'progress': round((ep + 1) / n_epochs, 4),
            'eta_s': round(elapsed / (ep + 1) * (n_epochs - ep - 1), 1),
            'Q': b64_slice(np.maximum(Q[::sx, ::sz], 1e-4).T, '<f4'), 'T': b64_slice(T[::sx, ::sz].T, '<f4'),
            'plume': b64_slice(plume[::sx, ::sz].T, '<f4'), 'phase': b64_slice(ph_s.T, 'u1'),
            'transmission_pct': round(100.0 * math.exp(-float(row['plume_tau'])), 2),
            'core_peak': round(float(core.max()) if core.size else T_AMBIENT, 2),
            'core_mean': round(float(core.mean()) if core.size else T_AMBIENT, 2),
            'ventral_peak': round(float(ven.max()) if ven.size else T_AMBIENT, 2),
            'ventral_mean': round(float(ven.mean()) if ven.size else T_AMBIENT, 2),
            'ablated_pct': round(100.0 * float(np.sum((ph_s == 3) & tissue)) / n_tissue, 2),
            'boiled_pct': round(100.0 * float(np.sum((ph_s == 2) & tissue)) / n_tissue, 2),
            'depth_um': round(row['depth_voxels'] * d * 1000.0, 1),
            'energy_j': {'incident': round(e_inc, 3), 'absorbed': round(e_abs, 3),
                         'reflected': round(e_refl, 3), 'transmitted': round(e_trans, 3)},
        }}
    yield {'event': 'done', 'data': {'elapsed_s': round(time.time() - t0, 1)}}
