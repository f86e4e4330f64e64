"""Voxel Monte Carlo photon transport on the GPU -- drop-in for the reference MC API.

Mirrors simulation/voxel_mc_3d.py:425-717 (`run_voxel_mc3d`) and
simulation/voxel_mc_metal.py:388-586 (`run_voxel_mc_metal`): same keyword arguments, same
returned keys (A_3d, Q_3d, Phi_3d, spectro, spectro_raw, energy_closure, ...), plus an exact
FP64 energy `ledger`. The photon kernel is bd_mc_trace in libbugdef.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from . import _lib
from ._device import is_gpu_available, require_device, to_dev

# Reference constants (simulation/voxel_mc_3d.py:28-30, voxel_mc_metal.py:407)
MC3D_ENERGY_CLOSURE_TOL = 0.01
MAX_EVENTS_CPU_SEMANTICS = 10_000_000
MAX_EVENTS_METAL_SEMANTICS = 50_000
# photons per kernel launch: beyond this the FP32 tally is folded into an FP64 map
PHOTON_BATCH = 1 << 22

is_metal_available = is_gpu_available  # drop-in name used by the reference callers

_CTX = {}


class McContext:
    """Owns a bd_mc context (photon queue + FP64 ledger partials) on one device."""

    def __init__(self, dev: torch.device):
        self.dev = dev
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            _lib.call("bd_mc_create", ctypes.byref(h))
        self.handle = h

    def __del__(self):
        try:
            if self.handle:
                _lib.load().bd_mc_destroy(self.handle)
        except Exception:
            pass


def mc_context(dev: torch.device) -> McContext:
    ctx = _CTX.get(dev.index)
    if ctx is None:
        ctx = McContext(dev)
        _CTX[dev.index] = ctx
    return ctx


def make_params(*, Nx, Ny, Nz, Lx, Ly, Lz, n_photons, spot_dia=0.5, theta_inc_deg=0.0, phi_inc_deg=0.0,
                beam_center=None, beam_profile='gaussian', launch_axis='z', n_ambient=1.0, r_max=0.0,
                seed=0, max_events=None, semantics='cpu', tally_fluence=True, photon_offset=0) -> _lib.McParams:
    """Launch parameters exactly as the reference derives them (voxel_mc_3d.py:599-625)."""
    sem = str(semantics).lower()
    if sem not in ('cpu', 'metal'):
        raise ValueError(f"semantics must be 'cpu' or 'metal', got {semantics!r}")
    axis = str(launch_axis).strip().lower()
    if axis not in ('z', 'x'):
        raise ValueError(f"launch_axis must be 'z' or 'x', got {launch_axis!r}")
    if beam_profile not in _lib.BEAM_PROFILES:
        raise ValueError(f"unknown beam_profile {beam_profile!r}")
    p = _lib.McParams()
    p.nx, p.ny, p.nz = int(Nx), int(Ny), int(Nz)
    p.launch_axis = 1 if axis == 'x' else 0
    dx, dy, dz = Lx / Nx, Ly / Ny, Lz / Nz
    p.dx, p.dy, p.dz = dx, dy, dz
    p.lx, p.ly, p.lz = float(Lx), float(Ly), float(Lz)
    th, ph = math.radians(theta_inc_deg), math.radians(phi_inc_deg)
    sin_th, cos_th, sin_ph, cos_ph = math.sin(th), math.cos(th), math.sin(ph), math.cos(ph)
    p.cos_ph, p.sin_ph = cos_ph, sin_ph
    # cos clamp: 0.05 on the CPU (voxel_mc_3d.py:386), 1e-6 on Metal (voxel_mc_metal.py:432)
    p.cos_th_safe = max(cos_th, 1e-6 if sem == 'metal' else 0.05)
    if axis == 'z':
        p.init_ux, p.init_uy, p.init_uz = sin_th * cos_ph, sin_th * sin_ph, cos_th
        xc, yc, zc = Lx / 2.0, Ly / 2.0, 0.0
        if beam_center is not None:
            xc, yc = float(beam_center[0]), float(beam_center[1])
    else:
        p.init_ux, p.init_uy, p.init_uz = cos_th, sin_th * cos_ph, sin_th * sin_ph
        xc, yc, zc = 0.0, Ly / 2.0, Lz / 2.0
        if beam_center is not None:
            yc, zc = float(beam_center[0]), float(beam_center[1])
    p.x_center, p.y_center, p.z_center = xc, yc, zc
    w0 = spot_dia / 2.0
    p.sigma_axis = w0 / 2.0
    p.beam_radius = w0
    p.beam_profile = _lib.BEAM_PROFILES[beam_profile]
    p.n_ambient = float(n_ambient)
    p.r_max_sq = float(r_max * r_max) if r_max > 0.0 else 0.0
    opts = 0
    if tally_fluence:
        opts |= _lib.MC_TALLY_FLUENCE
    if sem == 'metal':
        opts |= _lib.MC_METAL_SEMANTICS
    p.options = opts
    p.n_photons = int(n_photons)
    p.photon_offset = int(photon_offset)
    if max_events is None:
        max_events = MAX_EVENTS_METAL_SEMANTICS if sem == 'metal' else MAX_EVENTS_CPU_SEMANTICS
    p.max_events = int(max_events)
    p.seed = int(seed) & ((1 << 64) - 1)
    return p


def layers_to_grids(layers_config, Nx, Ny, Nz, Lx, Ly, Lz, launch_axis='z'):
    """Planar layer stack -> property grids by the cell-centre rule (voxel_mc_3d.py:517-548)."""
    mu_a = np.zeros((Nx, Ny, Nz)); mu_s = np.zeros((Nx, Ny, Nz))
    g = np.zeros((Nx, Ny, Nz)); n = np.ones((Nx, Ny, Nz))
    if layers_config is None:
        return mu_a, mu_s, g, n
    if str(launch_axis).strip().lower() == 'x':
        dx = Lx / Nx
        centres = np.linspace(dx / 2.0, Lx - dx / 2.0, Nx)
        start = 0.0
        for lay in layers_config:
            m = (centres >= start) & (centres < lay['z_end'])
            if np.any(m):
                mu_a[m, :, :] = lay['mu_a']; mu_s[m, :, :] = lay['mu_s']
                g[m, :, :] = lay['g']; n[m, :, :] = lay['n']
            start = lay['z_end']
    else:
        dz = Lz / Nz
        centres = np.linspace(dz / 2.0, Lz - dz / 2.0, Nz)
        start = 0.0
        for lay in layers_config:
            m = (centres >= start) & (centres < lay['z_end'])
            if np.any(m):
                mu_a[:, :, m] = lay['mu_a']; mu_s[:, :, m] = lay['mu_s']
                g[:, :, m] = lay['g']; n[:, :, m] = lay['n']
            start = lay['z_end']
    return mu_a, mu_s, g, n


def pack_props(mu_a, mu_s, g, n, dev, out=None, plume_mu_ext=None, flags=None, ratio_a=0.0, ratio_s=0.0,
               g_plume=0.8, stream=None) -> torch.Tensor:
    """float4 {mu_t, mu_a/mu_t, g, n} per voxel on the device (bd_mc_pack_props)."""
    ts = [to_dev(a, dev) for a in (mu_a, mu_s, g, n)]
    nv = ts[0].numel()
    if out is None:
        out = torch.empty(nv * 4, device=dev, dtype=torch.float32)
    _lib.call("bd_mc_pack_props", *(_lib.ptr(t) for t in ts), _lib.ptr(plume_mu_ext), _lib.ptr(flags),
              float(ratio_a), float(ratio_s), float(g_plume), int(nv), _lib.ptr(out), _lib.stream_ptr(stream))
    return out


def trace(params: _lib.McParams, props: torch.Tensor, A: torch.Tensor, L=None, lat_depth=None, ledger=None,
          flags=None, stream=None) -> torch.Tensor:
    """Enqueue one bd_mc_trace launch; returns the (device) FP64 ledger tensor."""
    dev = props.device
    if ledger is None:
        ledger = torch.zeros(_lib.LEDGER_LEN, device=dev, dtype=torch.float64)
    ctx = mc_context(dev)
    _lib.call("bd_mc_trace", ctx.handle, ctypes.byref(params), _lib.ptr(props), _lib.ptr(flags), _lib.ptr(A),
              _lib.ptr(L), _lib.ptr(lat_depth), _lib.ptr(ledger), _lib.stream_ptr(stream))
    return ledger


def run_voxel_mc_gpu(power: float = 1.0, pulse_duration: float = 0.20, n_photons: int = 100_000,
                     Lx: float = 2.0, Ly: float = 2.0, Lz: float = 1.0, Nx: int = 40, Ny: int = 40, Nz: int = 50,
                     custom_3d_props: dict = None, layers_config: list = None, theta_inc_deg: float = 0.0,
                     phi_inc_deg: float = 0.0, spot_dia: float = 0.50, beam_center: tuple = None,
                     n_ambient: float = 1.0, r_max: float = 0.0, base_seed: int = None, max_steps: int = None,
                     beam_profile: str = 'gaussian', launch_axis: str = 'z', semantics: str = 'cpu',
                     tally_fluence: bool = True, device=None) -> dict:
    """GPU voxel MC with the signature of run_voxel_mc_metal (voxel_mc_metal.py:388-408).

    `max_steps` caps events per photon (default 1e7 with CPU semantics, 50,000 with Metal
    semantics); weight left at the cap is reported in the ledger's TRUNCATED channel.
    """
    dev = require_device(device)
    if custom_3d_props is not None:
        mu_a, mu_s, g, n = (custom_3d_props[k] for k in ('mu_a', 'mu_s', 'g', 'n'))
    else:
        mu_a, mu_s, g, n = layers_to_grids(layers_config, Nx, Ny, Nz, Lx, Ly, Lz, launch_axis)
    if tuple(np.shape(mu_a)) != (Nx, Ny, Nz):
        raise ValueError(f"property grids have shape {np.shape(mu_a)}, expected {(Nx, Ny, Nz)}")
    seed = int(base_seed) if base_seed is not None else int(np.random.randint(1, 2 ** 31 - 1))
    nvox = Nx * Ny * Nz
    axis = str(launch_axis).strip().lower()
    n_depth = Nz if axis == 'z' else Nx
    with torch.cuda.device(dev):
        props = pack_props(mu_a, mu_s, g, n, dev)
        A = torch.zeros(nvox, device=dev, dtype=torch.float32)
        L = torch.zeros(nvox, device=dev, dtype=torch.float32) if tally_fluence else None
        latz = torch.zeros(n_depth, device=dev, dtype=torch.float64)
        ledger_sum = torch.zeros(_lib.LEDGER_LEN, device=dev, dtype=torch.float64)
        multi = n_photons > PHOTON_BATCH
        A64 = torch.zeros(nvox, device=dev, dtype=torch.float64) if multi else None
        L64 = torch.zeros(nvox, device=dev, dtype=torch.float64) if (multi and tally_fluence) else None
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        done = 0
        while done < n_photons or (n_photons == 0 and done == 0):
            nb = min(PHOTON_BATCH, n_photons - done)
            p = make_params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=Lz, n_photons=nb, spot_dia=spot_dia,
                            theta_inc_deg=theta_inc_deg, phi_inc_deg=phi_inc_deg, beam_center=beam_center,
                            beam_profile=beam_profile, launch_axis=launch_axis, n_ambient=n_ambient, r_max=r_max,
                            seed=seed, max_events=max_steps, semantics=semantics, tally_fluence=tally_fluence,
                            photon_offset=done)
            led = trace(p, props, A, L, latz)
            ledger_sum += led
            if multi:
                _lib.call("bd_fold_f32_to_f64", _lib.ptr(A), _lib.ptr(A64), nvox, _lib.stream_ptr())
                if L is not None:
                    _lib.call("bd_fold_f32_to_f64", _lib.ptr(L), _lib.ptr(L64), nvox, _lib.stream_ptr())
            done += nb
            if n_photons == 0:
                break
        _lib.call("bd_stream_sync", _lib.stream_ptr())
        elapsed = max(time.perf_counter() - t0, 1e-6)
        A_raw = (A64 if multi else A.double()).reshape(Nx, Ny, Nz).cpu().numpy()
        if tally_fluence:
            L_raw = (L64 if multi else L.double()).reshape(Nx, Ny, Nz).cpu().numpy()
        else:
            L_raw = np.zeros((Nx, Ny, Nz))
        led = ledger_sum.cpu().numpy()
        lat_z = latz.cpu().numpy()
    return _results(power, n_photons, Lx, Ly, Lz, Nx, Ny, Nz, A_raw, L_raw, led, lat_z, elapsed, axis, seed)


def _results(power, n_photons, Lx, Ly, Lz, Nx, Ny, Nz, A_raw, L_raw, led, lat_z, elapsed, axis, seed):
    """Normalisation and result dict of voxel_mc_3d.py:657-717."""
    dx, dy, dz = Lx / Nx, Ly / Ny, Lz / Nz
    N = float(max(n_photons, 1))
    R_spec = led[_lib.LEDGER_SPECULAR] / N
    R_diff = led[_lib.LEDGER_DIFFUSE] / N
    T_tot = led[_lib.LEDGER_TRANSMITTED] / N
    Lat = led[_lib.LEDGER_LATERAL] / N
    A_tot = (led[_lib.LEDGER_ABSORBED] + led[_lib.LEDGER_ABSORBED_VOID]) / N
    R_tot = R_spec + R_diff
    closure = R_tot + A_tot + T_tot + Lat
    exact = (R_tot + A_tot + T_tot + Lat + (led[_lib.LEDGER_TRUNCATED] + led[_lib.LEDGER_ROULETTE_LOSS]
                                            - led[_lib.LEDGER_ROULETTE_GAIN]) / N)
    if n_photons > 0 and abs(closure - 1.0) > MC3D_ENERGY_CLOSURE_TOL:
        import warnings
        warnings.warn(f"Voxel MC energy closure {closure:.5f} deviates from 1 by more than "
                      f"{MC3D_ENERGY_CLOSURE_TOL:.3f}", RuntimeWarning)
    vol = dx * dy * dz
    return {
        'grid_x': np.linspace(dx / 2.0, Lx - dx / 2.0, Nx),
        'grid_y': np.linspace(dy / 2.0, Ly - dy / 2.0, Ny),
        'grid_z': np.linspace(dz / 2.0, Lz - dz / 2.0, Nz),
        'dx': dx, 'dy': dy, 'dz': dz, 'Nx': Nx, 'Ny': Ny, 'Nz': Nz,
        'A_3d': A_raw / N,
        'lateral_escape_z': lat_z / N,
        'Q_3d': (A_raw / N) * (power / vol),
        'Phi_3d': (L_raw / N) / vol,
        'spectro': {
            'R_spec': round(R_spec * 100.0, 2), 'R_diff': round(R_diff * 100.0, 2),
            'R_tot': round(R_tot * 100.0, 2), 'Absorption': round(A_tot * 100.0, 2),
            'Transmission': round(T_tot * 100.0, 2), 'Lateral_loss': round(Lat * 100.0, 2),
        },
        'energy_closure': float(closure),
        'ledger_closure': float(exact),
        'ledger': led.copy(),
        'spectro_raw': {'R_spec': R_spec, 'R_diff': R_diff, 'Absorption': A_tot, 'Transmission': T_tot,
                        'Lateral_loss': Lat},
        'launch_axis': axis,
        'elapsed_seconds': round(elapsed, 4),
        'photons_per_sec': int(n_photons / elapsed),
        'photon_steps': float(led[_lib.LEDGER_COLLISIONS] + led[_lib.LEDGER_CROSSINGS]),
        'seed': seed,
        'engine': 'gpu',
    }


def run_voxel_mc3d(power: float = 1.0, pulse_duration: float = 0.20, n_photons: int = 200000,
                   spot_dia: float = 0.50, theta_inc_deg: float = 0.0, phi_inc_deg: float = 0.0,
                   Lx: float = 4.0, Ly: float = 4.0, Lz: float = 2.42, Nx: int = 80, Ny: int = 80, Nz: int = 60,
                   r_max: float = 0.0, layers_config: list = None, custom_3d_props: dict = None,
                   launch_axis: str = 'z', beam_center=None, beam_profile: str = 'gaussian',
                   engine: str = 'auto', base_seed: int = None, semantics: str = 'cpu', device=None) -> dict:
    """Signature of simulation/voxel_mc_3d.py:425-445. engine 'auto' and 'gpu' run the CUDA
    kernel; this package ships no CPU engine, so engine='cpu' raises ValueError."""
    eng = str(engine).strip().lower()
    if eng not in ('auto', 'gpu', 'cpu'):
        raise ValueError(f"Unknown engine='{engine}'. Valid options: 'auto', 'gpu', 'cpu'.")
    if eng == 'cpu':
        raise ValueError("engine='cpu' is not provided by bug_defense_b200 (GPU-only build); "
                         "use engine='gpu' or 'auto'")
    return run_voxel_mc_gpu(power=power, pulse_duration=pulse_duration, n_photons=n_photons, Lx=Lx, Ly=Ly,
                            Lz=Lz, Nx=Nx, Ny=Ny, Nz=Nz, custom_3d_props=custom_3d_props,
                            layers_config=layers_config, theta_inc_deg=theta_inc_deg, phi_inc_deg=phi_inc_deg,
                            spot_dia=spot_dia, beam_center=beam_center, n_ambient=1.0, r_max=r_max,
                            base_seed=base_seed, beam_profile=beam_profile, launch_axis=launch_axis,
                            semantics=semantics, device=device)


run_voxel_mc_metal = run_voxel_mc_gpu  # drop-in name (voxel_mc_metal.py:388)
