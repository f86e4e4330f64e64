"""ORACLE -- test infrastructure only (never imported by bug_defense_b200).

CPU restatement of the reference's CPU path in FP64 (plain C in oracle/orc.c, OpenMP),
exposed with the reference's own function names and argument meaning:

  thermal3d_step_explicit     simulation/voxel_thermal_3d.py:30-112
  apply_latent_heat_plateau   simulation/voxel_thermal_3d.py:115-143
  accumulate_arrhenius        simulation/coupled_ablation.py:33-40
  accumulate_char             simulation/coupled_ablation.py:43-58
  diffuse_plume_step          simulation/plume.py:18-80
  update_phase_properties     simulation/coupled_ablation.py:77-180
  run_voxel_mc3d              simulation/voxel_mc_3d.py:425-717 (FP64, Philox RNG, seedable)

Pinned against tests/golden/ fixtures generated by running the reference itself
(tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import time
from ctypes import POINTER, Structure, c_double, c_int, c_int64, c_uint8, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liborc.so"


def build(force: bool = False) -> Path:
    """gcc -O3 -fopenmp -shared oracle/orc.c -> oracle/liborc.so"""
    src = HERE / "orc.c"
    if not force and LIB.exists() and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    tmp = str(LIB) + ".tmp"
    # x86-64-v3 (AVX2/FMA): every B200 host has it; -ffast-math matches the reference's numba
    # kernels, which are all compiled with fastmath=True
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffast-math", "-fopenmp", "-shared", "-fPIC", "-std=gnu11", "-o", tmp,
           str(src), "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


class OrcArr(Structure):
    _fields_ = [("p", c_void_p), ("len", c_int64)]


class OrcMcParams(Structure):
    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int), ("launch_axis", c_int), ("beam_profile", c_int),
        ("metal", c_int),
        ("dx", c_double), ("dy", c_double), ("dz", c_double), ("lx", c_double), ("ly", c_double), ("lz", c_double),
        ("ux0", c_double), ("uy0", c_double), ("uz0", c_double), ("cos_ph", c_double), ("sin_ph", c_double),
        ("cos_th_safe", c_double), ("xc", c_double), ("yc", c_double), ("zc", c_double), ("sigma", c_double),
        ("radius", c_double), ("n_amb", c_double), ("rmax2", c_double),
        ("n_photons", c_int64), ("offset", c_int64), ("max_events", c_int64), ("seed", c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        P = c_void_p
        L.orc_philox4x32_10.argtypes = [POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32)]
        L.orc_thermal_step.argtypes = [P, P, P, P, P, c_int, c_int, c_int, c_double, c_double, c_double,
                                       c_double, c_double, c_double, c_int, c_int]
        L.orc_plateau.argtypes = [P, P, P, P, c_double, c_int64, P, c_double]
        L.orc_arrhenius.argtypes = [P, P, P, c_double, c_double, c_double, c_int64]
        L.orc_char.argtypes = [P, P, P, P, c_double, c_double, c_double, c_int64]
        L.orc_plume_step.argtypes = [P, P, P, c_int, c_int, c_int, c_double, c_double, c_double, c_double,
                                     c_double, c_double, c_double, c_double]
        L.orc_phase_update.argtypes = [P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, POINTER(OrcArr), c_int, c_int,
                                       POINTER(OrcArr), c_double, c_int, c_int, c_int, c_double, P, c_int64]
        L.orc_mc_trace.argtypes = [POINTER(OrcMcParams), P, P, P, P, P, P, P, P, c_int]
        L.orc_max_threads.restype = c_int
        L.orc_set_threads.argtypes = [c_int]
        _lib = L
    return _lib


def _p(a):
    return c_void_p(a.ctypes.data) if a is not None else c_void_p(None)


def _f64(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous, "oracle arrays must be C-contiguous float64"
    return _p(a)


def _u8(a):
    b = np.ascontiguousarray(a).view(np.uint8) if np.asarray(a).dtype == np.bool_ else np.ascontiguousarray(a, dtype=np.uint8)
    return b


def philox4x32_10(ctr, key):
    c = (c_uint32 * 4)(*ctr)
    k = (c_uint32 * 2)(*key)
    o = (c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def thermal3d_step_explicit(T, T_new, Q, k_grid, rho_cp_grid, Nx, Ny, Nz, dx, dy, dz, dt, h_eff, t_ambient,
                            is_active, bc_mode=0):
    lib().orc_thermal_step(_f64(T), _f64(T_new), _f64(Q), _f64(k_grid), _f64(rho_cp_grid), Nx, Ny, Nz, dx, dy,
                           dz, dt, h_eff, t_ambient, int(bool(is_active)), int(bc_mode))


def apply_latent_heat_plateau(T, H_acc, rho_cp_grid, ablated, t_abl, Nx, Ny, Nz, dry, t_void):
    a, d = _u8(ablated), _u8(dry)
    lib().orc_plateau(_f64(T), _f64(H_acc), _f64(rho_cp_grid), _p(a), t_abl, Nx * Ny * Nz, _p(d), t_void)


def accumulate_arrhenius(T, Omega, ablated, A, Ea_over_R, dt, Nx, Ny, Nz):
    a = _u8(ablated)
    lib().orc_arrhenius(_f64(T), _f64(Omega), _p(a), A, Ea_over_R, dt, Nx * Ny * Nz)


def accumulate_char(T, chi, dry, ablated, A, Ea_over_R, dt, Nx, Ny, Nz):
    a, d = _u8(ablated), _u8(dry)
    lib().orc_char(_f64(T), _f64(chi), _p(d), _p(a), A, Ea_over_R, dt, Nx * Ny * Nz)


def diffuse_plume_step(C, C_new, void_mask, Nx, Ny, Nz, dx, dy, dz, dt, D_xy, D_z, vz, decay):
    v = _u8(void_mask)
    lib().orc_plume_step(_f64(C), _f64(C_new), _p(v), Nx, Ny, Nz, dx, dy, dz, dt, D_xy, D_z, vz, decay)


def plume_policy(dt, dx, dy, dz, D_xy, D_z, vz, tau_linger, policy):
    """(n_steps, dt_step, decay_step) per substep; the same rules as bd_plume_steps_per_substep."""
    idx2, idy2, idz2 = 1 / dx ** 2, 1 / dy ** 2, 1 / dz ** 2
    decays = tau_linger > 0 and math.isfinite(tau_linger)
    if policy in ('as_given', 'cpu'):
        return 1, dt, (math.exp(-dt / tau_linger) if decays else 1.0)
    if policy == 'metal':
        dr = float(np.float32(D_xy) * (np.float32(idx2) + np.float32(idy2)) + np.float32(D_z) * np.float32(idz2))
        dtp = min(dt, 0.45 / (2.0 * dr)) if dr > 1e-6 else dt
        return 1, dtp, (math.exp(-dt / tau_linger) if decays else 1.0)
    if policy == 'subcycle':
        rate = 2.0 * (D_xy * (idx2 + idy2) + D_z * idz2) + max(0.0, vz) / dz
        n = max(1, int(math.ceil(dt * rate / 0.9 - 1e-9)))
        return n, dt / n, (math.exp(-(dt / n) / tau_linger) if decays else 1.0)
    raise ValueError(policy)


def _arr(v, N):
    if np.ndim(v) == 0:
        a = np.array([float(v)], dtype=np.float64)
    else:
        a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel())
        assert a.size in (1, N)
    return a


def update_phase_properties(H_acc, h_lat, T, chi, dry, ablated, mu_a, mu_s, g, n, k_grid, rho_cp_grid, wet_mu_a,
                            wet_k, wet_rho_cp, ds, cs, cs_chi_remove, alpha_max_stable):
    """ds: dict mu_a mu_s g n k rho_cp t_remove (scalars or arrays); cs: None or dict with any of
    mu_a mu_s k rho_cp and t_remove. dry is updated in place (bool or uint8); returns to_remove (bool)."""
    N = H_acc.size
    keep = []
    dsa = (OrcArr * 7)()
    for q, key in enumerate(('mu_a', 'mu_s', 'g', 'n', 'k', 'rho_cp', 't_remove')):
        a = _arr(ds[key], N); keep.append(a)
        dsa[q] = OrcArr(a.ctypes.data, a.size)
    csa = (OrcArr * 5)()
    has = {}
    dummy = np.zeros(1); keep.append(dummy)
    for q, key in enumerate(('mu_a', 'mu_s', 'k', 'rho_cp', 't_remove')):
        if cs is not None and key in cs:
            a = _arr(cs[key], N); keep.append(a)
            csa[q] = OrcArr(a.ctypes.data, a.size)
            has[key] = 1
        else:
            csa[q] = OrcArr(dummy.ctypes.data, 1)
            has[key] = 0
    d8 = np.ascontiguousarray(dry, dtype=np.uint8)
    a8 = _u8(ablated)
    rem = np.zeros(N, dtype=np.uint8)
    lib().orc_phase_update(_f64(H_acc), _f64(h_lat), _f64(T), _f64(chi), _p(d8), _p(a8), _f64(mu_a), _f64(mu_s),
                           _f64(g), _f64(n), _f64(k_grid), _f64(rho_cp_grid), _f64(wet_mu_a), _f64(wet_k),
                           _f64(wet_rho_cp), dsa, int(cs is not None), has['mu_a'], csa, float(cs_chi_remove),
                           has['mu_s'], has['k'], has['rho_cp'], float(alpha_max_stable), _p(rem), N)
    dry[...] = d8.reshape(np.shape(dry)).astype(np.asarray(dry).dtype)
    return rem.reshape(np.shape(H_acc)).astype(bool)


BEAM = {'gaussian': 0, 'tophat': 1, 'kim_exp_disk': 2, 'kim_gauss_disk': 3}


def run_voxel_mc3d(power=1.0, pulse_duration=0.20, n_photons=200000, spot_dia=0.50, theta_inc_deg=0.0,
                   phi_inc_deg=0.0, Lx=4.0, Ly=4.0, Lz=2.42, Nx=80, Ny=80, Nz=60, r_max=0.0, layers_config=None,
                   custom_3d_props=None, launch_axis='z', beam_center=None, beam_profile='gaussian', seed=1,
                   semantics='cpu', n_chunks=None, tally_fluence=True, max_events=10_000_000, photon_offset=0):
    """FP64 restatement of run_voxel_mc3d (voxel_mc_3d.py:425-717) with a seedable Philox RNG.
    Photon p draws from the Philox stream (seed, photon_offset + p), as the GPU tracer does."""
    dx, dy, dz = Lx / Nx, Ly / Ny, Lz / Nz
    axis = launch_axis.strip().lower()
    if custom_3d_props is not None:
        grids = [np.ascontiguousarray(custom_3d_props[k], dtype=np.float64) for k in ('mu_a', 'mu_s', 'g', 'n')]
    else:
        grids = [np.zeros((Nx, Ny, Nz)), np.zeros((Nx, Ny, Nz)), np.zeros((Nx, Ny, Nz)), np.ones((Nx, Ny, Nz))]
        if layers_config is not None:
            if axis == 'z':
                centres = np.linspace(dz / 2.0, Lz - dz / 2.0, Nz)
            else:
                centres = np.linspace(dx / 2.0, Lx - dx / 2.0, Nx)
            start = 0.0
            for lay in layers_config:
                m = (centres >= start) & (centres < lay['z_end'])
                for grid, key in zip(grids, ('mu_a', 'mu_s', 'g', 'n')):
                    if axis == 'z':
                        grid[:, :, m] = lay[key]
                    else:
                        grid[m, :, :] = lay[key]
                start = lay['z_end']
    P = OrcMcParams()
    P.nx, P.ny, P.nz = Nx, Ny, Nz
    P.launch_axis = 1 if axis == 'x' else 0
    P.beam_profile = BEAM[beam_profile]
    P.metal = 1 if semantics == 'metal' else 0
    P.dx, P.dy, P.dz, P.lx, P.ly, P.lz = dx, dy, dz, Lx, Ly, Lz
    th, ph = math.radians(theta_inc_deg), math.radians(phi_inc_deg)
    P.cos_ph, P.sin_ph = math.cos(ph), math.sin(ph)
    P.cos_th_safe = max(math.cos(th), 1e-6 if semantics == 'metal' else 0.05)
    if axis == 'z':
        P.ux0, P.uy0, P.uz0 = math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)
        P.xc, P.yc, P.zc = Lx / 2.0, Ly / 2.0, 0.0
        if beam_center is not None:
            P.xc, P.yc = float(beam_center[0]), float(beam_center[1])
    else:
        P.ux0, P.uy0, P.uz0 = math.cos(th), math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph)
        P.xc, P.yc, P.zc = 0.0, Ly / 2.0, Lz / 2.0
        if beam_center is not None:
            P.yc, P.zc = float(beam_center[0]), float(beam_center[1])
    w0 = spot_dia / 2.0
    P.sigma, P.radius = w0 / 2.0, w0
    P.n_amb = 1.0
    P.rmax2 = r_max * r_max if r_max > 0 else 0.0
    P.n_photons, P.offset, P.max_events, P.seed = int(n_photons), int(photon_offset), int(max_events), int(seed)
    nv = Nx * Ny * Nz
    if n_chunks is None:
        budget = 512 * 1024 ** 2  # MC3D_SCORING_MEMORY_BUDGET_BYTES (voxel_mc_3d.py:28, :621-625)
        n_chunks = max(1, min(max_threads(), max(1, budget // max(16 * nv, 1)), max(1, int(n_photons) // 5000)))
    A = np.zeros(nv); L = np.zeros(nv) if tally_fluence else None
    latz = np.zeros(Nz if axis == 'z' else Nx); led = np.zeros(16)
    t0 = time.perf_counter()
    lib().orc_mc_trace(ctypes.byref(P), *(_p(gr) for gr in grids), _p(A), _p(L), _p(latz), _p(led), int(n_chunks))
    elapsed = time.perf_counter() - t0
    N = float(max(n_photons, 1))
    R_spec, R_diff, T_t, Lat = led[1] / N, led[2] / N, led[3] / N, led[4] / N
    A_tot = (led[5] + led[6]) / N
    vol = dx * dy * dz
    A3 = A.reshape(Nx, Ny, Nz)
    return {
        'A_3d': A3 / N, 'Q_3d': A3 / N * (power / vol),
        'Phi_3d': (L.reshape(Nx, Ny, Nz) / N / vol) if L is not None else None,
        'lateral_escape_z': latz / N, 'ledger': led,
        'spectro_raw': {'R_spec': R_spec, 'R_diff': R_diff, 'Absorption': A_tot, 'Transmission': T_t,
                        'Lateral_loss': Lat},
        'energy_closure': R_spec + R_diff + A_tot + T_t + Lat,
        'elapsed_seconds': elapsed, 'photons_per_sec': n_photons / max(elapsed, 1e-9),
        'n_chunks': n_chunks, 'engine': 'oracle',
    }
