"""Fused ablation substep on the GPU -- drop-in for MetalAblationContext.

Mirrors simulation/metal_ablation_solver.py:285-455 (constructor, set_state,
advance_substeps, get_state, get_plume). One substep = bioheat stencil + latent-heat plateau
+ Arrhenius damage + char kinetics (bd_ablation_advance) and, when a plume is configured,
plume transport in the void domain (bd_plume_advance). The plume does not feed back into the
thermal fields inside a substep (metal_ablation_solver.py:193-240 only reads plume buffers), so
it runs as its own kernel sequence over the same substeps.

Semantic switches (defaults reproduce the reference CPU solvers, the parity reference):
  bc:               'series' (voxel_thermal_3d.py:97,105) or 'metal' (metal_ablation_solver.py:141,150)
  plume_dt_policy:  'as_given' (plume.py:79), 'metal' (dt clamp, metal_ablation_solver.py:235-237)
                    or 'subcycle' (stable sub-steps of dt/n_sub)
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._device import is_gpu_available, require_device, to_dev

is_metal_available = is_gpu_available

_BC = {'series': _lib.BC_SERIES, 'cpu': _lib.BC_SERIES, 'metal': _lib.BC_METAL}
_PLUME_POLICY = {'as_given': _lib.PLUME_DT_AS_GIVEN, 'cpu': _lib.PLUME_DT_AS_GIVEN,
                 'metal': _lib.PLUME_DT_METAL, 'subcycle': _lib.PLUME_DT_SUBCYCLE}


def plume_params_struct(shape, dx, dy, dz, dt, D_xy, D_z, vz, tau_linger, policy='as_given', n_sub=0):
    p = _lib.PlumeParams()
    p.nx, p.ny, p.nz = (int(v) for v in shape)
    if policy not in _PLUME_POLICY:
        raise ValueError(f"plume_dt_policy must be one of {sorted(_PLUME_POLICY)}, got {policy!r}")
    p.dt_policy = _PLUME_POLICY[policy]
    p.dx, p.dy, p.dz, p.dt = float(dx), float(dy), float(dz), float(dt)
    p.D_xy, p.D_z, p.vz = float(D_xy), float(D_z), float(vz)
    tau = float(tau_linger)
    p.tau_linger = tau if (tau > 0.0 and np.isfinite(tau)) else 0.0
    p.n_sub = int(n_sub)
    return p


def plume_steps_per_substep(p: _lib.PlumeParams):
    n = ctypes.c_int(0)
    dt = ctypes.c_float(0.0)
    _lib.call("bd_plume_steps_per_substep", ctypes.byref(p), ctypes.byref(n), ctypes.byref(dt))
    return int(n.value), float(dt.value)


class GpuAblationContext:
    """Device-resident coupled ablation state (constructor of metal_ablation_solver.py:290-302)."""

    def __init__(self, Nx, Ny, Nz, dx, dy, dz, dt_sub, h_eff, t_ambient, t_abl, t_void, arrhenius=None,
                 char_params=None, plume_params=None, bc='series', plume_dt_policy='as_given', device=None):
        self.dev = require_device(device)
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self.dt = float(dt_sub)
        self.h_eff, self.t_ambient = float(h_eff), float(t_ambient)
        self.t_abl, self.t_void = float(t_abl), float(t_void)
        if bc not in _BC:
            raise ValueError(f"bc must be 'series' or 'metal', got {bc!r}")
        self.bc = _BC[bc]
        self.has_arrhenius = arrhenius is not None
        self.arr_A = float(arrhenius[0]) if arrhenius is not None else 0.0
        self.arr_Ea_over_R = float(arrhenius[1]) if arrhenius is not None else 0.0
        self.has_char = char_params is not None
        self.char_A = float(char_params[0]) if char_params is not None else 0.0
        self.char_Ea_over_R = float(char_params[1]) if char_params is not None else 0.0
        self.has_plume = plume_params is not None
        if self.has_plume:
            # key fallbacks of metal_ablation_solver.py:321-328
            d_fb = float(plume_params.get('D', plume_params.get('D_plume', 0.5)))
            self.plume_D_xy = float(plume_params.get('D_xy', d_fb))
            self.plume_D_z = float(plume_params.get('D_z', d_fb))
            self.plume_vz = float(plume_params.get('vz', plume_params.get('v_drift', 15.0)))
            self.plume_tau = float(plume_params.get('tau_linger', 0.0))
        else:
            self.plume_D_xy = self.plume_D_z = self.plume_vz = self.plume_tau = 0.0
        self.plume_dt_policy = plume_dt_policy
        shape = (self.Nx, self.Ny, self.Nz)
        z = lambda dt=torch.float32: torch.zeros(shape, device=self.dev, dtype=dt)
        self.T_a, self.T_b = z(), z()
        self.H_acc, self.Omega, self.chi = z(), z(), z()
        self.Q, self.k, self.rho = z(), z(), z()
        self.flags = z(torch.uint8)
        self.P_a, self.P_b = z(), z()

    def set_state(self, T, H_acc, Omega, chi, dry, ablated, Q, k_grid, rho_cp_grid, plume=None, plume_void=None):
        """Upload state (metal_ablation_solver.py:381-397); plume_void defaults to `ablated`."""
        d, s = self.dev, self.T_a.shape
        self.T_a.copy_(to_dev(T, d).reshape(s))
        self.H_acc.copy_(to_dev(H_acc, d).reshape(s))
        self.Omega.copy_(to_dev(Omega, d).reshape(s))
        self.chi.copy_(to_dev(chi, d).reshape(s))
        self.Q.copy_(to_dev(Q, d).reshape(s))
        self.k.copy_(to_dev(k_grid, d).reshape(s))
        self.rho.copy_(to_dev(rho_cp_grid, d).reshape(s))
        abl = to_dev(ablated, d, torch.uint8).reshape(s)
        dry_t = to_dev(dry, d, torch.uint8).reshape(s)
        vd = to_dev(plume_void, d, torch.uint8).reshape(s) if plume_void is not None else None
        _lib.call("bd_pack_flags", _lib.ptr(abl), _lib.ptr(dry_t), _lib.ptr(vd), int(abl.numel()),
                  _lib.ptr(self.flags), _lib.stream_ptr())
        if plume is not None:
            self.P_a.copy_(to_dev(plume, d).reshape(s))

    def _abl_params(self, is_active):
        p = _lib.AblationParams()
        p.nx, p.ny, p.nz = self.Nx, self.Ny, self.Nz
        p.is_active = int(bool(is_active))
        p.dx, p.dy, p.dz, p.dt = self.dx, self.dy, self.dz, self.dt
        p.h_eff, p.t_ambient, p.t_abl, p.t_void = self.h_eff, self.t_ambient, self.t_abl, self.t_void
        p.bc_mode = self.bc
        p.has_arrhenius, p.arr_A, p.arr_Ea_over_R = int(self.has_arrhenius), self.arr_A, self.arr_Ea_over_R
        p.has_char, p.char_A, p.char_Ea_over_R = int(self.has_char), self.char_A, self.char_Ea_over_R
        p.q_scale = 1.0
        p.zero_src_in_ablated = 0
        return p

    def plume_struct(self):
        return plume_params_struct((self.Nx, self.Ny, self.Nz), self.dx, self.dy, self.dz, self.dt,
                                   self.plume_D_xy, self.plume_D_z, self.plume_vz, self.plume_tau,
                                   self.plume_dt_policy)

    def advance_substeps(self, n_substeps: int, is_active: int = 1):
        """n fused substeps (metal_ablation_solver.py:399-437)."""
        if n_substeps <= 0:
            return
        p = self._abl_params(is_active)
        with torch.cuda.device(self.dev):
            st = _lib.stream_ptr()
            _lib.call("bd_ablation_advance", ctypes.byref(p), _lib.ptr(self.T_a), _lib.ptr(self.T_b),
                      int(n_substeps), _lib.ptr(self.H_acc), _lib.ptr(self.Omega if self.has_arrhenius else None),
                      _lib.ptr(self.chi if self.has_char else None), _lib.ptr(self.flags), _lib.ptr(self.Q),
                      _lib.ptr(self.k), _lib.ptr(self.rho), st)
            if n_substeps % 2 == 1:
                self.T_a, self.T_b = self.T_b, self.T_a
            if self.has_plume:
                pp = self.plume_struct()
                in_b = ctypes.c_int(0)
                _lib.call("bd_plume_advance", ctypes.byref(pp), _lib.ptr(self.P_a), _lib.ptr(self.P_b),
                          int(n_substeps), _lib.ptr(self.flags), ctypes.byref(in_b), st)
                if in_b.value:
                    self.P_a, self.P_b = self.P_b, self.P_a

    def get_state(self):
        """(T, H_acc, Omega, chi) as float64 numpy arrays (metal_ablation_solver.py:439-446)."""
        return tuple(t.double().cpu().numpy() for t in (self.T_a, self.H_acc, self.Omega, self.chi))

    def get_plume(self, out_arr=None):
        buf = self.P_a.cpu().numpy()
        if out_arr is not None:
            out_arr[:] = buf
            return out_arr
        return buf.copy()


MetalAblationContext = GpuAblationContext
