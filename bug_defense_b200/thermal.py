"""Explicit bioheat stencil on the GPU -- drop-in for the reference thermal solvers.

Mirrors simulation/voxel_thermal_metal.py (MetalThermalContext :288-383,
run_thermal3d_substeps_metal :179-285) and simulation/voxel_thermal_3d.py
(VoxelThermalSolver3D :146-309). The stencil is bd_thermal_advance in libbugdef.so.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from ._device import is_gpu_available, require_device, to_dev

CFL_SAFETY_FACTOR = 0.40  # simulation/voxel_thermal_3d.py:27

is_metal_available = is_gpu_available


def _params(Nx, Ny, Nz, dx, dy, dz, dt, h_eff, t_ambient, is_active, bc_mode=_lib.BC_SERIES, q_scale=1.0):
    p = _lib.ThermalParams()
    p.nx, p.ny, p.nz = int(Nx), int(Ny), int(Nz)
    p.is_active = int(bool(is_active))
    p.dx, p.dy, p.dz, p.dt = float(dx), float(dy), float(dz), float(dt)
    p.h_eff, p.t_ambient = float(h_eff), float(t_ambient)
    p.bc_mode = int(bc_mode)
    p.q_scale = float(q_scale)
    return p


class GpuThermalContext:
    """Persistent device context for the 3-D transient thermal stencil.

    Same constructor and methods as MetalThermalContext (voxel_thermal_metal.py:294-383).
    get_T_view() returns a zero-copy float32 *device* tensor view of the current field.
    """

    def __init__(self, Nx, Ny, Nz, dx, dy, dz, dt, k_grid, rho_cp_grid, h_eff=0.0, t_ambient=20.0, device=None):
        self.dev = require_device(device)
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self.dt, self.h_eff, self.t_ambient = float(dt), float(h_eff), float(t_ambient)
        shape = (self.Nx, self.Ny, self.Nz)
        self.k = to_dev(k_grid, self.dev).reshape(shape)
        self.rho = to_dev(rho_cp_grid, self.dev).reshape(shape)
        self.T_a = torch.zeros(shape, device=self.dev, dtype=torch.float32)
        self.T_b = torch.zeros(shape, device=self.dev, dtype=torch.float32)
        self.Q = torch.zeros(shape, device=self.dev, dtype=torch.float32)

    def set_T(self, T):
        self.T_a.copy_(to_dev(T, self.dev).reshape(self.T_a.shape))

    def set_Q(self, Q):
        self.Q.copy_(to_dev(Q, self.dev).reshape(self.Q.shape))

    def advance(self, n_substeps: int, is_active: int = 1):
        if n_substeps <= 0:
            return
        p = _params(self.Nx, self.Ny, self.Nz, self.dx, self.dy, self.dz, self.dt, self.h_eff, self.t_ambient,
                    is_active)
        with torch.cuda.device(self.dev):
            _lib.call("bd_thermal_advance", ctypes.byref(p), _lib.ptr(self.T_a), _lib.ptr(self.T_b),
                      int(n_substeps), _lib.ptr(self.Q), _lib.ptr(self.k), _lib.ptr(self.rho), _lib.stream_ptr())
        if n_substeps % 2 == 1:
            self.T_a, self.T_b = self.T_b, self.T_a

    def get_T(self) -> np.ndarray:
        return self.T_a.double().cpu().numpy()

    def get_T_view(self) -> torch.Tensor:
        return self.T_a


MetalThermalContext = GpuThermalContext


def run_thermal3d_substeps_gpu(T, Q, k_grid, rho_cp_grid, Nx, Ny, Nz, dx, dy, dz, dt, n_substeps, h_eff=0.0,
                               t_ambient=20.0, is_active=1, device=None) -> np.ndarray:
    """Signature of run_thermal3d_substeps_metal (voxel_thermal_metal.py:179-195); returns float64."""
    ctx = GpuThermalContext(Nx, Ny, Nz, dx, dy, dz, dt, k_grid, rho_cp_grid, h_eff, t_ambient, device=device)
    ctx.set_T(T)
    ctx.set_Q(Q)
    ctx.advance(int(n_substeps), int(is_active))
    return ctx.get_T()


run_thermal3d_substeps_metal = run_thermal3d_substeps_gpu


class VoxelThermalSolver3D:
    """Mirror of simulation/voxel_thermal_3d.py:146-309 with the stencil on the GPU."""

    def __init__(self, grid_x, grid_y, grid_z, k_grid, rho_cp_grid, h_conv=15.0, emissivity=0.95, t_ambient=20.0):
        self.grid_x, self.grid_y, self.grid_z = grid_x, grid_y, grid_z
        self.Nx, self.Ny, self.Nz = len(grid_x), len(grid_y), len(grid_z)
        self.dx = float(grid_x[1] - grid_x[0]) if self.Nx > 1 else 0.05
        self.dy = float(grid_y[1] - grid_y[0]) if self.Ny > 1 else 0.05
        self.dz = float(grid_z[1] - grid_z[0]) if self.Nz > 1 else 0.04
        # unit heuristics of voxel_thermal_3d.py:169-180
        self.k_grid = k_grid * 1e-3 if np.max(k_grid) > 0.05 else np.array(k_grid, copy=True)
        self.rho_cp_grid = rho_cp_grid * 1e-9 if np.max(rho_cp_grid) > 100.0 else np.array(rho_cp_grid, copy=True)
        sigma_sb = 5.670374e-8
        h_rad = 4.0 * sigma_sb * emissivity * (t_ambient + 273.15) ** 3
        self.h_eff = (h_conv + h_rad) * 1e-6
        self.t_ambient = float(t_ambient)

    def cfl_conditioned_rho_cp(self, dt: float) -> np.ndarray:
        inv_d2 = 1.0 / self.dx ** 2 + 1.0 / self.dy ** 2 + 1.0 / self.dz ** 2
        alpha_max = CFL_SAFETY_FACTOR / (dt * inv_d2)
        rho = self.rho_cp_grid.copy()
        alpha = self.k_grid / np.maximum(rho, 1e-12)
        bad = alpha > alpha_max
        if np.any(bad):
            rho[bad] = self.k_grid[bad] / alpha_max
        return rho

    def solve(self, Q_3d, pulse_duration=0.20, total_time=1.00, dt=0.001, snapshot_times=None, engine='auto'):
        eng = str(engine).strip().lower()
        if eng == 'cpu':
            raise ValueError("engine='cpu' is not provided by bug_defense_b200 (GPU-only build)")
        n_steps = int(round(total_time / dt))
        ctx = GpuThermalContext(self.Nx, self.Ny, self.Nz, self.dx, self.dy, self.dz, dt, self.k_grid,
                                self.cfl_conditioned_rho_cp(dt), self.h_eff, self.t_ambient)
        ctx.set_T(np.full((self.Nx, self.Ny, self.Nz), self.t_ambient))
        ctx.set_Q(Q_3d)
        if snapshot_times is None:
            snapshot_times = [0.0, pulse_duration, total_time]
        targets = sorted({round(float(t), 4) for t in snapshot_times})
        mx, my, mz = self.Nx // 2, self.Ny // 2, self.Nz // 2
        snaps, centre, surface, times = {}, [], [], []
        t0 = time.time()
        for step in range(n_steps + 1):
            cur = round(step * dt, 4)
            v = ctx.get_T_view()
            pair = torch.stack([v[mx, my, mz], v[mx, my, 0]]).cpu().numpy()
            centre.append(float(pair[0])); surface.append(float(pair[1])); times.append(cur)
            if cur in targets:
                snaps[cur] = ctx.get_T()
            if step < n_steps:
                ctx.advance(1, int(cur < pulse_duration))
        return {
            'snapshots': snaps, 'time_history': np.array(times), 'center_history': np.array(centre),
            'surface_history': np.array(surface), 'solve_time': round(time.time() - t0, 3),
            'peak_surface_T': max(surface), 'peak_center_T': max(centre), 'engine': 'gpu',
        }
