"""ORACLE -- test infrastructure only: FP64 CPU restatement of CoupledAblationEngine.step_epoch
(simulation/coupled_ablation.py:440-617, CPU thermal path :507-544) on the C kernels of
oracle/orc.c, with the reference's host logic (removal :628-660, void mask :619-626, plume
inject/sync plume.py:292-366) in numpy. Used as the parity reference and as the timed CPU port
(bench.py --impl reference / cpu_baseline); never imported by the product."""
from __future__ import annotations

import math
import time

import numpy as np

from . import (accumulate_arrhenius, accumulate_char, apply_latent_heat_plateau, diffuse_plume_step, plume_policy,
               run_voxel_mc3d, thermal3d_step_explicit, update_phase_properties)

K_AIR = 0.026e-3
RHO_CP_AIR = 1.206e-6
R_GAS = 8.314
EXTINCTION_MAP = {10600: (0.15, 0.05, 0.075), 1940: (0.375, 0.15, 0.18), 1470: (0.45, 0.20, 0.22),
                  1064: (0.675, 0.60, 0.33), 532: (1.275, 0.80, 0.63), 450: (1.80, 1.00, 0.90),
                  320: (2.40, 1.20, 1.20)}


class OracleEngine:
    def __init__(self, optical_props, k_grid, rho_cp_grid, h_lat_grid, Lx, Ly, Lz, power, spot_dia, t_abl,
                 t_ambient=20.0, dt_epoch=0.01, dt_sub=5e-5, n_photons=100000, h_eff=0.0, r_max=0.0,
                 beam_center=None, stability_factor=0.35, k_void=K_AIR, rho_cp_void=RHO_CP_AIR, arrhenius=None,
                 beam_profile='gaussian', dry_state=None, char_state=None, plume_closure=None, theta_inc_deg=0.0,
                 phi_inc_deg=0.0, initial_dry_mask=None, initial_ablated_mask=None, air_gap_range=None,
                 wavelength_nm=10600.0, seed=1, plume_dt_policy='as_given', mc_stream='oracle', bc='series',
                 semantics='cpu', **_ignored):
        self.optical = {k: np.array(optical_props[k], dtype=np.float64, copy=True) for k in ('mu_a', 'mu_s', 'g', 'n')}
        self.Nx, self.Ny, self.Nz = self.optical['mu_a'].shape
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.dx, self.dy, self.dz = self.Lx / self.Nx, self.Ly / self.Ny, self.Lz / self.Nz
        self.voxel_vol = self.dx * self.dy * self.dz
        self.power, self.spot_dia, self.t_abl, self.t_ambient = float(power), float(spot_dia), float(t_abl), float(t_ambient)
        self.dt_epoch, self.dt_sub = float(dt_epoch), float(dt_sub)
        self.n_substeps = max(1, int(round(self.dt_epoch / self.dt_sub)))
        self.n_photons, self.h_eff, self.r_max = int(n_photons), float(h_eff), float(r_max)
        self.beam_center, self.beam_profile = beam_center, beam_profile
        self.theta_inc_deg, self.phi_inc_deg = float(theta_inc_deg), float(phi_inc_deg)
        self.seed = int(seed)
        self.k_grid = np.array(k_grid, dtype=np.float64, copy=True)
        self.rho_cp_grid = np.array(rho_cp_grid, dtype=np.float64, copy=True)
        self.h_lat = np.array(h_lat_grid, dtype=np.float64, copy=True)
        inv_d2 = 1 / self.dx ** 2 + 1 / self.dy ** 2 + 1 / self.dz ** 2
        self.alpha_max_stable = stability_factor / (self.dt_sub * inv_d2)
        bad = self.k_grid / np.maximum(self.rho_cp_grid, 1e-12) > self.alpha_max_stable
        self.rho_cp_grid[bad] = self.k_grid[bad] / self.alpha_max_stable
        self.k_void = float(k_void)
        self.rho_cp_void = max(float(rho_cp_void), self.k_void / self.alpha_max_stable)
        shape = (self.Nx, self.Ny, self.Nz)
        self.T = np.full(shape, self.t_ambient); self._T_next = np.empty_like(self.T)
        self.H_acc = np.zeros(shape); self.ablation_time = np.full(shape, -1.0)
        if initial_ablated_mask is not None:
            self.ablated = np.array(initial_ablated_mask, dtype=np.bool_, copy=True)
            self.ablation_time[self.ablated] = 0.0
            for key, v in (('mu_a', 0.0), ('mu_s', 0.0), ('g', 0.0), ('n', 1.0)):
                self.optical[key][self.ablated] = v
            self.k_grid[self.ablated] = self.k_void
            self.rho_cp_grid[self.ablated] = self.rho_cp_void
            self.T[self.ablated] = self.t_ambient
        else:
            self.ablated = np.zeros(shape, dtype=np.bool_)
        self.Q = np.zeros(shape)
        self.arrhenius = None if arrhenius is None else (float(arrhenius[0]), float(arrhenius[1]) / R_GAS)
        self.Omega = np.zeros(shape)
        self.T_peak = np.full(shape, self.t_ambient)
        self.dry_state = dict(dry_state) if dry_state is not None else None
        self.dry = (np.array(initial_dry_mask, dtype=np.bool_, copy=True) if initial_dry_mask is not None
                    else np.zeros(shape, dtype=np.bool_))
        self._wet = None
        if self.dry_state is not None:
            if isinstance(self.dry_state.get('rho_cp'), np.ndarray):
                self.dry_state['rho_cp'] = np.maximum(self.dry_state['rho_cp'], self.k_grid / self.alpha_max_stable)
            self._wet = (self.optical['mu_a'].copy(), self.k_grid.copy(), self.rho_cp_grid.copy())
        self.t_void = float(np.max(self.dry_state['t_remove'])) if self.dry_state is not None else self.t_abl
        self.char_state = char_state
        self.chi = np.zeros(shape)
        if char_state is not None:
            self._char = (float(char_state['A']), float(char_state['Ea']) / R_GAS)
            if 't_remove' in char_state:
                self.t_void = float(np.max(char_state['t_remove']))
        else:
            self._char = None
        self.air_gap_range = air_gap_range
        self.plume = None
        if plume_closure is not None and plume_closure.get('enabled', True):
            pc = plume_closure
            wl = float(pc.get('wavelength_nm', wavelength_nm))
            mu_a_max, mu_s_max, dmu = EXTINCTION_MAP.get(int(round(wl)), (0.30, 0.15, 0.15))
            if pc.get('mu_a_max', pc.get('mu_max')) is not None:
                mu_a_max = float(pc.get('mu_a_max', pc.get('mu_max')))
            d_over = pc.get('delta_mu_per_voxel', pc.get('delta_mu'))
            D_plume = float(pc.get('D_plume', pc.get('D', 2.0)))
            self.plume = dict(
                mu_a_max=mu_a_max, mu_s_max=mu_s_max, mu_max=mu_a_max + mu_s_max,
                delta_mu=float(d_over) if d_over is not None else dmu,
                D_xy=float(pc['D_xy']) if 'D_xy' in pc else D_plume, D_z=float(pc['D_z']) if 'D_z' in pc else D_plume,
                v=float(pc.get('v_drift', pc.get('vz', 80.0))), tau=float(pc.get('tau_linger_s', 0.00875)),
                raw=np.zeros(shape), mu_ext=np.zeros(shape))
        self.plume_dt_policy = plume_dt_policy
        # 'engine': epoch e traces photon p on the Philox stream (seed, (e << 32) + p), the streams of
        # the GPU engine's epoch e (k_epoch_begin), so the two MC tallies are correlated samples
        self.mc_stream = mc_stream
        # z-wall flux of the fused substep (0: series half-cell + h_eff, 1: Metal -h_eff (T - T_amb)) and
        # the MC semantics (the CPU or the Metal tracer's thresholds)
        self.bc_mode = {'series': 0, 'cpu': 0, 'metal': 1}[bc]
        self.semantics = semantics
        self.last_mc = None
        self._init_ds_cs()
        self.t = 0.0
        self.epoch = 0

    def _init_ds_cs(self):
        self._ds = None
        if self.dry_state is not None:
            self._ds = {}
            for k in ('mu_a', 'mu_s', 'g', 'n', 'k', 'rho_cp', 't_remove'):
                if k in self.dry_state:
                    v = self.dry_state[k]
                elif k == 't_remove':
                    v = self.t_abl
                elif k in self.optical:
                    v = self.optical[k].copy()
                else:
                    v = 0.0
                self._ds[k] = v
        self._cs = None
        self._cs_chi = 1.0
        if self.char_state is not None:
            cs = self.char_state
            self._cs = {k: cs[k] for k in ('mu_a', 'mu_s', 'k', 'rho_cp') if k in cs}
            self._cs['t_remove'] = cs.get('t_remove', self.dry_state.get('t_remove', self.t_abl)
                                          if self.dry_state else self.t_abl)
            self._cs_chi = float(cs.get('chi_remove', 1.0))

    def compute_void_mask(self):
        vm = self.ablated.copy()
        if self.air_gap_range is not None:
            k0, k1 = self.air_gap_range
            if k0 > 0 and np.any(self.ablated[:, :, k0 - 1]):
                vm[:, :, k0:k1] = True
        return vm

    def _mu_plume(self):
        p = self.plume
        ra = p['mu_a_max'] / max(1e-6, p['mu_max']); rs = p['mu_s_max'] / max(1e-6, p['mu_max'])
        return p['mu_ext'] * ra, p['mu_ext'] * rs

    def load_state(self, st: dict):
        """Overwrite the evolving state with `st` (float64 / bool arrays, e.g. another engine's
        state after an epoch), so one epoch of both engines can be compared from the same start.
        Keys: T H_acc chi dry ablated mu_a mu_s g n k_grid rho_cp_grid wet_mu_a wet_k wet_rho_cp T_peak
        ablation_time t epoch, optionally Omega, and plume_raw plume_mu_ext when there is a plume."""
        c = lambda a, dt=np.float64: np.array(a, dtype=dt, copy=True).reshape(self.T.shape)
        self.T, self.H_acc, self.chi = c(st['T']), c(st['H_acc']), c(st['chi'])
        if 'Omega' in st:
            self.Omega = c(st['Omega'])
        self.dry, self.ablated = c(st['dry'], np.bool_), c(st['ablated'], np.bool_)
        for key in ('mu_a', 'mu_s', 'g', 'n'):
            self.optical[key] = c(st[key])
        self.k_grid, self.rho_cp_grid = c(st['k_grid']), c(st['rho_cp_grid'])
        if self._wet is not None:
            self._wet = (c(st['wet_mu_a']), c(st['wet_k']), c(st['wet_rho_cp']))
        self.T_peak, self.ablation_time = c(st['T_peak']), c(st['ablation_time'])
        self.t, self.epoch = float(st['t']), int(st['epoch'])
        if self.plume is not None:
            self.plume['raw'], self.plume['mu_ext'] = c(st['plume_raw']), c(st['plume_mu_ext'])
        self._T_next = np.empty_like(self.T)

    def step_epoch(self, absorbed_map=None, threads=None, capture=None) -> dict:
        """One epoch. `capture` (a dict) receives copies of T, H_acc, chi, dry and ablated after the
        substeps and before the epoch-end phase update (the state the removal rule reads)."""
        t0 = time.perf_counter()
        if self.power > 0.0:
            if absorbed_map is None:
                opt = self.optical
                if self.plume is not None and np.any(self.plume['mu_ext'] > 0):
                    ma, ms = self._mu_plume()
                    opt = {k: v.copy() for k, v in self.optical.items()}
                    opt['mu_a'] = self.optical['mu_a'] + ma
                    opt['mu_s'] = self.optical['mu_s'] + ms
                    opt['g'][(self.plume['mu_ext'] > 0.001) & self.ablated] = 0.80
                if self.mc_stream == 'engine':
                    stream = dict(seed=self.seed, photon_offset=(self.epoch + 1) << 32)
                else:
                    stream = dict(seed=self.seed * 1_000_003 + self.epoch)
                mc = run_voxel_mc3d(power=self.power, n_photons=self.n_photons, spot_dia=self.spot_dia, Lx=self.Lx,
                                    Ly=self.Ly, Lz=self.Lz, Nx=self.Nx, Ny=self.Ny, Nz=self.Nz, r_max=self.r_max,
                                    custom_3d_props=opt, beam_center=self.beam_center, beam_profile=self.beam_profile,
                                    theta_inc_deg=self.theta_inc_deg, phi_inc_deg=self.phi_inc_deg,
                                    semantics=self.semantics, **stream)
                self.last_mc = mc
                A = mc['A_3d']
                absorbed, closure = float(A.sum()), float(mc['energy_closure'])
            else:
                A = absorbed_map
                absorbed, closure = float(np.sum(A)), 1.0
            self.Q = A * (self.power / self.voxel_vol)
            Qth = self.Q.copy()
            Qth[self.ablated] = 0.0
        else:
            self.Q = np.zeros_like(self.T); Qth = self.Q
            absorbed, closure = 0.0, 1.0
        t_opt = time.perf_counter() - t0
        t1 = time.perf_counter()
        Nx, Ny, Nz = self.Nx, self.Ny, self.Nz
        void = self.compute_void_mask() if self.plume is not None else self.ablated
        T, Tn = self.T, self._T_next
        if self.plume is not None:
            p = self.plume
            n_sub, dtp, decay = plume_policy(self.dt_sub, self.dx, self.dy, self.dz, p['D_xy'], p['D_z'], p['v'],
                                             p['tau'], self.plume_dt_policy)
            P, Pn = p['raw'], np.empty_like(p['raw'])
        for _ in range(self.n_substeps):
            thermal3d_step_explicit(T, Tn, Qth, self.k_grid, self.rho_cp_grid, Nx, Ny, Nz, self.dx, self.dy, self.dz,
                                    self.dt_sub, self.h_eff, self.t_ambient, True, self.bc_mode)
            apply_latent_heat_plateau(Tn, self.H_acc, self.rho_cp_grid, self.ablated, self.t_abl, Nx, Ny, Nz,
                                      self.dry, self.t_void)
            if self.arrhenius is not None:
                accumulate_arrhenius(Tn, self.Omega, self.ablated, self.arrhenius[0], self.arrhenius[1],
                                     self.dt_sub, Nx, Ny, Nz)
            if self._char is not None:
                accumulate_char(Tn, self.chi, self.dry, self.ablated, self._char[0], self._char[1], self.dt_sub,
                                Nx, Ny, Nz)
            if self.plume is not None:
                for _s in range(n_sub):
                    diffuse_plume_step(P, Pn, void, Nx, Ny, Nz, self.dx, self.dy, self.dz, dtp, p['D_xy'], p['D_z'],
                                       p['v'], decay)
                    P, Pn = Pn, P
            T, Tn = Tn, T
        self.T, self._T_next = T, Tn
        if self.plume is not None:
            self.plume['raw'] = P
        np.maximum(self.T_peak, self.T, out=self.T_peak)
        t_th = time.perf_counter() - t1
        if capture is not None:
            capture.update(T=self.T.copy(), H_acc=self.H_acc.copy(), chi=self.chi.copy(), dry=self.dry.copy(),
                           ablated=self.ablated.copy())
        self.t += self.dt_epoch
        self.epoch += 1
        if self.dry_state is None:
            rem = (~self.ablated) & (self.H_acc >= self.h_lat) & (self.T >= self.t_abl)
        else:
            dry8 = self.dry.view(np.uint8)
            rem = update_phase_properties(self.H_acc, self.h_lat, self.T, self.chi, dry8, self.ablated,
                                          self.optical['mu_a'], self.optical['mu_s'], self.optical['g'],
                                          self.optical['n'], self.k_grid, self.rho_cp_grid, self._wet[0], self._wet[1],
                                          self._wet[2], self._ds, self._cs, self._cs_chi, self.alpha_max_stable)
        n_new = self._remove(rem)
        if self.plume is not None:
            vm = self.compute_void_mask()
            p = self.plume
            p['raw'][~vm] = 0.0
            p['mu_ext'] = p['mu_max'] * np.tanh(p['raw'] / p['mu_max']) if p['mu_max'] > 0 else p['raw'].copy()
            p['mu_ext'][~vm] = 0.0
            ma, _ = self._mu_plume()
            tau = float(np.sum(ma[Nx // 2, Ny // 2, :]) * self.dz)
            peak = float(np.max(ma))
            mean = float(np.mean(ma[self.ablated])) if np.any(self.ablated) else 0.0
        else:
            tau, peak, mean = 0.0, 0.0, 0.0
        return {'epoch': self.epoch, 'time_s': self.t, 'n_new': n_new, 'absorbed_frac': absorbed,
                'mc_energy_closure': closure, 't_optical_s': t_opt, 't_thermal_s': t_th,
                'plume_transmission': math.exp(-tau), 'plume_tau': tau, 'plume_peak_mu_a': peak,
                'plume_mean_mu_a': mean}

    def _remove(self, newly) -> int:
        n_new = int(np.sum(newly))
        if n_new > 0:
            self.ablated[newly] = True
            self.dry[newly] = False
            self.chi[newly] = 0.0
            self.ablation_time[newly] = self.t
            for key, v in (('mu_a', 0.0), ('mu_s', 0.0), ('g', 0.0), ('n', 1.0)):
                self.optical[key][newly] = v
            self.k_grid[newly] = self.k_void
            self.rho_cp_grid[newly] = self.rho_cp_void
            self.T[newly] = self.t_void
            self.H_acc[newly] = 0.0
            if self.air_gap_range is not None:
                k0, k1 = self.air_gap_range
                if k0 > 0:
                    cols = self.ablated[:, :, k0 - 1] & ~self.ablated[:, :, k0]
                    if np.any(cols):
                        ix, iy = np.where(cols)
                        self.ablated[ix, iy, k0:k1] = True
                        self.ablation_time[ix, iy, k0:k1] = self.t
            if self.plume is not None:
                vm = self.compute_void_mask()
                self.plume['raw'][newly] += self.plume['delta_mu']
                self.plume['raw'][~vm] = 0.0
        return n_new
