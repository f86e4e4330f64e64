"""Device-resident coupled laser-tissue epoch -- drop-in for CoupledAblationEngine.

Same constructor keywords and step_epoch() diagnostics as
simulation/coupled_ablation.py:183-667. The host-side set-up (CFL conditioning, initial
ablated overrides, dry/char parameter caching) is the reference's, in float64 numpy; after it
every field lives on the GPU in float32 and one epoch (MC -> 20 fused substeps -> plume ->
phase/removal/plume-sync) is enqueued by bd_engine_step_epoch with no host round trip.
State attributes (T, H_acc, chi, dry, ablated, Q, optical, ...) are read lazily (one D2H copy
per access); assigning a whole array uploads it.

Extensions (keywords the reference does not have):
  seed             Philox key of the photon streams (reproducible MC)
  plume_dt_policy  'subcycle' (default: stable sub-steps), 'metal' (dt clamp of
                   metal_ablation_solver.py:235-237) or 'as_given' (plume.py:79 as called by
                   coupled_ablation.py:533-538)
  bc               'series' (voxel_thermal_3d.py:97,105) or 'metal' (metal_ablation_solver.py:141,150)
  semantics        'cpu' or 'metal' deltas of the photon tracer
  tally_fluence    also tally the track-length estimator for Phi
  use_graphs       replay each epoch stage as a captured CUDA graph (default) or launch directly
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._device import require_device, to_dev
from .ablation import plume_params_struct
from .plume import PlumeField, from_closure
from .voxel_mc import make_params

K_AIR = 0.026e-3       # W/(mm K)       coupled_ablation.py:28
RHO_CP_AIR = 1.206e-6  # J/(mm^3 K)     coupled_ablation.py:29
R_GAS = 8.314          # J/(mol K)      coupled_ablation.py:30


class _LazyOptical(dict):
    """engine.optical['mu_a'] etc. read from the device on access."""

    def __init__(self, eng):
        super().__init__()
        self._eng = eng

    def __getitem__(self, key):
        t = self._eng._opt_t[key]
        return t.double().cpu().numpy()

    def __setitem__(self, key, value):
        self._eng._opt_t[key].copy_(to_dev(value, self._eng.dev).reshape(self._eng.shape))

    def keys(self):
        return ('mu_a', 'mu_s', 'g', 'n')

    def items(self):
        return [(k, self[k]) for k in self.keys()]

    def __contains__(self, key):
        return key in ('mu_a', 'mu_s', 'g', 'n')

    def __iter__(self):
        return iter(self.keys())


class CoupledAblationEngine:
    def __init__(self, optical_props: dict, k_grid, rho_cp_grid, h_lat_grid, Lx: float, Ly: float, Lz: float,
                 power: float, spot_dia: float, t_abl: float, t_ambient: float = 20.0, dt_epoch: float = 0.01,
                 dt_sub: float = 5e-5, n_photons: int = 100000, h_eff: float = 0.0, r_max: float = 0.0,
                 beam_center=None, stability_factor: float = 0.35, k_void: float = K_AIR,
                 rho_cp_void: float = RHO_CP_AIR, arrhenius=None, beam_profile: str = 'gaussian', dry_state=None,
                 char_state=None, plume_closure=None, theta_inc_deg: float = 0.0, phi_inc_deg: float = 0.0,
                 initial_dry_mask=None, initial_ablated_mask=None, air_gap_range=None,
                 wavelength_nm: float = 10600.0, mc_engine: str = 'auto', thermal_engine: str = 'auto',
                 seed=None, plume_dt_policy: str = 'subcycle', bc: str = 'series', semantics: str = 'cpu',
                 tally_fluence: bool = True, use_graphs: bool = True, device=None):
        for name, eng in (('mc_engine', mc_engine), ('thermal_engine', thermal_engine)):
            e = str(eng).strip().lower()
            if e == 'cpu':
                raise ValueError(f"{name}='cpu' is not provided by bug_defense_b200 (GPU-only build)")
            if e not in ('auto', 'gpu'):
                raise ValueError(f"Unknown {name}='{eng}'. Valid options: 'auto', 'gpu', 'cpu'.")
        self.dev = require_device(device)
        self.mc_engine, self.thermal_engine = mc_engine, thermal_engine
        self.use_gpu_thermal = True

        # ---- set-up in float64, exactly as coupled_ablation.py:232-303, but on the device: the
        # inputs are uploaded once and every step (stability clamp, void properties, wet copies) is
        # the same IEEE float64 arithmetic as the host version, rounded to float32 at the end ----
        d = self.dev

        def h64(a):
            if isinstance(a, torch.Tensor):
                return a.to(device=d, dtype=torch.float64).clone()
            return to_dev(a, d, torch.float64)

        def hbool(a):
            if isinstance(a, torch.Tensor):
                return a.to(device=d).bool()
            return to_dev(a, d, torch.bool)

        optical = {key: h64(optical_props[key]) for key in ('mu_a', 'mu_s', 'g', 'n')}
        self.Nx, self.Ny, self.Nz = optical['mu_a'].shape
        self.shape = (self.Nx, self.Ny, self.Nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.dx, self.dy, self.dz = self.Lx / self.Nx, self.Ly / self.Ny, self.Lz / self.Nz
        self.voxel_vol = self.dx * self.dy * self.dz
        self._power = float(power)
        self.spot_dia = float(spot_dia)
        self.t_abl, self.t_ambient = float(t_abl), float(t_ambient)
        self.dt_epoch, self.dt_sub = float(dt_epoch), float(dt_sub)
        self.n_substeps = max(1, int(round(self.dt_epoch / self.dt_sub)))
        self.n_photons = int(n_photons)
        self.h_eff, self.r_max = float(h_eff), float(r_max)
        self._beam_center = beam_center
        self.beam_profile = beam_profile
        self.theta_inc_deg, self.phi_inc_deg = float(theta_inc_deg), float(phi_inc_deg)
        self.semantics = semantics
        self.tally_fluence = bool(tally_fluence)
        self.use_graphs = bool(use_graphs)
        self.seed = int(seed) if seed is not None else int(np.random.randint(1, 2 ** 31 - 1))

        k, rho, h_lat = h64(k_grid), h64(rho_cp_grid), h64(h_lat_grid)
        inv_d2 = 1.0 / self.dx ** 2 + 1.0 / self.dy ** 2 + 1.0 / self.dz ** 2
        self.alpha_max_stable = stability_factor / (self.dt_sub * inv_d2)
        alpha = k / torch.clamp(rho, min=1e-12)
        unstable = alpha > self.alpha_max_stable
        self._cfl_mask = unstable
        rho = torch.where(unstable, k / self.alpha_max_stable, rho)
        self.k_void = float(k_void)
        self.rho_cp_void = max(float(rho_cp_void), self.k_void / self.alpha_max_stable)

        ablation_time = torch.full(self.shape, -1.0, device=d, dtype=torch.float32)
        if initial_ablated_mask is not None:
            ablated = hbool(initial_ablated_mask).reshape(self.shape)
            ablation_time.masked_fill_(ablated, 0.0)
            for key, v in (('mu_a', 0.0), ('mu_s', 0.0), ('g', 0.0), ('n', 1.0)):
                optical[key].masked_fill_(ablated, v)
            k.masked_fill_(ablated, self.k_void)
            rho.masked_fill_(ablated, self.rho_cp_void)
        else:
            ablated = torch.zeros(self.shape, dtype=torch.bool, device=d)
        self.arrhenius = None if arrhenius is None else (float(arrhenius[0]), float(arrhenius[1]) / R_GAS)
        dry = (hbool(initial_dry_mask).reshape(self.shape) if initial_dry_mask is not None
               else torch.zeros(self.shape, dtype=torch.bool, device=d))
        self.dry_state = dict(dry_state) if dry_state is not None else None
        wet = None
        if self.dry_state is not None:
            rc = self.dry_state.get('rho_cp')
            if isinstance(rc, (np.ndarray, torch.Tensor)):
                self.dry_state['rho_cp'] = torch.maximum(h64(rc), k / self.alpha_max_stable)
            wet = (optical['mu_a'], k, rho)
        self.t_void = float(np.max(self.dry_state['t_remove'])) if self.dry_state is not None else self.t_abl
        self.char_state = char_state
        if char_state is not None:
            self._arrhenius_char = (float(char_state['A']), float(char_state['Ea']) / R_GAS)
            if 't_remove' in char_state:
                self.t_void = float(np.max(char_state['t_remove']))
        else:
            self._arrhenius_char = None
        self.air_gap_range = tuple(air_gap_range) if air_gap_range is not None else None
        self.wavelength_nm = float(wavelength_nm)

        # ---- device fields (float32) ----
        f32 = lambda t: t.to(torch.float32).reshape(self.shape).contiguous()
        z32 = lambda: torch.zeros(self.shape, device=d, dtype=torch.float32)
        self._opt_t = {key: f32(optical[key]) for key in ('mu_a', 'mu_s', 'g', 'n')}
        self._k, self._rho, self._h_lat = f32(k), f32(rho), f32(h_lat)
        self._T = torch.full(self.shape, self.t_ambient, device=d, dtype=torch.float32)
        self._T_alt = z32()
        self._H = z32()
        self._Omega = z32()
        self._chi = z32()
        self._T_peak = torch.full(self.shape, self.t_ambient, device=d, dtype=torch.float32)
        self._abl_time = ablation_time
        self._flags = (ablated.to(torch.uint8) * _lib.FLAG_ABLATED) | (dry.to(torch.uint8) * _lib.FLAG_DRY)
        self._wet = tuple(f32(w) for w in wet) if wet is not None else None
        self._A = z32()
        self._L = z32() if self.tally_fluence else None
        self._props = torch.zeros(self.Nx * self.Ny * self.Nz * 4, device=d, dtype=torch.float32)
        self._latz = torch.zeros(self.Nz, device=d, dtype=torch.float64)
        self._keep = []
        del optical, k, rho, h_lat, alpha

        # plume (diffusion model, point injection)
        self.plume_closure = plume_closure
        self.plume = None
        if plume_closure is not None:
            if isinstance(plume_closure, PlumeField):
                self.plume = plume_closure
                if self.plume.raw is None:
                    self.plume.raw = z32(); self.plume.mu_ext = z32(); self.plume.device = d
            elif isinstance(plume_closure, dict) and plume_closure.get('enabled', True):
                self.plume = from_closure(plume_closure, self.shape, self.dx, self.dy, self.dz, self.wavelength_nm, d)
        self._P_alt = z32() if self.plume is not None else None
        self.plume_dt_policy = plume_dt_policy
        self.bc = bc

        self._desc = self._build_desc()
        h = ctypes.c_void_p()
        _lib.call("bd_engine_create", ctypes.byref(self._desc), ctypes.byref(h))
        self._handle = h
        # initial epoch-end pass: void bits and packed MC properties of the first epoch
        self._init_flags_and_props()
        self.t = 0.0
        self.epoch = 0
        self.last_mc = None
        self._last_power = 0.0
        # host work that may run while the device finishes an enqueued epoch (weak references to
        # bound methods, run by _diag just before it blocks on the epoch's diagnostics)
        self._wait_hooks = []

    @property
    def cfl_conditioned_mask(self) -> np.ndarray:
        """Voxels whose rho_cp was raised to keep the explicit step stable (coupled_ablation.py:246-250)."""
        return self._cfl_mask.cpu().numpy()

    # ------------------------------------------------------------------------------
    def _gref(self, v):
        if v is None:
            return _lib.GridRef(None, 0.0, 0)
        if isinstance(v, torch.Tensor):
            if v.numel() == 1:
                return _lib.GridRef(None, float(v.reshape(-1)[0]), 0)
        elif np.ndim(v) == 0 or np.size(v) == 1:
            return _lib.GridRef(None, float(np.asarray(v).ravel()[0]), 0)
        t = to_dev(v, self.dev).reshape(-1)
        self._keep.append(t)
        return _lib.GridRef(t.data_ptr(), 0.0, 0)

    def _ds_value(self, key, optical_t):
        """_init_ds_cs_arrays (coupled_ablation.py:409-438): dry-state value or its fallback."""
        ds = self.dry_state
        if key in ds:
            return ds[key]
        if key == 't_remove':
            return self.t_abl
        if key in ('mu_a', 'mu_s', 'g', 'n'):
            return optical_t[key].double().cpu().numpy()
        return 0.0

    def _build_desc(self) -> _lib.EngineDesc:
        P = _lib.ptr
        D = _lib.EngineDesc()
        ph = D.phase
        ph.nx, ph.ny, ph.nz = self.Nx, self.Ny, self.Nz
        ph.single_stage = int(self.dry_state is None)
        ph.apply_removal = 1
        ph.t_abl = self.t_abl
        ph.alpha_max_stable = self.alpha_max_stable
        ph.k_void, ph.rho_cp_void, ph.t_void = self.k_void, self.rho_cp_void, self.t_void
        self._ds_t = {}
        if self.dry_state is not None:
            for key, fld in (('mu_a', 'ds_mu_a'), ('mu_s', 'ds_mu_s'), ('g', 'ds_g'), ('n', 'ds_n'), ('k', 'ds_k'),
                             ('rho_cp', 'ds_rho_cp'), ('t_remove', 'ds_t_remove')):
                ref = self._gref(self._ds_value(key, self._opt_t))
                if ref.ptr:
                    self._ds_t[key] = self._keep[-1]
                setattr(ph, fld, ref)
        cs = self.char_state
        ph.has_char_state = int(cs is not None)
        ph.cs_chi_remove = 1.0
        if cs is not None:
            for key, fld, flag in (('mu_a', 'cs_mu_a', 'has_cs_mu_a'), ('mu_s', 'cs_mu_s', 'has_cs_mu_s'),
                                   ('k', 'cs_k', 'has_cs_k'), ('rho_cp', 'cs_rho_cp', 'has_cs_rho_cp')):
                if key in cs:
                    setattr(ph, fld, self._gref(cs[key]))
                    setattr(ph, flag, 1)
            t_rem = cs.get('t_remove', self.dry_state.get('t_remove', self.t_abl) if self.dry_state else self.t_abl)
            ph.cs_t_remove = self._gref(t_rem)
            ph.cs_chi_remove = float(cs.get('chi_remove', 1.0))
        if self.air_gap_range is not None:
            ph.gap_k0, ph.gap_k1 = int(self.air_gap_range[0]), int(self.air_gap_range[1])
        else:
            ph.gap_k0, ph.gap_k1 = 0, 0
        pl = self.plume
        ph.has_plume = int(pl is not None)
        if pl is not None:
            ph.plume_delta_mu = pl.delta_mu
            ph.plume_mu_max = pl.mu_max
            ph.plume_ratio_a, ph.plume_ratio_s = pl.ratio_a, pl.ratio_s
            ph.plume_g = 0.80
            ph.plume, ph.mu_ext = P(pl.raw), P(pl.mu_ext)
        ph.T, ph.H_acc, ph.chi = P(self._T), P(self._H), P(self._chi)
        ph.mu_a, ph.mu_s, ph.g, ph.n = (P(self._opt_t[key]) for key in ('mu_a', 'mu_s', 'g', 'n'))
        ph.k, ph.rho_cp, ph.T_peak, ph.ablation_time = P(self._k), P(self._rho), P(self._T_peak), P(self._abl_time)
        ph.h_lat = P(self._h_lat)
        if self._wet is not None:
            ph.wet_mu_a, ph.wet_k, ph.wet_rho_cp = (P(w) for w in self._wet)
        ph.flags = P(self._flags)
        ph.props = P(self._props)

        sp = D.substep
        sp.nx, sp.ny, sp.nz = self.Nx, self.Ny, self.Nz
        sp.dx, sp.dy, sp.dz, sp.dt = self.dx, self.dy, self.dz, self.dt_sub
        sp.h_eff, sp.t_ambient, sp.t_abl, sp.t_void = self.h_eff, self.t_ambient, self.t_abl, self.t_void
        sp.bc_mode = {'series': _lib.BC_SERIES, 'cpu': _lib.BC_SERIES, 'metal': _lib.BC_METAL}[self.bc]
        if self.arrhenius is not None:
            sp.has_arrhenius, sp.arr_A, sp.arr_Ea_over_R = 1, self.arrhenius[0], self.arrhenius[1]
        if self._arrhenius_char is not None:
            sp.has_char, sp.char_A, sp.char_Ea_over_R = 1, self._arrhenius_char[0], self._arrhenius_char[1]
        D.n_substeps = self.n_substeps
        if pl is not None:
            D.has_plume_transport = 1
            D.plume = plume_params_struct(self.shape, self.dx, self.dy, self.dz, self.dt_sub, pl.D_xy, pl.D_z,
                                          pl.v_drift, pl.tau_linger, self.plume_dt_policy)
            D.plume_alt = P(self._P_alt)
        else:
            D.plume = plume_params_struct(self.shape, self.dx, self.dy, self.dz, self.dt_sub, 0, 0, 0, 0)
        D.mc = self._mc_params()
        D.T_alt, D.A, D.L = P(self._T_alt), P(self._A), P(self._L)
        D.omega = P(self._Omega) if self.arrhenius is not None else P(None)
        D.lat_depth = P(self._latz)
        D.dt_epoch = self.dt_epoch
        D.voxel_volume = self.voxel_vol
        return D

    def _mc_params(self):
        return make_params(Nx=self.Nx, Ny=self.Ny, Nz=self.Nz, Lx=self.Lx, Ly=self.Ly, Lz=self.Lz,
                           n_photons=self.n_photons, spot_dia=self.spot_dia, theta_inc_deg=self.theta_inc_deg,
                           phi_inc_deg=self.phi_inc_deg, beam_center=self._beam_center,
                           beam_profile=self.beam_profile, launch_axis='z', n_ambient=1.0, r_max=self.r_max,
                           seed=self.seed, semantics=self.semantics, tally_fluence=self.tally_fluence)

    def _init_flags_and_props(self):
        # bd_engine_create already ran the initial void / plume / packed-property pass
        _lib.call("bd_engine_set_time", self._handle, 0.0, 0, _lib.stream_ptr())

    # ------------------------------------------------------------------------------
    @property
    def power(self):
        return self._power

    @power.setter
    def power(self, v):
        self._power = float(v)

    @property
    def beam_center(self):
        return self._beam_center

    @beam_center.setter
    def beam_center(self, v):
        self._beam_center = v
        self._sync_mc()

    def _sync_mc(self):
        if getattr(self, '_handle', None):
            mp = self._mc_params()
            _lib.call("bd_engine_set_mc", self._handle, ctypes.byref(mp))

    def switch_wavelength(self, wavelength_nm: float, optical: dict = None, dry_state: dict = None,
                          power: float = None):
        """Mid-run wavelength switch of the dual-wavelength runner
        (run_dual_permutation_suite.py:254-283): intact (non-ablated) voxels take the new optical
        properties and dry-state optics, the wet copies restart from the current optics, the plume
        takes the new wavelength's extinction constants (plume.py:270-278) and re-derives its
        extinction; the packed MC properties follow before the next epoch. Arrays are full grids."""
        intact = ((self._flags & _lib.FLAG_ABLATED) == 0)
        if optical is not None:
            for key in ('mu_a', 'mu_s', 'g', 'n'):
                new = to_dev(optical[key], self.dev).reshape(self.shape)
                self._opt_t[key].copy_(torch.where(intact, new, self._opt_t[key]))
        if dry_state is not None and self.dry_state is not None:
            for key in ('mu_a', 'mu_s', 'g', 'n'):
                if key in dry_state and key in self._ds_t:
                    t = self._ds_t[key].view(self.shape)
                    t.copy_(torch.where(intact, to_dev(dry_state[key], self.dev).reshape(self.shape), t))
        if self._wet is not None:
            self._wet[0].view(self.shape).copy_(self._opt_t['mu_a'])
            self._wet[1].view(self.shape).copy_(self._k)
            self._wet[2].view(self.shape).copy_(self._rho)
        if self.plume is not None:
            self.plume.set_wavelength(wavelength_nm)
            pl = self.plume
            _lib.call("bd_engine_set_plume_optics", self._handle, float(pl.mu_max), float(pl.ratio_a),
                      float(pl.ratio_s), float(pl.delta_mu))
        self.wavelength_nm = float(wavelength_nm)
        if power is not None:
            self.power = power
        _lib.call("bd_engine_refresh_props", self._handle, _lib.stream_ptr())

    def step_epoch(self, absorbed_map=None) -> dict:
        """Advance one coupled epoch; returns the diagnostics of coupled_ablation.py:605-617.

        absorbed_map (optional, shape of the grid): fraction of launched weight absorbed per
        voxel to use instead of running the MC this epoch (a fixed heat source)."""
        opts = 0
        if absorbed_map is not None:
            # the engine's tally holds absorbed weight for n_photons launched photons
            tally = np.asarray(absorbed_map, dtype=np.float64) * max(self.n_photons, 1)
            self._A.copy_(to_dev(tally, self.dev).reshape(self.shape))
            opts |= _lib.EPOCH_SKIP_MC
        self._enqueue(opts)
        return self._diag(absorbed_map)

    # run the plume stage after the substeps on the caller's stream instead of beside MC + substeps
    # on the engine's own plume stream (same results; the stages share no data within an epoch)
    serial_plume = False

    def _enqueue(self, opts=0):
        if not self.use_graphs:
            opts |= _lib.EPOCH_NO_GRAPH
        if self.serial_plume:
            opts |= _lib.EPOCH_SERIAL_PLUME
        _lib.call("bd_engine_step_epoch", self._handle, float(self._power), int(opts), _lib.stream_ptr())
        self._last_power = self._power

    def step_epochs(self, n: int) -> dict:
        """n epochs with a single host synchronisation; returns the last epoch's diagnostics."""
        for _ in range(int(n)):
            self._enqueue(0)
        return self._diag(None)

    def _run_wait_hooks(self):
        live = []
        for ref in self._wait_hooks:
            fn = ref()
            if fn is not None:
                fn()
                live.append(ref)
        self._wait_hooks = live

    def _diag(self, absorbed_map):
        if self._wait_hooks:
            self._run_wait_hooks()
        dg = _lib.EpochDiag()
        _lib.call("bd_engine_read_diag", self._handle, ctypes.byref(dg), _lib.stream_ptr())
        self.t = dg.time_s
        self.epoch = int(dg.epoch)
        led = np.array(dg.ledger[:])
        laser = self._last_power > 0.0
        if laser and absorbed_map is None:
            N = float(max(self.n_photons, 1))
            absorbed = (led[_lib.LEDGER_ABSORBED] + led[_lib.LEDGER_ABSORBED_VOID]) / N
            closure = (led[1] + led[2] + led[3] + led[4]) / N + absorbed
            self.last_mc = {'engine': 'gpu', 'ledger': led, 'energy_closure': closure}
        elif laser:
            absorbed = float(np.sum(absorbed_map))
            closure = 1.0
        else:
            absorbed, closure = 0.0, 1.0
        if self.plume is not None:
            tau = float(dg.plume_tau)
            peak = float(dg.plume_peak_mu_a)
            mean = float(dg.plume_ablated_sum / dg.n_ablated) if dg.n_ablated > 0 else 0.0
        else:
            tau, peak, mean = 0.0, 0.0, 0.0
        return {
            'epoch': self.epoch, 'time_s': self.t, 'n_new': int(dg.n_new), 'absorbed_frac': absorbed,
            'mc_energy_closure': closure, 't_optical_s': dg.t_optical_ms * 1e-3, 't_thermal_s': dg.t_thermal_ms * 1e-3,
            'plume_transmission': float(math.exp(-tau)), 'plume_tau': tau, 'plume_peak_mu_a': peak,
            'plume_mean_mu_a': mean, 't_epoch_end_s': dg.t_epoch_end_ms * 1e-3, 'ledger': led,
            'n_void': int(dg.n_void), 'void_zlimit': int(dg.void_zlimit),
        }

    # ---- lazily-read state (host float64 / bool copies) -----------------------------
    def _get(self, t):
        return t.double().cpu().numpy()

    T = property(lambda s: s._get(s._T), lambda s, v: s._T.copy_(to_dev(v, s.dev).reshape(s.shape)))
    H_acc = property(lambda s: s._get(s._H), lambda s, v: s._H.copy_(to_dev(v, s.dev).reshape(s.shape)))
    Omega = property(lambda s: s._get(s._Omega))
    chi = property(lambda s: s._get(s._chi))
    T_peak = property(lambda s: s._get(s._T_peak))
    ablation_time = property(lambda s: s._get(s._abl_time))
    k_grid = property(lambda s: s._get(s._k))
    rho_cp_grid = property(lambda s: s._get(s._rho))
    h_lat = property(lambda s: s._get(s._h_lat))

    @property
    def ablated(self):
        return ((self._flags & _lib.FLAG_ABLATED) != 0).cpu().numpy()

    @property
    def dry(self):
        return ((self._flags & _lib.FLAG_DRY) != 0).cpu().numpy()

    @property
    def optical(self):
        return _LazyOptical(self)

    @property
    def Q_opt(self):
        if self._last_power <= 0.0:
            return np.zeros(self.shape)
        scale = self._last_power / (max(self.n_photons, 1) * self.voxel_vol)
        return self._A.double().cpu().numpy() * scale

    @property
    def Q(self):
        return self.Q_opt

    @property
    def Phi(self):
        if self._last_power <= 0.0 or self._L is None:
            return np.zeros(self.shape)
        return self._L.double().cpu().numpy() / (max(self.n_photons, 1) * self.voxel_vol)

    def compute_void_mask(self) -> np.ndarray:
        """coupled_ablation.py:619-626"""
        vm = self.ablated.copy()
        if self.air_gap_range is not None:
            k0, k1 = self.air_gap_range
            if k0 > 0 and np.any(vm[:, :, k0 - 1]):
                vm[:, :, k0:k1] = True
        return vm

    def centerline_depth_mm(self, ix: int = None, iy: int = None, k_surface: int = 0) -> float:
        """coupled_ablation.py:662-667"""
        ix = self.Nx // 2 if ix is None else ix
        iy = self.Ny // 2 if iy is None else iy
        col = ((self._flags[ix, iy, k_surface:] & _lib.FLAG_ABLATED) != 0).cpu().numpy()
        idx = np.where(col)[0]
        return float((idx.max() + 1) * self.dz) if idx.size else 0.0

    def __del__(self):
        try:
            if getattr(self, '_handle', None):
                _lib.load().bd_engine_destroy(self._handle)
                self._handle = None
        except Exception:
            pass
