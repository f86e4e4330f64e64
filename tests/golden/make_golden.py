"""Generate the golden fixtures in tests/golden/ by running the REFERENCE implementation.

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py [/path/to/reference]

Imports simulation/* from the reference tree (default /root/reference) and records inputs and
outputs of its CPU (numba) kernels, its coupled engine with the MC replaced by a fixed
absorbed map, and Monte Carlo statistics with batch standard errors. The fixtures are
committed; tests never import the reference at run time.
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
sys.path.insert(0, str(REF / "knowledge" / "simulation_lit_comparison" / "code"))
sys.path.insert(0, str(OUT))

from simulation.voxel_thermal_3d import _thermal3d_step_explicit, _apply_latent_heat_plateau  # noqa: E402
from simulation.coupled_ablation import (_accumulate_arrhenius, _accumulate_char,  # noqa: E402
                                         _update_phase_properties_numba, CoupledAblationEngine)
from simulation.plume import _diffuse_plume_step_numba, MultispectralPlumeField  # noqa: E402
from simulation.voxel_mc_3d import run_voxel_mc3d  # noqa: E402
import simulation.coupled_ablation as ca  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(OUT / name, **arrays)
    print("wrote", name, sum(np.asarray(a).nbytes for a in arrays.values()) // 1024, "KiB raw")


# ---------------------------------------------------------------------------------------
def thermal_fixtures():
    rng = np.random.default_rng(11)
    cases = {}
    # heterogeneous random grid, series BC (voxel_thermal_3d.py:30-112)
    Nx, Ny, Nz = 13, 11, 9
    T0 = rng.uniform(20, 120, (Nx, Ny, Nz)); Q = rng.uniform(0, 900, (Nx, Ny, Nz))
    k = rng.uniform(2e-4, 6e-4, (Nx, Ny, Nz)); rho = rng.uniform(1.5e-3, 4e-3, (Nx, Ny, Nz))
    p = dict(dx=0.03, dy=0.025, dz=0.02, dt=2e-5, h_eff=15e-6, t_amb=20.0)
    T = T0.copy(); Tn = np.empty_like(T); outs = []
    for s in range(10):
        _thermal3d_step_explicit(T, Tn, Q, k, rho, Nx, Ny, Nz, p['dx'], p['dy'], p['dz'], p['dt'], p['h_eff'],
                                 p['t_amb'], True)
        T, Tn = Tn, T
        if s in (0, 9):
            outs.append(T.copy())
    save("thermal_random.npz", T0=T0, Q=Q, k=k, rho=rho, T1=outs[0], T10=outs[1],
         params=json.dumps(p))
    # the two-strata case of tests/test_gpu_thermal.py:16-50 (large h_eff exercises the BC)
    Nx, Ny, Nz = 12, 12, 10
    T0 = np.full((Nx, Ny, Nz), 25.0); Q = np.zeros_like(T0); Q[4:8, 4:8, 0:3] = 800.0
    k = np.full_like(T0, 0.25e-3); k[:, :, 5:] = 0.5e-3
    rho = np.full_like(T0, 1.8e-3); rho[:, :, 5:] = 3.5e-3
    p = dict(dx=0.05, dy=0.05, dz=0.03, dt=2e-5, h_eff=12.0, t_amb=25.0)
    T = T0.copy(); Tn = np.empty_like(T)
    for _ in range(10):
        _thermal3d_step_explicit(T, Tn, Q, k, rho, Nx, Ny, Nz, 0.05, 0.05, 0.03, 2e-5, 12.0, 25.0, 1)
        T, Tn = Tn, T
    save("thermal_strata.npz", T0=T0, Q=Q, k=k, rho=rho, T10=T, params=json.dumps(p))


def fused_fixtures():
    # tests/test_gpu_thermal.py:76-136 configuration + a boiling/ablated/dry random case
    for name, seed in (("fused_strata.npz", None), ("fused_random.npz", 5)):
        if seed is None:
            Nx, Ny, Nz = 14, 14, 12
            T0 = np.full((Nx, Ny, Nz), 25.0); Q = np.zeros_like(T0); Q[5:9, 5:9, 0:3] = 750.0
            k = np.full_like(T0, 0.3e-3); k[:, :, 6:] = 0.5e-3
            rho = np.full_like(T0, 2.0e-3); rho[:, :, 6:] = 3.5e-3
            dry = np.zeros(T0.shape, bool); dry[6:8, 6:8, 0:2] = True
            abl = np.zeros(T0.shape, bool)
            H0 = np.zeros_like(T0); chi0 = np.zeros_like(T0)
            p = dict(dx=0.03, dy=0.03, dz=0.02, dt=2.5e-5, h_eff=15e-6, t_amb=20.0, t_abl=100.0, t_void=20.0,
                     arr_A=1e7, arr_EaR=65000.0 / 8.314, char_A=1e7, char_EaR=65000.0 / 8.314, n=30)
        else:
            rng = np.random.default_rng(seed)
            Nx, Ny, Nz = 12, 10, 16
            T0 = rng.uniform(60, 140, (Nx, Ny, Nz)); Q = rng.uniform(0, 3000, (Nx, Ny, Nz))
            k = rng.uniform(2e-4, 6e-4, T0.shape); rho = rng.uniform(1.5e-3, 4e-3, T0.shape)
            dry = rng.uniform(size=T0.shape) < 0.2; abl = rng.uniform(size=T0.shape) < 0.15
            H0 = np.where(rng.uniform(size=T0.shape) < 0.5, rng.uniform(0, 0.05, T0.shape), 0.0)
            chi0 = rng.uniform(0, 0.5, T0.shape)
            p = dict(dx=0.03, dy=0.03, dz=0.03, dt=3e-5, h_eff=15e-6, t_amb=20.0, t_abl=100.0, t_void=120.0,
                     arr_A=3e5, arr_EaR=5000.0, char_A=1e7, char_EaR=65000.0 / 8.314, n=25)
        T = T0.copy(); Tn = np.empty_like(T); H = H0.copy(); Om = np.zeros_like(T); chi = chi0.copy()
        for _ in range(p['n']):
            _thermal3d_step_explicit(T, Tn, Q, k, rho, Nx, Ny, Nz, p['dx'], p['dy'], p['dz'], p['dt'], p['h_eff'],
                                     p['t_amb'], 1)
            _apply_latent_heat_plateau(Tn, H, rho, abl, p['t_abl'], Nx, Ny, Nz, dry, p['t_void'])
            _accumulate_arrhenius(Tn, Om, abl, p['arr_A'], p['arr_EaR'], p['dt'], Nx, Ny, Nz)
            _accumulate_char(Tn, chi, dry, abl, p['char_A'], p['char_EaR'], p['dt'], Nx, Ny, Nz)
            T, Tn = Tn, T
        save(name, T0=T0, Q=Q, k=k, rho=rho, dry=dry, ablated=abl, H0=H0, chi0=chi0, T=T, H=H, Omega=Om,
             chi=chi, params=json.dumps(p))


def plume_fixtures():
    rng = np.random.default_rng(3)
    Nx, Ny, Nz = 15, 13, 11
    C0 = (rng.uniform(0, 1, (Nx, Ny, Nz)) * (rng.uniform(size=(Nx, Ny, Nz)) < 0.5)).astype(np.float32)
    vd = rng.uniform(size=(Nx, Ny, Nz)) < 0.75
    p = dict(dx=0.03, dy=0.03, dz=0.02, dt=1e-5, D_xy=1.0, D_z=2.0, vz=5.0, decay=float(np.exp(-1e-5 / 0.01)),
             n=10)
    C = C0.copy(); Cn = np.empty_like(C)
    for _ in range(p['n']):
        _diffuse_plume_step_numba(C, Cn, vd, Nx, Ny, Nz, p['dx'], p['dy'], p['dz'], p['dt'], p['D_xy'], p['D_z'],
                                  p['vz'], p['decay'])
        C, Cn = Cn, C
    save("plume_random.npz", C0=C0, void=vd, C10=C, params=json.dumps(p))
    # tests/test_plume.py:230-266: anisotropic point-source diffusion, 20 steps of 2e-5
    pl = MultispectralPlumeField(shape=(31, 31, 31), dx_mm=0.02, dy_mm=0.02, dz_mm=0.02, model='diffusion', D_xy=1.0,
                                 D_z=4.0, v_drift=0.0, tau_linger_s=float('inf'), blast_expansion=False)
    newly = np.zeros((31, 31, 31), bool); newly[15, 15, 15] = True
    pl.inject(newly)
    for _ in range(20):
        pl.diffuse_substep(np.ones((31, 31, 31), bool), dt_sub=2e-5)
    save("plume_aniso.npz", field=pl.raw_field.copy(), delta_mu=np.float64(pl.delta_mu))


def phase_fixtures():
    rng = np.random.default_rng(21)
    shape = (20, 10, 10); N = 2000
    for name, with_char in (("phase_char.npz", True), ("phase_nochar.npz", False)):
        H = np.where(rng.uniform(size=shape) < 0.6, rng.uniform(0, 3.0, shape), 0.0)
        h_lat = rng.uniform(0.5, 2.5, shape)
        T = rng.uniform(20, 450, shape)
        chi = rng.uniform(0, 1, shape)
        dry = rng.uniform(size=shape) < 0.35
        abl = rng.uniform(size=shape) < 0.1
        mu_a = rng.uniform(0.1, 20, shape); mu_s = rng.uniform(1, 40, shape)
        g = rng.uniform(0.7, 0.95, shape); n = rng.uniform(1.3, 1.6, shape)
        kk = rng.uniform(2e-4, 6e-4, shape); rho = rng.uniform(1e-3, 4e-3, shape)
        wet = (mu_a.copy(), kk.copy(), rho.copy())
        ds = dict(mu_a=rng.uniform(0.1, 5, shape), mu_s=rng.uniform(1, 30, shape), g=rng.uniform(0.7, 0.9, shape),
                  n=rng.uniform(1.3, 1.6, shape), k=rng.uniform(1e-4, 5e-4, shape),
                  rho_cp=rng.uniform(1e-3, 3e-3, shape), t_remove=350.0)
        cs = dict(mu_a=15.0, mu_s=20.0, k=0.35e-3, rho_cp=2.0e-3, t_remove=350.0) if with_char else None
        alpha_max = 0.35 / (5e-5 * 3 / 0.015 ** 2)
        ins = dict(H=H, h_lat=h_lat, T=T, chi=chi, dry=dry, ablated=abl, mu_a=mu_a, mu_s=mu_s, g=g, n=n, k=kk,
                   rho=rho)
        ins = {kname: v.copy() for kname, v in ins.items()}
        arr = lambda v: np.array([v], dtype=np.float64) if np.ndim(v) == 0 else np.ascontiguousarray(v.ravel())
        dsa = {kname: arr(v) for kname, v in ds.items()}
        dummy = np.zeros(1)
        csa = {kname: arr(v) for kname, v in cs.items()} if cs else {}
        rem = np.empty(shape, dtype=np.bool_)
        dry_w = dry.copy()
        _update_phase_properties_numba(
            H, h_lat, T, chi, dry_w, abl, mu_a, mu_s, g, n, kk, rho, wet[0], wet[1], wet[2],
            dsa['mu_a'], dsa['mu_s'], dsa['g'], dsa['n'], dsa['k'], dsa['rho_cp'], dsa['t_remove'],
            cs is not None, cs is not None, csa.get('mu_a', dummy), csa.get('mu_s', dummy), csa.get('k', dummy),
            csa.get('rho_cp', dummy), csa.get('t_remove', dummy), 0.95, cs is not None, cs is not None,
            cs is not None, alpha_max, rem)
        save(name, **{f"in_{kname}": v for kname, v in ins.items()},
             wet_mu_a=wet[0], wet_k=wet[1], wet_rho=wet[2],
             **{f"ds_{kname}": np.asarray(v, dtype=np.float64) for kname, v in ds.items()},
             **({f"cs_{kname}": np.float64(v) for kname, v in cs.items()} if cs else {}),
             alpha_max=np.float64(alpha_max), out_H=H, out_dry=dry_w, out_mu_a=mu_a, out_mu_s=mu_s, out_g=g, out_n=n,
             out_k=kk, out_rho=rho, out_remove=rem)


# ---------------------------------------------------------------------------------------
def engine_scenario():
    """Small coupled geometry: air on top, dry cuticle, subelytral air gap, wet tissue below."""
    Nx, Ny, Nz = 16, 16, 40
    d = 0.03
    shape = (Nx, Ny, Nz)
    mu_a = np.zeros(shape); mu_s = np.zeros(shape); g = np.zeros(shape); n = np.ones(shape)
    k = np.full(shape, 0.026e-3); rho = np.full(shape, 1.206e-6); h_lat = np.full(shape, 1e12)
    dry = np.zeros(shape, bool); abl0 = np.zeros(shape, bool)
    abl0[:, :, :4] = True
    layers = [(4, 8, 12.0, 20.0, 0.88, 1.56, 0.28e-3, 2.4e-3, 0.0, True),
              (8, 14, 0.0, 0.0, 0.0, 1.0, 0.026e-3, 1.206e-6, 1e12, False),
              (14, 24, 0.4, 12.0, 0.9, 1.46, 0.32e-3, 2.8e-3, 1.2, False),
              (24, 40, 1.0, 10.0, 0.93, 1.40, 0.5e-3, 3.65e-3, 1.6, False)]
    for k0, k1, ma, ms, gg, nn, kv, rv, hl, isdry in layers:
        mu_a[:, :, k0:k1] = ma; mu_s[:, :, k0:k1] = ms; g[:, :, k0:k1] = gg; n[:, :, k0:k1] = nn
        k[:, :, k0:k1] = kv; rho[:, :, k0:k1] = rv; h_lat[:, :, k0:k1] = hl; dry[:, :, k0:k1] = isdry
    # fixed absorbed-weight map (fraction of launched weight per voxel): Gaussian x Beer-Lambert
    x = (np.arange(Nx) + 0.5) * d - Nx * d / 2; y = (np.arange(Ny) + 0.5) * d - Ny * d / 2
    zc = (np.arange(Nz) + 0.5) * d
    rr = x[:, None] ** 2 + y[None, :] ** 2
    A = np.exp(-rr / (2 * 0.09 ** 2))[:, :, None] * np.exp(-zc / 0.25)[None, None, :]
    A[abl0] = 0.0
    A[:, :, 8:14] = 0.0
    A *= 0.6 / A.sum()
    cfg = dict(Lx=Nx * d, Ly=Ny * d, Lz=Nz * d, power=30.0, spot_dia=0.3, t_abl=100.0, t_ambient=20.0,
               dt_epoch=1e-3, dt_sub=5e-5, n_photons=1000, h_eff=15e-6, air_gap_range=[8, 14],
               wavelength_nm=532.0, epochs_on=45, epochs_off=10)
    char_state = dict(A=1.0e7, Ea=65000.0, mu_a=15.0, mu_s=20.0, k=0.35e-3, rho_cp=2.0e-3, t_remove=350.0,
                      chi_remove=0.95)
    plume = {'model': 'diffusion', 'D_xy': 1.0, 'D_z': 2.0, 'v_drift': 0.0, 'tau_linger_s': float('inf'),
             'blast_expansion': False}
    return dict(mu_a=mu_a, mu_s=mu_s, g=g, n=n, k=k, rho=rho, h_lat=h_lat, dry=dry, ablated=abl0, A=A), cfg, \
        char_state, plume


def engine_fixture():
    arrays, cfg, char_state, plume = engine_scenario()
    A = arrays['A']

    def fixed_mc(power, n_photons, spot_dia, Lx, Ly, Lz, Nx, Ny, Nz, **kw):
        vol = (Lx / Nx) * (Ly / Ny) * (Lz / Nz)
        return {'Q_3d': A * power / vol, 'Phi_3d': np.zeros_like(A), 'A_3d': A.copy(), 'energy_closure': 1.0}

    saved = ca.run_voxel_mc3d
    ca.run_voxel_mc3d = fixed_mc
    try:
        opt = {kname: arrays[kname].copy() for kname in ('mu_a', 'mu_s', 'g', 'n')}
        dry_state = {'mu_a': opt['mu_a'].copy(), 'mu_s': opt['mu_s'].copy(), 'g': opt['g'].copy(),
                     'n': opt['n'].copy(), 'k': arrays['k'].copy(), 'rho_cp': arrays['rho'].copy(), 't_remove': 350.0}
        eng = CoupledAblationEngine(
            optical_props=opt, k_grid=arrays['k'].copy(), rho_cp_grid=arrays['rho'].copy(),
            h_lat_grid=arrays['h_lat'].copy(), Lx=cfg['Lx'], Ly=cfg['Ly'], Lz=cfg['Lz'], power=cfg['power'],
            spot_dia=cfg['spot_dia'], t_abl=cfg['t_abl'], t_ambient=cfg['t_ambient'], dt_epoch=cfg['dt_epoch'],
            dt_sub=cfg['dt_sub'], n_photons=cfg['n_photons'], h_eff=cfg['h_eff'], dry_state=dry_state,
            char_state=dict(char_state), plume_closure=dict(plume), initial_dry_mask=arrays['dry'].copy(),
            initial_ablated_mask=arrays['ablated'].copy(), air_gap_range=tuple(cfg['air_gap_range']),
            wavelength_nm=cfg['wavelength_nm'], mc_engine='cpu', thermal_engine='cpu')
        diags = []
        snaps = {}
        for ep in range(cfg['epochs_on'] + cfg['epochs_off']):
            if ep == cfg['epochs_on']:
                eng.power = 0.0
            dg = eng.step_epoch()
            diags.append([dg['epoch'], dg['n_new'], dg['absorbed_frac'], dg['plume_transmission'], dg['plume_tau'],
                          dg['plume_peak_mu_a'], dg['plume_mean_mu_a']])
            if ep + 1 in (15, 30, cfg['epochs_on'] + cfg['epochs_off']):
                snaps[ep + 1] = dict(T=eng.T.copy(), H=eng.H_acc.copy(), chi=eng.chi.copy(), dry=eng.dry.copy(),
                                     ablated=eng.ablated.copy(), plume=eng.plume.raw_field.copy(),
                                     mu_ext=eng.plume.mu_ext_plume.copy(), mu_a=eng.optical['mu_a'].copy(),
                                     mu_s=eng.optical['mu_s'].copy(), k=eng.k_grid.copy(), rho=eng.rho_cp_grid.copy(),
                                     T_peak=eng.T_peak.copy(), ablation_time=eng.ablation_time.copy())
    finally:
        ca.run_voxel_mc3d = saved
    out = {f"in_{kname}": v for kname, v in arrays.items()}
    out['diag'] = np.array(diags, dtype=np.float64)
    for ep, sn in snaps.items():
        for kname, v in sn.items():
            out[f"ep{ep}_{kname}"] = v
    out['cfg'] = json.dumps(cfg); out['char_state'] = json.dumps(char_state); out['plume'] = json.dumps(
        {kname: (v if v != float('inf') else 'inf') for kname, v in plume.items()})
    out['snap_epochs'] = np.array(sorted(snaps))
    save("engine_fixedQ.npz", **out)


# ---------------------------------------------------------------------------------------
def mc_fixtures():
    import verification_benchmarks as vb
    res = {}
    from mc_cases import mc_cases
    for name, kw, nb, npb in mc_cases():
        rows = [run_voxel_mc3d(n_photons=npb, engine='cpu', **kw) for _ in range(nb)]
        keys = ('R_spec', 'R_diff', 'Absorption', 'Transmission', 'Lateral_loss')
        st = {}
        for key in keys:
            v = np.array([r['spectro_raw'][key] for r in rows])
            st[key] = [float(v.mean()), float(v.std(ddof=1) / np.sqrt(nb))]
        depth_axis = (0, 1) if kw.get('launch_axis', 'z') == 'z' else (1, 2)
        prof = np.array([r['A_3d'].sum(axis=depth_axis) for r in rows])
        res[name] = dict(stats=st, batches=nb, photons_per_batch=npb,
                         depth_profile=prof.mean(axis=0).tolist(),
                         depth_profile_se=(prof.std(axis=0, ddof=1) / np.sqrt(nb)).tolist(),
                         closure=float(np.mean([r['energy_closure'] for r in rows])))
        print(name, {key: round(v[0], 5) for key, v in st.items()})
    # analytic / canonical values (verification_benchmarks.py:28-29, :32-51, :102-151)
    n_, mu_a, d = 1.5, 1.0, 0.5
    R = ((n_ - 1) / (n_ + 1)) ** 2
    e1, e2 = np.exp(-mu_a * d), np.exp(-2 * mu_a * d)
    th = np.radians(45.0); stt = np.sin(th) / 1.5; ct = np.sqrt(1 - stt ** 2); ci = np.cos(th)
    R45 = 0.5 * (((ci - 1.5 * ct) / (ci + 1.5 * ct)) ** 2 + ((ct - 1.5 * ci) / (ct + 1.5 * ci)) ** 2)
    res['analytic'] = dict(
        slab_matched_Rd=vb.SLAB_MATCHED_RD, slab_matched_Tt=vb.SLAB_MATCHED_TT,
        semi_infinite_isotropic_Rd_a09=vb.semi_infinite_isotropic_rd(0.9),
        fresnel_slab_T=float((1 - R) ** 2 * e1 / (1 - R ** 2 * e2)),
        fresnel_slab_Rd=float(R * (1 - R) ** 2 * e2 / (1 - R ** 2 * e2)), fresnel_slab_Rspec=float(R),
        oblique45_T=float((1 - R45) * np.exp(-1.0 * 1.0 / ct)), oblique45_Rspec=float(R45),
        semi_infinite_mismatched_Rtot=0.2600)
    with open(OUT / "mc_stats.json", "w") as f:
        json.dump(res, f, indent=1)
    print("wrote mc_stats.json")


if __name__ == "__main__":
    which = sys.argv[2:] or ["thermal", "fused", "plume", "phase", "engine", "mc"]
    for w in which:
        globals()[f"{w}_fixtures" if w != "engine" else "engine_fixture"]()
