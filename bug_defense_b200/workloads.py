"""Seeded synthetic workloads with the shapes and value distributions of the benchmark configs.

There is no dataset: every property is drawn once per layer, uniformly within the published
ranges, from numpy.random.default_rng(seed), and is constant within a layer. Layers are assigned
to voxels by the cell-centre rule (simulation/voxel_mc_3d.py:527-536).

  single_epoch_stack(seed)  64x64x128 at 15 um: one 20k-photon epoch + 20 substeps, no ablation
  full_coupled_run(seed)    200x200x128 stack + 64 air slices on top (the plume region) = 200x200x192;
                            boiling, char, ablation, plume; 150k photons per epoch
  crater_sample(seed)       a random crater on the 200x200x128 stack (denoiser training / evaluation)
"""
from __future__ import annotations

import math

import numpy as np

DX = 0.015  # mm
# (name, thickness in um) from the dorsal surface down
STACK = [("exocuticle", 60.0), ("endocuticle", 120.0), ("air_gap", 300.0), ("fat", 400.0),
         ("hemolymph", 200.0), ("muscle", 600.0), ("ventral_cuticle", 150.0)]
H_LAT_WATER_J_PER_KG = 2.26e6


def _draw_layers(rng):
    """Optical (532 nm) and thermal properties, one draw per layer."""
    out = {}
    for name, _ in STACK:
        if name == "air_gap":
            out[name] = dict(mu_a=0.0, mu_s=0.0, g=0.0, n=1.0, k=0.026e-3, rho_cp=1.206e-6, water=0.0)
            continue
        if "cuticle" in name:
            opt = dict(mu_a=rng.uniform(5, 30), mu_s=rng.uniform(10, 40), g=rng.uniform(0.85, 0.90), n=1.56)
        elif name == "fat":
            opt = dict(mu_a=rng.uniform(0.05, 0.5), mu_s=rng.uniform(10, 20), g=0.90, n=1.46)
        elif name == "hemolymph":
            opt = dict(mu_a=rng.uniform(0.1, 1.0), mu_s=rng.uniform(1, 5), g=0.90, n=1.35)
        else:  # muscle
            opt = dict(mu_a=rng.uniform(0.2, 2.0), mu_s=rng.uniform(5, 15), g=0.93, n=1.40)
        k = rng.uniform(0.2, 0.6) * 1e-3                      # W/m/K -> W/mm/K
        rho = rng.uniform(1000, 1300)                          # kg/m^3
        c = rng.uniform(1.7, 3.8) * 1e3                        # J/kg/K
        water = rng.uniform(0.05, 0.8)
        opt.update(k=k, rho_cp=rho * c * 1e-9, rho=rho, water=water)
        out[name] = opt
    return out


def _layer_index(nz_tissue, n_air_top):
    """Layer name per z slice (cell-centre rule), air above the stack."""
    names = []
    edges = np.cumsum([t for _, t in STACK]) * 1e-3  # mm
    for k in range(n_air_top + nz_tissue):
        if k < n_air_top:
            names.append("top_air")
            continue
        zc = (k - n_air_top + 0.5) * DX
        idx = int(np.searchsorted(edges, zc, side="right"))
        names.append(STACK[idx][0] if idx < len(STACK) else "below")
    return names


def single_epoch_stack(seed: int = 0, nx: int = 64, ny: int = 64, nz: int = 128):
    """64x64x128 stack (1830 um of tissue = 122 voxels; the 6 remaining slices are ambient air on top,
    initial-ablated), 532 nm, Gaussian 0.5 mm spot at 22 deg, 40 W, 20k photons, 20 x 50 us."""
    rng = np.random.default_rng(seed)
    lay = _draw_layers(rng)
    n_tissue = int(round(sum(t for _, t in STACK) * 1e-3 / DX))
    n_air = nz - n_tissue
    return _build(lay, nx, ny, n_air, n_tissue, wet_ablation=False) | dict(
        power=40.0, spot_dia=0.5, theta_inc_deg=22.0, n_photons=20_000, n_substeps=20, dt_sub=5e-5, seed=seed)


def full_coupled_run(seed: int = 0, nx: int = 200, ny: int = 200, nz: int = 128, n_plume_air: int = 64, device=None):
    """200x200x128 stack with 64 air slices prepended for the plume (200x200x192), boiling at 100 C with
    2.26 MJ/kg x water fraction, cuticle dry with removal at 350 C, char A ~ U(1e10, 1e12)/s,
    Ea ~ U(1.5e5, 2e5) J/mol, plume D ~ U(10, 50) mm^2/s, extinction ~ U(0.5, 5)/mm per unit
    concentration (injected per ablated voxel); 150k photons per 1 ms epoch, 200 on / 800 off."""
    rng = np.random.default_rng(seed)
    lay = _draw_layers(rng)
    n_tissue = int(round(sum(t for _, t in STACK) * 1e-3 / DX))
    n_air = nz - n_tissue + n_plume_air
    geo = _build(lay, nx, ny, n_air, n_tissue, wet_ablation=True, device=device)
    char_A = float(rng.uniform(1e10, 1e12))
    char_Ea = float(rng.uniform(1.5e5, 2.0e5))
    D = float(rng.uniform(10.0, 50.0))
    ext = float(rng.uniform(0.5, 5.0))
    geo.update(
        power=40.0, spot_dia=0.5, theta_inc_deg=22.0, n_photons=150_000, dt_sub=5e-5, dt_epoch=1e-3,
        epochs_total=1000, epochs_on=200, t_abl=100.0, t_ambient=25.0, h_eff=15e-6, seed=seed,
        char_state=dict(A=char_A, Ea=char_Ea, mu_a=15.0, mu_s=20.0, k=0.35e-3, rho_cp=2.0e-3, t_remove=350.0,
                        chi_remove=0.95),
        plume_closure=dict(model='diffusion', D_xy=D, D_z=D, v_drift=0.0, tau_linger_s=float('inf'),
                           blast_expansion=False, delta_mu_per_voxel=ext, wavelength_nm=532.0),
        plume_D=D, plume_extinction=ext)
    return geo


def _build(lay, nx, ny, n_air, n_tissue, wet_ablation, device=None):
    """Layer properties per z slice, expanded to full (nx, ny, nz) grids: float64 numpy arrays, or
    float64 torch tensors built on `device` (the per-instance builder of a campaign, no host grids)."""
    nz = n_air + n_tissue
    names = _layer_index(n_tissue, n_air)
    shape = (nx, ny, nz)
    col = {key: np.full(nz, v, dtype=np.float64) for key, v in (("mu_a", 0.0), ("mu_s", 0.0), ("g", 0.0), ("n", 1.0),
                                                                ("k", 0.026e-3), ("rho_cp", 1.206e-6),
                                                                ("h_lat", 1e12))}
    dry_z = np.zeros(nz, bool)
    abl_z = np.zeros(nz, bool)
    gap = [kk for kk, nm in enumerate(names) if nm == "air_gap"]
    for kk, nm in enumerate(names):
        if nm == "top_air":
            abl_z[kk] = True
            continue
        if nm == "below":
            continue
        p = lay[nm]
        for key in ("mu_a", "mu_s", "g", "n", "k", "rho_cp"):
            col[key][kk] = p[key]
        if nm == "air_gap":
            continue
        if "cuticle" in nm:
            dry_z[kk] = wet_ablation
            col["h_lat"][kk] = 0.0 if wet_ablation else 1e12
        elif wet_ablation:
            col["h_lat"][kk] = H_LAT_WATER_J_PER_KG * p["rho"] * p["water"] * 1e-9
    if device is None:
        grid = lambda c: np.broadcast_to(c, shape).copy()
    else:
        import torch
        dev = torch.device(device)
        grid = lambda c: torch.as_tensor(c, device=dev).expand(shape).contiguous()
    optical = {key: grid(col[key]) for key in ("mu_a", "mu_s", "g", "n")}
    k, rho_cp, h_lat = grid(col["k"]), grid(col["rho_cp"]), grid(col["h_lat"])
    Lx, Ly, Lz = nx * DX, ny * DX, nz * DX
    return dict(shape=shape, Lx=Lx, Ly=Ly, Lz=Lz, optical=optical, k_grid=k, rho_cp_grid=rho_cp, h_lat_grid=h_lat,
                dry_mask=grid(dry_z), ablated_mask=grid(abl_z), air_gap_range=(gap[0], gap[-1] + 1) if gap else None,
                layers=lay, layer_names=names, n_air_top=n_air,
                dry_state=dict(**{key: grid(col[key]) for key in ("mu_a", "mu_s", "g", "n", "k", "rho_cp")},
                               t_remove=350.0))


def engine_kwargs(geo: dict) -> dict:
    """Keyword arguments of CoupledAblationEngine for a full_coupled_run geometry."""
    return dict(optical_props=geo["optical"], k_grid=geo["k_grid"], rho_cp_grid=geo["rho_cp_grid"],
                h_lat_grid=geo["h_lat_grid"], Lx=geo["Lx"], Ly=geo["Ly"], Lz=geo["Lz"], power=geo["power"],
                spot_dia=geo["spot_dia"], t_abl=geo["t_abl"], t_ambient=geo["t_ambient"],
                dt_epoch=geo["dt_epoch"], dt_sub=geo["dt_sub"], n_photons=geo["n_photons"], h_eff=geo["h_eff"],
                theta_inc_deg=geo["theta_inc_deg"], dry_state=geo["dry_state"], char_state=geo["char_state"],
                plume_closure=geo["plume_closure"], initial_dry_mask=geo["dry_mask"],
                initial_ablated_mask=geo["ablated_mask"], air_gap_range=geo["air_gap_range"],
                wavelength_nm=532.0, seed=geo["seed"] + 1)


def single_epoch_kwargs(geo: dict, seed: int = 1) -> dict:
    """CoupledAblationEngine keyword arguments of the single-epoch stack (single_epoch_stack): the
    same optics, conduction and beam, with boiling and removal out of reach (t_abl 1e9 C, h_lat
    1e12 J/mm^3, no dry / char state) and no plume, so an epoch is one MC pass + 20 substeps."""
    return dict(optical_props=geo["optical"], k_grid=geo["k_grid"], rho_cp_grid=geo["rho_cp_grid"],
                h_lat_grid=geo["h_lat_grid"], Lx=geo["Lx"], Ly=geo["Ly"], Lz=geo["Lz"], power=geo["power"],
                spot_dia=geo["spot_dia"], t_abl=1e9, t_ambient=25.0, dt_epoch=geo["n_substeps"] * geo["dt_sub"],
                dt_sub=geo["dt_sub"], n_photons=geo["n_photons"], h_eff=15e-6, theta_inc_deg=geo["theta_inc_deg"],
                initial_ablated_mask=geo["ablated_mask"], wavelength_nm=532.0, seed=seed)


def crater_sample(seed: int, nx: int = 200, ny: int = 200, nz: int = 128, device=None) -> dict:
    """One random crater geometry on the full-resolution stack (the denoiser's training and
    evaluation inputs): layer properties drawn as for full_coupled_run, then a paraboloid crater of
    depth U(0, 0.9) mm and radius U(0.08, 0.45) mm near the beam axis (none in 15% of samples) is
    emptied (void optics, ablated + void flags), a charred rim of 0-3 voxels takes char optics and
    the dry flag, and half of the craters hold a uniform plume absorption U(0, 1.5)/mm.
    Built on the device with torch; returns fp32 optical grids, flag bytes and the beam geometry
    (Gaussian 0.5 mm spot at 22 deg, centre of the face)."""
    import torch
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(seed)
    lay = _draw_layers(rng)
    n_tissue = int(round(sum(t for _, t in STACK) * 1e-3 / DX))
    n_air = nz - n_tissue
    names = _layer_index(n_tissue, n_air)
    zp = {key: np.zeros(nz) for key in ("mu_a", "mu_s", "g")}
    zp["n"] = np.ones(nz)
    abl_z = np.zeros(nz, bool)
    dry_z = np.zeros(nz, bool)
    for kk, nm in enumerate(names):
        if nm == "top_air":
            abl_z[kk] = True
        elif nm != "below":
            dry_z[kk] = "cuticle" in nm          # cuticle starts dry, as in full_coupled_run
            for key in ("mu_a", "mu_s", "g", "n"):
                zp[key][kk] = lay[nm][key]
    shape = (nx, ny, nz)
    grids = {k: torch.as_tensor(v, dtype=torch.float32, device=dev).expand(shape).contiguous() for k, v in zp.items()}
    fz = np.where(abl_z, 0x05, 0) | np.where(dry_z, 0x02, 0)
    flags = torch.as_tensor(fz.astype(np.uint8), device=dev).expand(shape).contiguous()
    Lx, Ly = nx * DX, ny * DX
    x = (torch.arange(nx, device=dev, dtype=torch.float32) + 0.5) * DX
    y = (torch.arange(ny, device=dev, dtype=torch.float32) + 0.5) * DX
    z = (torch.arange(nz, device=dev, dtype=torch.float32) + 0.5) * DX
    z0 = n_air * DX
    has = rng.random() >= 0.15
    depth = float(rng.uniform(0.0, 0.9)) if has else 0.0
    radius = float(rng.uniform(0.08, 0.45))
    xc = Lx / 2 + float(rng.uniform(-0.1, 0.1))
    yc = Ly / 2 + float(rng.uniform(-0.1, 0.1))
    rim = int(rng.integers(0, 4))
    plume = float(rng.uniform(0.0, 1.5)) if rng.random() < 0.5 else 0.0
    char_mu_a, char_mu_s = float(rng.uniform(10, 30)), float(rng.uniform(10, 30))
    r2 = ((x[:, None] - xc) ** 2 + (y[None, :] - yc) ** 2) / (radius * radius)
    floor = z0 + depth * torch.clamp(1.0 - r2, min=0.0)                 # crater floor per column
    zz = z[None, None, :]
    crater = (zz < floor[:, :, None]) & (zz >= z0) & (r2[:, :, None] < 1.0) if depth > 0 else torch.zeros(
        shape, dtype=torch.bool, device=dev)
    if rim > 0 and depth > 0:
        shell = (zz < floor[:, :, None] + rim * DX) & (zz >= z0) & (r2[:, :, None] < (1.0 + rim * DX / radius) ** 2)
        shell &= ~crater & (grids["mu_s"] > 0)
        grids["mu_a"][shell] = char_mu_a
        grids["mu_s"][shell] = char_mu_s
        grids["g"][shell] = 0.9
        grids["n"][shell] = 1.56
        flags[shell] |= 0x02
    grids["mu_a"][crater] = plume
    grids["mu_s"][crater] = 0.0
    grids["g"][crater] = 0.8
    grids["n"][crater] = 1.0
    flags[crater] |= 0x05
    return dict(shape=shape, Lx=Lx, Ly=Ly, Lz=nz * DX, mu_a=grids["mu_a"], mu_s=grids["mu_s"], g=grids["g"],
                n=grids["n"], flags=flags, spot_dia=0.5, theta_inc_deg=22.0, depth=depth, radius=radius, rim=rim,
                plume=plume, seed=seed)
