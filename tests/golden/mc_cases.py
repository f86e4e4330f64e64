"""Monte Carlo cases shared by make_golden.py (run on the reference) and the tests.

Each case: (name, run_voxel_mc3d keyword arguments, batches, photons per batch). Geometries
follow the reference tests and verification tier they are named after.
"""
import numpy as np


def mc_cases():
    """(name, kwargs, batches, photons per batch) -- reference run_voxel_mc3d(engine='cpu')."""
    cases = []
    Nx, Ny, Nz = 30, 30, 40
    mua = np.zeros((Nx, Ny, Nz)); mus = np.zeros_like(mua); g = np.zeros_like(mua); n = np.zeros_like(mua)
    for z0, z1, a, s, gg, nn in ((0, 10, 0.6, 16.0, 0.85, 1.52), (10, 24, 0.05, 4.0, 0.8, 1.34),
                                  (24, 40, 0.7, 18.0, 0.88, 1.42)):
        mua[:, :, z0:z1] = a; mus[:, :, z0:z1] = s; g[:, :, z0:z1] = gg; n[:, :, z0:z1] = nn
    props3 = dict(mu_a=mua, mu_s=mus, g=g, n=n)
    # tests/test_gpu_mc.py:40-126
    cases.append(("multilayer_oblique", dict(power=10.0, Lx=2.0, Ly=2.0, Lz=1.0, Nx=Nx, Ny=Ny, Nz=Nz,
                                             custom_3d_props=props3, theta_inc_deg=30.0, phi_inc_deg=45.0,
                                             spot_dia=0.40, beam_center=(1.0, 1.0)), 10, 50_000))
    # tests/test_gpu_mc.py:14-38
    cube = {kname: np.full((20, 20, 25), v) for kname, v in (('mu_a', 0.2), ('mu_s', 10.0), ('g', 0.8), ('n', 1.4))}
    cases.append(("homogeneous_cube", dict(power=5.0, Lx=1.0, Ly=1.0, Lz=1.0, Nx=20, Ny=20, Nz=25,
                                           custom_3d_props=cube, spot_dia=0.20), 10, 30_000))
    # verification_benchmarks.py:67-84 (V1a/V1b)
    cases.append(("slab_v1", dict(spot_dia=0.01, Lx=20.0, Ly=20.0, Lz=0.2, Nx=20, Ny=20, Nz=10,
                                  layers_config=[{'z_end': 0.2, 'mu_a': 1.0, 'mu_s': 9.0, 'g': 0.75, 'n': 1.0}]),
                  10, 50_000))
    # verification_benchmarks.py:102-128 (V1c/d/e)
    cases.append(("fresnel_slab_v1c", dict(spot_dia=0.01, Lx=2.0, Ly=2.0, Lz=0.55, Nx=4, Ny=4, Nz=11,
                                           layers_config=[{'z_end': 0.5, 'mu_a': 1.0, 'mu_s': 0.0, 'g': 0.0,
                                                           'n': 1.5},
                                                          {'z_end': 0.55, 'mu_a': 0.0, 'mu_s': 0.0, 'g': 0.0,
                                                           'n': 1.0}]), 10, 40_000))
    # verification_benchmarks.py:131-151 (V1f)
    cases.append(("oblique_v1f", dict(spot_dia=0.2, theta_inc_deg=45.0, Lx=8.0, Ly=8.0, Lz=1.0, Nx=40, Ny=40,
                                      Nz=20, layers_config=[{'z_end': 1.0, 'mu_a': 1.0, 'mu_s': 0.0, 'g': 0.0,
                                                             'n': 1.5}]), 10, 40_000))
    # verification_benchmarks.py:154-174 (V2b)
    cases.append(("semi_infinite_v2b", dict(spot_dia=0.01, Lx=20.0, Ly=20.0, Lz=4.0, Nx=20, Ny=20, Nz=8,
                                            layers_config=[{'z_end': 4.0, 'mu_a': 1.0, 'mu_s': 9.0, 'g': 0.0,
                                                            'n': 1.5}]), 10, 40_000))
    # branch coverage: top-hat, Kim disks, r_max, launch along x
    small = {kname: np.full((16, 16, 20), v) for kname, v in (('mu_a', 0.5), ('mu_s', 12.0), ('g', 0.85), ('n', 1.38))}
    small['n'][:, :, 10:] = 1.45
    small['mu_a'][:, :, 10:] = 1.5
    base = dict(Lx=1.2, Ly=1.2, Lz=1.0, Nx=16, Ny=16, Nz=20, custom_3d_props=small, spot_dia=0.5,
                theta_inc_deg=20.0, phi_inc_deg=30.0)
    cases.append(("tophat", dict(base, beam_profile='tophat'), 10, 30_000))
    cases.append(("kim_exp_disk", dict(base, beam_profile='kim_exp_disk'), 10, 30_000))
    cases.append(("kim_gauss_disk_rmax", dict(base, beam_profile='kim_gauss_disk', r_max=0.4), 10, 30_000))
    smx = {kname: np.ascontiguousarray(np.transpose(v, (2, 1, 0))) for kname, v in small.items()}
    cases.append(("launch_x", dict(Lx=1.0, Ly=1.2, Lz=1.2, Nx=20, Ny=16, Nz=16, custom_3d_props=smx, spot_dia=0.5,
                                   theta_inc_deg=20.0, phi_inc_deg=30.0, launch_axis='x'), 10, 30_000))
    return cases




def case(name):
    for n, kw, nb, npb in mc_cases():
        if n == name:
            return kw, nb, npb
    raise KeyError(name)
