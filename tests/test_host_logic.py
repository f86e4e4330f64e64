"""Host-side logic that needs no GPU: launch-parameter derivation, layer rasterisation,
plume dt policy, phase map, plume parameter tables, engine argument validation."""
import math

import numpy as np
import pytest


def test_mc_params_follow_reference_derivation():
    from bug_defense_b200.voxel_mc import make_params
    p = make_params(Nx=20, Ny=30, Nz=40, Lx=2.0, Ly=3.0, Lz=1.0, n_photons=1000, spot_dia=0.4, theta_inc_deg=30.0,
                    phi_inc_deg=45.0, beam_center=(1.0, 1.2), seed=5)
    th, ph = math.radians(30), math.radians(45)
    # voxel_mc_3d.py:382-397, :612-618
    assert p.init_ux == pytest.approx(math.sin(th) * math.cos(ph))
    assert p.init_uz == pytest.approx(math.cos(th))
    assert p.cos_th_safe == pytest.approx(math.cos(th))
    assert p.sigma_axis == pytest.approx(0.1) and p.beam_radius == pytest.approx(0.2)
    assert (p.x_center, p.y_center) == pytest.approx((1.0, 1.2))
    assert p.max_events == 10_000_000 and p.options & 1
    px = make_params(Nx=20, Ny=30, Nz=40, Lx=2.0, Ly=3.0, Lz=1.0, n_photons=1, launch_axis='x', theta_inc_deg=89.9)
    assert px.launch_axis == 1 and px.cos_th_safe == pytest.approx(0.05)   # CPU clamp, voxel_mc_3d.py:386
    pm = make_params(Nx=2, Ny=2, Nz=2, Lx=1, Ly=1, Lz=1, n_photons=1, theta_inc_deg=89.9, semantics='metal')
    assert pm.cos_th_safe == pytest.approx(max(math.cos(math.radians(89.9)), 1e-6), rel=1e-5)
    assert pm.max_events == 50_000
    with pytest.raises(ValueError):
        make_params(Nx=2, Ny=2, Nz=2, Lx=1, Ly=1, Lz=1, n_photons=1, beam_profile='nope')
    with pytest.raises(ValueError):
        make_params(Nx=2, Ny=2, Nz=2, Lx=1, Ly=1, Lz=1, n_photons=1, launch_axis='y')


def test_layers_to_grids_cell_centre_rule():
    from bug_defense_b200.voxel_mc import layers_to_grids
    layers = [{'z_end': 0.06, 'mu_a': 5.0, 'mu_s': 10.0, 'g': 0.9, 'n': 1.5},
              {'z_end': 0.2, 'mu_a': 1.0, 'mu_s': 2.0, 'g': 0.8, 'n': 1.3}]
    mu_a, mu_s, g, n = layers_to_grids(layers, 2, 2, 10, 1.0, 1.0, 0.3)
    # cell centres 0.015, 0.045 (layer 0), 0.075..0.195 (layer 1), 0.225+ untouched
    assert list(mu_a[0, 0]) == [5.0, 5.0, 1.0, 1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0]
    assert n[0, 0, 9] == 1.0


def test_plume_policy_matches_oracle_rules():
    import oracle
    from bug_defense_b200 import _lib
    from bug_defense_b200.ablation import plume_params_struct
    for pol in ('as_given', 'metal', 'subcycle'):
        for D, vz in ((1.0, 0.0), (10.0, 0.0), (50.0, 5.0)):
            p = plume_params_struct((8, 8, 8), 0.015, 0.015, 0.015, 5e-5, D, D, vz, float('inf'), pol)
            n = __import__('ctypes').c_int(0); dt = __import__('ctypes').c_float(0)
            assert _lib.load().bd_plume_steps_per_substep(__import__('ctypes').byref(p), __import__('ctypes').byref(n),
                                                          __import__('ctypes').byref(dt)) == 0
            n_o, dt_o, dec = oracle.plume_policy(5e-5, 0.015, 0.015, 0.015, D, D, vz, float('inf'), pol)
            assert n.value == n_o
            assert dt.value == pytest.approx(dt_o, rel=1e-6)
            if pol == 'subcycle':
                # the sub-step is FTCS-stable: every stencil coefficient stays >= 0
                rate = 2 * (2 * D / 0.015 ** 2 + D / 0.015 ** 2) + vz / 0.015
                assert dt_o * rate <= 1.0


def test_phase_map_matches_reference_rules():
    from bug_defense_b200.phase import compute_phase_map
    T = np.array([20.0, 99.6, 50.0, 400.0, 30.0]); chi = np.array([0, 0, 0.2, 0.5, 0.0])
    dry = np.array([0, 0, 1, 1, 0], bool); abl = np.array([0, 0, 0, 1, 0], bool); H = np.array([0, 0, 0, 0, 0.1])
    ph = compute_phase_map(T, chi, dry, abl, H)
    assert list(ph) == [0, 2, 1, 3, 2]
    gap = np.array([0, 1, 0, 0, 0], bool)
    assert list(compute_phase_map(T, chi, dry, abl, H, is_air_gap=gap)) == [0, 3, 1, 3, 2]


def test_plume_field_parameters_follow_table():
    from bug_defense_b200.plume import PlumeField, from_closure
    p = PlumeField((4, 4, 4), wavelength_nm=532)
    assert p.mu_max == pytest.approx(1.275 + 0.80)
    assert p.delta_mu == pytest.approx(0.63)
    assert p.ratio_a == pytest.approx(1.275 / 2.075)
    q = PlumeField((4, 4, 4), wavelength_nm=777, mu_a_max=1.0, delta_mu_per_voxel=2.0)
    assert q.mu_max == pytest.approx(1.15) and q.delta_mu == 2.0
    c = from_closure({'model': 'diffusion', 'D_xy': 1.0, 'D_z': 2.0, 'v_drift': 0.0, 'tau_linger_s': float('inf'),
                      'blast_expansion': False}, (4, 4, 4), 0.015, 0.015, 0.015, 1470.0, None)
    assert (c.D_xy, c.D_z, c.v_drift) == (1.0, 2.0, 0.0) and c.mu_max == pytest.approx(0.65)
    with pytest.raises(NotImplementedError):
        PlumeField((4, 4, 4), model='separable')


def test_gpu_only_build_rejects_cpu_engine_and_missing_device():
    import torch
    from bug_defense_b200 import voxel_mc
    with pytest.raises(ValueError):
        voxel_mc.run_voxel_mc3d(n_photons=10, engine='cpu')
    with pytest.raises(ValueError):
        voxel_mc.run_voxel_mc3d(n_photons=10, engine='bogus')
    if not torch.cuda.is_available():
        # the product has no CPU fallback: without a device it raises
        with pytest.raises(RuntimeError):
            voxel_mc.run_voxel_mc3d(n_photons=10, engine='gpu', Nx=4, Ny=4, Nz=4)


def test_engine_wait_hooks_run_once_each_and_drop_dead_owners():
    """Host work registered with an engine (the Recorder's slot unpacking) runs each time the engine
    is about to block on an epoch's diagnostics; a hook whose owner was collected is dropped."""
    import gc
    import weakref
    from bug_defense_b200.coupled import CoupledAblationEngine

    calls = []

    class Owner:
        def __init__(self, tag):
            self.tag = tag

        def hook(self):
            calls.append(self.tag)

    eng = object.__new__(CoupledAblationEngine)      # host logic only: no device state
    eng._wait_hooks = []
    a, b = Owner("a"), Owner("b")
    eng._wait_hooks += [weakref.WeakMethod(a.hook), weakref.WeakMethod(b.hook)]
    eng._run_wait_hooks()
    assert calls == ["a", "b"]
    del b
    gc.collect()
    eng._run_wait_hooks()
    assert calls == ["a", "b", "a"] and len(eng._wait_hooks) == 1


def test_layered_grids_upload_as_columns_with_the_same_bits():
    """to_dev sends a grid that is one z column broadcast over x and y as that column and expands it
    on the device; any grid that differs anywhere (one bit, -0.0 against 0.0) is copied whole."""
    import torch
    from bug_defense_b200 import _device
    from bug_defense_b200._device import slice_column, to_dev
    rng = np.random.default_rng(3)
    nx, ny, nz = 48, 40, 64
    col = rng.normal(size=nz)
    col[5] = np.nan
    col[7] = -0.0
    layered = np.broadcast_to(col, (nx, ny, nz)).copy()
    assert slice_column(layered) is not None
    assert slice_column(np.broadcast_to(col, (nx, ny, nz))) is not None      # a broadcast view
    for ix, iy, kz in ((0, 1, 3), (nx - 1, ny - 1, nz - 1), (17, 23, 7), (nx // 2, ny // 2, 0)):
        other = layered.copy()
        other[ix, iy, kz] = 0.0 if kz == 7 else np.nextafter(other[ix, iy, kz], np.inf)
        assert slice_column(other) is None, (ix, iy, kz)
    assert slice_column(layered[:, :, ::2]) is None                           # not C-contiguous
    assert slice_column(np.ones((4, 4, 8))) is None                           # below the size floor
    mask = np.zeros((nx, ny, nz), bool)
    mask[:, :, 10:20] = True
    assert np.array_equal(slice_column(mask), mask[0, 0])
    before = dict(_device.upload_stats)
    for arr, dt in ((layered, torch.float64), (layered, torch.float32), (mask, torch.bool), (mask, torch.uint8),
                    (rng.normal(size=(nx, ny, nz)), torch.float64)):
        t = to_dev(arr, torch.device("cpu"), dt)
        want = torch.from_numpy(np.ascontiguousarray(arr)).to(dt)
        assert t.shape == arr.shape and t.dtype == dt and t.is_contiguous()
        assert torch.equal(t.view(torch.uint8), want.contiguous().view(torch.uint8))
    assert _device.upload_stats["column_grids"] - before["column_grids"] == 4
    assert _device.upload_stats["full_grids"] - before["full_grids"] == 1
    assert _device.upload_stats["bytes"] - before["bytes"] == 2 * nz * 8 + 2 * nz + nx * ny * nz * 8
