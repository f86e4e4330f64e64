"""The allocation-free photon-transport entry point (bd_mc_trace_noalloc) gives the same results
as bd_mc_trace. It exists for callers that must not allocate device memory while running (a
fixed-latency control loop, or a host framework that owns all device memory); its scratch lives
in a static device array shared by every call, so this test also checks that a second call in a
row starts from a cleared state. The file is collected last (see conftest.py)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(torch, voxel_mc, dev):
    nx, ny, nz = 24, 24, 30
    mu_a = np.full((nx, ny, nz), 0.8); mu_s = np.full((nx, ny, nz), 14.0)
    g = np.full((nx, ny, nz), 0.88); n = np.full((nx, ny, nz), 1.40)
    mu_a[:, :, :6] = 12.0; n[:, :, :6] = 1.56; mu_s[:, :, 6:12] = 3.0; n[:, :, 6:12] = 1.35
    props = voxel_mc.pack_props(mu_a, mu_s, g, n, dev)
    p = voxel_mc.make_params(Nx=nx, Ny=ny, Nz=nz, Lx=1.2, Ly=1.2, Lz=1.5, n_photons=60_000, spot_dia=0.4,
                             theta_inc_deg=22.0, seed=2024)
    return (nx, ny, nz), props, p


def _outputs(torch, shape, dev):
    nv = shape[0] * shape[1] * shape[2]
    return (torch.zeros(nv, device=dev, dtype=torch.float32), torch.zeros(nv, device=dev, dtype=torch.float32),
            torch.zeros(shape[2], device=dev, dtype=torch.float64),
            torch.zeros(16, device=dev, dtype=torch.float64))


def test_noalloc_entry_point_matches_allocating_one_on_two_calls(gpu):
    """Two calls in a row, the first with more photons (a larger grid: more ledger rows of the
    shared array in use) than the second, each against bd_mc_trace with the same parameters."""
    import torch
    from bug_defense_b200 import _lib, voxel_mc
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    shape, props, p = _setup(torch, voxel_mc, dev)
    lib = _lib.load()
    for n_photons in (200_000, 40_000):
        p.n_photons = n_photons
        A0, L0, z0, led0 = _outputs(torch, shape, dev)
        voxel_mc.trace(p, props, A0, L0, z0, led0)   # existing entry point, bd_mc_trace
        A1, L1, z1, led1 = _outputs(torch, shape, dev)
        rc = lib.bd_mc_trace_noalloc(ctypes.byref(p), _lib.ptr(props), None, _lib.ptr(A1), _lib.ptr(L1),
                                     _lib.ptr(z1), _lib.ptr(led1), _lib.stream_ptr())
        _lib.check(rc, "bd_mc_trace_noalloc")
        torch.cuda.synchronize()
        a, b = led0.cpu().numpy(), led1.cpu().numpy()
        assert a[0] == n_photons
        # same photon streams: counts identical, FP64 weights equal up to summation order
        np.testing.assert_array_equal(a[[0, 10, 11, 12]], b[[0, 10, 11, 12]])
        np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-9)
        # the same photon histories; this entry point sums the absorbed map with FP32 atomics while
        # bd_mc_trace sums it exactly in fixed point, so the maps differ by FP32 rounding of the sums
        np.testing.assert_allclose(A1.cpu().numpy(), A0.cpu().numpy(), rtol=1e-4, atol=1e-6)
        np.testing.assert_allclose(L1.cpu().numpy(), L0.cpu().numpy(), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(z1.cpu().numpy(), z0.cpu().numpy(), rtol=1e-12, atol=1e-9)


def test_noalloc_entry_point_rejects_bad_arguments(gpu):
    import torch
    from bug_defense_b200 import _lib, voxel_mc
    dev = torch.device("cuda", 0)
    shape, props, p = _setup(torch, voxel_mc, dev)
    A1, L1, z1, led1 = _outputs(torch, shape, dev)
    lib = _lib.load()
    rc = lib.bd_mc_trace_noalloc(ctypes.byref(p), _lib.ptr(props), None, None, None, None, _lib.ptr(led1),
                                 _lib.stream_ptr())
    assert rc == _lib.BD_ERR_INVALID_ARG and "required" in _lib.last_error()
