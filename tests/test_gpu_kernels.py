"""GPU parity of the deterministic kernels against fixtures produced by the reference CPU path.

Tolerances: the GPU computes in FP32 and the reference in FP64. Temperatures agree to
<= 1e-4 relative (the stencil bar), enthalpy / damage / char to the reference test's own
absolute bounds (tests/test_gpu_thermal.py:133-136 of the reference: 1e-5)."""
import ctypes
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["thermal_random.npz", "thermal_strata.npz"])
def test_thermal_stencil_matches_reference(gpu, golden, name):
    g = golden(name)
    p = json.loads(str(g["params"]))
    Nx, Ny, Nz = g["T0"].shape
    T = gpu.run_thermal3d_substeps_gpu(g["T0"], g["Q"], g["k"], g["rho"], Nx, Ny, Nz, p["dx"], p["dy"], p["dz"],
                                       p["dt"], 10, p["h_eff"], p["t_amb"], 1)
    assert T.dtype == np.float64 and T.shape == g["T10"].shape
    rel = np.max(np.abs(T - g["T10"]) / np.abs(g["T10"]))
    assert rel <= 1e-4, rel
    if "T1" in g:
        T1 = gpu.run_thermal3d_substeps_gpu(g["T0"], g["Q"], g["k"], g["rho"], Nx, Ny, Nz, p["dx"], p["dy"], p["dz"],
                                            p["dt"], 1, p["h_eff"], p["t_amb"], 1)
        assert np.max(np.abs(T1 - g["T1"]) / np.abs(g["T1"])) <= 1e-5


def test_thermal_context_api(gpu, golden):
    g = golden("thermal_strata.npz")
    p = json.loads(str(g["params"]))
    Nx, Ny, Nz = g["T0"].shape
    ctx = gpu.MetalThermalContext(Nx, Ny, Nz, p["dx"], p["dy"], p["dz"], p["dt"], g["k"], g["rho"], p["h_eff"],
                                  p["t_amb"])
    ctx.set_T(g["T0"]); ctx.set_Q(g["Q"])
    ctx.advance(3, 1); ctx.advance(7, 1)   # odd + odd substep counts exercise the ping-pong
    np.testing.assert_allclose(ctx.get_T(), g["T10"], rtol=1e-4)
    assert float(ctx.get_T_view()[4, 4, 0]) == pytest.approx(g["T10"][4, 4, 0], rel=1e-4)
    ctx.set_T(g["T0"]); ctx.advance(4, 0)  # passive: no source, the field stays at 25 with T_amb 25
    np.testing.assert_allclose(ctx.get_T(), 25.0, atol=1e-4)


@pytest.mark.parametrize("name", ["fused_strata.npz", "fused_random.npz"])
def test_fused_ablation_matches_reference(gpu, golden, name):
    g = golden(name)
    p = json.loads(str(g["params"]))
    Nx, Ny, Nz = g["T0"].shape
    ctx = gpu.MetalAblationContext(Nx, Ny, Nz, p["dx"], p["dy"], p["dz"], p["dt"], p["h_eff"], p["t_amb"], p["t_abl"],
                                   p["t_void"], arrhenius=(p["arr_A"], p["arr_EaR"]),
                                   char_params=(p["char_A"], p["char_EaR"]))
    ctx.set_state(g["T0"], g["H0"], np.zeros_like(g["T0"]), g["chi0"], g["dry"], g["ablated"], g["Q"], g["k"], g["rho"])
    ctx.advance_substeps(p["n"], is_active=1)
    T, H, Om, chi = ctx.get_state()
    assert np.max(np.abs(T - g["T"]) / np.abs(g["T"])) <= 1e-4
    # enthalpy banking amplifies FP32 temperature rounding by rho_cp; bound relative to its scale
    assert np.max(np.abs(H - g["H"])) <= 1e-5 + 1e-4 * np.max(np.abs(g["H"]))
    assert np.max(np.abs(Om - g["Omega"])) <= 1e-5 + 1e-4 * np.max(np.abs(g["Omega"]))
    assert np.max(np.abs(chi - g["chi"])) <= 1e-5
    # masks are inputs here: plateau held exactly at t_abl where it binds
    wet = ~g["dry"] & ~g["ablated"]
    at_plateau = wet & (g["T"] == p["t_abl"])
    assert np.all(T[at_plateau] == np.float32(p["t_abl"]))


def test_plume_transport_matches_reference(gpu, golden):
    g = golden("plume_random.npz")
    p = json.loads(str(g["params"]))
    Nx, Ny, Nz = g["C0"].shape
    tau = -p["dt"] / np.log(p["decay"])
    ctx = gpu.MetalAblationContext(Nx, Ny, Nz, p["dx"], p["dy"], p["dz"], p["dt"], 0.0, 20.0, 100.0, 300.0,
                                   plume_params={'D_xy': p["D_xy"], 'D_z': p["D_z"], 'vz': p["vz"], 'tau_linger': tau},
                                   plume_dt_policy='as_given')
    z = np.zeros((Nx, Ny, Nz))
    ctx.set_state(np.full_like(z, 20.0), z, z, z, np.zeros_like(g["void"]), np.zeros_like(g["void"]), z, z,
                  np.full_like(z, 1e-3), plume=g["C0"], plume_void=g["void"])
    ctx.advance_substeps(p["n"], is_active=0)
    C = ctx.get_plume()
    np.testing.assert_allclose(C, g["C10"], rtol=1e-4, atol=1e-6)
    assert np.all(C[~g["void"]] == 0.0)


def test_plume_anisotropic_point_source(gpu, golden):
    """tests/test_plume.py:230-286 of the reference: ratio val_z/val_x within 1e-3 of the CPU."""
    g = golden("plume_aniso.npz")
    shape = (31, 31, 31)
    ctx = gpu.MetalAblationContext(31, 31, 31, 0.02, 0.02, 0.02, 2e-5, 10.0, 20.0, 100.0, 300.0,
                                   plume_params={'D_xy': 1.0, 'D_z': 4.0, 'vz': 0.0, 'tau_linger': float('inf')},
                                   plume_dt_policy='as_given')
    p0 = np.zeros(shape, np.float32); p0[15, 15, 15] = float(g["delta_mu"])
    z = np.zeros(shape); ones = np.ones(shape, np.uint8)
    ctx.set_state(np.full(shape, 20.0), z, z, z, ones, ones, z, z, z, plume=p0)
    ctx.advance_substeps(20, is_active=1)
    field = ctx.get_plume()
    ref = g["field"]
    np.testing.assert_allclose(field, ref, rtol=1e-4, atol=1e-9)
    assert (field[15, 15, 17] / field[17, 15, 15]) == pytest.approx(ref[15, 15, 17] / ref[17, 15, 15], rel=1e-3)
    assert field[15, 15, 17] > 2.0 * field[17, 15, 15]


def test_plume_leaves_thermal_state_bit_identical(gpu):
    """tests/test_plume.py:182-227 of the reference: the plume channel does not perturb T/H/Omega/chi."""
    Nx, Ny, Nz = 12, 12, 10
    k = np.full((Nx, Ny, Nz), 0.3e-3); rho = np.full((Nx, Ny, Nz), 2.0e-3)
    Q = np.zeros((Nx, Ny, Nz)); Q[4:8, 4:8, 2:6] = 50.0
    dry = np.zeros((Nx, Ny, Nz), np.uint8); abl = np.zeros((Nx, Ny, Nz), np.uint8); abl[5:7, 5:7, 0:3] = 1
    T0 = np.full((Nx, Ny, Nz), 25.0); z = np.zeros((Nx, Ny, Nz))
    args = (Nx, Ny, Nz, 0.03, 0.03, 0.02, 5e-5, 10.0, 20.0, 100.0, 300.0)
    kw = dict(arrhenius=(1e4, 5000.0 / 8.314), char_params=(1e3, 4000.0 / 8.314))
    c1 = gpu.MetalAblationContext(*args, **kw)
    c1.set_state(T0, z, z, z, dry, abl, Q, k, rho)
    c1.advance_substeps(50, is_active=1)
    c2 = gpu.MetalAblationContext(*args, plume_params={'D': 0.5, 'vz': 15.0, 'tau_linger': 0.010}, **kw)
    p = np.zeros((Nx, Ny, Nz), np.float32); p[5:7, 5:7, 1] = 10.0
    c2.set_state(T0, z, z, z, dry, abl, Q, k, rho, plume=p)
    c2.advance_substeps(50, is_active=1)
    for a, b in zip(c1.get_state(), c2.get_state()):
        assert np.max(np.abs(a - b)) == 0.0


@pytest.mark.parametrize("name", ["phase_char.npz", "phase_nochar.npz"])
def test_phase_update_matches_reference(gpu, golden, name):
    """Epoch-end phase kernel through the C ABI (removal off, to_remove mask out)."""
    import torch
    from bug_defense_b200 import _lib
    g = golden(name)
    ins = {k[3:]: g[k] for k in g.files if k.startswith("in_")}
    shape = ins["T"].shape
    dev = torch.device("cuda")
    f = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev).contiguous()
    fields = {k: f(v) for k, v in ins.items() if k not in ("dry", "ablated")}
    flags = torch.tensor((ins["ablated"].astype(np.uint8) * _lib.FLAG_ABLATED) | (ins["dry"].astype(np.uint8) *
                                                                                 _lib.FLAG_DRY), device=dev)
    wet = [f(g[k]) for k in ("wet_mu_a", "wet_k", "wet_rho")]
    keep = []

    def gref(v):
        if np.ndim(v) == 0:
            return _lib.GridRef(None, float(v), 0)
        t = f(v).reshape(-1); keep.append(t)
        return _lib.GridRef(t.data_ptr(), 0.0, 0)

    D = _lib.EngineDesc()
    ph = D.phase
    ph.nx, ph.ny, ph.nz = shape
    ph.single_stage, ph.apply_removal = 0, 0
    ph.t_abl, ph.alpha_max_stable, ph.cs_chi_remove = 100.0, float(g["alpha_max"]), 0.95
    P = _lib.ptr
    ph.T, ph.H_acc, ph.chi = P(fields["T"]), P(fields["H"]), P(fields["chi"])
    ph.mu_a, ph.mu_s, ph.g, ph.n = P(fields["mu_a"]), P(fields["mu_s"]), P(fields["g"]), P(fields["n"])
    ph.k, ph.rho_cp, ph.h_lat = P(fields["k"]), P(fields["rho"]), P(fields["h_lat"])
    ph.wet_mu_a, ph.wet_k, ph.wet_rho_cp = (P(w) for w in wet)
    for key in ("mu_a", "mu_s", "g", "n", "k", "rho_cp", "t_remove"):
        setattr(ph, f"ds_{key}", gref(g[f"ds_{key}"]))
    has_cs = "cs_mu_a" in g.files
    if has_cs:
        ph.has_char_state = ph.has_cs_mu_a = ph.has_cs_mu_s = ph.has_cs_k = ph.has_cs_rho_cp = 1
        for key in ("mu_a", "mu_s", "k", "rho_cp", "t_remove"):
            setattr(ph, f"cs_{key}", gref(float(g[f"cs_{key}"])))
    rem = torch.zeros(shape, dtype=torch.uint8, device=dev)
    ph.flags, ph.to_remove = P(flags), P(rem)
    Talt = torch.zeros_like(fields["T"]); A = torch.zeros_like(fields["T"])
    D.T_alt, D.A, D.voxel_volume, D.dt_epoch = P(Talt), P(A), 1.0, 1e-3
    h = ctypes.c_void_p()
    _lib.call("bd_engine_create", ctypes.byref(D), ctypes.byref(h))
    try:
        _lib.call("bd_engine_epoch_end", h, _lib.stream_ptr())
        torch.cuda.synchronize()
    finally:
        _lib.load().bd_engine_destroy(h)
    # masks: exact, except where the FP32 comparison sits at a threshold
    T = ins["T"]
    near = (np.abs(T - 350.0) < 0.01) | (np.abs(ins["H"] - ins["h_lat"]) < 1e-6 * ins["h_lat"])
    if has_cs:
        near |= np.abs(ins["chi"] - 0.95) < 1e-6
    got_rem = rem.cpu().numpy().astype(bool)
    assert np.all((got_rem == g["out_remove"]) | near)
    got_dry = ((flags & _lib.FLAG_DRY) != 0).cpu().numpy()
    assert np.all((got_dry == g["out_dry"]) | near)
    for k_in, k_out in (("H", "out_H"), ("mu_a", "out_mu_a"), ("mu_s", "out_mu_s"), ("g", "out_g"), ("n", "out_n"),
                        ("k", "out_k"), ("rho", "out_rho")):
        got = fields[k_in].double().cpu().numpy()
        # FP32 interpolation: error relative to the magnitudes interpolated between
        scale = max(np.max(np.abs(g[k_out])), np.max(np.abs(ins[k_in])))
        ok = np.isclose(got, g[k_out], rtol=2e-6, atol=4e-7 * scale) | near
        assert np.all(ok), (k_in, np.max(np.abs(got - g[k_out])))


@pytest.mark.parametrize("shape", [(20, 18, 24), (9, 35, 68)])
def test_plume_tma_path_matches_oracle(gpu, orc, shape):
    """Grids with nz % 4 == 0 take the TMA-staged plume kernel; compare with the FP64 oracle
    (itself pinned to the reference plume step) over 15 steps with drift and decay."""
    rng = np.random.default_rng(sum(shape))
    Nx, Ny, Nz = shape
    vd = rng.uniform(size=shape) < 0.8
    C0 = (rng.uniform(0, 1, shape) * vd).astype(np.float32)
    dx, dy, dz, dt, Dxy, Dz, vz, tau = 0.03, 0.025, 0.02, 1e-5, 1.5, 2.5, 4.0, 0.02
    ctx = gpu.MetalAblationContext(Nx, Ny, Nz, dx, dy, dz, dt, 0.0, 20.0, 100.0, 300.0,
                                   plume_params={'D_xy': Dxy, 'D_z': Dz, 'vz': vz, 'tau_linger': tau},
                                   plume_dt_policy='as_given')
    z = np.zeros(shape)
    ctx.set_state(np.full(shape, 20.0), z, z, z, np.zeros(shape, np.uint8), np.zeros(shape, np.uint8), z, z,
                  np.full(shape, 1e-3), plume=C0, plume_void=vd)
    ctx.advance_substeps(15, is_active=0)
    got = ctx.get_plume()
    C = C0.astype(np.float64); Cn = np.empty_like(C)
    decay = float(np.exp(-dt / tau))
    for _ in range(15):
        orc.diffuse_plume_step(C, Cn, vd, Nx, Ny, Nz, dx, dy, dz, dt, Dxy, Dz, vz, decay)
        C, Cn = Cn, C
    np.testing.assert_allclose(got, C, rtol=1e-4, atol=1e-6)
    assert np.all(got[~vd] == 0.0)


@pytest.mark.parametrize("shape", [(20, 18, 24), (7, 33, 64)])
def test_thermal_tma_path_matches_oracle(gpu, orc, shape):
    """Grids with nz % 4 == 0 take the TMA-staged stencil; compare with the FP64 oracle over 12 steps."""
    rng = np.random.default_rng(7 + sum(shape))
    Nx, Ny, Nz = shape
    T0 = rng.uniform(20, 120, shape); Q = rng.uniform(0, 900, shape)
    k = rng.uniform(2e-4, 6e-4, shape); rho = rng.uniform(1.5e-3, 4e-3, shape)
    dx, dy, dz, dt, h, ta = 0.03, 0.025, 0.02, 2e-5, 15e-6, 20.0
    got = gpu.run_thermal3d_substeps_gpu(T0, Q, k, rho, Nx, Ny, Nz, dx, dy, dz, dt, 12, h, ta, 1)
    T, Tn = T0.copy(), np.empty_like(T0)
    for _ in range(12):
        orc.thermal3d_step_explicit(T, Tn, Q, k, rho, Nx, Ny, Nz, dx, dy, dz, dt, h, ta, 1)
        T, Tn = Tn, T
    assert np.max(np.abs(got - T) / np.abs(T)) <= 1e-5
