"""Pin the oracle (oracle/orc.c) against fixtures produced by the reference itself.

Deterministic kernels must agree to FP64 round-off; the Monte Carlo statistically (3.5 combined
standard errors: the reference CPU MC uses numba's unseeded np.random) and against the
analytic / canonical values of the reference's verification tier.
"""
import json

import numpy as np
import pytest


def test_philox_known_answers(orc):
    # Random123 known-answer vectors for Philox-4x32-10
    assert orc.philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert orc.philox4x32_10([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert orc.philox4x32_10([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


@pytest.mark.parametrize("name", ["thermal_random.npz", "thermal_strata.npz"])
def test_thermal_step_matches_reference(orc, golden, name):
    g = golden(name)
    p = json.loads(str(g["params"]))
    T = g["T0"].copy(); Tn = np.empty_like(T)
    Nx, Ny, Nz = T.shape
    for s in range(10):
        orc.thermal3d_step_explicit(T, Tn, g["Q"], g["k"], g["rho"], Nx, Ny, Nz, p["dx"], p["dy"], p["dz"], p["dt"],
                                    p["h_eff"], p["t_amb"], 1)
        T, Tn = Tn, T
        if s == 0 and "T1" in g:
            np.testing.assert_allclose(T, g["T1"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(T, g["T10"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("name", ["fused_strata.npz", "fused_random.npz"])
def test_fused_substeps_match_reference(orc, golden, name):
    g = golden(name)
    p = json.loads(str(g["params"]))
    T = g["T0"].copy(); Tn = np.empty_like(T); H = g["H0"].copy(); Om = np.zeros_like(T); chi = g["chi0"].copy()
    Nx, Ny, Nz = T.shape
    for _ in range(p["n"]):
        orc.thermal3d_step_explicit(T, Tn, g["Q"], g["k"], g["rho"], Nx, Ny, Nz, p["dx"], p["dy"], p["dz"], p["dt"],
                                    p["h_eff"], p["t_amb"], 1)
        orc.apply_latent_heat_plateau(Tn, H, g["rho"], g["ablated"], p["t_abl"], Nx, Ny, Nz, g["dry"], p["t_void"])
        orc.accumulate_arrhenius(Tn, Om, g["ablated"], p["arr_A"], p["arr_EaR"], p["dt"], Nx, Ny, Nz)
        orc.accumulate_char(Tn, chi, g["dry"], g["ablated"], p["char_A"], p["char_EaR"], p["dt"], Nx, Ny, Nz)
        T, Tn = Tn, T
    np.testing.assert_allclose(T, g["T"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(H, g["H"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(Om, g["Omega"], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(chi, g["chi"], rtol=1e-10, atol=1e-13)


def test_plume_step_matches_reference(orc, golden):
    g = golden("plume_random.npz")
    p = json.loads(str(g["params"]))
    C = g["C0"].astype(np.float64); Cn = np.empty_like(C)
    Nx, Ny, Nz = C.shape
    for _ in range(p["n"]):
        orc.diffuse_plume_step(C, Cn, g["void"], Nx, Ny, Nz, p["dx"], p["dy"], p["dz"], p["dt"], p["D_xy"], p["D_z"],
                               p["vz"], p["decay"])
        C, Cn = Cn, C
    # the reference field is float32: agreement to float32 round-off
    np.testing.assert_allclose(C, g["C10"], rtol=2e-5, atol=1e-6)
    assert np.all(C[~g["void"]] == 0.0)


@pytest.mark.parametrize("name", ["phase_char.npz", "phase_nochar.npz"])
def test_phase_update_matches_reference(orc, golden, name):
    g = golden(name)
    ins = {k[3:]: g[k].copy() for k in g.files if k.startswith("in_")}
    ds = {k[3:]: g[k] for k in g.files if k.startswith("ds_")}
    cs = {k[3:]: float(g[k]) for k in g.files if k.startswith("cs_")} or None
    dry = ins["dry"].copy()
    rem = orc.update_phase_properties(ins["H"], ins["h_lat"], ins["T"], ins["chi"], dry, ins["ablated"],
                                      ins["mu_a"], ins["mu_s"], ins["g"], ins["n"], ins["k"], ins["rho"],
                                      g["wet_mu_a"], g["wet_k"], g["wet_rho"], ds, cs, 0.95, float(g["alpha_max"]))
    np.testing.assert_array_equal(rem, g["out_remove"])
    np.testing.assert_array_equal(dry, g["out_dry"])
    for k_in, k_out in (("H", "out_H"), ("mu_a", "out_mu_a"), ("mu_s", "out_mu_s"), ("g", "out_g"), ("n", "out_n"),
                        ("k", "out_k"), ("rho", "out_rho")):
        np.testing.assert_allclose(ins[k_in], g[k_out], rtol=1e-12, atol=1e-15, err_msg=k_in)


# --------------------------------------------------------------------------------------
def _mc_case(name):
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent / "golden"))
    import importlib
    mg = importlib.import_module("mc_cases")
    return mg.case(name)


MC_CASES = ["multilayer_oblique", "homogeneous_cube", "slab_v1", "fresnel_slab_v1c", "oblique_v1f",
            "semi_infinite_v2b", "tophat", "kim_exp_disk", "kim_gauss_disk_rmax", "launch_x"]


@pytest.mark.parametrize("name", MC_CASES)
def test_oracle_mc_matches_reference_statistics(orc, golden, name):
    stats = golden("mc_stats.json")[name]
    kw, nb, npb = _mc_case(name)
    n = nb * npb
    r = orc.run_voxel_mc3d(n_photons=n, seed=1234, **kw)
    for key, (mean, se) in stats["stats"].items():
        # oracle SE for the same photon count equals the batch SE of the golden (same n)
        tol = 3.5 * np.sqrt(2.0) * se + 1e-9
        assert abs(r["spectro_raw"][key] - mean) <= tol, (key, r["spectro_raw"][key], mean, tol)
    led = r["ledger"]
    exact = (led[1] + led[2] + led[3] + led[4] + led[5] + led[6] + led[9] + led[8] - led[7]) / led[0]
    assert abs(exact - 1.0) < 1e-9
    prof = r["A_3d"].sum(axis=(0, 1) if kw.get("launch_axis", "z") == "z" else (1, 2))
    ref = np.array(stats["depth_profile"])
    if ref.sum() > 0:
        assert np.corrcoef(prof, ref)[0, 1] > 0.995


def test_oracle_mc_analytic_values(orc, golden):
    an = golden("mc_stats.json")["analytic"]
    kw, nb, npb = _mc_case("fresnel_slab_v1c")
    r = orc.run_voxel_mc3d(n_photons=400_000, seed=7, **kw)["spectro_raw"]
    assert r["R_spec"] == pytest.approx(an["fresnel_slab_Rspec"], abs=1e-12)
    assert abs(r["Transmission"] - an["fresnel_slab_T"]) < 4 * np.sqrt(an["fresnel_slab_T"] * (1 - an["fresnel_slab_T"]) / 4e5)
    assert abs(r["R_diff"] - an["fresnel_slab_Rd"]) < 4 * np.sqrt(an["fresnel_slab_Rd"] * (1 - an["fresnel_slab_Rd"]) / 4e5)
    kw, nb, npb = _mc_case("oblique_v1f")
    r = orc.run_voxel_mc3d(n_photons=400_000, seed=8, **kw)["spectro_raw"]
    assert r["R_spec"] == pytest.approx(an["oblique45_Rspec"], abs=1e-12)
    assert abs(r["Transmission"] - an["oblique45_T"]) < 4 * np.sqrt(an["oblique45_T"] * (1 - an["oblique45_T"]) / 4e5)
    kw, nb, npb = _mc_case("slab_v1")
    r = orc.run_voxel_mc3d(n_photons=500_000, seed=9, **kw)["spectro_raw"]
    se = golden("mc_stats.json")["slab_v1"]["stats"]
    assert abs(r["R_diff"] - an["slab_matched_Rd"]) < 3 * np.sqrt(2) * se["R_diff"][1] + 1e-5
    assert abs(r["Transmission"] - an["slab_matched_Tt"]) < 3 * np.sqrt(2) * se["Transmission"][1] + 1e-5


def test_oracle_engine_matches_reference_engine(orc, golden):
    """oracle/engine.py restates CoupledAblationEngine (CPU path); same fixed source -> same run."""
    from oracle.engine import OracleEngine
    g = golden("engine_fixedQ.npz")
    cfg = json.loads(str(g["cfg"]))
    cs = json.loads(str(g["char_state"]))
    pl = {k: (float('inf') if v == 'inf' else v) for k, v in json.loads(str(g["plume"])).items()}
    opt = {k: g[f"in_{k}"] for k in ("mu_a", "mu_s", "g", "n")}
    ds = {'mu_a': g["in_mu_a"].copy(), 'mu_s': g["in_mu_s"].copy(), 'g': g["in_g"].copy(), 'n': g["in_n"].copy(),
          'k': g["in_k"].copy(), 'rho_cp': g["in_rho"].copy(), 't_remove': 350.0}
    eng = OracleEngine(optical_props=opt, k_grid=g["in_k"], rho_cp_grid=g["in_rho"], h_lat_grid=g["in_h_lat"],
                       Lx=cfg["Lx"], Ly=cfg["Ly"], Lz=cfg["Lz"], power=cfg["power"], spot_dia=cfg["spot_dia"],
                       t_abl=cfg["t_abl"], t_ambient=cfg["t_ambient"], dt_epoch=cfg["dt_epoch"], dt_sub=cfg["dt_sub"],
                       n_photons=cfg["n_photons"], h_eff=cfg["h_eff"], dry_state=ds, char_state=cs, plume_closure=pl,
                       initial_dry_mask=g["in_dry"], initial_ablated_mask=g["in_ablated"],
                       air_gap_range=tuple(cfg["air_gap_range"]), wavelength_nm=cfg["wavelength_nm"])
    diag = []
    for ep in range(cfg["epochs_on"] + cfg["epochs_off"]):
        if ep == cfg["epochs_on"]:
            eng.power = 0.0
        d = eng.step_epoch(absorbed_map=g["in_A"])
        diag.append([d['epoch'], d['n_new'], d['absorbed_frac'], d['plume_transmission'], d['plume_tau'],
                     d['plume_peak_mu_a'], d['plume_mean_mu_a']])
        e = ep + 1
        if e in set(int(x) for x in g["snap_epochs"]):
            np.testing.assert_array_equal(eng.ablated, g[f"ep{e}_ablated"])
            np.testing.assert_array_equal(eng.dry, g[f"ep{e}_dry"])
            np.testing.assert_allclose(eng.T, g[f"ep{e}_T"], rtol=1e-9, atol=1e-9)
            np.testing.assert_allclose(eng.chi, g[f"ep{e}_chi"], rtol=1e-9, atol=1e-12)
            np.testing.assert_allclose(eng.plume['raw'], g[f"ep{e}_plume"], rtol=1e-5, atol=1e-6)
            np.testing.assert_allclose(eng.ablation_time, g[f"ep{e}_ablation_time"], atol=1e-12)
    diag = np.array(diag)
    np.testing.assert_array_equal(diag[:, :2], g["diag"][:, :2])
    np.testing.assert_allclose(diag[:, 2:], g["diag"][:, 2:], rtol=1e-5, atol=1e-7)
