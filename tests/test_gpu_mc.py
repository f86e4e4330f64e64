"""GPU photon transport vs the reference CPU MC (statistics recorded from the reference) and vs
the FP64 oracle on the SAME Philox photon streams (correlated sampling: much tighter)."""
import numpy as np
import pytest

from test_oracle_golden import MC_CASES, _mc_case

pytestmark = pytest.mark.gpu


# The reference's 400k-photon sample of the 45 deg refraction slab (verification_benchmarks.py:131-151)
# records T = 0.30701 +- 0.00041, 3.4 of its standard errors above the exact value 0.30561 (Fresnel
# entrance split, Beer-Lambert along the refracted path, no Fresnel at the far face); the FP64
# oracle with 8e6 photons lands on the exact value. That case is judged against the exact T and A.
EXACT = {"oblique_v1f": ("oblique45_T", "Transmission", "Absorption")}
GPU_FACTOR = 10   # GPU photons per reference photon: the combined SE is the reference's x sqrt(1.1)


@pytest.mark.parametrize("name", MC_CASES)
def test_gpu_mc_matches_reference_statistics(gpu, orc, golden, name):
    """R / A / T / lateral within 3 combined standard errors of the reference's batch statistics."""
    stats = golden("mc_stats.json")[name]
    an = golden("mc_stats.json")["analytic"]
    kw, nb, npb = _mc_case(name)
    n = nb * npb
    r = gpu.run_voxel_mc3d(n_photons=GPU_FACTOR * n, base_seed=4321, **kw)
    assert r["engine"] == "gpu"
    means = {key: mean for key, (mean, se) in stats["stats"].items()}
    if name in EXACT:
        key_an, key_t, key_a = EXACT[name]
        means[key_t] = an[key_an]
        means[key_a] = 1.0 - an[key_an] - an["oblique45_Rspec"]
    for key, (_, se) in stats["stats"].items():
        # deterministic channels (R_spec, and channels no photon reaches) differ by FP32 rounding only
        tol = 3.0 * se * np.sqrt(1.0 + 1.0 / GPU_FACTOR) + 1e-6
        assert abs(r["spectro_raw"][key] - means[key]) <= tol, (key, r["spectro_raw"][key], means[key], tol)
    # FP64 ledger closes to round-off once roulette and truncation are accounted
    assert abs(r["ledger_closure"] - 1.0) < 1e-9
    assert abs(r["energy_closure"] - 1.0) < 0.01
    axis = (0, 1) if kw.get("launch_axis", "z") == "z" else (1, 2)
    prof = r["A_3d"].sum(axis=axis)
    ref = np.array(stats["depth_profile"])
    if ref.sum() > 0:
        assert np.corrcoef(prof, ref)[0, 1] > 0.995
    # same photon streams in the FP64 oracle: FP32 vs FP64 arithmetic only
    g = gpu.run_voxel_mc3d(n_photons=n, base_seed=4321, **kw)
    o = orc.run_voxel_mc3d(n_photons=n, seed=4321, **kw)
    for key in stats["stats"]:
        assert abs(g["spectro_raw"][key] - o["spectro_raw"][key]) < 2e-3, key
    assert np.allclose(g["A_3d"].sum(), o["A_3d"].sum(), rtol=2e-3)


def test_gpu_mc_specular_is_exact_fresnel(gpu, golden):
    """tests/test_gpu_mc.py:105-114 of the reference: R_spec equals the unpolarised Fresnel value."""
    an = golden("mc_stats.json")["analytic"]
    kw, _, _ = _mc_case("oblique_v1f")
    r = gpu.run_voxel_mc3d(n_photons=200_000, base_seed=3, **kw)
    assert r["spectro_raw"]["R_spec"] == pytest.approx(an["oblique45_Rspec"], abs=2e-6)
    T = an["oblique45_T"]
    assert abs(r["spectro_raw"]["Transmission"] - T) < 4 * np.sqrt(T * (1 - T) / 2e5)


def test_gpu_mc_canonical_slab(gpu, golden):
    """V1a/V1b of the reference verification tier: Rd 0.09739, Tt 0.66096 (van de Hulst)."""
    an = golden("mc_stats.json")["analytic"]
    kw, _, _ = _mc_case("slab_v1")
    r = gpu.run_voxel_mc3d(n_photons=1_000_000, base_seed=11, **kw)["spectro_raw"]
    se = golden("mc_stats.json")["slab_v1"]["stats"]
    assert abs(r["R_diff"] - an["slab_matched_Rd"]) < 3 * se["R_diff"][1] * np.sqrt(0.5) + 1e-4
    assert abs(r["Transmission"] - an["slab_matched_Tt"]) < 3 * se["Transmission"][1] * np.sqrt(0.5) + 1e-4


def test_gpu_mc_batches_fold_into_fp64(gpu):
    """Photon counts above one launch are folded into an FP64 map; totals stay consistent."""
    from bug_defense_b200 import voxel_mc
    cube = {k: np.full((8, 8, 10), v) for k, v in (('mu_a', 1.0), ('mu_s', 5.0), ('g', 0.8), ('n', 1.4))}
    old = voxel_mc.PHOTON_BATCH
    voxel_mc.PHOTON_BATCH = 50_000
    try:
        r = gpu.run_voxel_mc3d(n_photons=175_000, base_seed=9, Lx=1, Ly=1, Lz=1, Nx=8, Ny=8, Nz=10,
                               custom_3d_props=cube, spot_dia=0.3)
    finally:
        voxel_mc.PHOTON_BATCH = old
    one = gpu.run_voxel_mc3d(n_photons=175_000, base_seed=9, Lx=1, Ly=1, Lz=1, Nx=8, Ny=8, Nz=10,
                             custom_3d_props=cube, spot_dia=0.3)
    # identical photon streams (offsets continue across batches): same totals to FP32 tally noise
    assert r["A_3d"].sum() == pytest.approx(one["A_3d"].sum(), rel=1e-5)
    assert r["ledger"][0] == 175_000 and abs(r["ledger_closure"] - 1) < 1e-9


def test_gpu_mc_zero_photons_and_bad_args(gpu):
    r = gpu.run_voxel_mc3d(n_photons=0, Nx=4, Ny=4, Nz=4, Lx=1, Ly=1, Lz=1)
    assert r["A_3d"].sum() == 0.0
    with pytest.raises(ValueError):
        gpu.run_voxel_mc3d(n_photons=10, Nx=4, Ny=4, Nz=4, Lx=1, Ly=1, Lz=1, custom_3d_props={
            'mu_a': np.zeros((3, 4, 4)), 'mu_s': np.zeros((3, 4, 4)), 'g': np.zeros((3, 4, 4)), 'n': np.ones((3, 4, 4))})
