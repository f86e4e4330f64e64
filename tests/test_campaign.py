"""Campaign set-up on the CPU: chromophore spectra, the 24 instance descriptions and the per-wavelength
optics of an instance (no GPU needed)."""
import numpy as np
import pytest

from bug_defense_b200 import campaign as cp


def test_spectra_shapes_follow_the_published_forms():
    nm = np.array(cp.WAVELENGTHS_NM, dtype=float)
    w = cp.water_mua(nm)
    # water: weak in the visible, the 980 nm band above 1064 nm, strong 1470/1940/2940 nm bands
    assert w[0] < w[1] < w[2] < w[4] < w[3] < w[5] < w[6] < w[7]
    assert 1000.0 < w[7] < 2000.0                        # ~12,000 /cm at 2940 nm, in 1/mm
    m = cp.melanin_mua(nm)
    assert np.all(np.diff(m) < 0) and m[0] == pytest.approx(51.9 * 0.9 ** -3.5)
    b = cp.baseline_tissue_mua(nm)
    assert np.all(np.diff(b) <= 0) and b[-1] == pytest.approx(0.0244, rel=1e-3)
    with pytest.raises(ValueError):
        cp.water_mua(100.0)


def test_campaign_has_24_seeded_instances():
    a = cp.campaign_instances(3)
    b = cp.campaign_instances(3)
    assert len(a) == 24 and a == b
    assert {i["wavelength_nm"] for i in a} == set(float(x) for x in cp.WAVELENGTHS_NM)
    assert {i["power"] for i in a} == set(cp.POWERS_W)
    assert all(50.0 <= i["pulse_ms"] <= 400.0 for i in a)
    assert len({i["tissue_seed"] for i in a}) == 24


def test_instance_optics_scale_from_532nm():
    from bug_defense_b200 import workloads
    inst = dict(cp.campaign_instances(0)[1], grid=(8, 8, 128), n_plume_air=8)
    base = workloads.full_coupled_run(inst["tissue_seed"], nx=8, ny=8, nz=128, n_plume_air=8)
    g532 = cp.instance_geometry(dict(inst, wavelength_nm=532.0))
    np.testing.assert_allclose(g532["optical"]["mu_a"], base["optical"]["mu_a"], rtol=1e-12)
    np.testing.assert_allclose(g532["optical"]["mu_s"], base["optical"]["mu_s"], rtol=1e-12)
    g2940 = cp.instance_geometry(dict(inst, wavelength_nm=2940.0))
    tissue = base["optical"]["mu_a"] > 0
    assert np.all(g2940["optical"]["mu_a"][tissue] > 10 * base["optical"]["mu_a"][tissue])
    assert np.all(g2940["optical"]["mu_s"][tissue] < base["optical"]["mu_s"][tissue])
    air = ~tissue
    assert np.all(g2940["optical"]["mu_a"][air] == 0)
    assert g2940["plume_closure"]["wavelength_nm"] == 2940.0
    assert g2940["epochs_on"] == int(round(inst["pulse_ms"]))
