"""Mid-run wavelength switch (run_dual_permutation_suite.py:254-283): intact voxels take the new
optics, ablated voxels keep theirs, the plume takes the new extinction constants, and the next
epoch's MC sees exactly the properties a fresh packing of the new state would give."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_switch_wavelength_repacks_properties(gpu):
    import torch
    from bug_defense_b200 import campaign, voxel_mc
    inst = dict(campaign.campaign_instances(2, grid=(32, 32, 128), n_plume_air=16)[1], n_photons=40_000)
    eng = campaign.make_engine(inst)
    eng.power = 80.0
    eng.step_epochs(8)
    n_void0 = eng.step_epochs(1)["n_void"]
    abl = eng.ablated
    assert abl.sum() > (eng.Nx * eng.Ny * 16)          # a crater below the plume air
    old = {k: eng.optical[k] for k in ("mu_a", "mu_s", "g", "n")}
    geo2 = campaign.instance_geometry(dict(inst, wavelength_nm=1064.0))
    eng.switch_wavelength(1064.0, optical=geo2["optical"], dry_state=geo2["dry_state"], power=60.0)
    torch.cuda.synchronize()
    abl = eng.ablated
    for k in ("mu_a", "mu_s", "g", "n"):
        want = np.where(abl, old[k], geo2["optical"][k])
        np.testing.assert_allclose(eng.optical[k], want, rtol=1e-6)
    assert eng.plume.wavelength == 1064.0 and eng.power == 60.0
    # packed MC properties = a fresh packing of the switched optics with the plume extinction
    pl = eng.plume
    ref = voxel_mc.pack_props(*(eng._opt_t[k] for k in ("mu_a", "mu_s", "g", "n")), eng.dev, plume_mu_ext=pl.mu_ext,
                              flags=eng._flags, ratio_a=pl.ratio_a, ratio_s=pl.ratio_s, g_plume=0.8)
    got = eng._props.view(-1)
    assert torch.allclose(got, ref.view(-1), rtol=1e-6, atol=1e-7)
    # the refresh pass adds no plume and no diagnostics; the run continues normally
    d = eng.step_epochs(2)
    assert d["n_void"] >= n_void0 and abs(d["mc_energy_closure"] - 1.0) < 0.01
