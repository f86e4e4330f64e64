"""What the trained denoiser gains over the method without it.

On held-out random craters (seeds never used in training), a 15k-photon absorbed map is scored by
relative L2 against a many-photon reference: the committed network must remove most of the noise
of the raw 15k-photon map and do at least as well as plain Monte Carlo with 10x the photons. The
network's output stays a map of the same physical quantity: zero where nothing absorbs, and its
total absorbed fraction close to the reference's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_network_beats_ten_times_the_photons(gpu):
    from bug_defense_b200 import denoise, workloads
    den = denoise.Denoiser.load()
    rows = []
    for k in range(4):
        s = workloads.crater_sample(910_000 + k)
        ref, props, _ = denoise.mc_map(s, 30_000_000, 100 + k)
        lo, _, _ = denoise.mc_map(s, denoise.LO_PHOTONS, 200 + k, props=props)
        plain, _, _ = denoise.mc_map(s, 10 * denoise.LO_PHOTONS, 300 + k, props=props)
        out = den(lo, props, s["flags"])
        mu_a = s["mu_a"]
        assert float(out[mu_a == 0].abs().max()) == 0.0
        assert abs(float(out.double().sum() / ref.double().sum()) - 1.0) < 0.05
        rows.append((denoise.relative_l2(lo, ref), denoise.relative_l2(out, ref), denoise.relative_l2(plain, ref)))
    noisy, den_err, plain_err = np.mean(rows, axis=0)
    print(f"DENOISER rel L2 noisy {noisy:.4f} denoised {den_err:.4f} plain10x {plain_err:.4f}")
    assert den_err < 0.4 * noisy
    assert den_err <= plain_err
