"""Absorbed-power maps against 10^8-photon FP64 maps of the reference CPU Monte Carlo.

Fixtures: tests/golden/mc_ref_<seed>.npz, made by tests/golden/make_mc_ref_map.py, which runs the
reference's run_voxel_mc3d(engine='cpu') (numba, FP64 accumulation, voxel_mc_3d.py:377-380) with
10^8 photons in 10 batches on two held-out denoiser craters (workloads.crater_sample) of the
full-resolution 200x200x128 stack, 22 deg Gaussian beam of 0.5 mm.

  * 10^8 GPU photons (FP32 transport, exact fixed-point tally, FP64 ledger): the reflected,
    absorbed, transmitted and lateral fractions within 3 combined standard errors of the
    reference's batch statistics, and a per-voxel relative L2 distance to the reference map that
    is no larger than the Monte Carlo noise of the two maps (estimated from two independent GPU
    halves): no FP32 bias above the noise of 10^8 photons.
  * The plain 150k-photon epoch map and the denoised 15k-photon map (the trained network), each
    scored by relative L2 against the reference map over several photon seeds and reported; the
    network must remove at least half of the 15k-photon map's distance to the FP64 oracle. Whether
    it also beats the plain 150k-photon map depends on the crater (reported, not asserted).
The geometry is built on the CPU exactly as for the fixture and moved to the GPU.
"""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEEDS = (900_000, 900_005)
KEYS = ("R_diff", "Absorption", "Transmission", "Lateral_loss")


def load_ref(golden, seed):
    z = golden(f"mc_ref_{seed}.npz")
    meta = json.loads(str(z["meta"]))
    return z["q"], meta


def rel_l2_vs_ref(a, q, meta) -> float:
    """||a - ref|| / ||ref|| over the whole grid; ref = q * scale inside the stored box, 0 outside."""
    import torch
    lo, hi = meta["lo"], meta["hi"]
    a = a.double()
    ref = torch.as_tensor(q.astype(np.float64), device=a.device) * meta["scale"]
    inside = a[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
    d2 = float(((inside - ref) ** 2).sum()) + float((a ** 2).sum() - (inside ** 2).sum())
    return float(np.sqrt(d2 / meta["norm2"]))


def _sample(seed):
    import torch
    from bug_defense_b200 import workloads
    s = workloads.crater_sample(seed, device="cpu")
    dev = torch.device("cuda", torch.cuda.current_device())
    return {k: (v.to(dev) if isinstance(v, torch.Tensor) else v) for k, v in s.items()}


@pytest.mark.parametrize("seed", SEEDS)
def test_1e8_photon_map_matches_reference_fp64_map(gpu, golden, seed):
    from bug_defense_b200 import _lib, denoise
    q, meta = load_ref(golden, seed)
    s = _sample(seed)
    assert list(s["shape"]) == meta["shape"]
    half = meta["n_photons"] // 2
    a1, props, led1 = denoise.mc_map(s, half, 31 * seed + 1)
    a2, _, led2 = denoise.mc_map(s, half, 31 * seed + 2, props=props)
    a = 0.5 * (a1 + a2)
    led = (led1 + led2).cpu().numpy()
    n = float(meta["n_photons"])
    closure = (led[1:7].sum() + led[8] + led[9] - led[7]) / led[0]
    assert led[0] == n and abs(closure - 1.0) < 1e-9
    frac = dict(R_diff=led[_lib.LEDGER_DIFFUSE] / n, Transmission=led[_lib.LEDGER_TRANSMITTED] / n,
                Lateral_loss=led[_lib.LEDGER_LATERAL] / n,
                Absorption=(led[_lib.LEDGER_ABSORBED] + led[_lib.LEDGER_ABSORBED_VOID]) / n)
    report = dict(seed=seed, fractions={})
    for key in KEYS:
        st = meta["spectro"][key]
        # binomial standard error of the GPU fraction at the same photon count
        se_g = np.sqrt(max(frac[key] * (1 - frac[key]), 1e-30) / n)
        se = np.hypot(st["se"], se_g)
        report["fractions"][key] = [frac[key], st["mean"], float((frac[key] - st["mean"]) / se)]
        assert abs(frac[key] - st["mean"]) <= 3.0 * se, (key, frac[key], st["mean"], se)
    rel = rel_l2_vs_ref(a, q, meta)
    # one 5e7-photon half against the other differs by sqrt(2) sigma(5e7) = 2 sigma(1e8); the GPU
    # 1e8 map against the reference 1e8 map then differs by sqrt(2) sigma(1e8) when neither is biased
    halves = float((a1.double() - a2.double()).norm() / a.double().norm())
    expect = halves / np.sqrt(2.0)
    report.update(rel_l2_gpu_1e8_vs_ref=rel, expected_noise=expect)
    print("REFMAP " + json.dumps(report))
    assert rel <= 1.25 * expect + 2e-4, (rel, expect)


@pytest.mark.parametrize("seed", SEEDS)
def test_denoised_and_plain_maps_against_fp64_oracle(gpu, golden, seed):
    from bug_defense_b200 import denoise
    q, meta = load_ref(golden, seed)
    s = _sample(seed)
    den = denoise.Denoiser.load()
    plain, noisy, out = [], [], []
    props = None
    for r in range(4):
        a_pl, props, _ = denoise.mc_map(s, 150_000, 1000 * seed + 2 * r, props=props)
        a_lo, _, _ = denoise.mc_map(s, denoise.LO_PHOTONS, 1000 * seed + 2 * r + 1, props=props)
        plain.append(rel_l2_vs_ref(a_pl, q, meta))
        noisy.append(rel_l2_vs_ref(a_lo, q, meta))
        out.append(rel_l2_vs_ref(den(a_lo, props, s["flags"]), q, meta))
    res = dict(seed=seed, plain_150k=float(np.mean(plain)), noisy_15k=float(np.mean(noisy)),
               denoised_15k=float(np.mean(out)))
    print("REFMAP " + json.dumps(res))
    assert res["denoised_15k"] < 0.5 * res["noisy_15k"], res
