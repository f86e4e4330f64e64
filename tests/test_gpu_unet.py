"""The denoiser network on the GPU (bd_unet_*) against the float64 oracle (oracle/unet.py):
forward output, training loss, every layer's weight and bias gradients, and the Adam update.

The oracle rounds the stored activations to bf16 where the GPU stores them, and uses the bf16
weights the tensor cores see, so remaining differences come from FP32 accumulation order and
rounding-boundary flips: the forward map is held to 1% of its scale, gradients to 3% (relative L2
per tensor)."""
import numpy as np
import pytest

from oracle import unet as ou

pytestmark = pytest.mark.gpu

SHAPE = (8, 8, 16)
SCALE = 1e3


def _bf(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(torch.bfloat16).to(torch.float64).numpy()


def _problem(seed=0):
    import torch
    from bug_defense_b200 import voxel_mc
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", 0)
    mu_a = rng.uniform(0.05, 8.0, SHAPE)
    mu_a[:, :, :3] = 0.0                                     # air on top
    mu_s = rng.uniform(1.0, 30.0, SHAPE)
    mu_s[:, :, :3] = 0.0
    g = np.full(SHAPE, 0.9); n = np.full(SHAPE, 1.4)
    flags = np.zeros(SHAPE, np.uint8)
    flags[:, :, :3] = 0x01
    flags[2:5, 2:5, 3:6] = 0x02
    a = (rng.random(SHAPE) * 1e-3 * (mu_a > 0)).astype(np.float32)
    target = (rng.random(SHAPE) * 1e-3 * (mu_a > 0)).astype(np.float32)
    props = voxel_mc.pack_props(mu_a, mu_s, g, n, dev)
    pv = props.view(-1, 4).cpu().numpy()
    mu_a32 = (pv[:, 0] * pv[:, 1]).astype(np.float32)
    mu_s32 = np.maximum(pv[:, 0] - mu_a32, np.float32(0)).astype(np.float32)
    f4, mask = ou.features(a.astype(np.float64), mu_a32.reshape(SHAPE).astype(np.float64),
                           mu_s32.reshape(SHAPE).astype(np.float64), flags, SCALE)
    x16 = _bf(ou.expand_z(f4))
    p = ou.init_params(seed)
    L, _, _ = ou.unpack(p)
    L = [(w, rng.normal(0, 0.05, w.shape[1])) for w, _ in L]
    p32 = ou.pack(L, rng.normal(0, 0.3, 16), 0.05).astype(np.float32)
    # the oracle sees what the kernels see: bf16 convolution weights, fp32 biases and head
    Lq, hw, hb = ou.unpack(p32.astype(np.float64))
    p_or = ou.pack([(_bf(w), b) for w, b in Lq], hw, hb)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    return dict(p32=p32, p_or=p_or, x16=x16, a=a, mask=mask, target=target, props=props, flags=t(flags),
                a_dev=t(a), target_dev=t(target))


def test_network_forward_matches_oracle(gpu):
    from bug_defense_b200 import denoise
    P = _problem(1)
    net = denoise.UNet(SHAPE, training=False, params=P["p32"])
    pred = net.forward(P["a_dev"], P["props"], P["flags"], scale=SCALE).cpu().numpy()
    ref, _ = ou.forward(P["p_or"], P["x16"], P["a"].astype(np.float64), P["mask"], SCALE, bf16=_bf)
    err = np.abs(pred - ref).max()
    assert err <= 1e-2 * np.abs(ref).max(), err
    assert np.all(pred[P["mask"] == 0] == 0)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def test_network_gradients_match_oracle(gpu):
    from bug_defense_b200 import denoise
    P = _problem(2)
    norm = 1.0 / np.prod(SHAPE)
    net = denoise.UNet(SHAPE, training=True, params=P["p32"])
    net.forward_backward(P["a_dev"], P["props"], P["flags"], P["target_dev"], scale=SCALE, loss_norm=norm)
    loss = net.read_loss()
    grads = net.grads().cpu().numpy().astype(np.float64)
    _, cache = ou.forward(P["p_or"], P["x16"], P["a"].astype(np.float64), P["mask"], SCALE, bf16=_bf)
    loss_ref, g_ref = ou.backward(P["p_or"], cache, P["target"].astype(np.float64), norm, bf16=_bf)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    Lg, hwg, hbg = ou.unpack(grads)
    Lr, hwr, hbr = ou.unpack(g_ref)
    for i, ((wg, bg), (wr, br)) in enumerate(zip(Lg, Lr)):
        if i == 0:
            wg, wr = wg[:, :, :12], wr[:, :, :12]
        assert _rel(wg, wr) < 3e-2, (i, _rel(wg, wr))
        assert _rel(bg, br) < 3e-2, (i, _rel(bg, br))
    assert _rel(hwg, hwr) < 1e-2 and abs(hbg - hbr) <= 1e-2 * abs(hbr) + 1e-9


def test_adam_update_and_descent(gpu):
    from bug_defense_b200 import denoise
    P = _problem(3)
    net = denoise.UNet(SHAPE, training=True, params=P["p32"])
    net.forward_backward(P["a_dev"], P["props"], P["flags"], P["target_dev"], scale=SCALE)
    l0 = net.read_loss()
    g = net.grads().cpu().numpy().astype(np.float64)
    net.adam(1e-3)
    p1 = net.params().cpu().numpy().astype(np.float64)
    m = 0.1 * g; v = 0.001 * g * g
    want = P["p32"].astype(np.float64) - 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    np.testing.assert_allclose(p1, want, rtol=1e-5, atol=1e-7)
    for _ in range(40):
        net.forward_backward(P["a_dev"], P["props"], P["flags"], P["target_dev"], scale=SCALE)
        net.adam(1e-3)
    net.forward_backward(P["a_dev"], P["props"], P["flags"], P["target_dev"], scale=SCALE)
    assert net.read_loss() < 0.5 * l0
