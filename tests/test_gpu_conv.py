"""Denoiser convolution layers on the tensor cores against the float64 oracle (oracle/unet.py).

Inputs and weights are bf16-representable, so the kernels' only differences from the oracle are
FP32 accumulation order and the bf16 rounding of stored outputs: tolerance 1% of the output scale
(bf16 has an 8-bit significand; outputs are rounded once)."""
import numpy as np
import pytest

from oracle import unet as ou

pytestmark = pytest.mark.gpu

SHAPE = (6, 10, 20)       # interior; 17 tiles of 128 rows, several CTAs
COARSE = (4, 6, 10)       # coarse level of the upsampling modes (fine = 8 x 12 x 20)


def _bf(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(torch.bfloat16).to(torch.float64).numpy()


def _rand(rng, shape, scale=1.0, positive_frac=None):
    a = rng.normal(0.0, scale, size=shape)
    if positive_frac is not None:
        a = np.where(rng.random(shape) < positive_frac, np.abs(a), -np.abs(a))
    return _bf(a)


def _dev(a, dtype=None):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype or torch.float32)


def _pad(a):
    from bug_defense_b200 import denoise
    return denoise.to_planes(_dev(a))


def _unpad(t, shape=SHAPE):
    from bug_defense_b200 import denoise
    return denoise.from_planes(t, shape).double().cpu().numpy()


def _zeros(channels, shape=SHAPE):
    from bug_defense_b200 import denoise
    return denoise.zeros_planes(channels, shape)


def _close(got, ref, frac=1e-2):
    scale = max(np.abs(ref).max(), 1e-6)
    err = np.abs(got - ref).max()
    assert err <= frac * scale, f"max err {err:.3e} vs scale {scale:.3e}"


def _weights(rng, taps, cin, cout):
    return _bf(rng.normal(0.0, 1.0 / np.sqrt(taps * cin), size=(taps, cout, cin)))


COMBOS = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 32), (32, 16), (16, 64), (64, 16)]


@pytest.mark.parametrize("cin,cout", COMBOS)
def test_forward_relu_matches_oracle(gpu, cin, cout):
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(cin * 100 + cout)
    x = _rand(rng, (cin,) + SHAPE)
    w = _weights(rng, 27, cin, cout)
    b = _bf(rng.normal(0, 0.1, cout))
    img = denoise.pack_weights(_dev(w), 27, cin, cout)
    out = _zeros(cout)
    denoise.conv3d(_lib.CONV_FWD_RELU, _pad(x), img, SHAPE, cin, cout, bias=_dev(b), out=out)
    ref = ou.relu(ou.conv(x, w) + b[:, None, None, None])
    _close(_unpad(out), ref)
    # the pad and margin rows stay zero
    nxp, nyp, nzp = (s + 2 for s in SHAPE)
    o = out.float()
    vol = o[:, :nxp * nyp * nzp].view(-1, nxp, nyp, nzp, 8)
    assert float(vol[:, 0].abs().max()) == 0.0 and float(vol[:, :, :, -1].abs().max()) == 0.0
    assert float(o[:, nxp * nyp * nzp:].abs().max()) == 0.0


def test_forward_nine_taps_z_packed(gpu):
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(9)
    f4 = _rand(rng, (4,) + SHAPE)
    x16 = ou.expand_z(f4)
    w = _weights(rng, 9, 16, 16)
    w[:, :, 12:] = 0.0
    img = denoise.pack_weights(_dev(w), 9, 16, 16)
    out = _zeros(16)
    denoise.conv3d(_lib.CONV_FWD_RELU, _pad(x16), img, SHAPE, 16, 16, taps=9, bias=_dev(np.zeros(16)), out=out)
    ref = ou.relu(ou.conv(x16, w, taps=9))
    _close(_unpad(out), ref)
    # the z-packed 9-tap form equals a 27-tap convolution of the 4 features
    w27 = np.zeros((27, 16, 4))
    for q in range(9):
        for j in range(3):
            w27[q * 3 + j] = w[q][:, 4 * j:4 * j + 4]
    np.testing.assert_allclose(ou.conv(f4, w27), ou.conv(x16, w, taps=9), rtol=1e-12, atol=1e-12)


def test_forward_output_slices_cover_64_by_64(gpu):
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(64)
    x = _rand(rng, (64,) + SHAPE)
    w = _weights(rng, 27, 64, 64)
    b = _bf(rng.normal(0, 0.1, 64))
    out = _zeros(64)
    xd, wd, bd = _pad(x), _dev(w), _dev(b)
    for off in (0, 32):
        img = denoise.pack_weights(wd, 27, 64, 64, n_off=off, n_slice=32)
        denoise.conv3d(_lib.CONV_FWD_RELU, xd, img, SHAPE, 64, 64, n_slice=32, n_off=off, bias=bd[off:off + 32],
                       out=out)
    _close(_unpad(out), ou.relu(ou.conv(x, w) + b[:, None, None, None]))


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 64), (64, 32), (32, 32)])
def test_data_gradient_raw_and_masked(gpu, cin, cout):
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(7 + cin + cout)
    gy = _rand(rng, (cout,) + SHAPE)
    w = _weights(rng, 27, cin, cout)
    act = _rand(rng, (cin,) + SHAPE, positive_frac=0.6)
    ref = ou.conv_data_grad(gy, w)
    wd = _dev(w)
    slices = [(0, cin)] if not (cout == 64 and cin == 64) else [(0, 32), (32, 32)]
    for mode in (_lib.CONV_BWD_RAW, _lib.CONV_BWD_MASK):
        out = _zeros(cin)
        for off, ns in slices:
            img = denoise.pack_weights(wd, 27, cin, cout, n_off=off, n_slice=ns, transpose=True)
            denoise.conv3d(mode, _pad(gy), img, SHAPE, cout, cin, n_slice=ns, n_off=off, out=out,
                           aux=_pad(act) if mode == _lib.CONV_BWD_MASK else None)
        want = ref if mode == _lib.CONV_BWD_RAW else ref * (act > 0)
        _close(_unpad(out), want)


@pytest.mark.parametrize("cin,cout", [(64, 32), (32, 16)])
def test_upsampling_forward_adds_skip(gpu, cin, cout):
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(11 + cin)
    fine = tuple(2 * s for s in COARSE)
    x = _rand(rng, (cin,) + COARSE)
    skip = _rand(rng, (cout,) + fine)
    w = _weights(rng, 27, cin, cout)
    b = _bf(rng.normal(0, 0.1, cout))
    img = denoise.pack_weights(_dev(w), 27, cin, cout)
    out = _zeros(cout, fine)
    oc = _zeros(cout, COARSE)
    denoise.conv3d(_lib.CONV_FWD_UPADD, _pad(x), img, COARSE, cin, cout, bias=_dev(b), out=out, out_coarse=oc,
                   aux=_pad(skip))
    u = ou.relu(ou.conv(x, w) + b[:, None, None, None])
    _close(_unpad(oc, COARSE), u)
    _close(_unpad(out, fine), ou.up(u) + skip)


@pytest.mark.parametrize("cin,cout", [(64, 32), (32, 16)])
def test_upsampling_gradient_adds_residual(gpu, cin, cout):
    """BWD_UPADD: the data gradient at the coarse level (cin here is the layer's cout) spread to the
    finer level as the average-pool adjoint, plus the residual gradient, gated by the activation."""
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(13 + cin)
    fine = tuple(2 * s for s in COARSE)
    g = _rand(rng, (cin,) + COARSE)
    w = _weights(rng, 27, cout, cin)           # forward layer cout -> cin at the coarse level
    resid = _rand(rng, (cout,) + fine)
    act = _rand(rng, (cout,) + fine, positive_frac=0.6)
    img = denoise.pack_weights(_dev(w), 27, cout, cin, transpose=True)
    out = _zeros(cout, fine)
    denoise.conv3d(_lib.CONV_BWD_UPADD, _pad(g), img, COARSE, cin, cout, out=out, aux=_pad(resid), aux2=_pad(act))
    dp = ou.conv_data_grad(g, w)
    _close(_unpad(out, fine), (resid + ou.up(dp) / 8.0) * (act > 0))


@pytest.mark.parametrize("train", [False, True])
def test_head_fuses_output_layer_and_loss(gpu, train):
    import torch
    from bug_defense_b200 import _lib, denoise
    rng = np.random.default_rng(21)
    x = _rand(rng, (16,) + SHAPE)
    w = _weights(rng, 27, 16, 16)
    b = _bf(rng.normal(0, 0.1, 16))
    head = rng.normal(0, 0.3, 17).astype(np.float32)
    a_noisy = rng.random(SHAPE).astype(np.float32) * 1e-3
    mask = (rng.random(SHAPE) < 0.8).astype(np.uint8)
    target = rng.random(SHAPE).astype(np.float32) * 1e-3
    scale, norm = 1e3, 1.0 / np.prod(SHAPE)
    img = denoise.pack_weights(_dev(w), 27, 16, 16)
    pred = torch.zeros(SHAPE, device="cuda")
    hg = torch.zeros(17, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    gout = _zeros(16)
    denoise.conv3d(_lib.CONV_FWD_HEAD, _pad(x), img, SHAPE, 16, 16, bias=_dev(b), head=_dev(head),
                   a_noisy=_dev(a_noisy), mask=_dev(mask, torch.uint8), scale=scale, loss_norm=norm, pred=pred,
                   target=_dev(target) if train else None, head_grad=hg if train else None,
                   loss=loss if train else None, grad_out=gout if train else None)
    h = ou.relu(ou.conv(x, w) + b[:, None, None, None])
    y = np.tensordot(head[:16].astype(np.float64), h, axes=([0], [0])) + head[16]
    p_s = (a_noisy * scale + y) * mask
    np.testing.assert_allclose(pred.cpu().numpy(), p_s / scale, rtol=1e-3, atol=1e-3 * np.abs(p_s / scale).max())
    if train:
        res = (p_s - target * scale) * mask
        np.testing.assert_allclose(float(loss.item()), float((res * res).sum()), rtol=1e-3)
        dy = 2 * res * norm
        ghw = np.tensordot(h, dy, axes=([1, 2, 3], [0, 1, 2]))
        np.testing.assert_allclose(hg.cpu().numpy()[:16], ghw, rtol=2e-3, atol=1e-3 * np.abs(ghw).max())
        np.testing.assert_allclose(hg.cpu().numpy()[16], dy.sum(), rtol=2e-3, atol=1e-6)
        _close(_unpad(gout), dy[None] * head[:16, None, None, None] * (h > 0))


@pytest.mark.parametrize("cout,cin,taps", [(16, 16, 9), (16, 16, 27), (32, 16, 27), (32, 32, 27), (64, 32, 27),
                                           (64, 64, 27), (32, 64, 27), (16, 32, 27)])
def test_weight_gradient_matches_oracle(gpu, cout, cin, taps):
    import torch
    from bug_defense_b200 import denoise
    rng = np.random.default_rng(cout * 7 + cin + taps)
    g = _rand(rng, (cout,) + SHAPE)
    x = _rand(rng, (cin,) + SHAPE)
    dw = torch.zeros((taps, cout, cin), device="cuda")
    denoise.conv3d_wgrad(_pad(g), _pad(x), dw, SHAPE, cin, cout, taps=taps)
    ref = ou.conv_wgrad(g, x, taps)
    _close(dw.double().cpu().numpy(), ref, frac=2e-3)
