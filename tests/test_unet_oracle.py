"""Pins the denoiser's CPU oracle (oracle/unet.py): its analytic gradients agree with central finite
differences of its own forward pass, and its layer adjoints satisfy <conv(x), g> = <x, conv^T(g)>.
The reference has no learned component, so this self-consistency is the oracle's pin."""
import numpy as np

from oracle import unet as ou


def _problem(seed=0, shape=(4, 4, 8)):
    rng = np.random.default_rng(seed)
    p = ou.init_params(seed)
    L, hw, hb = ou.unpack(p)
    L = [(w, rng.normal(0, 0.05, w.shape[1])) for w, _ in L]
    p = ou.pack(L, rng.normal(0, 0.5, 16), 0.1)
    a = rng.random(shape) * 1e-3
    mu_a = rng.random(shape) * 3
    mu_s = rng.random(shape) * 20
    flags = (rng.random(shape) < 0.1).astype(np.uint8)
    f4, mask = ou.features(a, mu_a, mu_s, flags, 1e3)
    x16 = ou.expand_z(f4)
    target = rng.random(shape) * 1e-3
    return p, x16, a, mask, target


def test_layer_adjoints():
    rng = np.random.default_rng(1)
    shape = (5, 6, 7)
    for taps, ci, co in [(27, 4, 3), (9, 8, 5)]:
        x = rng.normal(size=(ci,) + shape)
        g = rng.normal(size=(co,) + shape)
        w = rng.normal(size=(taps, co, ci))
        lhs = np.sum(ou.conv(x, w, taps) * g)
        np.testing.assert_allclose(lhs, np.sum(x * ou.conv_data_grad(g, w, taps)), rtol=1e-12)
        np.testing.assert_allclose(lhs, np.sum(w * ou.conv_wgrad(g, x, taps)), rtol=1e-12)
    x = rng.normal(size=(2, 4, 6, 8))
    y = rng.normal(size=(2, 2, 3, 4))
    np.testing.assert_allclose(np.sum(ou.pool(x) * y), np.sum(x * ou.up(y) / 8), rtol=1e-12)
    np.testing.assert_allclose(np.sum(ou.up(y) * x), np.sum(y * ou.pool_sum(x)), rtol=1e-12)


def test_gradients_match_finite_differences():
    p, x16, a, mask, target = _problem()
    norm = 1.0 / a.size
    _, cache = ou.forward(p, x16, a, mask, 1e3)
    loss, grad = ou.backward(p, cache, target, norm)
    assert loss > 0 and grad.shape == p.shape == (ou.n_params(),)

    def f(q):
        _, c = ou.forward(q, x16, a, mask, 1e3)
        return ou.backward(q, c, target, norm)[0] * norm

    rng = np.random.default_rng(2)
    offs, o = [], 0
    for t, ci, co in ou.LAYERS:
        offs.append((o, t * ci * co, co))
        o += t * ci * co + co
    picks = []
    for o, nw, nb in offs:
        picks += list(o + rng.choice(nw, 3, replace=False)) + [o + nw + int(rng.integers(nb))]
    picks += [o, o + 7, o + 16]
    eps = 1e-6
    for i in picks:
        if i < 9 * 16 * 16 and (i % 16) >= 12:
            continue  # weights of the always-zero input channels of the first layer
        d = np.zeros_like(p)
        d[i] = eps
        fd = (f(p + d) - f(p - d)) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(grad).max()) + 1e-4 * abs(fd), (i, fd, grad[i])


def test_untrained_network_returns_its_input():
    """init_params has a zero head: the residual network starts as the identity on the noisy map."""
    p = ou.init_params(3)
    rng = np.random.default_rng(3)
    shape = (4, 4, 4)
    a = rng.random(shape)
    f4, mask = ou.features(a, np.ones(shape), np.ones(shape), np.zeros(shape, np.uint8), 10.0)
    pred, _ = ou.forward(p, ou.expand_z(f4), a, mask, 10.0)
    np.testing.assert_allclose(pred, a, rtol=1e-12)
