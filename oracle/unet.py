"""CPU oracle for the absorbed-map denoiser: float64 numpy statement of its convolution layers and
of the whole U-Net, forward and backward.

TEST INFRASTRUCTURE ONLY. Only tests/, the smoke check and the benchmark's CPU leg may import it;
the product path (bug_defense_b200) never does.

The reference has no learned component (its absorbed maps come from plain Monte Carlo,
simulation/voxel_mc_3d.py:657-688), so there is no reference implementation to pin against: this
module is pinned instead by finite-difference checks of its own gradients (tests/test_unet_oracle.py),
and the GPU kernels are compared with it on identical bf16-representable inputs.

Arrays are natural-layout (channels, nx, ny, nz), z fastest. Taps are ordered
t = (dx+1)*9 + (dy+1)*3 + (dz+1) (27 taps) or t = (dx+1)*3 + (dy+1) (9 taps, z packed in channels);
weights are [taps][cout][cin].
"""
from __future__ import annotations

import numpy as np

# (taps, cin, cout) of the ten 3-D convolutions; the first sees the z-packed 16-channel input.
LAYERS = [(9, 16, 16), (27, 16, 16), (27, 16, 32), (27, 32, 32), (27, 32, 64), (27, 64, 64),
          (27, 64, 32), (27, 32, 32), (27, 32, 16), (27, 16, 16)]
HEAD = 16


def n_params() -> int:
    return sum(t * ci * co + co for t, ci, co in LAYERS) + HEAD + 1


def unpack(params: np.ndarray):
    """Flat parameter vector -> ([(W[T][cout][cin], b[cout]) per layer], head_w[16], head_b)."""
    out, o = [], 0
    for t, ci, co in LAYERS:
        w = params[o:o + t * co * ci].reshape(t, co, ci); o += t * co * ci
        b = params[o:o + co]; o += co
        out.append((w, b))
    hw = params[o:o + HEAD]; hb = params[o + HEAD]
    return out, hw, hb


def pack(layers, hw, hb) -> np.ndarray:
    parts = []
    for w, b in layers:
        parts += [np.asarray(w).ravel(), np.asarray(b).ravel()]
    parts += [np.asarray(hw).ravel(), np.asarray([hb]).ravel()]
    return np.concatenate(parts)


def tap_offsets(taps: int):
    if taps == 27:
        return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]
    return [(t // 3 - 1, t % 3 - 1, 0) for t in range(9)]


def _shifted(xp, d, shape):
    """Window of the zero-padded array xp (pad 1) holding x[v + d] for every interior v."""
    nx, ny, nz = shape
    dx, dy, dz = d
    return xp[:, 1 + dx:1 + dx + nx, 1 + dy:1 + dy + ny, 1 + dz:1 + dz + nz]


def conv(x, w, taps=27):
    """out[co](v) = sum_t sum_ci w[t][co][ci] x[ci](v + off_t), zero outside the volume."""
    shape = x.shape[1:]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1)))
    out = np.zeros((w.shape[1],) + shape)
    for t, d in enumerate(tap_offsets(taps)):
        out += np.tensordot(w[t], _shifted(xp, d, shape), axes=([1], [0]))
    return out


def conv_data_grad(gy, w, taps=27):
    """d/dx of sum(gy * conv(x, w)): dx[ci](u) = sum_t sum_co w[t][co][ci] gy[co](u - off_t)."""
    shape = gy.shape[1:]
    gp = np.pad(gy, ((0, 0), (1, 1), (1, 1), (1, 1)))
    out = np.zeros((w.shape[2],) + shape)
    for t, (dx, dy, dz) in enumerate(tap_offsets(taps)):
        out += np.tensordot(w[t].T, _shifted(gp, (-dx, -dy, -dz), shape), axes=([1], [0]))
    return out


def conv_wgrad(gy, x, taps=27):
    """dw[t][co][ci] = sum_v gy[co](v) x[ci](v + off_t)."""
    shape = x.shape[1:]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1)))
    return np.stack([np.tensordot(gy, _shifted(xp, d, shape), axes=([1, 2, 3], [1, 2, 3]))
                     for d in tap_offsets(taps)])


def pool(x):
    c, nx, ny, nz = x.shape
    return x.reshape(c, nx // 2, 2, ny // 2, 2, nz // 2, 2).mean(axis=(2, 4, 6))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def pool_sum(x):
    c, nx, ny, nz = x.shape
    return x.reshape(c, nx // 2, 2, ny // 2, 2, nz // 2, 2).sum(axis=(2, 4, 6))


def relu(x):
    return np.maximum(x, 0.0)


def features(a_noisy, mu_a, mu_s, flags, scale):
    """The four per-voxel input features: scaled noisy map, log1p(mu_a), log1p(mu_s)/4 and the
    tissue state (0 void or ablated, 0.5 dry, 1 wet); plus the absorber mask (mu_a > 0)."""
    void = (flags & 0x05) != 0
    dry = (flags & 0x02) != 0
    state = np.where(void, 0.0, np.where(dry, 0.5, 1.0))
    f = np.stack([a_noisy * scale, np.log1p(mu_a), 0.25 * np.log1p(mu_s), state])
    return f, (mu_a > 0).astype(np.float64)


def expand_z(f4):
    """(4, nx, ny, nz) features -> (16, ...) channels [f(z-1), f(z), f(z+1), 0]."""
    c, nx, ny, nz = f4.shape
    fp = np.pad(f4, ((0, 0), (0, 0), (0, 0), (1, 1)))
    out = np.zeros((16, nx, ny, nz))
    for j in range(3):
        out[4 * j:4 * j + 4] = fp[:, :, :, j:j + nz]
    return out


def forward(params, x16, a_noisy, mask, scale, bf16=None):
    """Network forward. bf16 (optional) rounds every stored activation the way the GPU stores it.
    Returns the denoised map (input units) and the cache for backward."""
    rnd = bf16 if bf16 is not None else (lambda a: a)
    L, hw, hb = unpack(params)
    c = {}
    a1 = rnd(relu(conv(x16, L[0][0], 9) + L[0][1][:, None, None, None]))
    s0 = rnd(relu(conv(a1, L[1][0]) + L[1][1][:, None, None, None]))
    p0 = rnd(pool(s0))
    a3 = rnd(relu(conv(p0, L[2][0]) + L[2][1][:, None, None, None]))
    s1 = rnd(relu(conv(a3, L[3][0]) + L[3][1][:, None, None, None]))
    p1 = rnd(pool(s1))
    a5 = rnd(relu(conv(p1, L[4][0]) + L[4][1][:, None, None, None]))
    a6 = rnd(relu(conv(a5, L[5][0]) + L[5][1][:, None, None, None]))
    u7 = relu(conv(a6, L[6][0]) + L[6][1][:, None, None, None])
    t7 = rnd(up(u7) + s1)
    u7 = rnd(u7)
    a8 = rnd(relu(conv(t7, L[7][0]) + L[7][1][:, None, None, None]))
    u9 = relu(conv(a8, L[8][0]) + L[8][1][:, None, None, None])
    t9 = rnd(up(u9) + s0)
    u9 = rnd(u9)
    h = relu(conv(t9, L[9][0]) + L[9][1][:, None, None, None])
    y = np.tensordot(hw, h, axes=([0], [0])) + hb
    pred_s = (a_noisy * scale + y) * mask
    c.update(x16=x16, a1=a1, s0=s0, p0=p0, a3=a3, s1=s1, p1=p1, a5=a5, a6=a6, u7=u7, t7=t7, a8=a8, u9=u9,
             t9=t9, h=h, mask=mask, pred_s=pred_s, scale=scale)
    return pred_s / scale, c


def backward(params, c, target, loss_norm, bf16=None):
    """Loss = sum over voxels of (pred*scale - target*scale)^2 * mask; returns (loss, gradient of
    loss * loss_norm with respect to the flat parameters)."""
    rnd = bf16 if bf16 is not None else (lambda a: a)
    L, hw, hb = unpack(params)
    G = [None] * len(L)
    res = (c["pred_s"] - target * c["scale"]) * c["mask"]
    loss = float(np.sum(res * res))
    dy = 2.0 * res * loss_norm
    h = c["h"]
    ghw = np.tensordot(h, dy, axes=([1, 2, 3], [0, 1, 2]))
    ghb = float(dy.sum())
    g10 = rnd(dy[None] * hw[:, None, None, None] * (h > 0))

    def layer(i, g, x, taps=27):
        G[i] = (conv_wgrad(g, x, taps), g.sum(axis=(1, 2, 3)))

    layer(9, g10, c["t9"])
    dt9 = rnd(conv_data_grad(g10, L[9][0]))
    g9 = rnd(pool_sum(dt9) * (c["u9"] > 0))
    layer(8, g9, c["a8"])
    g8 = rnd(conv_data_grad(g9, L[8][0]) * (c["a8"] > 0))
    layer(7, g8, c["t7"])
    dt7 = rnd(conv_data_grad(g8, L[7][0]))
    g7 = rnd(pool_sum(dt7) * (c["u7"] > 0))
    layer(6, g7, c["a6"])
    g6 = rnd(conv_data_grad(g7, L[6][0]) * (c["a6"] > 0))
    layer(5, g6, c["a5"])
    g5 = rnd(conv_data_grad(g6, L[5][0]) * (c["a5"] > 0))
    layer(4, g5, c["p1"])
    g4 = rnd((dt7 + up(conv_data_grad(g5, L[4][0])) / 8.0) * (c["s1"] > 0))
    layer(3, g4, c["a3"])
    g3 = rnd(conv_data_grad(g4, L[3][0]) * (c["a3"] > 0))
    layer(2, g3, c["p0"])
    g2 = rnd((dt9 + up(conv_data_grad(g3, L[2][0])) / 8.0) * (c["s0"] > 0))
    layer(1, g2, c["a1"])
    g1 = rnd(conv_data_grad(g2, L[1][0]) * (c["a1"] > 0))
    layer(0, g1, c["x16"], taps=9)
    return loss, pack(G, ghw, ghb)


def init_params(seed=0):
    """He-normal weights, zero biases, zero head (the untrained network returns its input)."""
    rng = np.random.default_rng(seed)
    layers = []
    for t, ci, co in LAYERS:
        fan_in = t * ci if t == 27 else 9 * 12
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), size=(t, co, ci))
        if t == 9:
            w[:, :, 12:] = 0.0
        layers.append((w, np.zeros(co)))
    return pack(layers, np.zeros(HEAD), 0.0)
