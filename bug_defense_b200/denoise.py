"""Learned denoiser for low-photon absorbed-power maps.

The reference has no learned component: its absorbed maps are plain Monte Carlo tallies
(simulation/voxel_mc_3d.py:657-688, simulation/voxel_mc_metal.py:555-586), and every epoch of
CoupledAblationEngine.step_epoch pays for the photon count that makes them smooth enough
(coupled_ablation.py:454-468). This module adds a small 3-D U-Net (3 levels, 16/32/64 channels,
BF16 tensor-core convolutions with FP32 accumulation) that maps a map traced with few photons,
plus the optical properties and tissue state, to an estimate of the many-photon map. Plain MC stays
the fallback and the reference for its error.

Volumes on the device are bf16 "8-channel planes" with a one-voxel zero pad (see
include/bugdef.h, "Absorbed-map denoiser"). This module holds the layer-level wrappers of the C ABI
(used by the tests and by the network driver) and the Denoiser / training front end.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

# (taps, cin, cout) of the ten 3-D convolutions; the first sees the z-packed 16-channel input
LAYERS = [(9, 16, 16), (27, 16, 16), (27, 16, 32), (27, 32, 32), (27, 32, 64), (27, 64, 64),
          (27, 64, 32), (27, 32, 32), (27, 32, 16), (27, 16, 16)]
HEAD = 16
N_PARAMS = sum(t * ci * co + co for t, ci, co in LAYERS) + HEAD + 1


def _torch():
    import torch
    return torch


def plane_rows(nx: int, ny: int, nz: int) -> int:
    """Rows per 8-channel plane of a level: padded rows plus the zero margin (bd_conv_plane_rows)."""
    return int(_lib.load().bd_conv_plane_rows(int(nx), int(ny), int(nz)))


def zeros_planes(channels: int, shape, device="cuda"):
    """Zeroed plane-layout volume: (channels/8, R, 8) bf16."""
    torch = _torch()
    return torch.zeros((channels // 8, plane_rows(*shape), 8), dtype=torch.bfloat16, device=device)


def to_planes(x):
    """(C, nx, ny, nz) tensor -> plane-layout bf16 volume (C/8, R, 8) with a zero pad and margin."""
    torch = _torch()
    c, nx, ny, nz = x.shape
    out = zeros_planes(c, (nx, ny, nz), x.device)
    vol = out[:, :(nx + 2) * (ny + 2) * (nz + 2)].view(c // 8, nx + 2, ny + 2, nz + 2, 8)
    vol[:, 1:-1, 1:-1, 1:-1, :] = x.reshape(c // 8, 8, nx, ny, nz).permute(0, 2, 3, 4, 1).to(torch.bfloat16)
    return out


def from_planes(t, shape):
    """Plane-layout volume -> (C, nx, ny, nz) float32 (interior only)."""
    nx, ny, nz = shape
    cb = t.shape[0]
    vol = t[:, :(nx + 2) * (ny + 2) * (nz + 2)].view(cb, nx + 2, ny + 2, nz + 2, 8)
    return vol[:, 1:-1, 1:-1, 1:-1, :].permute(0, 4, 1, 2, 3).reshape(cb * 8, nx, ny, nz).float()


def image_bytes(taps: int, k_channels: int, n_slice: int) -> int:
    return int(_lib.load().bd_conv_image_bytes(taps, k_channels, n_slice))


def pack_weights(w, taps, cin, cout, n_off=0, n_slice=None, transpose=False, stream=None):
    """FP32 [taps][cout][cin] device tensor -> bf16 weight image for one output slice."""
    torch = _torch()
    n_slice = n_slice if n_slice is not None else (cin if transpose else cout)
    k = cout if transpose else cin
    img = torch.empty(image_bytes(taps, k, n_slice) // 2, dtype=torch.bfloat16, device=w.device)
    _lib.call("bd_conv_pack_weights", taps, cin, cout, n_off, n_slice, int(transpose), _lib.ptr(w.contiguous()),
              _lib.ptr(img), _lib.stream_ptr(stream))
    return img


def conv3d(mode, inp, wimage, shape, cin, cout_total, n_slice=None, n_off=0, taps=27, bias=None, out=None,
           out_coarse=None, aux=None, aux2=None, head=None, stream=None, **head_args):
    """One convolution layer through bd_conv3d (synchronous). `shape` is the interior size of the
    level the convolution runs on; volumes are plane-layout bf16 (see to_planes)."""
    c = _lib.ConvCall()
    c.nx, c.ny, c.nz = shape
    c.cin, c.cout_total = cin, cout_total
    c.n_off, c.n_slice = n_off, n_slice if n_slice is not None else cout_total
    c.taps, c.mode = taps, mode
    c.input, c.wimage, c.bias = _lib.ptr(inp), _lib.ptr(wimage), _lib.ptr(bias)
    c.out, c.out_coarse, c.aux, c.aux2 = _lib.ptr(out), _lib.ptr(out_coarse), _lib.ptr(aux), _lib.ptr(aux2)
    c.head = _lib.ptr(head)
    for name in ("a_noisy", "mask", "pred", "target", "head_grad", "loss", "grad_out"):
        setattr(c, name, _lib.ptr(head_args.get(name)))
    c.scale = float(head_args.get("scale", 1.0))
    c.loss_norm = float(head_args.get("loss_norm", 1.0))
    _lib.call("bd_conv3d", ctypes.byref(c), _lib.stream_ptr(stream))


def conv3d_wgrad(grad, act, dw, shape, cin, cout, taps=27, stream=None):
    """dw[t][co][ci] += sum_v grad[v][co] act[v + off_t][ci] (synchronous)."""
    nx, ny, nz = shape
    _lib.call("bd_conv3d_wgrad", nx, ny, nz, cin, cout, taps, _lib.ptr(grad), _lib.ptr(act), _lib.ptr(dw),
              _lib.stream_ptr(stream))


class UNet:
    """Device-resident denoiser network (bd_unet_*): parameters, activations and, with
    training=True, gradients and Adam moments, for one grid shape (multiples of 4)."""

    def __init__(self, shape, training: bool = False, params=None, device=None):
        torch = _torch()
        self.shape = tuple(int(s) for s in shape)
        self.training = bool(training)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("bd_unet_create", *self.shape, int(self.training), ctypes.byref(h))
        self._h = h
        self.n_params = int(_lib.load().bd_unet_param_count())
        assert self.n_params == N_PARAMS
        if params is not None:
            self.set_params(params)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.load().bd_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params, stream=None):
        torch = _torch()
        p = torch.as_tensor(params, dtype=torch.float32).to(self.device).contiguous()
        if p.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.numel()}")
        self._staged = p
        _lib.call("bd_unet_set_params", self._h, _lib.ptr(p), _lib.stream_ptr(stream))

    def params(self, stream=None):
        torch = _torch()
        out = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        _lib.call("bd_unet_get_params", self._h, _lib.ptr(out), _lib.stream_ptr(stream))
        return out

    def grads(self, stream=None):
        torch = _torch()
        out = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        _lib.call("bd_unet_get_grads", self._h, _lib.ptr(out), _lib.stream_ptr(stream))
        return out

    def forward(self, a_noisy, props, flags=None, scale: float = 1e4, out=None, stream=None):
        """Denoised absorbed map (same units and layout as a_noisy: fp32, nx*ny*nz, z fastest)."""
        torch = _torch()
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        _lib.call("bd_unet_forward", self._h, _lib.ptr(a_noisy), _lib.ptr(props), _lib.ptr(flags), float(scale),
                  _lib.ptr(out), _lib.stream_ptr(stream))
        return out

    def forward_backward(self, a_noisy, props, flags, target, scale: float = 1e4, loss_norm=None, pred=None,
                         stream=None):
        torch = _torch()
        if pred is None:
            pred = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        norm = loss_norm if loss_norm is not None else 1.0 / float(np.prod(self.shape))
        _lib.call("bd_unet_forward_backward", self._h, _lib.ptr(a_noisy), _lib.ptr(props), _lib.ptr(flags),
                  _lib.ptr(target), float(scale), float(norm), _lib.ptr(pred), _lib.stream_ptr(stream))
        return pred

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, stream=None):
        _lib.call("bd_unet_adam", self._h, float(lr), float(beta1), float(beta2), float(eps), _lib.stream_ptr(stream))

    def read_loss(self, stream=None) -> float:
        v = ctypes.c_double(0.0)
        _lib.call("bd_unet_read_loss", self._h, ctypes.byref(v), _lib.stream_ptr(stream))
        return float(v.value)


def init_params(seed: int = 0):
    """He-normal convolution weights, zero biases and a zero head: the untrained residual network
    returns the noisy map unchanged (numpy float32 vector)."""
    rng = np.random.default_rng(seed)
    parts = []
    for t, ci, co in LAYERS:
        fan_in = t * ci if t == 27 else 9 * 12
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), size=(t, co, ci))
        if t == 9:
            w[:, :, 12:] = 0.0      # the first layer's input channels 12-15 are always zero
        parts += [w.ravel(), np.zeros(co)]
    parts += [np.zeros(HEAD), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)


# --------------------------------------------------------------------------- data, training, use

SCALE = 1e4          # absorbed fraction per voxel -> network range (hot cuticle voxels ~1)
LO_PHOTONS = 15_000
HI_PHOTONS = 1_500_000


def mc_map(sample: dict, n_photons: int, seed: int, props=None, stream=None):
    """Absorbed map (fraction of launched weight per voxel, fp32 on the device) of `n_photons`
    traced through a crater_sample geometry; returns (map, packed props, FP64 ledger)."""
    torch = _torch()
    from . import voxel_mc
    nx, ny, nz = sample["shape"]
    dev = sample["mu_a"].device
    if props is None:
        props = voxel_mc.pack_props(sample["mu_a"], sample["mu_s"], sample["g"], sample["n"], dev, stream=stream)
    A = torch.zeros(nx * ny * nz, dtype=torch.float32, device=dev)
    ledger = torch.zeros(_lib.LEDGER_LEN, dtype=torch.float64, device=dev)
    done = 0
    while done < n_photons:          # launches of at most 2^24 photons (exact fixed-point tallies)
        nb = min(1 << 24, n_photons - done)
        p = voxel_mc.make_params(Nx=nx, Ny=ny, Nz=nz, Lx=sample["Lx"], Ly=sample["Ly"], Lz=sample["Lz"],
                                 n_photons=nb, spot_dia=sample["spot_dia"], theta_inc_deg=sample["theta_inc_deg"],
                                 seed=seed, tally_fluence=False, photon_offset=done)
        ledger += voxel_mc.trace(p, props, A, flags=sample["flags"], stream=stream)
        done += nb
    A.mul_(1.0 / n_photons)
    return A.view(nx, ny, nz), props, ledger


def relative_l2(a, ref) -> float:
    """||a - ref|| / ||ref|| over the whole map (FP64 sums)."""
    a = a.double().flatten(); ref = ref.double().flatten()
    return float(((a - ref).norm() / ref.norm()).item())


def train(n_pairs: int = 2000, epochs: int = 2, shape=(200, 200, 128), lr: float = 1e-3, seed: int = 0,
          lo: int = LO_PHOTONS, hi: int = HI_PHOTONS, params=None, log_every: int = 100, log=print):
    """Train the denoiser on the GPU with its own kernels: for each of n_pairs random craters
    (workloads.crater_sample, seeds seed*1e6 + i) trace a lo- and a hi-photon map with fresh MC
    seeds every epoch, run forward + backward and one Adam step (cosine-decayed lr). Returns the
    trained FP32 parameters (numpy) and a history of (step, mean loss)."""
    torch = _torch()
    from . import workloads
    net = UNet(shape, training=True, params=params if params is not None else init_params(seed))
    total = n_pairs * epochs
    hist, acc, cnt, step = [], 0.0, 0, 0
    for ep in range(epochs):
        for i in range(n_pairs):
            s = workloads.crater_sample(seed * 1_000_000 + i, *shape)
            base = (seed * 1_000_003 + ep * 7919 + i) * 2
            a_lo, props, _ = mc_map(s, lo, base)
            a_hi, _, _ = mc_map(s, hi, base + 1, props=props)
            net.forward_backward(a_lo, props, s["flags"], a_hi, scale=SCALE)
            lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(total, 1)))
            net.adam(lr_t)
            step += 1
            if step % log_every == 0 or step == total:
                acc += net.read_loss(); cnt += 1
                hist.append((step, acc / cnt))
                log(f"step {step}/{total} loss {acc / cnt:.5g}")
                acc, cnt = 0.0, 0
    out = net.params().cpu().numpy()
    net.close()
    return out, hist


class Denoiser:
    """Trained absorbed-map denoiser: `den(a_noisy, props, flags)` returns the denoised map.
    Weights load from an .npz written by save(); the network is fully convolutional and runs on
    any grid whose dims are multiples of 4."""

    def __init__(self, params, scale: float = SCALE, meta: dict | None = None):
        self.params = np.asarray(params, dtype=np.float32)
        self.scale = float(scale)
        self.meta = dict(meta or {})
        self._nets = {}

    @classmethod
    def load(cls, path=None):
        from pathlib import Path
        p = Path(path) if path is not None else DEFAULT_WEIGHTS
        if not p.exists():
            raise FileNotFoundError(f"denoiser weights not found: {p}")
        z = np.load(p, allow_pickle=False)
        meta = {k: z[k].item() if z[k].ndim == 0 else z[k].tolist() for k in z.files if k not in ("params",)}
        return cls(z["params"], float(z["scale"]) if "scale" in z.files else SCALE, meta)

    def save(self, path, **meta):
        np.savez_compressed(path, params=self.params, scale=np.float64(self.scale),
                            **{k: np.asarray(v) for k, v in meta.items()})

    def net(self, shape, device=None):
        key = (tuple(shape), str(device))
        if key not in self._nets:
            self._nets[key] = UNet(shape, training=False, params=self.params, device=device)
        return self._nets[key]

    def __call__(self, a_noisy, props, flags=None, out=None, stream=None):
        shape = tuple(a_noisy.shape) if a_noisy.dim() == 3 else None
        if shape is None:
            raise ValueError("a_noisy must be a (nx, ny, nz) device tensor")
        return self.net(shape, a_noisy.device).forward(a_noisy, props, flags, scale=self.scale, out=out,
                                                       stream=stream)


def _default_weights():
    from pathlib import Path
    return Path(__file__).resolve().parent / "weights" / "denoiser.npz"


DEFAULT_WEIGHTS = _default_weights()


def main(argv=None):
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="train the absorbed-map denoiser on the GPU")
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=2)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--shape", type=int, nargs=3, default=[200, 200, 128])
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--log", default=None)
    ap.add_argument("--samples", type=int, default=8)
    a = ap.parse_args(argv)
    if a.cmd == "evaluate":
        res = evaluate(Denoiser.load(a.out), n_samples=a.samples)
        print(json.dumps(res))
        if a.log:
            from pathlib import Path
            Path(a.log).write_text(json.dumps(res, indent=1) + "\n")
        return
    t0 = time.time()
    lines = []

    def log(msg):
        line = f"[{time.time() - t0:8.1f}s] {msg}"
        print(line, flush=True)
        lines.append(line)

    params, hist = train(n_pairs=a.pairs, epochs=a.epochs, shape=tuple(a.shape), lr=a.lr, seed=a.seed, log=log)
    from pathlib import Path
    Path(a.out).parent.mkdir(parents=True, exist_ok=True)
    Denoiser(params).save(a.out, shape=np.asarray(a.shape), pairs=a.pairs, epochs=a.epochs, lr=a.lr, seed=a.seed,
                          lo_photons=LO_PHOTONS, hi_photons=HI_PHOTONS, train_seconds=time.time() - t0)
    if a.log:
        Path(a.log).write_text("\n".join(lines) + "\n" + json.dumps({"history": hist}) + "\n")



def evaluate(den: "Denoiser", n_samples: int = 8, seed0: int = 900_000, ref_photons: int = 100_000_000,
             lo: int = LO_PHOTONS, plain: int = 150_000, shape=(200, 200, 128), timing_reps: int = 10) -> dict:
    """Held-out comparison on random craters (seeds seed0 + k): relative L2 against a ref_photons
    map of the noisy lo-photon map, the denoised lo-photon map and the plain `plain`-photon map,
    plus CUDA-event times of each path (MC of lo photons + network, MC of plain photons)."""
    torch = _torch()
    from . import workloads
    rows = []
    for k in range(n_samples):
        s = workloads.crater_sample(seed0 + k, *shape)
        ref, props, _ = mc_map(s, ref_photons, 7 * k + 1)
        a_lo, _, _ = mc_map(s, lo, 7 * k + 2, props=props)
        a_pl, _, _ = mc_map(s, plain, 7 * k + 3, props=props)
        out = den(a_lo, props, s["flags"])
        rows.append(dict(seed=seed0 + k, depth=s["depth"], noisy=relative_l2(a_lo, ref), denoised=relative_l2(out, ref),
                         plain=relative_l2(a_pl, ref)))

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        for _ in range(timing_reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / timing_reps

    s = workloads.crater_sample(seed0, *shape)
    a_lo, props, _ = mc_map(s, lo, 11)
    out = torch.empty(shape, dtype=torch.float32, device=a_lo.device)
    t_mc_lo = timed(lambda: mc_map(s, lo, 12, props=props))
    t_net = timed(lambda: den(a_lo, props, s["flags"], out=out))
    t_mc_plain = timed(lambda: mc_map(s, plain, 13, props=props))
    mean = lambda key: float(np.mean([r[key] for r in rows]))
    return dict(samples=rows, rel_l2_noisy=mean("noisy"), rel_l2_denoised=mean("denoised"), rel_l2_plain=mean("plain"),
                ms_mc_lo=t_mc_lo, ms_net=t_net, ms_mc_plain=t_mc_plain,
                ms_denoised_path=t_mc_lo + t_net, speedup_vs_plain=t_mc_plain / (t_mc_lo + t_net),
                lo_photons=lo, plain_photons=plain, ref_photons=ref_photons, shape=list(shape))


if __name__ == "__main__":
    main()
