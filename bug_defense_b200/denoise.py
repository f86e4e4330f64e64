"""Learned denoiser for low-photon absorbed-power maps.

The reference has no learned component: its absorbed maps are plain Monte Carlo tallies
(simulation/voxel_mc_3d.py:657-688, simulation/voxel_mc_metal.py:555-586), and every epoch of
CoupledAblationEngine.step_epoch pays for the photon count that makes them smooth enough
(coupled_ablation.py:454-468). This module adds a small 3-D U-Net (3 levels, 16/32/64 channels,
BF16 tensor-core convolutions with FP32 accumulation) that maps a map traced with few photons,
plus the optical properties and tissue state, to an estimate of the many-photon map. Plain MC stays
the fallback and the judge of its error.

Volumes on the device are channels-last bf16 rows with a one-voxel zero pad (see
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


def to_padded(x, dtype=None):
    """(C, nx, ny, nz) tensor -> contiguous (nx+2, ny+2, nz+2, C) bf16 tensor with a zero pad."""
    torch = _torch()
    dtype = dtype or torch.bfloat16
    c, nx, ny, nz = x.shape
    out = torch.zeros((nx + 2, ny + 2, nz + 2, c), dtype=dtype, device=x.device)
    out[1:-1, 1:-1, 1:-1, :] = x.permute(1, 2, 3, 0).to(dtype)
    return out


def from_padded(xp):
    """(nx+2, ny+2, nz+2, C) -> (C, nx, ny, nz) float32 (interior only)."""
    return xp[1:-1, 1:-1, 1:-1, :].permute(3, 0, 1, 2).float()


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
    level the convolution runs on; tensors are padded channels-last bf16 (see to_padded)."""
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
