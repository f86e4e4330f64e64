"""Device selection and host<->device helpers (torch is only the memory/stream plumbing)."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib


def is_gpu_available() -> bool:
    """True when a CUDA device and libbugdef.so are usable.

    Mirrors is_metal_available() (simulation/voxel_mc_metal.py:23-38): it never raises.
    """
    try:
        if not torch.cuda.is_available():
            return False
        return _lib.device_count() > 0
    except Exception:
        return False


def require_device(device=None) -> torch.device:
    """Return the CUDA device to use or raise RuntimeError (no CPU fallback exists)."""
    if not torch.cuda.is_available():
        raise RuntimeError("bug_defense_b200 needs a CUDA device (sm_100a); none is available")
    _lib.load()
    if device is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError(f"device must be a CUDA device, got {device!r}")
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
    _lib.check(_lib.load().bd_device_init(dev.index), "bd_device_init")
    return dev


def to_dev(a, dev, dtype=torch.float32) -> torch.Tensor:
    """Contiguous device copy of a numpy array / scalar / tensor."""
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=dtype).contiguous()
    arr = np.ascontiguousarray(a)
    if dtype == torch.float32 and arr.dtype == np.float64:
        # upload as is and round on the device (the same IEEE round-to-nearest as numpy's astype)
        return torch.from_numpy(arr).to(dev).to(torch.float32)
    if dtype == torch.uint8:
        arr = arr.astype(np.uint8, copy=False)
    elif dtype == torch.float32:
        arr = arr.astype(np.float32, copy=False)
    elif dtype == torch.float64:
        arr = arr.astype(np.float64, copy=False)
    return torch.from_numpy(arr).to(dev)


def full_grid(value, shape, dev, dtype=torch.float32) -> torch.Tensor:
    """A property given as a scalar or as a per-voxel array, as a device grid."""
    if np.ndim(value) == 0:
        return torch.full(shape, float(value), device=dev, dtype=dtype)
    t = to_dev(value, dev, dtype)
    if tuple(t.shape) != tuple(shape):
        t = t.reshape(shape)
    return t
