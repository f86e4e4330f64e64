"""Tissue phase classification and the char-state constants of the production runners.

CHAR_STATE: simulation/run_multispectral_matrix.py:69-78 (same physical constants).
compute_phase_map: simulation/run_multispectral_matrix.py:168-192, here on device tensors
(accepts numpy arrays too) so the per-epoch recording needs no full-grid host copy.
"""
from __future__ import annotations

import numpy as np
import torch

T_ABL_CUTICLE = 350.0

CHAR_STATE = {
    'A': 1.0e7,
    'Ea': 65000.0,
    'mu_a': 15.0,
    'mu_s': 20.0,
    'k': 0.35e-3,
    'rho_cp': 2.0e-3,
    't_remove': T_ABL_CUTICLE,
    'chi_remove': 0.95,
}


def compute_phase_map(T, chi, dry, ablated, H_acc, is_air_gap=None):
    """0 intact, 1 charred (dry & chi >= 0.10), 2 boiling (T >= 99.5 or H > 0), 3 ablated/air."""
    as_np = isinstance(T, np.ndarray)
    tt = (lambda a: torch.as_tensor(a)) if as_np else (lambda a: a)
    T, chi, dry, ablated, H_acc = tt(T), tt(chi), tt(dry).bool(), tt(ablated).bool(), tt(H_acc)
    phase = torch.zeros(T.shape, dtype=torch.uint8, device=T.device)
    boiling = (T >= 99.5) | (H_acc > 0.0)
    charred = dry & (chi >= 0.10)
    if is_air_gap is not None:
        gap = tt(is_air_gap).bool()
        boiling = boiling & ~gap
        charred = charred & ~gap
    phase[boiling] = 2
    phase[charred] = 1
    phase[ablated] = 3
    if is_air_gap is not None:
        phase[gap] = 3
    return phase.numpy() if as_np else phase
