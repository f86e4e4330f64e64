"""Plume extinction field -- device-resident mirror of MultispectralPlumeField.

Parameter logic follows simulation/plume.py:142-290 (wavelength extinction table, ceilings,
delta_mu, D_xy/D_z/v_drift, tau_linger); the field itself lives on the GPU and is advanced by
bd_plume_advance (transport) and the engine's epoch-end kernel (injection + tanh saturation,
plume.py:292-366). Only the 'diffusion' model with point injection is provided.
"""
from __future__ import annotations

import numpy as np
import torch

# Mass-extinction table of the reference (plume.py:156-164): the same physical constants.
EXTINCTION_MAP = {
    10600: {'mu_a_max': 0.15, 'mu_s_max': 0.05, 'delta_mu': 0.075},
    1940: {'mu_a_max': 0.375, 'mu_s_max': 0.15, 'delta_mu': 0.18},
    1470: {'mu_a_max': 0.45, 'mu_s_max': 0.20, 'delta_mu': 0.22},
    1064: {'mu_a_max': 0.675, 'mu_s_max': 0.60, 'delta_mu': 0.33},
    532: {'mu_a_max': 1.275, 'mu_s_max': 0.80, 'delta_mu': 0.63},
    450: {'mu_a_max': 1.80, 'mu_s_max': 1.00, 'delta_mu': 0.90},
    320: {'mu_a_max': 2.40, 'mu_s_max': 1.20, 'delta_mu': 1.20},
}
_DEFAULT = {'mu_a_max': 0.30, 'mu_s_max': 0.15, 'delta_mu': 0.15}


class PlumeField:
    """Plume parameters + device fields (raw_field, mu_ext_plume as CUDA tensors)."""

    def __init__(self, shape, dx_mm=0.030, dy_mm=0.030, dz_mm=0.020, wavelength_nm=None, tau_linger_s=0.00875,
                 delta_mu_per_voxel=None, mu_a_max=None, model='diffusion', D_plume=2.0, D_xy=None, D_z=None,
                 v_drift=80.0, blast_expansion=False, device=None):
        self.shape = tuple(shape)
        self.dx, self.dy, self.dz = float(dx_mm), float(dy_mm), float(dz_mm)
        self.tau_linger = float(tau_linger_s)
        self.wavelength = float(wavelength_nm) if wavelength_nm is not None else 10600.0
        self.model = str(model).lower()
        if self.model != 'diffusion':
            raise NotImplementedError("only the 'diffusion' plume model is provided (plume.py:147-150)")
        if blast_expansion:
            raise NotImplementedError("blast_expansion=True (separable blast kernel, plume.py:306-327) is not "
                                      "provided; production runs use point injection")
        self.blast_expansion = False
        self.D_plume = float(D_plume)
        self.D_xy = float(D_xy) if D_xy is not None else self.D_plume
        self.D_z = float(D_z) if D_z is not None else self.D_plume
        self.v_drift = float(v_drift)
        self._set_optics(mu_a_max, delta_mu_per_voxel)
        self.device = device
        self.raw = torch.zeros(self.shape, device=device, dtype=torch.float32) if device is not None else None
        self.mu_ext = torch.zeros(self.shape, device=device, dtype=torch.float32) if device is not None else None

    def _set_optics(self, mu_a_max=None, delta_mu=None):
        cfg = EXTINCTION_MAP.get(int(round(self.wavelength)), _DEFAULT)
        self.mu_a_max = float(cfg.get('mu_a_max', 0.30))
        self.mu_s_max = float(cfg.get('mu_s_max', 0.25 * self.mu_a_max))
        self.mu_max = self.mu_a_max + self.mu_s_max
        if mu_a_max is not None:
            self.mu_a_max = float(mu_a_max)
            self.mu_max = self.mu_a_max + self.mu_s_max
        self.delta_mu = float(delta_mu) if delta_mu is not None else float(cfg.get('delta_mu', 0.15))

    def set_wavelength(self, wavelength_nm: float):
        """plume.py:270-278 (used by the dual-wavelength runner's mid-run switch)."""
        self.wavelength = float(wavelength_nm)
        self._set_optics()

    @property
    def ratio_a(self) -> float:
        return self.mu_a_max / max(1e-6, self.mu_max)

    @property
    def ratio_s(self) -> float:
        return self.mu_s_max / max(1e-6, self.mu_max)

    # host views (copies), as the reference exposes numpy arrays
    @property
    def raw_field(self) -> np.ndarray:
        return self.raw.cpu().numpy()

    @property
    def mu_ext_plume(self) -> np.ndarray:
        return self.mu_ext.cpu().numpy()

    @property
    def mu_a_plume(self) -> np.ndarray:
        return self.mu_ext_plume * np.float32(self.ratio_a)

    @property
    def mu_s_plume(self) -> np.ndarray:
        return self.mu_ext_plume * np.float32(self.ratio_s)

    def reset(self):
        self.raw.zero_()
        self.mu_ext.zero_()


def from_closure(closure: dict, shape, dx, dy, dz, wavelength_nm, device):
    """Build the plume from an engine `plume_closure` dict (coupled_ablation.py:324-362)."""
    wl = float(closure.get('wavelength_nm', wavelength_nm))
    D_plume = float(closure.get('D_plume', closure.get('D', 2.0)))
    return PlumeField(
        shape=shape, dx_mm=dx, dy_mm=dy, dz_mm=dz, wavelength_nm=wl,
        tau_linger_s=float(closure.get('tau_linger_s', 0.00875)),
        delta_mu_per_voxel=closure.get('delta_mu_per_voxel', closure.get('delta_mu')),
        mu_a_max=closure.get('mu_a_max', closure.get('mu_max')),
        model=str(closure.get('model', 'diffusion')).lower(), D_plume=D_plume,
        D_xy=float(closure['D_xy']) if 'D_xy' in closure else D_plume,
        D_z=float(closure['D_z']) if 'D_z' in closure else D_plume,
        v_drift=float(closure.get('v_drift', closure.get('vz', 80.0))),
        blast_expansion=bool(closure.get('blast_expansion', True)), device=device)


MultispectralPlumeField = PlumeField
PlumeAbsorptionField = PlumeField
