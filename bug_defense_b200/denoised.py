"""Coupled run with the learned denoiser forming each laser epoch's heat source.

The reference forms the source of a laser epoch from a plain Monte Carlo tally of n_photons
(coupled_ablation.py:454-478: run the MC on the current optics, Q = A P / V, zeroed in ablated
voxels). Here a laser epoch traces only `lo_photons` photons on the engine's current packed
properties (plume extinction included), passes the noisy map, the optics and the tissue state
through the trained network (denoise.Denoiser) and hands the denoised map to the engine as the
epoch's absorbed map, in place of its own MC (the engine's fixed-map path: the epoch's substeps,
phase update and plume run unchanged). Every `check_every` laser epochs the plain n_photons map is
traced as well, as two independent halves, and the two maps are compared by relative L2. With
independent errors E||den - plain||^2 = err_den^2 + err_plain^2, and the halves give
err_plain ~ sigma = ||h1 - h2|| / ||h1 + h2||, so the denoised map is at least as accurate as plain
MC while ||den - plain|| / ||plain|| <= sqrt(2) sigma: above that bound (or above a fixed
`threshold`, when one is given) the run falls back to plain MC for good (that epoch already uses the
plain map). Plain MC stays the judge of the network's error: the spot checks are returned with the
diagnostics.
"""
from __future__ import annotations

import math

from . import _lib


class DenoisedCoupledRun:
    """Drive a CoupledAblationEngine with denoised low-photon maps on laser epochs.

    engine: the engine (its n_photons is the plain photon count of the spot checks and fallback);
    denoiser: a denoise.Denoiser (default: the trained weights); lo_photons: photons per denoised
    epoch; check_every: laser epochs between spot checks (0: never); threshold: a fixed relative L2
    between the denoised and the plain map above which the run falls back to plain MC (None: the
    equal-error bound sqrt(2) sigma of the plain map's own noise)."""

    def __init__(self, engine, denoiser=None, lo_photons: int = 15_000, check_every: int = 20,
                 threshold: float | None = None):
        import torch
        from . import denoise
        self.eng = engine
        self.den = denoiser if denoiser is not None else denoise.Denoiser.load()
        self.lo_photons = int(lo_photons)
        self.check_every = int(check_every)
        self.threshold = None if threshold is None else float(threshold)
        self.fallen_back = False
        self.checks = []              # (epoch, relative L2 denoised vs plain, the bound it was held to)
        self.laser_epochs = 0
        dev = engine.dev
        self._A_lo = torch.zeros(engine.shape, dtype=torch.float32, device=dev)
        self._A_pl = torch.zeros(engine.shape, dtype=torch.float32, device=dev)
        self._A_pl2 = torch.zeros(engine.shape, dtype=torch.float32, device=dev)
        self._out = torch.empty(engine.shape, dtype=torch.float32, device=dev)
        self._ledger = torch.zeros(_lib.LEDGER_LEN, dtype=torch.float64, device=dev)
        self._enqueued = int(engine.epoch)

    def _trace(self, n_photons: int, A, offset: int):
        from . import voxel_mc
        p = self.eng._mc_params()
        p.n_photons = int(n_photons)
        p.photon_offset = int(offset)
        p.options &= ~_lib.MC_TALLY_FLUENCE
        A.zero_()
        self._ledger.zero_()
        voxel_mc.trace(p, self.eng._props, A, ledger=self._ledger, flags=self.eng._flags)
        return self._ledger

    def enqueue(self):
        """Enqueue one epoch; a spot-check epoch synchronises to compare the maps."""
        eng = self.eng
        e = self._enqueued + 1                    # the epoch being enqueued (1-based, as the engine counts)
        self._enqueued = e
        if eng.power <= 0.0 or self.fallen_back:
            eng._enqueue(0)
            return
        self.laser_epochs += 1
        # photon streams disjoint from the engine's own MC of the same epoch (offset (e << 32) + p)
        base = (e << 32) + (1 << 31)
        self._trace(self.lo_photons, self._A_lo, base)
        self._A_lo.mul_(1.0 / self.lo_photons)
        den = self.den(self._A_lo, eng._props, eng._flags, out=self._out)
        use = den
        if self.check_every > 0 and self.laser_epochs % self.check_every == 0:
            half = max(eng.n_photons // 2, 1)
            self._trace(half, self._A_pl, base + (1 << 30))
            self._trace(half, self._A_pl2, base + (1 << 30) + half)
            h1, h2 = self._A_pl.double(), self._A_pl2.double()
            plain = (h1 + h2) * (0.5 / half)
            sigma = float(((h1 - h2).norm() / (h1 + h2).norm()).item())
            rel = float(((den.double() - plain).norm() / plain.norm()).item())
            bound = self.threshold if self.threshold is not None else math.sqrt(2.0) * sigma
            self.checks.append((e, rel, bound))
            if rel > bound:
                self.fallen_back = True
                self._A_pl.copy_(plain)
                use = self._A_pl
        # the engine's tally holds absorbed weight for its n_photons launched photons
        eng._A.copy_(use)
        eng._A.mul_(float(max(eng.n_photons, 1)))
        eng._enqueue(_lib.EPOCH_SKIP_MC)

    def step_epoch(self) -> dict:
        """One epoch and its diagnostics (coupled_ablation.py:605-617 keys, plus the spot checks)."""
        self.enqueue()
        d = self.eng._diag(None)
        d['denoised'] = not self.fallen_back
        d['spot_checks'] = list(self.checks)
        return d
