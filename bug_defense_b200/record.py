"""Per-epoch recording of a coupled run without per-epoch host synchronisation.

The production runner pulls full 3-D fields from the engine after every epoch and slices them on
the host (knowledge/beetle/scripts/run_highres_knowledge_suite.py:271-306), then saves one npz per
run (:330-367). Here bd_engine_record fills a compact record slot on the device (xz slices of T,
Q, phase and plume absorption, crater depth, band peak temperatures, the epoch's diagnostics), the
slot is copied asynchronously into a ring of pinned host buffers, and filled slots are unpacked
while the engine waits for its next epoch (the engine's wait hook), when the ring wraps around, or
at finish(): the GPU never waits for the host, and a synchronising caller (step_epoch after every
epoch) does not leave the GPU idle while slots are unpacked.
"""
from __future__ import annotations

import ctypes
import math
import weakref

import numpy as np
import torch

from . import _lib

HEAD_BYTES = 256


class Recorder:
    """Record epochs of a CoupledAblationEngine.

    y: xz slice (default mid-y); ix: centreline column (default mid-x), or beam_ix: the centreline's
    x index in every slice (a tilted beam axis, the production runner's sampling line); k_surface:
    first slice below the ambient air (crater depth origin, and the origin of the record's grid_z);
    bands: three (k0, k1) z ranges for peak_T_dorsal, peak_T_core, peak_T_ventral; ring: pinned slots
    in flight."""

    def __init__(self, eng, y=None, ix=None, k_surface=0, bands=((0, 0), (0, 0), (0, 0)), ring: int = 16,
                 beam_ix=None):
        self.eng = eng
        self.nx, self.ny, self.nz = eng.shape
        self.y = self.ny // 2 if y is None else int(y)
        self.ix = self.nx // 2 if ix is None else int(ix)
        if beam_ix is None:
            self.line = np.full(self.nz, self.ix, dtype=np.int64)
        else:
            self.line = np.clip(np.asarray(beam_ix, dtype=np.int64).reshape(self.nz), 0, self.nx - 1)
        self.k_surface = int(k_surface)
        self.bands = [tuple(int(v) for v in b) for b in bands]
        self.slot_bytes = int(_lib.load().bd_record_slot_bytes(self.nx, self.nz))
        self.dev_slot = torch.empty(self.slot_bytes, dtype=torch.uint8, device=eng.dev)
        self.ring = [torch.empty(self.slot_bytes, dtype=torch.uint8, pin_memory=True) for _ in range(int(ring))]
        self.events = [torch.cuda.Event() for _ in self.ring]
        self.pending = [None] * len(self.ring)       # epoch index held by a ring slot
        self.n = 0
        self.drained = 0                             # slots are drained in record order
        hooks = getattr(eng, "_wait_hooks", None)
        if hooks is not None:
            hooks.append(weakref.WeakMethod(self._drain_filled))
        self.rows = {}
        gap = getattr(eng, "air_gap_range", None)
        self.gap = (int(gap[0]), int(gap[1])) if gap is not None else (0, 0)
        self.ratio_a = float(np.float32(eng.plume.ratio_a)) if getattr(eng, "plume", None) is not None else 0.0

    def _spec(self) -> _lib.RecordSpec:
        sp = _lib.RecordSpec()
        sp.y, sp.k_surface = self.y, self.k_surface
        for b, (k0, k1) in enumerate(self.bands):
            sp.band_k0[b], sp.band_k1[b] = k0, k1
        sp.gap_k0, sp.gap_k1 = self.gap
        laser = self.eng._last_power > 0.0 and self.eng.n_photons > 0
        sp.q_scale = float(self.eng._last_power / (self.eng.n_photons * self.eng.voxel_vol)) if laser else 0.0
        sp.plume_ratio_a = self.ratio_a
        return sp

    def record(self, stream=None):
        """Enqueue the record of the epoch the engine just enqueued (no synchronisation)."""
        st = stream if stream is not None else torch.cuda.current_stream(self.eng.dev)
        i = self.n % len(self.ring)
        if self.pending[i] is not None:
            self._drain(i)
        sp = self._spec()
        _lib.call("bd_engine_record", self.eng._handle, ctypes.byref(sp), _lib.ptr(self.dev_slot),
                  _lib.stream_ptr(st))
        with torch.cuda.stream(st):
            self.ring[i].copy_(self.dev_slot, non_blocking=True)
        self.events[i].record(st)
        self.pending[i] = self.n
        self.n += 1

    def _drain_filled(self):
        """Unpack every recorded slot (the engine calls this after enqueuing an epoch, before it
        blocks: the slots' copies precede that epoch, so the waits end while the epoch runs)."""
        while self.drained < self.n:
            i = self.drained % len(self.ring)
            if self.pending[i] is not None:
                self._drain(i)
            self.drained += 1

    def _drain(self, i):
        self.events[i].synchronize()
        buf = self.ring[i].numpy()
        head = _lib.RecordHead.from_buffer_copy(buf[:ctypes.sizeof(_lib.RecordHead)].tobytes())
        n = self.nx * self.nz
        f = buf[HEAD_BYTES:HEAD_BYTES + 12 * n].view(np.float32)
        ph = buf[HEAD_BYTES + 12 * n:HEAD_BYTES + 13 * n]
        self.rows[self.pending[i]] = dict(
            time_s=head.time_s, epoch=head.epoch, plume_tau=head.plume_tau, n_new=head.n_new, n_void=head.n_void,
            absorbed_weight=head.absorbed_weight, peak_T=list(head.peak_T), depth_voxels=head.depth_voxels,
            T=f[:n].reshape(self.nx, self.nz).copy(), Q=f[n:2 * n].reshape(self.nx, self.nz).copy(),
            plume=f[2 * n:3 * n].reshape(self.nx, self.nz).copy(), phase=ph.reshape(self.nx, self.nz).copy())
        self.pending[i] = None

    def finish(self):
        for i in range(len(self.ring)):
            if self.pending[i] is not None:
                self._drain(i)
        self.drained = self.n
        return self.arrays()

    def arrays(self) -> dict:
        """The runner's per-epoch series (run_highres_knowledge_suite.py:280-306) for recorded epochs."""
        eps = sorted(self.rows)
        R = [self.rows[e] for e in eps]
        dz = self.eng.dz
        zs = np.arange(self.nz)
        return dict(
            times=np.array([r["time_s"] for r in R]),
            centerline_T=np.array([r["T"][self.line, zs] for r in R], dtype=np.float32),
            centerline_Q=np.array([r["Q"][self.line, zs] for r in R], dtype=np.float32),
            centerline_phase=np.array([r["phase"][self.line, zs] for r in R], dtype=np.uint8),
            xz_T=np.array([r["T"] for r in R], dtype=np.float32),
            xz_Q=np.array([r["Q"] for r in R], dtype=np.float32),
            xz_phase=np.array([r["phase"] for r in R], dtype=np.uint8),
            xz_plume=np.array([r["plume"] for r in R], dtype=np.float32),
            plume_trans=np.array([math.exp(-r["plume_tau"]) for r in R]),
            peak_T_dorsal=np.array([r["peak_T"][0] for r in R]),
            peak_T_core=np.array([r["peak_T"][1] for r in R]),
            peak_T_ventral=np.array([r["peak_T"][2] for r in R]),
            crater_depths_mm=np.array([r["depth_voxels"] * dz for r in R]),
        )

    def record_arrays(self, arrays=None, gap_k0=None, **meta) -> dict:
        """The runner's whole record (run_highres_knowledge_suite.py:330-367): the per-epoch series, the
        grids (grid_z from -k_surface dz at the top of the grid to the bottom, 0 = dorsal surface), the
        time of the first ablated voxel in the mid-y slice just above the air gap (t_perforation_s,
        slice gap_k0 - 1, default the engine's air gap) and of the first core-band peak at or above
        99.5 C (t_core_boil_s), None when never, the grid constants and the caller's metadata."""
        eng = self.eng
        a = self.finish() if arrays is None else arrays
        k0 = gap_k0 if gap_k0 is not None else (self.gap[0] if self.gap[1] > self.gap[0] else None)
        t = np.asarray(a["times"])
        perf = np.flatnonzero((a["xz_phase"][:, :, k0 - 1] == 3).any(axis=1)) if k0 else np.zeros(0, int)
        boil = np.flatnonzero(np.asarray(a["peak_T_core"]) >= 99.5)
        top = self.k_surface * eng.dz
        return dict(a, grid_x=np.linspace(0, eng.Lx, eng.Nx), grid_y=np.linspace(0, eng.Ly, eng.Ny),
                    grid_z=np.linspace(-top, eng.Nz * eng.dz - top, eng.Nz),
                    t_perforation_s=float(t[perf[0]]) if perf.size else None,
                    t_core_boil_s=float(t[boil[0]]) if boil.size else None,
                    NX=eng.Nx, NY=eng.Ny, NZ=eng.Nz, DX=eng.dx, DY=eng.dy, DZ=eng.dz, dt_epoch=eng.dt_epoch, **meta)

    def save_npz(self, path, **meta):
        """np.savez_compressed of record_arrays(): the keys of the runner's record, with the caller's
        metadata (wavelength_nm, power_w, ...)."""
        np.savez_compressed(path, **self.record_arrays(**meta))
