"""Batched campaign: many independent coupled runs (wavelength x power x pulse schedule) on one GPU.

The reference runs its campaigns one simulation per subprocess (run_highres_knowledge_suite.py:633-654,
run_single_highres :187-410; run_multispectral_matrix.py; the dual-wavelength runner
run_dual_permutation_suite.py:254-283). Here every instance is a device-resident
CoupledAblationEngine with its own CUDA stream; each epoch is a captured CUDA graph per stage, and
the instances' epochs are enqueued round-robin so their kernels overlap on the GPU (the crater
geometries diverge per instance, so the instances never share state). The launch shapes are
picked once per campaign by `autotune` on a throwaway engine of the real workload.

Per-layer optical properties follow a seeded chromophore mix, scaled from the 532 nm draw:
    mu_a(l) = mu_a(532) * mix(l) / mix(532),  mix = w * water + m * melanin + (1 - w - m) * baseline
    mu_s(l) = mu_s(532) * (l / 532) ** -b
with published spectral forms (restated, not the reference's tables): water absorption anchors from
the Hale & Querry / Segelstein / Pope & Fry compilations interpolated log-linearly, the melanin power
law 519 (l / 500 nm) ** -3.5 /cm and the bloodless-tissue baseline 0.244 + 85.3 exp(-(l - 154) / 66.2)
/cm (S. L. Jacques, Phys. Med. Biol. 58 (2013) R37). The reference's basis.py:90-160 provides the
same three spectra (water_mua, melanin_mua, baseline_tissue_mua) from its own tables.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

WAVELENGTHS_NM = (450, 532, 808, 980, 1064, 1470, 1940, 2940)
POWERS_W = (20.0, 40.0, 80.0)
EPOCHS_TOTAL = 1000          # 1 s of 1 ms epochs

# water absorption coefficient (1/cm) at anchor wavelengths (nm), literature values
_WATER_ANCHORS = np.array([
    (400, 6.6e-5), (450, 9.2e-5), (500, 2.5e-4), (532, 4.5e-4), (600, 2.2e-3), (700, 6.5e-3),
    (750, 2.6e-2), (808, 2.0e-2), (900, 6.8e-2), (980, 4.8e-1), (1064, 1.4e-1), (1200, 1.04),
    (1300, 1.2), (1450, 31.0), (1470, 30.0), (1550, 10.0), (1700, 6.0), (1800, 8.0), (1940, 120.0),
    (2100, 27.0), (2500, 50.0), (2800, 2600.0), (2940, 12000.0), (3000, 11000.0)])


def water_mua(nm):
    """Water absorption coefficient in 1/mm (log-linear interpolation between anchors)."""
    nm = np.asarray(nm, dtype=np.float64)
    lo, hi = _WATER_ANCHORS[0, 0], _WATER_ANCHORS[-1, 0]
    if np.any(nm < lo) or np.any(nm > hi):
        raise ValueError(f"water_mua: wavelength outside {lo:.0f}-{hi:.0f} nm")
    return np.exp(np.interp(nm, _WATER_ANCHORS[:, 0], np.log(_WATER_ANCHORS[:, 1]))) * 0.1


def melanin_mua(nm):
    """Melanosome absorption in 1/mm: 519 (nm / 500) ** -3.5 per cm."""
    return 51.9 * (np.asarray(nm, dtype=np.float64) / 500.0) ** -3.5


def baseline_tissue_mua(nm):
    """Bloodless protein / tissue baseline in 1/mm: 0.244 + 85.3 exp(-(nm - 154) / 66.2) per cm."""
    return 0.1 * (0.244 + 85.3 * np.exp(-(np.asarray(nm, dtype=np.float64) - 154.0) / 66.2))


def layer_mix(rng, layer_name: str, water: float) -> dict:
    """Seeded chromophore fractions of one layer: its water fraction, melanin in the cuticle."""
    mel = float(rng.uniform(0.005, 0.05)) if "cuticle" in layer_name else 0.0
    return dict(water=float(water), melanin=mel, protein=max(0.0, 1.0 - water - mel),
                b_mie=float(rng.uniform(0.9, 1.5)))


def mix_mua(mix: dict, nm: float) -> float:
    return (mix["water"] * float(water_mua(nm)) + mix["melanin"] * float(melanin_mua(nm))
            + mix["protein"] * float(baseline_tissue_mua(nm)))


def campaign_instances(seed: int = 0, wavelengths=WAVELENGTHS_NM, powers=POWERS_W, grid=(200, 200, 128),
                       n_plume_air: int = 64):
    """The 8 wavelengths x 3 powers = 24 instance descriptions: one tissue draw per instance (seed
    seed*1000 + i), a pulse length U(50, 400) ms, and its chromophore mix."""
    rng = np.random.default_rng(seed)
    out = []
    i = 0
    for nm in wavelengths:
        for p in powers:
            out.append(dict(index=i, wavelength_nm=float(nm), power=float(p),
                            pulse_ms=float(rng.uniform(50.0, 400.0)), tissue_seed=seed * 1000 + i,
                            mix_seed=seed * 1000 + 500 + i, grid=tuple(grid), n_plume_air=n_plume_air))
            i += 1
    return out


def instance_geometry(inst: dict, device=None) -> dict:
    """full_coupled_run geometry of an instance with its optics moved from 532 nm to its wavelength;
    with `device` the grids are built there (torch float64) and never exist on the host."""
    from . import workloads
    nx, ny, nz = inst["grid"]
    geo = workloads.full_coupled_run(inst["tissue_seed"], nx=nx, ny=ny, nz=nz, n_plume_air=inst["n_plume_air"],
                                     device=device)
    nm = inst["wavelength_nm"]
    rng = np.random.default_rng(inst["mix_seed"])
    names = geo["layer_names"]
    nz = geo["shape"][2]                       # tissue stack plus the prepended plume air
    mixes = {}
    for kk, name in enumerate(names):
        if name in ("top_air", "below", "air_gap") or name in mixes:
            continue
        mixes[name] = layer_mix(rng, name, geo["layers"][name]["water"])
    scale_a = np.ones(nz)
    scale_s = np.ones(nz)
    for kk, name in enumerate(names):
        if name in mixes:
            m = mixes[name]
            scale_a[kk] = mix_mua(m, nm) / mix_mua(m, 532.0)
            scale_s[kk] = (nm / 532.0) ** -m["b_mie"]
    if device is not None:
        import torch
        scale_a = torch.as_tensor(scale_a, device=torch.device(device))
        scale_s = torch.as_tensor(scale_s, device=torch.device(device))
    for key, sc in (("mu_a", scale_a), ("mu_s", scale_s)):
        geo["optical"][key] = geo["optical"][key] * sc[None, None, :]
        geo["dry_state"][key] = geo["dry_state"][key] * sc[None, None, :]
    # char: broadband carbon absorption ~ 1/lambda, scattering ~ lambda^-1.2
    geo["char_state"] = dict(geo["char_state"], mu_a=geo["char_state"]["mu_a"] * (532.0 / nm),
                             mu_s=geo["char_state"]["mu_s"] * (532.0 / nm) ** 1.2)
    geo["plume_closure"] = dict(geo["plume_closure"], wavelength_nm=nm)
    geo["power"] = inst["power"]
    geo["epochs_on"] = int(round(inst["pulse_ms"]))
    geo["wavelength_nm"] = nm
    geo["mixes"] = mixes
    return geo


def make_engine(inst: dict, device=None, use_graphs: bool = True):
    from .coupled import CoupledAblationEngine
    from .workloads import engine_kwargs
    import torch
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    geo = instance_geometry(inst, device=dev)
    kw = engine_kwargs(geo)
    kw.update(wavelength_nm=geo["wavelength_nm"], power=geo["power"], use_graphs=use_graphs, device=device,
              tally_fluence=False)
    if inst.get("n_photons"):
        kw["n_photons"] = int(inst["n_photons"])
    eng = CoupledAblationEngine(**kw)
    eng.epochs_on = geo["epochs_on"]
    eng.laser_power = geo["power"]
    return eng


def _stage_ms(eng, n_epochs: int, laser: bool) -> np.ndarray:
    from . import _lib
    import ctypes
    eng.power = eng.laser_power if laser else 0.0
    _lib.call("bd_engine_timing", eng._handle, 1)
    for _ in range(n_epochs):
        eng._enqueue(0)
    ms = (ctypes.c_double * 4)()
    n = ctypes.c_int64(0)
    _lib.call("bd_engine_timing_read", eng._handle, ms, ctypes.byref(n))
    _lib.call("bd_engine_timing", eng._handle, 0)
    return np.array(ms[:]) / max(int(n.value), 1)


def _epoch_ms(eng, n_epochs: int, laser: bool) -> float:
    """Whole-epoch time (ms, device events) over n_epochs: with the plume stage beside MC and the
    substeps, a stage's span is not what a launch shape should minimise."""
    import torch
    eng.power = eng.laser_power if laser else 0.0
    st = torch.cuda.current_stream(eng.dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(n_epochs):
        eng._enqueue(0)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / max(n_epochs, 1)


def autotune(inst, epochs_per_trial: int = 6, candidates=None, device=None, log=None) -> dict:
    """Pick launch shapes by timing them on a throwaway engine of the real workload: `inst` is a
    campaign instance dict or a callable returning an engine with a `laser_power` attribute.
    MC CTAs per SM (photons per thread) are timed by whole laser-on epochs; x-planes per CTA of the
    fused substep kernel by whole epochs with the laser off (the void domain does not change between
    trials): the plume stage runs beside MC and the substeps, so a shape that slows its own stage
    but leaves the plume more room can win. The plume kernel and the direct kernel's x-planes per CTA are searched
    together, also by laser-off epochs; the compact kernel chooses its x-planes per stage on the
    device. Sets
    the winning values process-wide (bd_tune_set) and returns the choices with every trial's time
    (ms per epoch)."""
    from . import _lib
    cand = dict(candidates or {})
    cand.setdefault(_lib.TUNE_MC_BLOCKS_PER_SM, [1, 2, 3, 4, 6, 8])
    cand.setdefault(_lib.TUNE_STENCIL_XC, [1, 2, 4, 8, 16])
    cand.setdefault(_lib.TUNE_PLUME_KERNEL, [_lib.PLUME_KERNEL_DIRECT, _lib.PLUME_KERNEL_COMPACT])
    cand.setdefault(_lib.TUNE_PLUME_XC, [2, 3, 4, 6])
    cand.setdefault(_lib.TUNE_STENCIL_CAP, [0, 1, 2])
    names = {_lib.TUNE_MC_BLOCKS_PER_SM: "mc_ctas_per_sm", _lib.TUNE_STENCIL_XC: "stencil_xc",
             _lib.TUNE_PLUME_XC: "plume_xc", _lib.TUNE_PLUME_KERNEL: "plume_kernel",
             _lib.TUNE_STENCIL_CAP: "stencil_cap"}
    eng = inst() if callable(inst) else make_engine(inst, device=device)
    eng.step_epochs(3)                       # warm-up: graphs, caches, a first crater
    out = {"trials": {}}

    def trial(settings, mc=False):
        for knob, v in settings:
            _lib.call("bd_tune_set", int(knob), int(v))
        _stage_ms(eng, 1, laser=mc)          # re-capture the stage graphs for the new shape
        # whole epochs: the stages run beside each other, so a stage's own time is not what matters
        return _epoch_ms(eng, epochs_per_trial, laser=mc)

    def single(knob, mc):
        trials = []
        for v in cand[knob]:
            t = trial([(knob, v)], mc=mc)
            trials.append((int(v), t))
            if log:
                log(f"autotune {names[knob]}={v}: {t:.3f} ms/epoch")
        best = min(trials, key=lambda t: t[1])[0]
        _lib.call("bd_tune_set", int(knob), int(best))
        out[names[knob]] = best
        out["trials"][names[knob]] = trials

    # laser-off trials first, on the state the run starts from (they leave the void domain as it is);
    # the MC trials, whose laser epochs deepen the crater, come last
    single(_lib.TUNE_STENCIL_XC, False)
    single(_lib.TUNE_STENCIL_CAP, False)
    # plume kernel x x-planes per CTA (only the one-launch-per-step grid kernel takes the knob); the
    # candidates differ by a few per cent, so each is timed twice (forward, then reversed order) and
    # keeps its better time
    combos = [(int(kern), xc) for kern in cand[_lib.TUNE_PLUME_KERNEL]
              for xc in (cand[_lib.TUNE_PLUME_XC] if kern == _lib.PLUME_KERNEL_DIRECT else [None])]
    best_t = {}
    for order in (combos, combos[::-1]):
        for kern, xc in order:
            sets = [(_lib.TUNE_PLUME_KERNEL, kern)] + ([] if xc is None else [(_lib.TUNE_PLUME_XC, xc)])
            t = trial(sets)
            best_t[(kern, xc)] = min(t, best_t.get((kern, xc), float("inf")))
            if log:
                log(f"autotune plume_kernel={kern} plume_xc={xc}: {t:.3f} ms/epoch")
    trials = [(kern, xc, best_t[(kern, xc)]) for kern, xc in combos]
    kern, xc, _ = min(trials, key=lambda t: t[2])
    _lib.call("bd_tune_set", _lib.TUNE_PLUME_KERNEL, kern)
    if xc is not None:
        _lib.call("bd_tune_set", _lib.TUNE_PLUME_XC, xc)
    else:
        xv = ctypes.c_int(0)
        _lib.call("bd_tune_get", _lib.TUNE_PLUME_XC, ctypes.byref(xv))
        xc = xv.value
    out["plume_kernel"] = kern
    out["plume_xc"] = int(xc)
    out["trials"]["plume"] = [[k, x, t] for k, x, t in trials]
    single(_lib.TUNE_MC_BLOCKS_PER_SM, True)
    del eng
    return out


class Campaign:
    """Run many instances together: one engine per instance, epochs enqueued round-robin with no
    host synchronisation between them (diagnostics are read every `sync_every` epochs). The laser
    of instance i is on for its first epochs_on epochs.

    Every instance gets its own stream and runs its own plume stage beside its own MC and
    substeps. With `batch_plume` the instances' plume
    stages instead run as one batched stage (bd_plume_batch_run: one launch per FTCS step over the
    live units of every instance still stepping) on a stream of its own, beside the instances' MC and
    substeps, and each instance's epoch end waits for it. Same results; measured slower on the
    24-instance campaign (the batched stage streams every instance's field through L2 each step,
    where an instance's own stage keeps its field resident), so it is off by default."""

    def __init__(self, instances, device=None, use_graphs: bool = True, log=None, batch_plume: bool = False):
        import torch
        from . import _lib
        self.instances = list(instances)
        self.engines = []
        self.streams = []
        t0 = time.perf_counter()
        for inst in self.instances:
            eng = make_engine(inst, device=device, use_graphs=use_graphs)
            self.engines.append(eng)
            self.streams.append(torch.cuda.Stream(device=eng.dev))
            if log:
                log(f"instance {inst['index']}: {inst['wavelength_nm']:.0f} nm, {inst['power']:.0f} W, "
                    f"pulse {inst['pulse_ms']:.0f} ms")
        self.batch = None
        if batch_plume and len(self.engines) <= 32 and use_graphs:
            n = len(self.engines)
            arr = (ctypes.c_void_p * n)(*[e._handle for e in self.engines])
            h = ctypes.c_void_p()
            _lib.call("bd_plume_batch_create", arr, n, ctypes.byref(h))
            self.batch = h
            dev = self.engines[0].dev
            self.plume_stream = torch.cuda.Stream(device=dev, priority=-1)
            self.ev_prev = [torch.cuda.Event() for _ in self.engines]
            self.ev_plume = torch.cuda.Event()
        self.setup_s = time.perf_counter() - t0
        self.epoch = 0

    def close(self):
        """Release the batched plume stage (the engines stay usable)."""
        from . import _lib
        if self.batch is not None:
            import torch
            torch.cuda.synchronize(self.engines[0].dev)
            _lib.call("bd_plume_batch_destroy", self.batch)
            self.batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def enqueue(self, n_epochs: int):
        import torch
        from . import _lib
        for _ in range(int(n_epochs)):
            if self.batch is None:
                for eng, st in zip(self.engines, self.streams):
                    with torch.cuda.stream(st):
                        eng.power = eng.laser_power if self.epoch < eng.epochs_on else 0.0
                        eng._enqueue(0)
            else:
                # the batched plume stage starts once every instance's previous epoch has ended and
                # runs beside their MC and substeps; each instance's epoch end waits for it
                for eng, st, ev in zip(self.engines, self.streams, self.ev_prev):
                    ev.record(st)
                    with torch.cuda.stream(st):
                        eng.power = eng.laser_power if self.epoch < eng.epochs_on else 0.0
                        eng._enqueue(_lib.EPOCH_EXTERNAL_PLUME)
                for ev in self.ev_prev:
                    self.plume_stream.wait_event(ev)
                with torch.cuda.stream(self.plume_stream):
                    _lib.call("bd_plume_batch_run", self.batch, _lib.stream_ptr())
                self.ev_plume.record(self.plume_stream)
                for eng, st in zip(self.engines, self.streams):
                    st.wait_event(self.ev_plume)
                    with torch.cuda.stream(st):
                        _lib.call("bd_engine_epoch_finish", eng._handle, _lib.stream_ptr())
            self.epoch += 1

    def diagnostics(self):
        import torch
        out = []
        for eng, st in zip(self.engines, self.streams):
            with torch.cuda.stream(st):
                out.append(eng._diag(None))
        return out

    def run(self, n_epochs: int = EPOCHS_TOTAL, sync_every: int = 100):
        """Advance every instance n_epochs; returns the diagnostics of the last epoch per instance."""
        done = 0
        diags = None
        while done < n_epochs:
            k = min(sync_every, n_epochs - done)
            self.enqueue(k)
            done += k
            diags = self.diagnostics()
        return diags
