#!/usr/bin/env python
"""Benchmark: coupled 1 ms epochs/s of the full-resolution coupled laser-tissue run.

Workload (seeded synthetic, no dataset): 200x200x128 layered beetle stack + 64 air slices for the
plume (200x200x192 voxels at 15 um), 532 nm, 40 W Gaussian 0.5 mm spot at 22 deg, 150k photons per
laser epoch, 20 x 50 us substeps, boiling / char / ablation / plume (D, extinction, char kinetics
drawn from the seed). A step is one 1 ms epoch; the laser is on for the first 20 % of the timed
epochs (the 200-on / 800-off duty of the 1000-epoch production schedule) and off after.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: replicas only (independent instances, one per rank; no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "coupled 1 ms epochs/s (full-resolution coupled run)"
FALLBACK_HBM_GBS = 6650.0
LASER_DUTY = 0.2
POWER_W = 40.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--small", action="store_true", help="64x64x128 grid (profiling / smoke only, not a bench line)")
    ap.add_argument("--no-denoiser", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-full-run", action="store_true", help="skip the device-timed 1000-epoch schedule")
    ap.add_argument("--plume-kernel", type=int, default=None, choices=[4, 6],
                    help="plume kernel to use (4 direct, 6 direct over a compact unit list) instead of "
                         "the autotuner's choice")
    ap.add_argument("--batch-plume", action="store_true",
                    help="campaign: run the instances' plume stages as one batched stage (one launch per step)")
    ap.add_argument("--workload", default="coupled", choices=["coupled", "campaign"],
                    help="coupled: the headline run; campaign: 24 wavelength x power x pulse instances at once")
    return ap.parse_args()


def dist_env():
    from bug_defense_b200.replicas import dist_env as env
    return env()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured", d
    return FALLBACK_HBM_GBS, "fallback", {}


def l2_copy_gbs(dev, sizes_mb=(8, 16, 32), reps: int = 100) -> float:
    """Copy bandwidth of L2-resident buffer pairs (2 x 8, 16 or 32 MB; the L2 holds 126 MB): GB/s
    of bytes read + written by `reps` device-to-device copies replayed from one CUDA graph (no host
    launch cost), timed with CUDA events after a warm-up; the best of the sizes. The denominator of
    the plume step's L2 fraction (its void field stays in L2 between steps)."""
    import torch
    best = 0.0
    for mb in sizes_mb:
        a = torch.ones(mb * (1 << 20) // 4, dtype=torch.float32, device=dev)
        b = torch.empty_like(a)
        st = torch.cuda.Stream(dev)
        with torch.cuda.stream(st):
            for _ in range(5):
                b.copy_(a)
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            for _ in range(reps):
                b.copy_(a)
        for _ in range(2):
            g.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * a.numel() * 4 * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9)
        del g, a, b
    return best


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(float(r[2]) for r in rows), "reasons": reasons,
                "samples": len(rows)}


def _threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def cpu_port_phases(geo, kw, n_phase=10, plume=True, warm=True):
    """The oracle port (FP64 C restatement of the reference CPU path, all host threads) on the same
    workload: one untimed laser-on epoch when `warm`, then n_phase laser-on and n_phase laser-off
    epochs, each timed; returns the median of each phase (seconds)."""
    import oracle
    from oracle.engine import OracleEngine
    oracle.build()
    oracle.set_threads(_threads())
    kwp = dict(kw)
    if not plume:
        kwp["plume_closure"] = None
    eng = OracleEngine(**kwp, plume_dt_policy="subcycle")
    if warm:
        eng.power = POWER_W
        eng.step_epoch()
    t_on, t_off = [], []
    for _ in range(n_phase):
        eng.power = POWER_W
        t0 = time.perf_counter(); eng.step_epoch(); t_on.append(time.perf_counter() - t0)
    for _ in range(n_phase):
        eng.power = 0.0
        t0 = time.perf_counter(); eng.step_epoch(); t_off.append(time.perf_counter() - t0)
    return statistics.median(t_on), statistics.median(t_off)


def cpu_mc_alone(geo, n_photons, reps=3):
    """Photons/s of the oracle's FP64 MC alone (the reference's run_voxel_mc3d(engine='cpu')
    counterpart) on the workload's initial geometry: median of `reps` timed runs after a warm-up."""
    import numpy as np
    import oracle
    oracle.set_threads(_threads())
    opt = {k: np.asarray(v, dtype=np.float64) for k, v in geo["optical"].items()}
    kw = dict(power=POWER_W, n_photons=n_photons, spot_dia=geo["spot_dia"], Lx=geo["Lx"], Ly=geo["Ly"], Lz=geo["Lz"],
              Nx=geo["shape"][0], Ny=geo["shape"][1], Nz=geo["shape"][2], custom_3d_props=opt,
              theta_inc_deg=geo["theta_inc_deg"], tally_fluence=False)
    oracle.run_voxel_mc3d(seed=1, **dict(kw, n_photons=max(n_photons // 10, 1000)))
    ts = []
    for r in range(reps):
        t0 = time.perf_counter(); oracle.run_voxel_mc3d(seed=2 + r, **kw); ts.append(time.perf_counter() - t0)
    return n_photons / statistics.median(ts)


def full_run_rate(t_on, t_off):
    """Epochs/s of the 1000-epoch schedule (200 laser-on, 800 laser-off) from per-phase times."""
    return 1000.0 / (200.0 * t_on + 800.0 * t_off)


def cpu_port_baseline(geo, kw, n_phase=10):
    """Reported CPU baseline: medians over n_phase laser-on and n_phase laser-off epochs of the same
    workload on the oracle port, with and without the plume, plus the MC alone in photons/s; value =
    epochs/s at the benchmark's 20 % laser duty (1 / (0.2 t_on + 0.8 t_off)), with the plume."""
    t0 = time.perf_counter()
    ton, toff = cpu_port_phases(geo, kw, n_phase, plume=True)
    ton_np, toff_np = cpu_port_phases(geo, kw, n_phase, plume=False)
    mc_rate = cpu_mc_alone(geo, kw["n_photons"])
    per_epoch = LASER_DUTY * ton + (1 - LASER_DUTY) * toff
    return {"value": 1.0 / per_epoch, "unit": "epochs/s", "cores": _threads(), "kind": "port",
            "sample": f"median over {n_phase} laser-on + {n_phase} laser-off epochs (after one warm-up epoch) of the "
                      f"same workload on the FP64 C port of the reference CPU path (oracle/orc.c, OpenMP), with and "
                      f"without the plume, and the MC alone; value = 1 / (0.2 t_on + 0.8 t_off) with the plume",
            "t_on_s": round(ton, 4), "t_off_s": round(toff, 4),
            "without_plume": {"t_on_s": round(ton_np, 4), "t_off_s": round(toff_np, 4),
                              "epochs_per_s": round(1.0 / (LASER_DUTY * ton_np + (1 - LASER_DUTY) * toff_np), 4)},
            "full_run_epochs_per_s": round(full_run_rate(ton, toff), 4),
            "mc_photons_per_s": round(mc_rate, 1), "seconds": round(time.perf_counter() - t0, 1)}


def make_engine(geo, dev, seed_offset=0):
    from bug_defense_b200 import CoupledAblationEngine
    from bug_defense_b200.workloads import engine_kwargs
    kw = engine_kwargs(geo)
    kw["seed"] = kw["seed"] + seed_offset
    return CoupledAblationEngine(**kw, device=dev)


def algorithmic_bytes(eng, n_void):
    """Unique bytes each stage must move per launch (cache-ideal neighbours)."""
    nv = eng.Nx * eng.Ny * eng.Nz
    # fused substep over every voxel: T r+w 8, k 4, rho 4, source 4, flags 1, H r+w 8, chi r+w 8
    sub = nv * 37
    # plume step over the plume (void) domain: C r+w 8, neighbourhood byte 1
    plume = n_void * 9
    return {"substep": sub, "plume_step": plume}


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from bug_defense_b200 import _lib, workloads
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    geo = workloads.full_coupled_run(seed=args.seed) if not args.small else workloads.full_coupled_run(
        seed=args.seed, nx=64, ny=64)
    tuned = None
    if not args.no_autotune:
        # launch shapes picked on a throwaway engine of the same workload (outside the timed region)
        from bug_defense_b200 import campaign

        def probe():
            e = make_engine(geo, dev, seed_offset=1000 + rank)
            e.laser_power = POWER_W
            return e
        cand = None
        if args.plume_kernel is not None:
            cand = {_lib.TUNE_PLUME_KERNEL: [args.plume_kernel]}
        tuned = campaign.autotune(probe, candidates=cand)
        torch.cuda.synchronize()
        if rank == 0:
            print("autotune trials (ms per epoch):", json.dumps(tuned["trials"]), file=sys.stderr)
    if args.plume_kernel is not None:
        _lib.call("bd_tune_set", _lib.TUNE_PLUME_KERNEL, args.plume_kernel)
    from bug_defense_b200.replicas import replica_seed
    eng = make_engine(geo, dev, seed_offset=replica_seed(0, rank))
    K, W = int(args.steps), int(args.warmup)
    n_on = max(1, int(round(LASER_DUTY * K)))
    for _ in range(W):
        eng.power = POWER_W
        eng._enqueue(0)
    laser_diag = eng._diag(None) if W > 0 else None
    torch.cuda.synchronize()
    lib = _lib.load()
    lib.bd_engine_timing(eng._handle, 1)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(st)
        for s in range(K):
            eng.power = POWER_W if s < n_on else 0.0
            eng._enqueue(0)
        e1.record(st)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    stage = (ctypes.c_double * 4)()
    nep = ctypes.c_int64(0)
    _lib.check(lib.bd_engine_timing_read(eng._handle, stage, ctypes.byref(nep)))
    lib.bd_engine_timing(eng._handle, 0)
    stage_ms = list(stage)
    d = eng._diag(None)
    from bug_defense_b200.replicas import max_over_ranks
    ms = max_over_ranks(ms, device=dev)
    res = {"ms": ms, "K": K, "n_on": n_on, "stage_ms": stage_ms, "clocks": clk.summary(), "eng": eng, "geo": geo,
           "last_diag": d, "laser_diag": laser_diag, "tuned": tuned}
    return res


def e2e_run(args, geo, dev, K):
    """Same metric through the public API from host arrays: engine construction (upload of every
    field from host numpy), K epochs each returning the diagnostics dict, and the runner's per-epoch
    recording (xz slices of T, Q, phase and plume at mid-y, run_highres_knowledge_suite.py:280-306)
    through Recorder into pinned host memory."""
    import numpy as np
    import torch
    from bug_defense_b200.record import Recorder
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    from bug_defense_b200._device import upload_stats
    up0 = dict(upload_stats)
    e0.record(st)
    h0 = time.perf_counter()
    eng = make_engine(geo, dev, seed_offset=101)
    h1 = time.perf_counter()
    ec = torch.cuda.Event(enable_timing=True)
    ec.record(st)
    # bytes that crossed host->device (grids that are one z column broadcast over x and y travel as
    # that column) and the host input the constructor read
    h2d = upload_stats["bytes"] - up0["bytes"]
    host_in = sum(np.asarray(v).nbytes for v in (geo["optical"]["mu_a"], geo["optical"]["mu_s"], geo["optical"]["g"],
                                                 geo["optical"]["n"], geo["k_grid"], geo["rho_cp_grid"],
                                                 geo["h_lat_grid"], geo["dry_mask"], geo["ablated_mask"]))
    host_in += sum(np.asarray(geo["dry_state"][k]).nbytes for k in ("mu_a", "mu_s", "g", "n", "k", "rho_cp"))
    n_on = max(1, int(round(LASER_DUTY * K)))
    # the runner's per-epoch recording through the public Recorder: the device record kernel fills
    # a slot (xz slices of T, Q, phase and plume at mid-y, depth, band peaks) that is copied into a
    # pinned ring without a per-epoch synchronisation; step_epoch() returns the diagnostics dict
    rec = Recorder(eng, k_surface=geo["n_air_top"], ring=16)
    for s in range(K):
        eng.power = POWER_W if s < n_on else 0.0
        eng.step_epoch()
        rec.record()
    rec.finish()
    d2h = ctypes.sizeof(__import__("bug_defense_b200")._lib.EpochDiag) + rec.slot_bytes
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": K / (ms / 1e3), "unit": "epochs/s", "h2d_bytes_per_step": int(h2d / K),
            "d2h_bytes_per_step": int(d2h), "construct_ms": round(e0.elapsed_time(ec), 2),
            "construct_host_ms": round((h1 - h0) * 1e3, 2), "host_input_bytes": int(host_in),
            "construct_h2d_bytes": int(h2d),
            "column_grids": upload_stats["column_grids"] - up0["column_grids"],
            "full_grids": upload_stats["full_grids"] - up0["full_grids"],
            "epochs_ms": round(ec.elapsed_time(e1), 2), "note": "engine construction from host arrays + per-epoch diagnostics "
                                                     "and xz recording slices, amortised over the timed epochs"}


def full_run_leg(geo, dev):
    """The production schedule on the device: a fresh engine, 1000 epochs (200 laser-on at 40 W, then
    800 laser-off), enqueued without host synchronisation, timed by CUDA events (stage-graph capture
    included)."""
    import torch
    eng = make_engine(geo, dev, seed_offset=202)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for s in range(geo["epochs_total"]):
        eng.power = POWER_W if s < geo["epochs_on"] else 0.0
        eng._enqueue(0)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    d = eng._diag(None)
    return {"epochs": geo["epochs_total"], "laser_on_epochs": geo["epochs_on"], "ms": round(ms, 2),
            "epochs_per_s": round(geo["epochs_total"] / (ms / 1e3), 3), "void_zlimit_end": int(d["void_zlimit"]),
            "void_voxels_end": int(d["n_void"]),
            "crater_depth_mm_end": round(eng.centerline_depth_mm(k_surface=geo["n_air_top"]), 4)}


def ours_main(args):
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    r = run_ours(args, rank, world, local)
    eng, geo = r["eng"], r["geo"]
    K, ms = r["K"], r["ms"]
    value = K * world / (ms / 1e3)
    hbm, peak_kind, peaks = measured_peaks()
    # the plume domain grows as voxels are removed: average the first and last timed epochs
    n_void = 0.5 * (r["laser_diag"]["n_void"] + r["last_diag"]["n_void"]) if r["laser_diag"] else r["last_diag"]["n_void"]
    ab = algorithmic_bytes(eng, n_void)
    from bug_defense_b200.ablation import plume_steps_per_substep
    n_plume_sub, _ = plume_steps_per_substep(eng._desc.plume)
    stage = r["stage_ms"]
    stage_names = ["mc", "substeps", "plume", "epoch_end"]
    # dominant HBM-bound stage among the stencils
    launches_sub = eng.n_substeps * K
    launches_plume = eng.n_substeps * n_plume_sub * K
    per_launch = {"substeps": stage[1] / max(launches_sub, 1), "plume": stage[2] / max(launches_plume, 1)}
    dom = "substeps" if stage[1] >= stage[2] else "plume"
    bytes_per_launch = ab["substep"] if dom == "substeps" else ab["plume_step"]
    achieved = bytes_per_launch / (per_launch[dom] * 1e-3) / 1e9
    from bug_defense_b200 import _lib
    kv = ctypes.c_int(0)
    _lib.call("bd_tune_get", _lib.TUNE_PLUME_KERNEL, ctypes.byref(kv))
    plume_kernel = {4: "k_plume_direct_z", 6: "k_plume_direct_c"}.get(kv.value, "k_plume_step")
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        tj = json.loads(tf.read_text())
        key = {"substeps": "k_substep", "plume": plume_kernel.split("<")[0]}[dom]
        if key in tj:
            traffic = tj[key]["bytes_per_voxel"] * eng.Nx * eng.Ny * eng.Nz
    roof = {"bound": "hbm", "kernel": {"substeps": "k_substep<fused ablation>", "plume": plume_kernel}[dom],
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6650 GB/s", "algorithmic_bytes_per_launch": bytes_per_launch,
            "avg_launch_ms": round(per_launch[dom], 5),
            "units_per_launch": ("voxel-substeps" if dom == "substeps" else "plume (void) voxel-steps"),
            "void_voxels": int(n_void)}
    if dom == "plume":
        l2 = l2_copy_gbs(eng.dev)
        roof.update({"l2_peak": round(l2, 1), "l2_frac": round(achieved / l2, 4),
                     "l2_method": "best of 8, 16 and 32 MB device-to-device copies (L2-resident pairs), 100 "
                                  "copies replayed from one CUDA graph, read + written bytes / event time, "
                                  "measured in this run"})
    led = r["last_diag"]["ledger"]
    mc_ms = stage[0]
    photons = r["n_on"] * eng.n_photons
    mc = {"photons_per_s": photons / (mc_ms * 1e-3) if mc_ms > 0 else None,
          "mc_ms_per_laser_epoch": mc_ms / max(r["n_on"], 1)}
    if r["laser_diag"] is not None:
        from bug_defense_b200 import _lib as L_
        ld = r["laser_diag"]["ledger"]
        steps_per_epoch = float(ld[L_.LEDGER_COLLISIONS] + ld[L_.LEDGER_CROSSINGS])
        mc["photon_steps_per_laser_epoch"] = steps_per_epoch
        if mc_ms > 0:
            mc["photon_steps_per_s"] = steps_per_epoch * r["n_on"] / (mc_ms * 1e-3)
        lc = (ld[1:7].sum() + ld[8] + ld[9] - ld[7]) / max(ld[0], 1)
        mc["ledger_closure_minus_1"] = float(lc - 1.0)
        # issue-rate roof: SMs x 4 schedulers x 1 warp instruction per clock x 32 lanes / thread
        # instructions per photon-step (the count of one ncu capture, profiles/traffic.json)
        tf = ROOT / "profiles" / "traffic.json"
        ipp = json.loads(tf.read_text()).get("k_mc_trace", {}).get("thread_instructions_per_photon_step") \
            if tf.exists() else None
        if ipp and mc_ms > 0:
            import torch
            n_sm = torch.cuda.get_device_properties(eng.dev).multi_processor_count
            mhz = (r["clocks"] or {}).get("sm_mhz") or 1965.0
            roof_steps = n_sm * 4 * mhz * 1e6 * 32 / ipp
            mc["issue_roof_photon_steps_per_s"] = roof_steps
            mc["issue_roof_frac"] = round(mc["photon_steps_per_s"] / roof_steps, 4)
            mc["thread_instructions_per_photon_step"] = ipp
    # per epoch: begin + 3 epoch-end kernels + the plume stage's set-up (mask and z lists; with the
    # compact kernel the mask, bitmaps, unit counts, x-planes pick, z lists and unit list) + substeps +
    # plume steps; per laser epoch: MC, ledger reduction and tally finalisation
    plume_prep = 6 if kv.value == _lib.PLUME_KERNEL_COMPACT else 2
    gpu_launches = K * (1 + 3 + plume_prep + eng.n_substeps + eng.n_substeps * n_plume_sub) + r["n_on"] * 3
    out = {"metric": METRIC, "value": round(value, 3), "unit": "epochs/s", "n_gpus": world, "steps": K,
           "warmup": args.warmup, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (FP64 ledgers)", "data": "synthetic (seeded, reference config shapes)",
           "config": config_dict(geo, world, args.seed, n_plume_sub),
           "stage_ms_per_epoch": {n: round(v / K, 4) for n, v in zip(stage_names, stage)},
           "mc": mc, "roofline": roof, "clocks": r["clocks"], "gpu_launches": gpu_launches, "impl": "ours"}
    if r.get("tuned"):
        out["autotune"] = {k: v for k, v in r["tuned"].items() if k != "trials"}
    if rank == 0 and world == 1 and not args.no_e2e:
        import torch
        out["e2e"] = e2e_run(args, geo, torch.device("cuda", local), K)
    if rank == 0 and world == 1 and not args.small and not args.no_full_run:
        out["full_run"] = full_run_leg(geo, torch.device("cuda", local))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from bug_defense_b200.workloads import engine_kwargs
        out["cpu_baseline"] = cpu_port_baseline(geo, engine_kwargs(geo))
        if "full_run" in out:
            out["full_run"]["vs_cpu_port_full_run"] = round(
                out["full_run"]["epochs_per_s"] / out["cpu_baseline"]["full_run_epochs_per_s"], 2)
    if rank == 0 and world == 1 and not args.no_denoiser:
        out["denoiser"] = denoiser_leg()
        out["denoised_run"] = denoised_run_leg()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def denoiser_leg():
    """Denoised low-photon optical epoch vs the plain 150k-photon epoch on held-out random craters,
    both scored by relative L2 against a 1e8-photon map (outside the timed region)."""
    from bug_defense_b200 import denoise
    if not denoise.DEFAULT_WEIGHTS.exists():
        return {"unavailable": "no trained weights"}
    r = denoise.evaluate(denoise.Denoiser.load(), n_samples=3, ref_photons=100_000_000)
    keep = ("rel_l2_noisy", "rel_l2_denoised", "rel_l2_plain", "ms_mc_lo", "ms_net", "ms_mc_plain",
            "ms_denoised_path", "speedup_vs_plain", "lo_photons", "plain_photons", "ref_photons", "shape")
    out = {k: (round(v, 5) if isinstance(v, float) else v) for k, v in r.items() if k in keep}
    out["samples"] = len(r["samples"])
    out["workload"] = "random craters on the 200x200x128 stack (held-out seeds), GPU MC maps"
    return out


def denoised_run_leg(n_laser=10, check_every=5):
    """The denoised coupled run: the 532 nm and 1470 nm, 40 W runs at full resolution, laser-on epochs timed on the
    device with plain 150k-photon MC and with 15k photons through the denoiser (spot-checked against
    plain MC every `check_every` laser epochs), each on a fresh engine after 3 warm-up epochs."""
    import torch
    from bug_defense_b200 import campaign
    from bug_defense_b200.denoised import DenoisedCoupledRun
    insts = [i for i in campaign.campaign_instances(0) if i["power"] == 40.0 and i["wavelength_nm"] in (532.0, 1470.0)]
    out = []
    for inst in insts:
        row = {"wavelength_nm": inst["wavelength_nm"], "power_w": 40.0}
        for mode in ("plain", "denoised"):
            eng = campaign.make_engine(dict(inst, n_photons=150_000))
            eng.power = 40.0
            run = DenoisedCoupledRun(eng, check_every=check_every) if mode == "denoised" else None
            step = run.enqueue if run else (lambda: eng._enqueue(0))
            for _ in range(3):
                step()
            torch.cuda.synchronize()
            st = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(n_laser):
                step()
            e1.record(st)
            torch.cuda.synchronize()
            row[f"{mode}_ms_per_laser_epoch"] = round(e0.elapsed_time(e1) / n_laser, 3)
            if run:
                row["spot_checks"] = [{"rel_l2": round(r, 4), "bound": round(b, 4)} for _, r, b in run.checks]
                row["fell_back"] = run.fallen_back
            del eng, run
        row["speedup"] = round(row["plain_ms_per_laser_epoch"] / row["denoised_ms_per_laser_epoch"], 3)
        out.append(row)
    return {"runs": out, "laser_epochs_timed": n_laser,
            "note": "laser-on epochs of the full-resolution coupled run; the plume stage (one launch per FTCS "
                    "step, beside MC and the substeps) bounds the epoch, so a cheaper optical step shortens "
                    "the epoch only by what it removes from the plume stream's competition"}


def campaign_main(args):
    """24 instances (8 wavelengths x 3 powers, pulse U(50, 400) ms) of the full-resolution run at
    once; a step is one 1 ms epoch of every instance. Launch shapes from the autotuner."""
    import torch
    import torch.distributed as dist
    from bug_defense_b200 import campaign
    from bug_defense_b200.replicas import max_over_ranks, rank_share, sum_over_ranks
    rank, world, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    all_insts = campaign.campaign_instances(args.seed)
    if world > len(all_insts):
        raise ValueError(f"{world} ranks for {len(all_insts)} campaign instances")
    insts = rank_share(all_insts, rank, world)
    t0 = time.perf_counter()
    tuned = campaign.autotune(insts[0])
    t_tune = time.perf_counter() - t0
    camp = campaign.Campaign(insts, batch_plume=bool(args.batch_plume))
    camp.enqueue(args.warmup)
    camp.diagnostics()
    K = int(args.steps)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # every instance stream waits for ev0 and ev1 waits for every stream: device-timed makespan
    ev0.record()
    for st in camp.streams:
        st.wait_event(ev0)
    done = 0
    while done < K:
        k = min(100, K - done)
        camp.enqueue(k)
        done += k
    for st in camp.streams:
        torch.cuda.current_stream().wait_stream(st)
    ev1.record()
    torch.cuda.synchronize()
    # whole job: every rank's instances over the slowest rank's device-timed makespan
    ms = max_over_ranks(ev0.elapsed_time(ev1), device=dev)
    n_inst = int(sum_over_ranks(len(insts), device=dev))
    diags = camp.diagnostics()
    value = n_inst * K / (ms / 1e3)
    out = {"metric": "campaign instance-epochs/s (24 full-resolution instances at once)", "value": round(value, 3),
           "unit": "instance-epochs/s", "n_gpus": world, "steps": K, "warmup": args.warmup,
           "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
           "dtype": "f32 (FP64 ledgers)", "data": "synthetic (seeded, reference config shapes)",
           "config": {"workload": "campaign: 8 wavelengths x 3 powers, pulse U(50, 400) ms, 200x200x192 @ 15 um, "
                                  "150k photons per laser epoch", "instances": n_inst,
                      "parallelism": f"instances split over {world} rank(s)",
                      "plume_stage": ("batched: one launch per FTCS step over every instance's live units"
                                      if camp.batch is not None else "one stage per instance")},
           "autotune": {k: v for k, v in tuned.items()}, "autotune_s": round(t_tune, 1),
           "setup_s": round(camp.setup_s, 1),
           "void_voxels_end": [int(d["n_void"]) for d in diags],
           "impl": "ours"}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def config_dict(geo, world, seed, n_plume_sub):
    return {"workload": "full-resolution coupled run: 200x200x128 stack + 64 plume air slices "
                        "(200x200x192 @ 15 um), 150k photons/laser epoch, 20 x 50 us substeps, "
                        f"laser on for the first {int(LASER_DUTY * 100)} % of timed epochs",
            "voxels": int(np.prod(geo["shape"])), "photons_per_laser_epoch": int(geo["n_photons"]),
            "plume_D_mm2_s": round(geo["plume_D"], 3), "plume_steps_per_substep": n_plume_sub,
            "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (>= 30 MB per field)", "seed": seed}


def reference_main(args):
    """The reference's CPU path (the FP64 C port of it, all host threads) on the same workload and
    schedule as the repo arm: W untimed warm-up epochs with the laser on, then K timed epochs with the
    laser on for the first 20 %. Rank 0 only."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    import oracle
    from oracle import plume_policy
    from oracle.engine import OracleEngine
    from bug_defense_b200 import workloads
    geo = workloads.full_coupled_run(seed=args.seed)
    kw = workloads.engine_kwargs(geo)
    oracle.build()
    oracle.set_threads(_threads())
    eng = OracleEngine(**kw, plume_dt_policy="subcycle")
    p = eng.plume
    n_sub = plume_policy(eng.dt_sub, eng.dx, eng.dy, eng.dz, p["D_xy"], p["D_z"], p["v"], p["tau"], "subcycle")[0]
    K, W = int(args.steps), int(args.warmup)
    n_on = max(1, int(round(LASER_DUTY * K)))
    for _ in range(W):
        eng.power = POWER_W
        eng.step_epoch()
    t_on, t_off = [], []
    t0 = time.perf_counter()
    for s in range(K):
        eng.power = POWER_W if s < n_on else 0.0
        a = time.perf_counter()
        eng.step_epoch()
        (t_on if s < n_on else t_off).append(time.perf_counter() - a)
    sec = time.perf_counter() - t0
    value = K / sec
    cb = {"value": round(value, 5), "unit": "epochs/s", "cores": _threads(), "kind": "port",
          "sample": f"{W} warm-up + {K} timed epochs of the workload ({n_on} laser-on, {K - n_on} laser-off) on the FP64 "
                    f"C port of the reference CPU path (oracle/orc.c, OpenMP, {_threads()} threads)",
          "t_on_median_s": round(statistics.median(t_on), 4),
          "t_off_median_s": round(statistics.median(t_off), 4) if t_off else None}
    if t_off:
        cb["full_run_epochs_per_s"] = round(full_run_rate(statistics.median(t_on), statistics.median(t_off)), 4)
    out = {"metric": METRIC, "value": round(value, 5), "unit": "epochs/s", "n_gpus": world, "steps": K,
           "warmup": W, "ms_per_step": round(1e3 * sec / K, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, reference config shapes)",
           "config": config_dict(geo, world, args.seed, n_sub),
           "impl": "reference", "cpu_baseline": cb,
           "e2e": {"value": round(value, 5), "unit": "epochs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        reference_main(a)
    elif a.workload == "campaign":
        campaign_main(a)
    else:
        ours_main(a)
