#!/usr/bin/env python
"""Throughput of the B200 3-D elastic solver on its headline workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload size_cap|reference_default|two_layer_2d|survey_windows]

One bench step is one leapfrog time step (velocity + stress update, CPML, source and
receiver sampling) over the whole grid.  Default workload: the 300 x 300 x 400 grid at the
reference's 36 M-node size cap (vp gradient + seeded smoothed noise, 6-face 20-cell CPML,
Ricker 12 Hz, dt 0.6 ms, 300 receivers); the model (2.6 GB of fields and materials) is far
larger than the 126 MB L2, so no flush is needed between steps.

Printed: one JSON line with the throughput in Gcell-updates/s (active nodes incl. CPML,
excl. ghosts, per step), the HBM roofline of the step under the compulsory-traffic model
84 B/cell + 48 B/CPML-slab-cell, the end-to-end rate through the public API with host
buffers, and the CPU baseline (the oracle restatement on the host cores).

`--impl reference` runs the reference's own CUDA solver (cuda/Cuda_Seis3D.cu compiled
unmodified into oracle/_ref) through its own API on the same workload and device.
Multi-GPU (torchrun): every rank runs its own shot (independent units, no collective on
the data path: weak scaling); the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
WORLD = int(os.environ.get("WORLD_SIZE", "1"))
RANK = int(os.environ.get("RANK", "0"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))
# The GPU this process measures, as nvidia-smi names it (an index or a UUID).  nvidia-smi
# ignores CUDA_VISIBLE_DEVICES, so the clock sampler is given this name explicitly.
_VISIBLE = [d.strip() for d in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if d.strip()]
GPU_ID = (_VISIBLE[LOCAL_RANK] if LOCAL_RANK < len(_VISIBLE) else str(LOCAL_RANK)) if WORLD > 1 else \
    (_VISIBLE[0] if _VISIBLE else "0")
if WORLD > 1:
    # One GPU per rank; the ranks share nothing on the data path.
    os.environ["CUDA_VISIBLE_DEVICES"] = GPU_ID
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

METRIC = "3D elastic Gcell-updates/s & %HBM roofline; shots/h vs plain at 1e-3 trace err"
UNIT = "Gcell-updates/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------------------
# Clocks during the timed region.
# --------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: str):
        self.device_index = device_index
        self.samples = []
        self.proc = None
        self.window = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(1.0)

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), line.strip()))

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        t0, t1 = self.window or (0, float("inf"))
        rows = [s for t, s in self.samples if t0 - 0.15 <= t <= t1 + 0.15] or [s for _, s in self.samples[-3:]]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in rows:
            parts = [p.strip() for p in row.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------------------
# Workload.
# --------------------------------------------------------------------------------------
def make_shot(name: str, steps: int, api=None):
    """The workload's shot; `api` builds its context and source (this solver's host code by
    default; the reference arm passes the reference's own, oracle.ReferenceApi)."""
    from cmakepro_cuda_seissim_v2_b200 import models3d

    if name == "size_cap":
        shot = models3d.size_cap_shot(steps=steps, api=api)
    elif name == "reference_default":
        shot = models3d.reference_default_shot(steps=steps, api=api)
    else:
        raise SystemExit(f"unknown workload {name}")
    if WORLD > 1:
        # Independent shot per rank: move the source along x.
        shot.source.x3D = 20 + (shot.source.x3D + 37 * RANK) % (shot.context.nx3D - 40)
    return shot


STORAGE_LABELS = {"fp32": "fp32", "bf16_cpml": "fp32 fields and materials, bf16 CPML memories"}


def workload_config(shot, storage: str = "fp32") -> dict:
    """The `config` object of a 3-D line; both arms print the same one."""
    c = shot.context
    return {"workload": shot.name, "grid": [c.nx3D, c.ny3D, c.nz3D], "padded": [c.gx3D, c.gy3D, c.gz3D],
            "active_cells": shot.active_cells, "cpml_slab_cells": slab_cells(c), "pml": c.pml3D,
            "free_surface": bool(c.freeSurface3D), "dt_s": float(c.dt3D), "receivers": int(len(shot.receivers)),
            "gather_stride": int(shot.stride), "storage": STORAGE_LABELS[storage], "parallelism": f"shots{WORLD}",
            "l2": "inputs larger than L2 (fields+materials %.2f GB vs 126 MB)" % (
                12 * 4 * c.gx3D * c.gy3D * c.gz3D / 1e9)}


def slab_cells(c) -> int:
    """Active cells inside each axis's CPML slab, summed over axes."""
    nxa, nya, nza = c.gx3D - 8, c.gy3D - 8, c.gz3D - 8
    if c.reflecting3D:
        return 0
    p = c.pml3D
    return 2 * p * nya * nza + 2 * p * nxa * nza + (1 if c.freeSurface3D else 2) * p * nxa * nya


def step_bytes(c, storage: str = "fp32") -> int:
    """Compulsory HBM bytes of one step: 9 fields read+written, 3 materials read (84 B/cell)
    plus 6 CPML memories read+written per slab cell (48 B in FP32, 24 B in BF16)."""
    nact = (c.gx3D - 8) * (c.gy3D - 8) * (c.gz3D - 8)
    return 84 * nact + (24 if storage == "bf16_cpml" else 48) * slab_cells(c)


def measured_peak():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            peaks = json.load(f)
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic(workload: str):
    """DRAM bytes per step from the committed ncu summary of this workload, if any."""
    path = os.path.join(HERE, "profiles", f"traffic_{workload}.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# --------------------------------------------------------------------------------------
# Distributed plumbing (timing reduction only).
# --------------------------------------------------------------------------------------
def init_dist():
    if WORLD <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def reduce_max(dist, value: float) -> float:
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------------------
# CPU baseline: the oracle restatement (FP32, OpenMP over z planes) on the host cores.
# --------------------------------------------------------------------------------------
def cpu_baseline(shot, budget_s: float):
    import oracle

    threads = os.cpu_count() or 1
    o = oracle.CpuOracle(shot.context, 32, threads=threads)
    o.upload_model(shot.vp, shot.vs, shot.rho)
    t = time.perf_counter()
    o.step(shot.source, 0)
    one = time.perf_counter() - t
    n = max(1, min(200, int(budget_s / max(one, 1e-6))))
    t = time.perf_counter()
    o.run(shot.source, 1, n)
    dt = time.perf_counter() - t
    o.close()
    rate = shot.active_cells * n / dt / 1e9
    return {"value": round(rate, 5), "unit": UNIT, "cores": int(o.lib.oracle3d_max_threads()), "kind": "port",
            "sample": f"{shot.name}: {n} steps (after 1 untimed) of the FP32 oracle restatement, OpenMP over z planes, "
                      f"{dt:.1f} s"}


# --------------------------------------------------------------------------------------
# Our solver.
# --------------------------------------------------------------------------------------
STORAGE_MODES = {"fp32": 0, "bf16_cpml": 3}        # enum seis3d_storage
THIN_PML = 6                                       # CPML cells of the learned-boundary mode
E2E_REPEATS = 3
FULL_STEPS = {"size_cap": 2500, "reference_default": 2000}   # run length of one shot


def storage_check(shot, steps: int, storage: int) -> dict:
    """Trace change of a 16-bit storage mode: the whole shot (`steps` steps, the workload's
    receivers and stride) run in FP32 storage and in `storage`, gathers compared (relative L2)."""
    from cmakepro_cuda_seissim_v2_b200 import seis3d

    gathers = []
    for mode in (0, storage):
        s = seis3d.Session(shot.context, storage=mode, tune=True)
        s.upload_model(shot.vp, shot.vs, shot.rho)
        s.set_receivers(shot.receivers)
        s.gather_begin(shot.stride, steps // shot.stride)
        s.run_steps(shot.source, 0, steps)
        gathers.append(s.gather_fetch().astype(np.float64))
        s.release()
    a, b = gathers
    return {"steps": steps, "trace_rel_l2_vs_fp32_storage": float(np.linalg.norm(b - a) / np.linalg.norm(a))}


def run_ours(args, dist):
    import torch

    from cmakepro_cuda_seissim_v2_b200 import build, seis3d

    build.build()
    torch.cuda.init()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    shot = make_shot(args.workload, args.steps)
    c = shot.context
    # The z chunk is tuned at initialisation (timed on the zeroed fields) unless given.
    storage = STORAGE_MODES[args.storage]
    s = seis3d.Session(c, storage=storage, tile_y=args.tile_y, z_chunk=args.z_chunk, tune=args.z_chunk == 0)
    z_chunk = s.z_chunk()[1]
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.gather_begin(shot.stride, (args.warmup + args.steps) // shot.stride + 1)
    stream = torch.cuda.ExternalStream(s.views().stream3D)

    # Warm-up (W steps), then capture the step graph outside the timed region.
    s.run_steps(shot.source, 0, args.warmup)
    s.prepare_steps(shot.source)
    s.synchronize()

    sampler = ClockSampler(GPU_ID)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = s.views().kernelLaunches
    barrier(dist)
    torch.cuda.synchronize()
    w0 = time.time()
    e0.record(stream)
    s.run_steps(shot.source, args.warmup, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    barrier(dist)
    sampler.mark(w0, w1)
    sampler.stop()
    launches = s.views().kernelLaunches - launches0
    ms_local = e0.elapsed_time(e1)
    ms = reduce_max(dist, ms_local)
    gather = s.gather_fetch()
    finite = bool(np.all(np.isfinite(gather)))

    # Per-pass device times (untimed diagnostic, graph-free launches).
    passes = s.profile_steps(shot.source, args.warmup + args.steps, min(20, args.steps))

    cells = shot.active_cells
    value = WORLD * cells * args.steps / (ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    bytes_step = step_bytes(c, args.storage)
    achieved = bytes_step * args.steps / (ms_local / 1e3) / 1e9
    traffic = committed_traffic(args.workload) if args.storage == "fp32" else None

    # End to end through the public API with host buffers: model upload (H2D), reset,
    # K steps with the device gather, gather read-back (D2H).
    # Repeated E2E_REPEATS times, each a complete upload-run-read cycle; the median is
    # reported (a host-side stall of a second was seen once in four runs) with every sample.
    e2e = None
    if not args.no_e2e:
        walls = []
        for _ in range(E2E_REPEATS):
            barrier(dist)
            t = time.perf_counter()
            s.gather_end()
            s.upload_volumes(shot.vp, shot.vs, shot.rho)
            s.reset()
            s.gather_begin(shot.stride, args.steps // shot.stride)
            s.run_steps(shot.source, 0, args.steps)
            g2 = s.gather_fetch()
            walls.append(reduce_max(dist, time.perf_counter() - t))
        dt = float(np.median(walls))
        h2d = shot.vp.size * 3 * 4
        d2h = g2.size * 4
        e2e = {"value": round(WORLD * cells * args.steps / dt / 1e9, 4), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d // args.steps), "d2h_bytes_per_step": int(d2h // args.steps),
               "wall_s": round(dt, 4), "wall_s_samples": [round(w, 4) for w in walls],
               "statistic": "median of %d complete runs" % E2E_REPEATS,
               "path": "seis3d_upload_model (host volumes) + reset + gather_begin + run_steps + gather_fetch"}
    s.release()
    full_steps = FULL_STEPS[args.workload]
    shot_line = {"steps": full_steps, "shots_per_hour_per_gpu": round(3600.0 / (full_steps * ms / args.steps / 1e3), 1)}
    if args.storage != "fp32" and not args.no_storage_check:
        shot_line["storage_check"] = storage_check(shot, full_steps, storage)

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": WORLD, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(shot, args.storage),
        "launch": {"z_chunk": z_chunk, "z_chunk_tuned": args.z_chunk == 0, "tile": [32, 16]},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic.get("dram_bytes_per_step") if traffic else None,
                     "kernel": "one step = velocityPass + stressPass + step tail (free-surface images inside the passes)",
                     "bytes_per_step": bytes_step,
                     "model": "84 B/active cell + %d B/CPML slab cell" % (24 if args.storage == "bf16_cpml" else 48)},
        "passes_ms_per_step": {k: round(v / min(20, args.steps), 5) for k, v in passes.items()},
        "shot": shot_line,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": sampler.summary(),
        "gather_finite": finite,
    }
    return line, shot


# --------------------------------------------------------------------------------------
# Windowed multi-shot survey (shots/hour; not the headline line): the first `--shots` shots of
# the 600 x 200 x 600 survey, each on its cropped window, every shot run for `--steps` steps
# (the survey's 1500 by default) from a reset state.  Two arms on the same resident sessions:
# "plain" runs the shots one after another (seis3d_run_steps, wait, next shot); "batched"
# steps them together through seis3d_batch_run_steps with the tuner on.  Both record every
# 2nd step of every shot on the device; their gathers must be bit-identical.
# --------------------------------------------------------------------------------------
SURVEY_STRIDE = 2


def run_ours_survey(args):
    import torch

    from cmakepro_cuda_seissim_v2_b200 import build, models3d, seis3d

    build.build()
    torch.cuda.init()
    torch.cuda.set_device(0)
    steps = args.steps
    base = models3d.window_survey(steps=steps)
    # --thin-cpml: the same windows with the 6-cell CPML of the learned-boundary mode (with its
    # networks at the selected gain 0, i.e. the thin layer alone).
    survey = dataclasses.replace(base, pml=THIN_PML) if args.thin_cpml else base
    shots = survey.shots[:args.shots]
    storage = STORAGE_MODES[args.storage]
    sessions, sources = [], []
    for shot in shots:
        s = seis3d.Session(survey.context(shot), storage=storage, thin_cpml=args.thin_cpml)
        s.upload_volumes(*survey.window(shot))
        s.set_receivers(survey.receivers(shot))
        sessions.append(s)
        sources.append(survey.source(shot))
    samples = steps // SURVEY_STRIDE

    def restart():
        for s in sessions:
            s.gather_end()
            s.reset()
            s.gather_begin(SURVEY_STRIDE, samples)
        torch.cuda.synchronize()

    # Warm-up: W steps of every shot on its own, then the per-session step graphs exist.
    for s, src in zip(sessions, sources):
        s.gather_begin(SURVEY_STRIDE, samples)
        s.run_steps(src, 0, args.warmup)
        s.prepare_steps(src)
    for s in sessions:
        s.synchronize()
    sampler = ClockSampler(GPU_ID)
    sampler.start()

    # Plain: one shot after another.
    restart()
    w0 = time.time()
    plain_ms = 0.0
    launches0 = sum(s.views().kernelLaunches for s in sessions)
    for s, src in zip(sessions, sources):
        stream = torch.cuda.ExternalStream(s.views().stream3D)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.run_steps(src, 0, steps)
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
    plain_launches = sum(s.views().kernelLaunches for s in sessions) - launches0
    plain_gathers = [s.gather_fetch() for s in sessions]

    # Batched, tuned on its first steps (the tuning steps are part of the timed run).
    restart()
    batch = seis3d.Batch(sessions, tune=True)
    stream = torch.cuda.ExternalStream(batch.info()["stream"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.run_steps(sources, 0, steps)
    e1.record(stream)
    e1.synchronize()
    batch.synchronize()
    w1 = time.time()
    sampler.mark(w0, w1)
    sampler.stop()
    batch_ms = e0.elapsed_time(e1)
    info = batch.info()
    batch_gathers = [s.gather_fetch() for s in sessions]
    identical = all(np.array_equal(a, b) for a, b in zip(plain_gathers, batch_gathers))
    finite = all(bool(np.all(np.isfinite(g))) for g in batch_gathers)

    # End to end through the public API with host buffers: every window's model uploaded from
    # host memory, reset, the batched run (tuned already), every gather read back.
    windows = [survey.window(shot) for shot in shots]
    t = time.perf_counter()
    for s, w in zip(sessions, windows):
        s.gather_end()
        s.upload_volumes(*w)
        s.reset()
        s.gather_begin(SURVEY_STRIDE, samples)
    batch.run_steps(sources, 0, steps)
    batch.synchronize()
    e2e_gathers = [s.gather_fetch() for s in sessions]
    e2e_s = time.perf_counter() - t
    identical = identical and all(np.array_equal(a, b) for a, b in zip(plain_gathers, e2e_gathers))
    h2d = sum(sum(a.nbytes for a in w) for w in windows)
    d2h = sum(g.nbytes for g in e2e_gathers)
    batch.release()
    for s in sessions:
        s.release()

    # A 16-bit storage mode or the thin CPML is also measured against the plain FP32 form with
    # the 20-cell CPML: every shot so, one after another (the same timing as the plain arm), and
    # the batched gathers' change against those gathers.
    fp32 = None
    if storage != 0 or args.thin_cpml:
        fp32_ms, change = 0.0, 0.0
        for shot, src, g in zip(shots, sources, batch_gathers):
            f = seis3d.Session(base.context(shot))
            f.upload_volumes(*base.window(shot))
            f.set_receivers(base.receivers(shot))
            f.gather_begin(SURVEY_STRIDE, samples)
            f.run_steps(src, 0, args.warmup)
            f.prepare_steps(src)
            f.gather_end()
            f.reset()
            f.gather_begin(SURVEY_STRIDE, samples)
            stream = torch.cuda.ExternalStream(f.views().stream3D)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            f.run_steps(src, 0, steps)
            e1.record(stream)
            e1.synchronize()
            fp32_ms += e0.elapsed_time(e1)
            ref = f.gather_fetch().astype(np.float64)
            f.release()
            change = max(change, float(np.linalg.norm(g.astype(np.float64) - ref) / np.linalg.norm(ref)))
        fp32 = {"value": round(len(shots) * 3600.0 / (fp32_ms / 1e3), 1), "unit": "shots/h", "ms": round(fp32_ms, 2),
                "batched_speedup": round(fp32_ms / batch_ms, 4), "max_trace_rel_l2_vs_fp32": change}

    cells = sum(survey.active_cells(shot) for shot in shots)
    n = len(shots)
    value = n * 3600.0 / (batch_ms / 1e3)
    plain = n * 3600.0 / (plain_ms / 1e3)
    line = {
        "metric": "shots/h of the windowed survey (batched + tuned vs plain, %s)" % (
            ("FP32" if args.storage == "fp32" else args.storage) + (", 6-cell CPML" if args.thin_cpml else "")), "value": round(value, 1),
        "unit": "shots/h", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(batch_ms / steps, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": survey.name, "shots_timed": n, "windows": [list(q.size) for q in shots],
                   "active_cells_per_step": cells, "steps_per_shot": steps, "gather_stride": SURVEY_STRIDE,
                   "receivers_per_shot": 150, "storage": STORAGE_LABELS[args.storage], "cpml_cells": survey.pml,
                   "l2": "inputs larger than L2 (every window's fields and materials exceed 126 MB)"},
        "plain": {"value": round(plain, 1), "unit": "shots/h", "ms": round(plain_ms, 2),
                  "gcell_per_s": round(cells * steps / (plain_ms / 1e3) / 1e9, 3), "gpu_launches": plain_launches},
        "batched": {"ms": round(batch_ms, 2), "gcell_per_s": round(cells * steps / (batch_ms / 1e3) / 1e9, 3),
                    "speedup_vs_plain": round(plain_ms / batch_ms, 4), "shots_per_launch": info["shots_per_launch"],
                    "z_chunk": info["z_chunk"], "tuned_candidates": info["candidates"],
                    "tuned_ms_per_step": round(info["tuned_ms_per_step"], 4)},
        "gathers_identical": identical, "gather_finite": finite,
        "plain_fp32": fp32,
        "e2e": {"value": round(n * 3600.0 / e2e_s, 1), "unit": "shots/h", "h2d_bytes_per_step": int(h2d // steps),
                "d2h_bytes_per_step": int(d2h // steps), "wall_s": round(e2e_s, 3),
                "path": "seis3d_upload_model per window + reset + gather_begin + seis3d_batch_run_steps + "
                        "gather_fetch per shot"},
        "gpu_launches": int(info["kernel_launches"]),
        "clocks": sampler.summary(),
    }
    return line


def run_reference_survey(args):
    """The reference's own CUDA solver on the same windows, one shot after another through its
    API (initializeGpu3D per window, plane uploads, runStep3D per step): a bounded sample of
    `--reference-steps` steps of each timed shot, scaled to the full run length."""
    import oracle

    if oracle.reference_library() is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/libref3d.so is missing"}
    import torch

    from cmakepro_cuda_seissim_v2_b200 import models3d

    torch.cuda.init()
    survey = models3d.window_survey(steps=args.steps)
    shots = survey.shots[:args.shots]
    sample = min(args.reference_steps, args.steps)
    ms_total = 0.0
    for shot in shots:
        r = oracle.ReferenceSolver(survey.context(shot))
        r.upload_model(*survey.window(shot))
        r.set_receivers(survey.receivers(shot))
        r.run(survey.source(shot), 0, 3)
        r.synchronize()
        ms_total += r.time_steps(survey.source(shot), 3, sample) * args.steps / sample
        r.close()
    value = len(shots) * 3600.0 / (ms_total / 1e3)
    return {"impl": "reference", "metric": "shots/h of the windowed survey (batched + tuned vs plain, FP32)",
            "value": round(value, 1), "unit": "shots/h", "n_gpus": 1, "steps": args.steps, "warmup": 3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": survey.name, "shots_timed": len(shots)},
            "cpu_baseline": {"value": round(value, 1), "unit": "shots/h", "cores": 1, "kind": "reference",
                             "sample": f"reference CUDA solver, {sample} runStep3D calls per shot scaled to "
                                       f"{args.steps}", "device": "cuda:0"},
            "e2e": {"value": round(value, 1), "unit": "shots/h", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# --------------------------------------------------------------------------------------
# Reference arm: the reference's own CUDA solver built from its source.
# --------------------------------------------------------------------------------------
def run_reference(args):
    import oracle

    if oracle.reference_library() is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/libref3d.so (reference cuda/Cuda_Seis3D.cu built "
                                                    "from its source) is missing: run `make -C oracle` with the "
                                                    "reference tree"}
    import torch

    torch.cuda.init()
    # Context, padding and dt come from the reference's own host code: this process never
    # loads the B200 solver library.
    shot = make_shot(args.workload, args.steps, api=oracle.ReferenceApi())
    c = shot.context
    r = oracle.ReferenceSolver(c)
    r.upload_model(shot.vp, shot.vs, shot.rho)
    r.set_receivers(shot.receivers)
    r.run(shot.source, 0, args.warmup)
    r.synchronize()
    sampler = ClockSampler(GPU_ID)
    sampler.start()
    torch.cuda.synchronize()
    w0 = time.time()
    ms = r.time_steps(shot.source, args.warmup, args.steps)
    torch.cuda.synchronize()
    w1 = time.time()
    sampler.mark(w0, w1)
    sampler.stop()
    cells = shot.active_cells
    value = cells * args.steps / (ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    achieved = step_bytes(c) * args.steps / (ms / 1e3) / 1e9
    e2e = None
    if not args.no_e2e:
        # The reference's own loop: plane upload, reset, runStep3D per step and
        # sampleReceivers3D (D2H + stream sync) every `stride` steps (src/Seis3D_Sim.cpp:120-153);
        # the same statistic as the other arm (median of E2E_REPEATS complete runs).
        walls = []
        for _ in range(E2E_REPEATS):
            t = time.perf_counter()
            r.upload_model(shot.vp, shot.vs, shot.rho)
            r.reset()
            g = r.run_gather(shot.source, 0, args.steps, shot.stride)
            walls.append(time.perf_counter() - t)
        dt = float(np.median(walls))
        h2d = shot.vp.size * 3 * 4
        d2h = g.size * 4
        e2e = {"value": round(cells * args.steps / dt / 1e9, 4), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d // args.steps), "d2h_bytes_per_step": int(d2h // args.steps),
               "wall_s": round(dt, 4), "wall_s_samples": [round(w, 4) for w in walls],
               "statistic": "median of %d complete runs" % E2E_REPEATS,
               "path": "uploadModelPlane3D x nz + finishModelUpload3D + resetGpu3D + runStep3D per step + "
                       "sampleReceivers3D every stride steps"}
    r.close()
    mapped = [p for p in oracle.loaded_libraries() if os.path.basename(p).startswith("libseis")]
    if mapped:
        raise SystemExit(f"reference arm mapped this project's solver library: {mapped}")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(shot),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "model": "84 B/active cell + 48 B/CPML slab cell"},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"reference CUDA solver (cuda/Cuda_Seis3D.cu built unmodified, sm_100a) on "
                                   f"cuda:0, {args.steps} runStep3D calls driven by one host thread",
                         "device": "cuda:0"},
        "e2e": e2e,
        "clocks": sampler.summary(),
    }
    return line


# --------------------------------------------------------------------------------------
# 2-D P-SV workload (the 440 x 420 two-layer free-surface shot; not the headline line).
# --------------------------------------------------------------------------------------
BYTES_2D = 96  # 10 split fields read + written, 4 materials read, per active cell and step


def run_ours_2d(args):
    import torch

    from cmakepro_cuda_seissim_v2_b200 import build, models2d, seis2d

    build.build()
    torch.cuda.init()
    shot = models2d.two_layer_shot(max(args.steps + args.warmup, 1))
    c = shot.context
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, c)
    seis2d.gatherBegin(gpu, 0, 1, args.warmup + args.steps)
    seis2d.runGpuSimulationSteps(gpu, 0, args.warmup, c)
    seis2d.synchronize(gpu)
    stream = torch.cuda.ExternalStream(gpu.views().stream)
    sampler = ClockSampler(GPU_ID)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = gpu.kernelLaunches
    torch.cuda.synchronize()
    w0 = time.time()
    e0.record(stream)
    seis2d.runGpuSimulationSteps(gpu, args.warmup, args.steps, c)
    e1.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    sampler.mark(w0, w1)
    sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = gpu.kernelLaunches - launches0
    passes = seis2d.profileSteps(gpu, args.warmup + args.steps, min(50, args.steps), c)
    cells = shot.active_cells
    value = cells * args.steps / (ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    achieved = BYTES_2D * cells * args.steps / (ms / 1e3) / 1e9
    # End to end through the public API: context upload (initialize), the run with the
    # device gather, the gather read-back.
    t = time.perf_counter()
    seis2d.initializeGpuSimulation(gpu, c)
    seis2d.gatherBegin(gpu, 0, 1, args.steps)
    seis2d.runGpuSimulationSteps(gpu, 0, args.steps, c)
    gvx, gvz, _ = seis2d.gatherFetch(gpu, args.steps)
    dt = time.perf_counter() - t
    h2d = 4 * (c.rho.size * 4 + c.NX * 2 + c.NZ * 2 + c.dp_flat.size + c.wavelet.size) + 4 * c.num_rcv
    d2h = gvx.nbytes + gvz.nbytes
    seis2d.releaseGpuSimulation(gpu)
    line = {
        "metric": "2D P-SV Gcell-updates/s", "value": round(value, 4), "unit": "Gcell-updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 6),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": shot.name, "grid": [c.NX, c.NZ], "active_cells": cells, "npml": c.npml,
                   "scheme": "free surface + split-field PML (flag_type 3)", "receivers": int(c.num_rcv),
                   "l2": "working set 10 MB: L2-resident, no flush (launch- and latency-bound)"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": None,
                     "model": "96 B/active cell (10 split fields RW + 4 materials)"},
        "passes_ms_per_step": {k: round(v / min(50, args.steps), 6) for k, v in passes.items()},
        "e2e": {"value": round(cells * args.steps / dt / 1e9, 4), "unit": "Gcell-updates/s",
                "h2d_bytes_per_step": int(h2d // args.steps), "d2h_bytes_per_step": int(d2h // args.steps),
                "wall_s": round(dt, 4), "path": "initializeGpuSimulation + gatherBegin + run_steps + gatherFetch"},
        "gpu_launches": int(launches),
        "clocks": sampler.summary(),
    }
    return line, shot


# --------------------------------------------------------------------------------------
# Learned thin boundary (not the headline line): training on the solver's own lock-step
# thin/wide runs, then a held-out 300 x 50 x 300 layered model run with a 6-cell CPML and the
# networks, compared with the 20-cell CPML by reflected energy and traces (both against a
# 40-cell run), and timed against the 20-cell run as shots per hour.
# --------------------------------------------------------------------------------------
def run_learned_boundary(args):
    import torch

    from cmakepro_cuda_seissim_v2_b200 import build, learned_boundary as lb

    build.build()
    torch.cuda.init()
    t = time.perf_counter()
    net, gain, report = lb.train_boundary(models=args.lb_models, size=args.lb_size, steps=args.lb_steps,
                                          fraction=args.lb_fraction, rows_per_face=3_000_000,
                                          iterations=args.lb_iterations,
                                          batch=4096, lr=1e-3)
    train_s = time.perf_counter() - t
    model = lb.random_layered_model(300, 50, 300, 777)
    res = lb.evaluate(model, net, args.steps, gains=(gain,) if gain > 0 else (0.5,))
    dt_ms = res["dt_ms"]
    timing = {"thin+net": lb.step_time(model, 6, 200, dt_ms, net, gain if gain > 0 else 0.5),
              "thin": lb.step_time(model, 6, 200, dt_ms), "cpml20": lb.step_time(model, 20, 200, dt_ms)}
    net.release()
    shots = {k: 3600.0 / (v * args.steps / 1e3) for k, v in timing.items()}
    learned_key = [k for k in res if k.startswith("thin+net")][0]
    line = {
        "metric": "shots/h of a held-out 300x50x300 model: 6-cell CPML + learned boundary vs 20-cell CPML",
        "value": round(shots["thin+net"], 1), "unit": "shots/h", "n_gpus": 1, "steps": args.steps, "warmup": 10,
        "ms_per_step": round(timing["thin+net"], 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 solver, bf16 network", "data": "synthetic",
        "config": {"workload": "random layered 300x50x300 (seed 777), free surface, Ricker %.1f Hz" % model.frequency,
                   "training": dict({k: report[k] for k in ("models", "size", "steps", "rows", "iterations", "batch",
                                                             "collect_s", "train_s")}, fraction=args.lb_fraction),
                   "selected_gain": gain, "validation_energy": report["validation_energy"]},
        "shots_per_hour": {k: round(v, 1) for k, v in shots.items()},
        "errors_vs_cpml40": {k: {kk: vv for kk, vv in v.items() if kk != "ms"} for k, v in res.items()
                             if isinstance(v, dict) and "trace_rel_l2" in v},
        "learned_vs_thin": {"reflected_energy": round(res[learned_key]["reflected_energy"] /
                                                      res["thin"]["reflected_energy"], 4),
                            "trace_rel_l2": round(res[learned_key]["trace_rel_l2"] / res["thin"]["trace_rel_l2"], 4)},
        "train_wall_s": round(train_s, 1),
    }
    return line


def cpu_baseline_2d(shot, budget_s: float):
    import oracle

    o = oracle.CpuOracle2D(shot.context, 32)
    t = time.perf_counter()
    o.run(0, 10)
    one = (time.perf_counter() - t) / 10
    n = max(10, min(shot.steps, int(budget_s / max(one, 1e-6))))
    t = time.perf_counter()
    o.run(10, n)
    dt = time.perf_counter() - t
    o.close()
    return {"value": round(shot.active_cells * n / dt / 1e9, 5), "unit": "Gcell-updates/s",
            "cores": os.cpu_count() or 1, "kind": "port",
            "sample": f"{shot.name}: {n} steps (after 10 untimed) of the FP32 oracle restatement, OpenMP over rows, "
                      f"{dt:.1f} s"}


def run_reference_2d(args):
    import oracle

    if oracle.reference2d_library() is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/libref2d.so (reference CUDA_Kernels/Cuda_Check.cu "
                                                    "built from its source) is missing"}
    import torch

    from cmakepro_cuda_seissim_v2_b200 import models2d

    torch.cuda.init()
    shot = models2d.two_layer_shot(args.steps + args.warmup)
    c = shot.context
    r = oracle.ReferenceSolver2D(c)
    r.run(0, args.warmup)
    sampler = ClockSampler(GPU_ID)
    sampler.start()
    w0 = time.time()
    ms = r.time_steps(args.warmup, args.steps)
    w1 = time.time()
    sampler.mark(w0, w1)
    sampler.stop()
    r.close()
    cells = shot.active_cells
    value = cells * args.steps / (ms / 1e3) / 1e9
    # The reference loop with recording: one runGpuSimulationStep and one
    # recordReceiverStepOnGpu (two blocking D2H) per step (src/Seis2D/Workflow2D.inc:297-345).
    t = time.perf_counter()
    r = oracle.ReferenceSolver2D(c)
    r.run(0, args.steps, nrcv=c.num_rcv)
    dt = time.perf_counter() - t
    r.close()
    return {
        "impl": "reference", "metric": "2D P-SV Gcell-updates/s", "value": round(value, 4),
        "unit": "Gcell-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 6), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": {"workload": shot.name, "grid": [c.NX, c.NZ]},
        "cpu_baseline": {"value": round(value, 4), "unit": "Gcell-updates/s", "cores": 1, "kind": "reference",
                         "sample": f"reference CUDA_Kernels/Cuda_Check.cu built unmodified (--use_fast_math, sm_100a), "
                                   f"{args.steps} runGpuSimulationStep calls", "device": "cuda:0"},
        "e2e": {"value": round(cells * args.steps / dt / 1e9, 4), "unit": "Gcell-updates/s",
                "h2d_bytes_per_step": int(4 * c.rho.size * 4 // args.steps), "d2h_bytes_per_step": 8 * c.num_rcv,
                "wall_s": round(dt, 4), "path": "initializeGpuSimulation + (runGpuSimulationStep + "
                                                "recordReceiverStepOnGpu) per step"},
        "clocks": sampler.summary(),
    }


def main():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["size_cap", "reference_default", "two_layer_2d", "survey_windows",
                                          "learned_boundary"], default="size_cap")
    p.add_argument("--lb-models", type=int, default=24, help="learned_boundary: training models")
    p.add_argument("--lb-size", type=int, default=64, help="learned_boundary: training model side (cells)")
    p.add_argument("--lb-steps", type=int, default=300, help="learned_boundary: lock-step steps per model")
    p.add_argument("--lb-iterations", type=int, default=3000, help="learned_boundary: Adam steps per face")
    p.add_argument("--lb-fraction", type=float, default=0.1,
                   help="learned_boundary: fraction of boundary columns recorded per step (3M rows per face at most)")
    p.add_argument("--shots", type=int, default=8, help="survey_windows: shots timed (of 64)")
    p.add_argument("--reference-steps", type=int, default=100, help="survey_windows: reference sample per shot")
    p.add_argument("--storage", choices=sorted(STORAGE_MODES), default="fp32",
                   help="3-D workloads: fp32 (parity mode) or bf16_cpml (CPML memories in BF16)")
    p.add_argument("--no-storage-check", action="store_true",
                   help="16-bit storage: skip the whole-shot trace comparison with FP32 storage")
    p.add_argument("--thin-cpml", action="store_true",
                   help="survey_windows: the windows with the 6-cell CPML of the learned-boundary mode "
                        "(networks at gain 0), timed against the plain FP32 20-cell form")
    p.add_argument("--tile-y", type=int, default=0)
    p.add_argument("--z-chunk", type=int, default=0)
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    args = p.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")

    if args.workload == "two_layer_2d":
        # The 2-D shot is one small L2-resident grid: rank 0 alone measures it.
        if RANK != 0:
            return 0
        if args.impl == "reference":
            print(json.dumps(run_reference_2d(args)), flush=True)
            return 0
        line, shot = run_ours_2d(args)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_2d(shot, args.cpu_seconds)
        print(json.dumps(line), flush=True)
        return 0

    if args.workload == "learned_boundary":
        if RANK != 0:
            return 0
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned boundary and "
                                                                  "rejects CPML layers thinner than 8 cells"}))
            return 0
        print(json.dumps(run_learned_boundary(args)), flush=True)
        return 0

    if args.workload == "survey_windows":
        # One GPU holds the timed shots' windows; rank 0 alone measures them.
        if RANK != 0:
            return 0
        line = run_reference_survey(args) if args.impl == "reference" else run_ours_survey(args)
        print(json.dumps(line), flush=True)
        return 0

    if args.impl == "reference":
        if RANK != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0

    dist = init_dist()
    line, shot = run_ours(args, dist)
    if RANK == 0:
        if WORLD == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(shot, args.cpu_seconds)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
