"""Training and evaluation of the learned thin boundary (no reference counterpart).

Training data are the solver's own runs: for each seeded random layered model a thin-CPML
session and a 40-cell-CPML session of the same model are stepped in lock step, and after
every step the thin session's boundary columns are recorded with the wide minus thin
difference on their corrected cells as targets; the thin interior is then reset to the wide
one (seis3d_boundary_collect).  The networks are trained on the device by the library's own
forward/backward kernels (seis3d_boundary_train).

Evaluation runs one held-out model four ways: the thin CPML alone, the thin CPML with the
networks, the standard 20-cell CPML (the layer the thin forms must approach) and the 40-cell
CPML (the big-domain reference).  Errors against the 40-cell run: receiver traces (relative L2 over the
whole gather) and the reflected energy, sum over sampled times of |v - v_40|^2 over the
physical cells divided by the sum of |v_40|^2, plus the late/peak ratio of the physical-cell
velocity energy that tests/Seis3DBoundaryRegression.cpp:50-61 of the reference uses.
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np

from . import capi, models3d, seis3d


@dataclasses.dataclass
class BoundaryModel:
    """A seeded random layered model with its shot."""
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    frequency: float
    source: tuple[int, int, int]
    free_surface: bool


def random_layered_model(nx, ny, nz, seed, free_surface=True, layers=None, vmin=1500.0, vmax=5000.0,
                         fmin=10.0, fmax=25.0) -> BoundaryModel:
    """3-8 flat layers at seeded depths with vp drawn in [vmin, vmax] (increasing with depth
    more often than not), vs = vp / sqrt 3, Gardner density, a Ricker frequency in
    [fmin, fmax] and a source at a seeded position at least 6 cells inside every face."""
    u = models3d.splitmix64_uniform(32, seed) * 0.5 + 0.5
    count = layers or 3 + int(u[0] * 6)
    bounds = np.sort(u[1:count]) * nz
    velocity = vmin + (vmax - vmin) * u[10:10 + count]
    velocity = np.sort(velocity) if u[20] < 0.7 else velocity
    z = np.arange(nz)[:, None, None]
    index = np.zeros((nz, 1, 1), dtype=np.int64)
    for b in bounds:
        index += (z >= b).astype(np.int64)
    vp = np.broadcast_to(velocity[index], (nz, ny, nx))
    vp, vs, rho = models3d.elastic_from_vp(vp)
    frequency = fmin + (fmax - fmin) * u[21]
    src = (6 + int(u[22] * (nx - 12)), 6 + int(u[23] * (ny - 12)), 6 + int(u[24] * (nz - 12)))
    return BoundaryModel(vp, vs, rho, float(frequency), src, free_surface)


def context(model: BoundaryModel, pml: int, dt_ms: float | None = None, spacing: float = 10.0) -> capi.Context:
    nz, ny, nx = model.vp.shape
    c = seis3d.default_context(nx3D=nx, ny3D=ny, nz3D=nz, spacing3D=spacing, pml3D=pml,
                               freeSurface3D=int(model.free_surface), reflecting3D=0,
                               modelKind3D=capi.MODEL_IMPORTED, maxVp3D=float(model.vp.max()),
                               frequency3D=model.frequency)
    if dt_ms is not None:
        c.manualTimeStep3D = 1
        c.requestedDtMs3D = float(dt_ms)
    return seis3d.validate_thin_context3D(c)


def source(model: BoundaryModel) -> capi.Source:
    x, y, z = model.source
    return seis3d.default_source(x3D=x, y3D=y, z3D=z, kind3D=capi.SOURCE_EXPLOSION, amplitude3D=1.0e8)


def collect(dataset: seis3d.BoundaryDataset, model: BoundaryModel, steps: int, thin_pml: int = 6,
            wide_pml: int = 40, fraction: float = 1.0, seed: int = 0) -> None:
    """Lock-step runs of one model on a thin and a wide CPML, recording every step."""
    ct, cw = context(model, thin_pml), context(model, wide_pml)
    dt_ms = round(min(ct.dt3D, cw.dt3D) * 1e6) / 1e3
    ct, cw = context(model, thin_pml, dt_ms), context(model, wide_pml, dt_ms)
    thin = seis3d.Session(ct, thin_cpml=True)
    wide = seis3d.Session(cw, thin_cpml=True)
    try:
        for s in (thin, wide):
            s.upload_volumes(model.vp, model.vs, model.rho)
        dataset.begin_model()
        src = source(model)
        for n in range(steps):
            thin.run_step(src, n)
            wide.run_step(src, n)
            dataset.collect(thin, wide, fraction, seed * 1000003 + n)
        thin.synchronize()
    finally:
        thin.release()
        wide.release()


def train(net: seis3d.BoundaryNet, dataset: seis3d.BoundaryDataset, faces, iterations: int = 2000,
          batch: int = 4096, lr: float = 1e-3, seed: int = 0) -> dict:
    """Adam on every given face in rounds of 100 iterations; returns the loss history."""
    history = {f: [] for f in faces}
    for f in faces:
        done = 0
        while done < iterations:
            k = min(100, iterations - done)
            rate = lr * (0.3 if done >= 0.75 * iterations else 1.0)
            history[f].append(net.train(dataset, f, k, batch, rate, seed + done))
            done += k
    return history


@dataclasses.dataclass
class RunResult:
    gather: np.ndarray
    energy: list          # physical-cell velocity energy at the sampled steps
    fields: list          # physical-cell velocities at the sampled steps (for differences)
    ms: float             # device time of the run


def run(model: BoundaryModel, pml: int, steps: int, dt_ms: float, receivers, net=None, gain=1.0,
        every: int = 50) -> RunResult:
    c = context(model, pml, dt_ms)
    s = seis3d.Session(c, thin_cpml=True)
    try:
        s.upload_volumes(model.vp, model.vs, model.rho)
        s.set_receivers(receivers)
        if net is not None:
            seis3d.attach_boundary(s, net, gain)
        s.gather_begin(1, steps)
        src = source(model)
        nz, ny, nx = model.vp.shape
        sl = (slice(c.oz3D, c.oz3D + nz), slice(c.oy3D, c.oy3D + ny), slice(c.ox3D, c.ox3D + nx))
        energy, fields = [], []
        t = time.perf_counter()
        done = 0
        while done < steps:
            k = min(every, steps - done)
            s.run_steps(src, done, k)
            done += k
            v = [s.field(i)[sl].astype(np.float64) for i in range(3)]
            energy.append(float(sum(np.sum(a * a) for a in v)))
            fields.append(v)
        ms = (time.perf_counter() - t) * 1e3
        gather = s.gather_fetch()
    finally:
        s.release()
    return RunResult(gather, energy, fields, ms)


def evaluate(model: BoundaryModel, net: seis3d.BoundaryNet, steps: int, thin_pml: int = 6, standard_pml: int = 20,
             wide_pml: int = 40, gains=(1.0,), receivers=None, every: int = 50) -> dict:
    """Errors of thin, thin + network (each gain) and the 20-cell CPML against the wide run."""
    dts = [context(model, p).dt3D for p in (thin_pml, standard_pml, wide_pml)]
    dt_ms = round(min(dts) * 1e6) / 1e3
    nz, ny, nx = model.vp.shape
    if receivers is None:
        receivers = models3d.fit_receivers(nx, ny, 50, 3)
    wide = run(model, wide_pml, steps, dt_ms, receivers, every=every)

    def errors(r: RunResult) -> dict:
        num = den = 0.0
        for a, b in zip(r.fields, wide.fields):
            num += sum(float(np.sum((x - y) ** 2)) for x, y in zip(a, b))
            den += sum(float(np.sum(y * y)) for y in b)
        g = np.linalg.norm(r.gather.astype(np.float64) - wide.gather) / np.linalg.norm(wide.gather)
        peak = max(r.energy)
        return {"trace_rel_l2": float(g), "reflected_energy": num / den, "late_over_peak": r.energy[-1] / peak,
                "ms": r.ms}

    out = {"dt_ms": dt_ms, "steps": steps, "wide": {"late_over_peak": wide.energy[-1] / max(wide.energy),
                                                       "ms": wide.ms}}
    out["thin"] = errors(run(model, thin_pml, steps, dt_ms, receivers, every=every))
    out["cpml20"] = errors(run(model, standard_pml, steps, dt_ms, receivers, every=every))
    for gain in gains:
        out[f"thin+net@{gain:g}"] = errors(run(model, thin_pml, steps, dt_ms, receivers, net=net, gain=gain,
                                               every=every))
    return out


def step_time(model: BoundaryModel, pml: int, steps: int, dt_ms: float, net=None, gain: float = 1.0) -> float:
    """Device milliseconds per step (CUDA events around the solver's own launches, the
    network's correction included when attached)."""
    c = context(model, pml, dt_ms)
    s = seis3d.Session(c, thin_cpml=True, tune=True)
    try:
        s.upload_volumes(model.vp, model.vs, model.rho)
        if net is not None:
            seis3d.attach_boundary(s, net, gain)
        src = source(model)
        s.run_steps(src, 0, 10)
        return s.profile_steps(src, 10, steps)["step"] / steps
    finally:
        s.release()


def select_gain(net: seis3d.BoundaryNet, model: BoundaryModel, steps: int, gains=(0.0, 0.25, 0.5, 1.0),
                every: int = 50) -> tuple[float, dict]:
    """The gain (0 = the thin CPML alone, the fallback) with the least reflected energy on a
    validation model, and the energies of every candidate."""
    res = evaluate(model, net, steps, gains=tuple(g for g in gains if g > 0), every=every)
    energy = {0.0: res["thin"]["reflected_energy"]}
    for g in gains:
        if g > 0:
            energy[g] = res[f"thin+net@{g:g}"]["reflected_energy"]
    best = min(energy, key=energy.get)
    return best, energy


def train_boundary(models: int = 16, size: int = 64, steps: int = 300, fraction: float = 0.1,
                   rows_per_face: int = 3_000_000, iterations: int = 3000, batch: int = 4096, lr: float = 1e-3,
                   thin_pml: int = 6, wide_pml: int = 40, seed: int = 1000, validation_steps: int = 600,
                   log=None) -> tuple[seis3d.BoundaryNet, float, dict]:
    """Collect lock-step rows from `models` seeded random layered models of size^3 cells,
    train the per-face networks, and select their gain on a held-out validation model.
    Returns (networks, gain, report)."""
    t0 = time.perf_counter()
    data = seis3d.BoundaryDataset(rows_per_face)
    try:
        for m in range(models):
            collect(data, random_layered_model(size, size, size, seed + m), steps, thin_pml, wide_pml, fraction, m)
        rows = data.rows()
        t1 = time.perf_counter()
        net = seis3d.BoundaryNet(thin_pml, seed=seed)
        faces = [f for f in range(6) if rows[f] > 0]
        history = train(net, data, faces, iterations, batch, lr, seed)
        t2 = time.perf_counter()
    finally:
        data.release()
    validation = random_layered_model(96, 48, 96, seed + 100000)
    gain, energies = select_gain(net, validation, validation_steps)
    report = {"models": models, "size": size, "steps": steps, "rows": rows, "collect_s": round(t1 - t0, 2),
              "train_s": round(t2 - t1, 2), "iterations": iterations, "batch": batch,
              "loss_first": {f: history[f][0] for f in faces}, "loss_last": {f: history[f][-1] for f in faces},
              "gain": gain, "validation_energy": {f"{g:g}": e for g, e in energies.items()}}
    if log:
        log(report)
    return net, gain, report


def default_steps(model: BoundaryModel, extent_cells: int, spacing: float = 10.0, cfl_dt: float = 0.0005) -> int:
    """Steps for the slowest wave to cross the model once more than its size."""
    vmin = float(model.vs.min())
    return int(math.ceil(1.5 * extent_cells * spacing / vmin / cfl_dt))
