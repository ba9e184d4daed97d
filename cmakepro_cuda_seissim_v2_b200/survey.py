"""Multi-shot 3-D survey driver: the reference's shot sequence, receiver mesh and gather rules,
with the shots of a survey shared out over ranks (one GPU each).

Reference semantics kept here:

* ``receiver_mesh`` = configureReceivers3D (src/Seis3D/Acquisition3D.cpp:21-37): an X-by-Y
  surface mesh at one depth, x fastest, at most 300 channels, inside the model.
* ``sequence_shot`` = positionSequenceShot3D (:233-243): shot i of a rectangular spread sits at
  (ox + (i % nx) * dx, oy + (i // nx) * dy, oz); the whole spread must lie inside the model.
* ``check_gather`` = the checks of startGather3D (:188-212): source inside the model at depth
  >= 2, 1..32767 samples, stride 1..10000, a SEG-Y sample interval of at most 32767 us and a
  512 MiB host budget for one gather.

Shots are independent: ``partition_shots`` assigns them to ranks by estimated cost (cell
updates) with a longest-first greedy rule, every rank runs its own shots on its own GPU, and
``run_survey`` collects the finished gathers on rank 0 with one host-side gather of Python
objects at the end -- no collective touches the wavefields.  ``run_window_survey`` does the
same for surveys whose shots sit on cropped windows of a large model, running each rank's
shots in groups stepped together by one batched launch (``gpu_window_runner``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import capi

MAX_SEGY_SAMPLES = 32767
MAX_SEGY_INTERVAL_US = 32767
GATHER_BUDGET_BYTES = 512 * 1024 * 1024


@dataclass
class Survey3D:
    """Survey3D of the reference (include/Seis3D_Sim.h:36-45, same defaults): receiver mesh and
    shot spread in physical grid cells, CMP bin size and world origin in metres."""

    receiver_count: tuple[int, int] = (50, 3)
    receiver_spacing: tuple[int, int] = (5, 23)
    receiver_origin: tuple[int, int, int] = (27, 1, 0)
    shot_count: tuple[int, int] = (3, 2)
    shot_spacing: tuple[int, int] = (20, 20)
    shot_origin: tuple[int, int, int] = (24, 24, 12)
    cmp_bin_size: tuple[float, float] = (25.0, 25.0)
    world_origin: tuple[float, float] = (0.0, 0.0)


@dataclass
class ShotResult:
    index: int
    source: tuple[int, int, int]
    rank: int
    gather: np.ndarray                    # float32 [sample][receiver][vx, vy, vz]
    extra: dict = field(default_factory=dict)


def receiver_mesh(survey: Survey3D, context) -> list[tuple[int, int, int]]:
    """configureReceivers3D: validate and list the receivers, x fastest."""
    cx, cy = survey.receiver_count
    sx, sy = survey.receiver_spacing
    ox, oy, oz = survey.receiver_origin
    if cx < 1 or cy < 1 or cx > capi.MAX_RECEIVERS or cy > capi.MAX_RECEIVERS or cx * cy > capi.MAX_RECEIVERS \
            or sx < 1 or sy < 1:
        raise ValueError("Receiver mesh must have 1..300 total channels (X times Y) and positive spacing.")
    last_x, last_y = ox + (cx - 1) * sx, oy + (cy - 1) * sy
    if ox < 0 or oy < 0 or last_x >= context.nx3D or last_y >= context.ny3D or oz < 0 or oz >= context.nz3D:
        raise ValueError("Receiver mesh exceeds the model.")
    return [(ox + x * sx, oy + y * sy, oz) for y in range(cy) for x in range(cx)]


def shot_count(survey: Survey3D) -> int:
    return survey.shot_count[0] * survey.shot_count[1]


def sequence_shot(survey: Survey3D, context, index: int) -> tuple[int, int, int]:
    """positionSequenceShot3D: source cell of shot `index` of the spread."""
    nx, ny = survey.shot_count
    sx, sy = survey.shot_spacing
    ox, oy, oz = survey.shot_origin
    if nx < 1 or ny < 1 or nx > 100 or ny > 100 or sx < 1 or sy < 1:
        raise ValueError("Invalid 3D source spread.")
    last_x, last_y = ox + (nx - 1) * sx, oy + (ny - 1) * sy
    if ox < 1 or oy < 1 or last_x >= context.nx3D - 1 or last_y >= context.ny3D - 1 or oz < 2 \
            or oz >= context.nz3D - 1:
        raise ValueError("Source spread exceeds the 3D model.")
    if index < 0 or index >= nx * ny:
        raise ValueError("Shot index outside the spread.")
    return ox + (index % nx) * sx, oy + (index // nx) * sy, oz


def check_gather(context, source, stride: int, target_samples: int, receivers: int) -> None:
    """The checks of startGather3D before a gather is captured."""
    if source.x3D < 1 or source.x3D >= context.nx3D - 1 or source.y3D < 1 or source.y3D >= context.ny3D - 1 \
            or source.z3D < 2 or source.z3D >= context.nz3D - 1 or not np.isfinite(source.amplitude3D):
        raise ValueError("Place the source inside the model, at depth >=2, before capture.")
    if not all(np.isfinite(d) for d in source.direction3D):
        raise ValueError("Invalid source direction.")
    if target_samples < 1 or target_samples > MAX_SEGY_SAMPLES or stride < 1 or stride > 10000:
        raise ValueError("Gather sample count must be 1..32767 with stride 1..10000.")
    interval = round(float(context.dt3D) * 1e6) * stride
    if interval > MAX_SEGY_INTERVAL_US:
        raise ValueError("SEG-Y rev1 sample interval must not exceed 32767 us.")
    if target_samples * receivers * 3 * 4 > GATHER_BUDGET_BYTES:
        raise ValueError("Shot gather exceeds the 512 MiB CPU budget.")


def partition_shots(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-first greedy assignment of shots to `world` ranks by cost; ties go to the lower
    rank, and each rank's list keeps the survey order.  Deterministic, so every rank computes
    the same plan without communicating."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    load = [0.0] * world
    plan: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda q: (-float(costs[q]), q)):
        r = min(range(world), key=lambda q: (load[q], q))
        plan[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in plan]


ShotRunner = Callable[[int, tuple[int, int, int]], np.ndarray]


def run_survey(survey: Survey3D, context, runner: ShotRunner, costs: Sequence[float] | None = None,
               rank: int = 0, world: int = 1, dist=None) -> list[ShotResult] | None:
    """Runs this rank's share of the survey with `runner(index, source_cell) -> gather` and
    returns every shot's result, in survey order, on rank 0 (None on the other ranks).

    `dist` is torch.distributed (any backend with object gathers, e.g. gloo or nccl) when
    world > 1; the gathers are collected once, after every rank has finished its shots."""
    n = shot_count(survey)
    sources = [sequence_shot(survey, context, i) for i in range(n)]
    plan = partition_shots(costs if costs is not None else [1.0] * n, world)
    mine = [ShotResult(i, sources[i], rank, np.asarray(runner(i, sources[i]), dtype=np.float32)) for i in plan[rank]]
    return _collect(mine, n, rank, world, dist)


def _collect(mine: list[ShotResult], n: int, rank: int, world: int, dist) -> list[ShotResult] | None:
    """Every rank's finished shots onto rank 0, in survey order (one host-side object gather)."""
    if world == 1:
        return sorted(mine, key=lambda r: r.index)
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    results = sorted((r for part in gathered for r in part), key=lambda r: r.index)
    if [r.index for r in results] != list(range(n)):
        raise RuntimeError("survey gather is missing shots")
    return results


# A group runner steps several shots together and returns their gathers, in the given order.
GroupRunner = Callable[[Sequence[int]], Sequence[np.ndarray]]


def run_window_survey(survey, group_runner: GroupRunner, batch: int = 8, rank: int = 0, world: int = 1,
                      dist=None) -> list[ShotResult] | None:
    """A windowed survey (models3d.WindowSurvey) sharded over ranks: every rank takes its
    longest-first share by cost (active window cells x steps), runs it in groups of `batch`
    shots stepped together on its GPU (largest windows first, so each group holds windows of
    similar size), and rank 0 collects every gather in survey order."""
    if batch < 1:
        raise ValueError("batch must be >= 1")
    n = len(survey.shots)
    costs = [float(survey.active_cells(q)) * survey.steps for q in survey.shots]
    plan = partition_shots(costs, world)
    order = sorted(plan[rank], key=lambda i: (-costs[i], i))
    mine = []
    for k in range(0, len(order), batch):
        group = order[k:k + batch]
        gathers = group_runner(group)
        if len(gathers) != len(group):
            raise RuntimeError("the group runner returned the wrong number of gathers")
        for i, g in zip(group, gathers):
            mine.append(ShotResult(i, tuple(survey.shots[i].source), rank, np.asarray(g, dtype=np.float32),
                                   {"origin": survey.shots[i].origin, "size": survey.shots[i].size}))
    return _collect(mine, n, rank, world, dist)


def gpu_window_runner(survey, stride: int = 2, tune: bool = True) -> GroupRunner:
    """A group runner for this rank's GPU: per group, one session per window (cropped model
    uploaded, 150 receivers, device gather of survey.steps // stride samples), all stepped
    together by one seis3d batch (tuned on its first steps), gathers read back and the
    sessions released."""
    from . import seis3d

    def run(group: Sequence[int]) -> list[np.ndarray]:
        sessions, sources = [], []
        try:
            for i in group:
                shot = survey.shots[i]
                s = seis3d.Session(survey.context(shot))
                sessions.append(s)
                s.upload_volumes(*survey.window(shot))
                receivers = survey.receivers(shot)
                s.set_receivers(receivers)
                src = survey.source(shot)
                check_gather(s.context, src, stride, survey.steps // stride, len(receivers))
                s.gather_begin(stride, survey.steps // stride)
                sources.append(src)
            b = seis3d.Batch(sessions, tune=tune)
            try:
                b.run_steps(sources, 0, survey.steps)
                b.synchronize()
            finally:
                b.release()
            return [s.gather_fetch() for s in sessions]
        finally:
            for s in sessions:
                s.release()

    return run


def gpu_runner(context, vp, vs, rho, source_template, steps: int, stride: int, receivers,
               compact_rows: bool = False) -> ShotRunner:
    """A runner for this rank's GPU: one session, the model uploaded once, and per shot a
    reset, the source moved to the shot cell, a device-resident gather of `steps` steps and
    its read-back (the reference's frozen-gather capture, src/Seis3D_Sim.cpp:120-153)."""
    from . import seis3d

    session = seis3d.Session(context, compact_rows=compact_rows)
    session.upload_model(vp, vs, rho)
    session.set_receivers(receivers)
    samples = steps // stride

    def run(index: int, cell: tuple[int, int, int]) -> np.ndarray:
        source = seis3d.default_source()
        for name, _ in capi.Source._fields_:
            setattr(source, name, getattr(source_template, name))
        source.x3D, source.y3D, source.z3D = cell
        check_gather(session.context, source, stride, samples, len(receivers))
        session.reset()
        session.gather_begin(stride, samples)
        session.run_steps(source, 0, steps)
        gather = session.gather_fetch()
        session.gather_end()
        return gather

    run.session = session
    return run
