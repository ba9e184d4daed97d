"""Synthetic earth models, acquisition geometry and shot set-ups of the solver workloads.

The workloads are the reference session defaults and the configurations the solver is
measured on; every model is generated from a stated seed in FP64 and handed to the solver
as FP32 vp/vs/rho planes through the same plane-upload path as an imported ``.s3dm`` model
(src/Seis3D/ModelIo3D.cpp:68-77), so the reference solver and this one see bit-identical
materials.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import capi, seis3d


def gardner_density(vp: np.ndarray) -> np.ndarray:
    """Gardner's relation rho = 310 vp^0.25 (kg/m^3, vp in m/s)."""
    return 310.0 * np.power(vp, 0.25)


def elastic_from_vp(vp: np.ndarray):
    """vs = vp / sqrt(3) and Gardner density, computed in FP64 and rounded to FP32."""
    vp64 = np.asarray(vp, dtype=np.float64)
    return (vp64.astype(np.float32), (vp64 / math.sqrt(3.0)).astype(np.float32),
            gardner_density(vp64).astype(np.float32))


def splitmix64_uniform(count: int, seed: int) -> np.ndarray:
    """`count` counter-based SplitMix64 draws mapped to [-1, 1) in FP64."""
    with np.errstate(over="ignore"):
        z = (np.arange(count, dtype=np.uint64) + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def smooth_noise(shape, sigma: float, seed: int) -> np.ndarray:
    """White noise smoothed by a separable Gaussian (sigma in cells, truncated at 4 sigma),
    normalised to max |g| = 1; FP64."""
    from scipy.ndimage import gaussian_filter1d

    g = splitmix64_uniform(int(np.prod(shape)), seed).reshape(shape)
    for axis in range(len(shape)):
        g = gaussian_filter1d(g, sigma, axis=axis, mode="reflect", truncate=4.0)
    return g / np.max(np.abs(g))


def fit_receivers(nx: int, ny: int, count_x: int = 50, count_y: int = 3) -> np.ndarray:
    """Surface receiver mesh of fitSurvey3D + configureReceivers3D
    (src/Seis3D_Sim.cpp:42-56, src/Seis3D/Acquisition3D.cpp:21-32): [(x, y, 0)], y-major."""
    count_x = min(max(count_x, 1), min(capi.MAX_RECEIVERS, nx - 2))
    count_y = min(max(count_y, 1), min(capi.MAX_RECEIVERS // count_x, ny - 2))
    sx = max(1, (nx - 3) // max(1, count_x - 1))
    sy = max(1, (ny - 3) // max(1, count_y - 1))
    ox = nx // 2 if count_x == 1 else (nx - 1 - (count_x - 1) * sx) // 2
    oy = ny // 2 if count_y == 1 else (ny - 1 - (count_y - 1) * sy) // 2
    return np.array([(ox + i * sx, oy + j * sy, 0) for j in range(count_y) for i in range(count_x)], dtype=np.int32)


@dataclasses.dataclass
class Shot:
    """One shot: context, source, receivers, materials and run length."""

    name: str
    context: capi.Context
    source: capi.Source
    receivers: np.ndarray
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    steps: int
    stride: int

    @property
    def active_cells(self) -> int:
        c = self.context
        return (c.gx3D - 8) * (c.gy3D - 8) * (c.gz3D - 8)

    @property
    def samples(self) -> int:
        return self.steps // self.stride


def imported_context(nx, ny, nz, spacing, pml, free_surface, max_vp, frequency, dt_ms=None, api=None,
                     thin: bool = False) -> capi.Context:
    """Context of an imported model (modelKind Imported, maxVp from the data as
    inspectModel3D does: src/Seis3D/ModelIo3D.cpp:53-64).

    `api` supplies ``default_context`` and ``validate_context3D``: this solver's (the default)
    or any object with the same two calls, e.g. one backed by the reference's own host code.
    `thin` validates a CPML of 4..7 cells (sessions created with thin_cpml)."""
    api = api or seis3d
    c = api.default_context(nx3D=nx, ny3D=ny, nz3D=nz, spacing3D=spacing, pml3D=pml,
                            freeSurface3D=int(free_surface), reflecting3D=0, modelKind3D=capi.MODEL_IMPORTED,
                            maxVp3D=float(max_vp), frequency3D=float(frequency))
    if dt_ms is not None:
        c.manualTimeStep3D = 1
        c.requestedDtMs3D = float(dt_ms)
    return seis3d.validate_thin_context3D(c) if thin else api.validate_context3D(c)


def layered_model(nx, ny, nz, velocities, thickness=None):
    """Flat layers of equal (or given) thickness along z; returns vp [nz][ny][nx] FP64."""
    n = len(velocities)
    if thickness is None:
        bounds = [round(k * nz / n) for k in range(n + 1)]
    else:
        bounds = [0]
        for t in thickness:
            bounds.append(bounds[-1] + t)
    vp = np.empty((nz, ny, nx), dtype=np.float64)
    for k in range(n):
        vp[bounds[k]:bounds[k + 1]] = velocities[k]
    return vp


def reference_default_shot(steps: int = 2000, api=None) -> Shot:
    """300 x 50 x 300 reference-default workload: 5 flat 60-cell layers, vp 1800/2400/
    3000/3700/4500 m/s, vs = vp/sqrt3, Gardner density, free surface + 5-face 20-cell CPML,
    explosion Ricker 15 Hz at (150, 25, 10), dt 0.5 ms, every 2nd step recorded on the
    default 50 x 3 receiver spread."""
    nx, ny, nz = 300, 50, 300
    vp, vs, rho = elastic_from_vp(layered_model(nx, ny, nz, [1800, 2400, 3000, 3700, 4500]))
    c = imported_context(nx, ny, nz, 10.0, 20, True, float(vp.max()), 15.0, dt_ms=0.5, api=api)
    src = (api or seis3d).default_source(x3D=150, y3D=25, z3D=10, kind3D=capi.SOURCE_EXPLOSION, amplitude3D=1.0e8)
    return Shot("300x50x300 layered, free surface + 5-face CPML20", c, src, fit_receivers(nx, ny, 50, 3),
                vp, vs, rho, steps, 2)


def size_cap_shot(steps: int = 2500, seed: int = 20261203, api=None) -> Shot:
    """300 x 300 x 400 (36 M nodes, the reference's size cap) workload: vp linear
    2000 -> 4000 m/s with depth times (1 + 0.1 g), g a sigma = 8 smoothed seeded noise
    field (max |g| = 1), vs = vp/sqrt3, Gardner density, 6-face 20-cell CPML, Ricker 12 Hz
    at the session default (150, 150, 100), dt 0.6 ms, 300 receivers (20 x 15) at z = 0."""
    nx, ny, nz = 300, 300, 400
    depth = np.linspace(2000.0, 4000.0, nz)[:, None, None]
    g = smooth_noise((nz, ny, nx), 8.0, seed)
    vp, vs, rho = elastic_from_vp(depth * (1.0 + 0.1 * g))
    c = imported_context(nx, ny, nz, 10.0, 20, False, float(vp.max()), 12.0, dt_ms=0.6, api=api)
    src = (api or seis3d).default_source(x3D=150, y3D=150, z3D=100, kind3D=capi.SOURCE_EXPLOSION,
                                         amplitude3D=1.0e8)
    return Shot("300x300x400 gradient+noise, 6-face CPML20", c, src, fit_receivers(nx, ny, 20, 15),
                vp, vs, rho, steps, 1)


def small_shot(nx=40, ny=32, nz=36, pml=8, free_surface=True, steps=60, seed=7, layers=(2000, 2600, 3200),
               source=None, kind=capi.SOURCE_EXPLOSION, frequency=25.0, spacing=10.0) -> Shot:
    """Small layered + noise model for parity tests (finishes on the CPU oracle in
    seconds).  Receivers on a 5 x 3 surface spread plus a buried line."""
    vp = layered_model(nx, ny, nz, list(layers))
    vp = vp * (1.0 + 0.05 * splitmix64_uniform(nx * ny * nz, seed).reshape(nz, ny, nx))
    vp, vs, rho = elastic_from_vp(vp)
    c = imported_context(nx, ny, nz, spacing, pml, free_surface, float(vp.max()), frequency)
    sx, sy, sz = source if source is not None else (nx // 2, ny // 2, nz // 3)
    src = seis3d.default_source(x3D=sx, y3D=sy, z3D=sz, kind3D=kind, amplitude3D=1.0e8,
                                direction3D=(0.3, -0.5, 0.8))
    rec = list(map(tuple, fit_receivers(nx, ny, 5, 3)))
    rec += [(x, ny // 3, nz // 2) for x in range(2, nx - 2, 7)]
    return Shot(f"small {nx}x{ny}x{nz}", c, src, np.array(rec, dtype=np.int32), vp, vs, rho, steps, 1)


@dataclasses.dataclass
class WindowShot:
    """One shot of a windowed survey: the window's origin and size in the large model, the
    source cell inside the window and the run length."""

    index: int
    origin: tuple[int, int, int]
    size: tuple[int, int, int]
    source: tuple[int, int, int]


@dataclasses.dataclass
class WindowSurvey:
    """A large model and its shots, each simulated on a cropped window (free surface on top,
    5-face CPML around the window)."""

    name: str
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    shots: list
    spacing: float
    pml: int
    frequency: float
    dt_ms: float
    steps: int

    def window(self, shot: WindowShot):
        """(vp, vs, rho) of the shot's window, contiguous FP32 [z][y][x]."""
        (x0, y0, z0), (wx, wy, wz) = shot.origin, shot.size
        sl = (slice(z0, z0 + wz), slice(y0, y0 + wy), slice(x0, x0 + wx))
        return (np.ascontiguousarray(self.vp[sl]), np.ascontiguousarray(self.vs[sl]),
                np.ascontiguousarray(self.rho[sl]))

    def context(self, shot: WindowShot) -> capi.Context:
        vp = self.vp[shot.origin[2]:shot.origin[2] + shot.size[2], shot.origin[1]:shot.origin[1] + shot.size[1],
                     shot.origin[0]:shot.origin[0] + shot.size[0]]
        return imported_context(*shot.size, self.spacing, self.pml, True, float(vp.max()), self.frequency,
                                dt_ms=self.dt_ms, thin=self.pml < 8)

    def source(self, shot: WindowShot) -> capi.Source:
        x, y, z = shot.source
        return seis3d.default_source(x3D=x, y3D=y, z3D=z, kind3D=capi.SOURCE_EXPLOSION, amplitude3D=1.0e8)

    def receivers(self, shot: WindowShot) -> np.ndarray:
        """The 50 x 3 surface spread of the window (fewer on windows narrower than 52 x 5 cells)."""
        return fit_receivers(shot.size[0], shot.size[1], 50, 3)

    def active_cells(self, shot: WindowShot) -> int:
        wx, wy, wz = shot.size
        return (wx + 2 * self.pml) * (wy + 2 * self.pml) * (wz + self.pml)


def smooth_layered_model(nx, ny, nz, seed, layers=6, vmin=1800.0, vmax=4500.0, undulation=12.0):
    """Seeded smooth random layered model: (layer index [nz][ny][nx] uint8, vp of each layer).
    `layers` layers whose interfaces are mean depths plus smooth undulations (sigma 24 cells,
    amplitude `undulation` cells), velocities increasing from vmin to vmax with seeded jitter."""
    mean = np.sort(0.5 + 0.5 * splitmix64_uniform(layers - 1, seed)) * nz * 0.9
    jitter = 0.08 * splitmix64_uniform(layers, seed + 1)
    velocity = np.clip(np.linspace(vmin, vmax, layers) * (1.0 + jitter), vmin, vmax)
    velocity[0], velocity[-1] = vmin, vmax
    z = np.arange(nz, dtype=np.float32)[:, None, None]
    index = np.zeros((nz, ny, nx), np.uint8)
    for k in range(layers - 1):
        surface = (mean[k] + undulation * smooth_noise((ny, nx), 24.0, seed + 10 + k)).astype(np.float32)
        index += (z >= surface[None]).astype(np.uint8)
    return index, velocity


def window_survey(shots: int = 64, steps: int = 1500, seed: int = 20261204, nx: int = 600, ny: int = 200,
                  nz: int = 600, window_range: tuple[int, int] = (160, 320), pml: int = 20,
                  source_depth: int = 10) -> WindowSurvey:
    """600 x 200 x 600 smooth random layered model (dx 10 m, vp 1800-4500 m/s, vs = vp/sqrt3,
    Gardner density) with `shots` explosion shots on a seeded 8 x 8 grid of source positions,
    each on a window centred on its source with sides drawn uniformly from 160-320 cells (the
    y side at most the model's 200), free surface + 5-face CPML20, Ricker 15 Hz, dt 0.5 ms,
    1500 steps, 150 receivers per shot."""
    index, velocity = smooth_layered_model(nx, ny, nz, seed)
    tables = elastic_from_vp(velocity)
    vp, vs, rho = (t[index] for t in tables)
    draws = splitmix64_uniform(6 * shots, seed + 100).reshape(shots, 6)
    out = []
    for i in range(shots):
        gx, gy = i % 8, (i // 8) % 8
        sx = int(round(nx * 0.1 + nx * 0.8 * (gx + 0.5 + 0.3 * draws[i, 0]) / 8))
        sy = int(round(ny * 0.1 + ny * 0.8 * (gy + 0.5 + 0.3 * draws[i, 1]) / 8))
        lo, hi = window_range
        size = [min(int(lo + (hi - lo) * (0.5 + 0.5 * draws[i, 2 + a])), n) for a, n in enumerate((nx, ny, nz))]
        origin = [min(max(c - w // 2, 0), n - w) for c, w, n in zip((sx, sy, 0), size, (nx, ny, nz))]
        origin[2] = 0
        source = (min(max(sx - origin[0], 1), size[0] - 2), min(max(sy - origin[1], 1), size[1] - 2), source_depth)
        out.append(WindowShot(i, tuple(origin), tuple(size), source))
    return WindowSurvey(f"{nx}x{ny}x{nz} smooth layered, {shots} windowed shots {window_range[0]}-{window_range[1]} "
                        f"cells, FS + 5-face CPML{pml}",
                        vp, vs, rho, out, 10.0, pml, 15.0, 0.5, steps)
