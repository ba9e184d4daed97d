"""Synthetic 2-D P-SV workloads built with the reference's own set-up rules.

``two_layer_shot`` is the 2-D benchmark configuration: a 400 x 400 physical grid at 5 m with
a free surface on top and a 20-cell split-field PML on the other three sides, laid out as the
reference does (the free surface is grid row ``npml`` with air rows above it,
CUDA_Kernels/Cuda_Check.cu:894,519-522), so the grid is 440 x 420 and depths are counted
from row 20.  Two layers (depth < 200 cells: vp 2500, vs 1443, rho 2000; below: 3500, 2000,
2300), explosive 20 Hz Ricker (t0 = 1/f0) at grid (200, 40), dt = 0.5 ms, 2000 steps, 200
receivers on grid row 30 at x = 0, 2, ..., 398 recording vx, vz every step.

Every set-up quantity goes through the reference formulas (material fill of
setGridMaterial2D, PML profile of updatePmlDampingArrays, traction-free modulus and stencil
coefficients of setupTestContext, Ricker series of generateRickerWavelet).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import capi2d, seis2d


@dataclass
class Shot2D:
    context: seis2d.SimulationContext
    steps: int
    name: str

    @property
    def receivers(self) -> np.ndarray:
        return self.context.rcv_grid_idx

    @property
    def active_cells(self) -> int:
        """Cells a step updates: (NX - 8) x (NZ - 8), the interior the kernels cover."""
        return (self.context.NX - 8) * (self.context.NZ - 8)


def layered_context(NX: int, NZ: int, npml: int, h: float, dt: float, nt: int, layers, *, flag_type: int = 3,
                    up: bool = True, f0: float = 20.0, t0: float | None = None, src=(0, 0), src_type: int = 2,
                    src_amp: float = 1.0, src_angle: float = 0.0, receivers=()) -> seis2d.SimulationContext:
    """A context whose rows hold horizontal layers.

    ``layers`` is a list of (first depth row below the free surface, vp, vs, rho); rows above
    the free surface take the first layer.  ``src`` and ``receivers`` are grid (x, row)."""
    total = seis2d.checkedGridElementCount(NX, NZ)
    ctx = seis2d.SimulationContext(NX=NX, NZ=NZ, total_grid=total, h=float(np.float32(h)), dt=float(np.float32(dt)),
                                   nt=nt, npml=npml, flag_type=flag_type, upFlag=up)
    ctx.rho = np.zeros(total, np.float32)
    ctx.mu = np.zeros(total, np.float32)
    ctx.lambda_ = np.zeros(total, np.float32)
    ctx.lambda2mu = np.zeros(total, np.float32)
    fs = npml if (flag_type == 3 and up) else 0
    rows = np.arange(NZ) - fs
    for z in range(NZ):
        vp, vs, rho = layers[0][1:]
        for first, lvp, lvs, lrho in layers:
            if rows[z] >= first:
                vp, vs, rho = lvp, lvs, lrho
        rho32, vp32, vs32 = np.float32(rho), np.float32(vp), np.float32(vs)
        mu = rho32 * vs32 * vs32
        l2m = rho32 * vp32 * vp32
        sl = slice(z * NX, (z + 1) * NX)
        ctx.rho[sl] = rho32
        ctx.mu[sl] = mu
        ctx.lambda2mu[sl] = l2m
        ctx.lambda_[sl] = l2m - np.float32(2.0) * mu
    ctx.c1_h, ctx.c2_h, ctx.c3_h, ctx.c4_h = seis2d.stencil_coefficients(h)
    seis2d.updatePmlDampingArrays(ctx)
    seis2d.freeSurfaceModulus(ctx)
    if t0 is None:
        t0 = float(np.float32(1.0) / np.float32(f0))
    ctx.wavelet = seis2d.generateRickerWavelet(nt, ctx.dt, f0, t0)
    ctx.src_z_idx = int(src[1])
    ctx.src_idx = int(src[1]) * NX + int(src[0])
    ctx.src_type = src_type
    ctx.src_amp = src_amp
    ctx.src_angle = src_angle
    rcv = np.asarray([z * NX + x for x, z in receivers], dtype=np.int32)
    ctx.rcv_grid_idx = rcv
    ctx.num_rcv = int(rcv.size)
    return ctx


def two_layer_shot(steps: int = 2000) -> Shot2D:
    npml = 20
    ctx = layered_context(440, 420, npml, 5.0, 0.0005, steps,
                          [(0, 2500.0, 1443.0, 2000.0), (200, 3500.0, 2000.0, 2300.0)],
                          f0=20.0, src=(200, npml + 20), src_type=capi2d.EXPLOSIVE,
                          receivers=[(x, npml + 10) for x in range(0, 400, 2)])
    return Shot2D(ctx, steps, "two_layer_440x420")


def small_shot2d(flag_type: int = 3, up: bool = True, steps: int = 200, src_type: int = capi2d.EXPLOSIVE,
                 size=(120, 100), npml: int = 12) -> Shot2D:
    """A small layered case of the same construction for parity tests."""
    NX, NZ = size
    fs = npml if (flag_type == 3 and up) else 0
    ctx = layered_context(NX, NZ, npml, 5.0, 0.0005, steps,
                          [(0, 2200.0, 1200.0, 1900.0), (30, 3000.0, 1700.0, 2200.0), (55, 3600.0, 2050.0, 2350.0)],
                          f0=25.0, src=(NX // 2 + 3, fs + 14), src_type=src_type, src_angle=30.0,
                          receivers=[(x, fs + 6) for x in range(0, NX, 3)] + [(NX // 3, fs + 40), (NX - 9, NZ - 9)],
                          flag_type=flag_type, up=up)
    return Shot2D(ctx, steps, f"small_{NX}x{NZ}_type{flag_type}{'fs' if up else ''}")
