"""2-D cases of the reference's solver regression (tests/SolverRegression.cpp), restated for
both the CPU oracle and the CUDA solver."""
import numpy as np

from cmakepro_cuda_seissim_v2_b200 import seis2d


def make_context(scheme: int, free_surface: bool = False, size: int = 96, density: float = 1000.0):
    """makeContext (SolverRegression.cpp:22-49): uniform medium, zero damping profiles, 700
    steps of a 200 Hz Ricker at dt = 0.1 ms, one receiver 8 cells right of the source."""
    f = np.float32
    n = size * size
    ctx = seis2d.SimulationContext(NX=size, NZ=size, total_grid=n, h=1.0, dt=float(f(0.0001)), nt=700, npml=16,
                                   flag_type=scheme, upFlag=free_surface)
    ctx.c1_h, ctx.c2_h, ctx.c3_h, ctx.c4_h = (float(f(w)) for w in seis2d.kStaggeredDerivativeWeights)
    d = f(density)
    ctx.rho = np.full(n, d, f)
    ctx.mu = np.full(n, d * f(1000.0) * f(1000.0), f)
    ctx.lambda2mu = np.full(n, d * f(2000.0) * f(2000.0), f)
    ctx.lambda_ = np.full(n, d * f(2000000.0), f)
    ctx.dp_flat = np.full(size, d * f(3000000.0), f)
    ctx.dx, ctx.dx_half, ctx.dz, ctx.dz_half = (np.zeros(size, f) for _ in range(4))
    steps = np.arange(ctx.nt, dtype=f)
    phase = f(3.14159265358979323846) * f(200.0) * (steps * f(ctx.dt) - f(0.005))
    ctx.wavelet = ((f(1.0) - f(2.0) * phase * phase) * np.exp(-phase * phase)).astype(f)
    ctx.src_idx = (size // 2) * size + size // 2
    ctx.src_z_idx = size // 2
    ctx.src_amp = 1.0
    ctx.src_type = 0
    ctx.num_rcv = 1
    ctx.rcv_grid_idx = np.array([ctx.src_idx + 8], np.int32)
    return ctx


def add_pml(ctx):
    """The damping profile of checkPmlReflection (SolverRegression.cpp:182-190)."""
    f = np.float32
    m = f(3.0) * f(2000.0) * f(16.12) * f(3.5) / (f(2.0) * f(ctx.npml))
    for i in range(ctx.npml):
        whole = m * f(np.power(f((ctx.npml - i) / f(ctx.npml)), f(2.5)))
        half = m * f(np.power(f((ctx.npml - i - f(0.5)) / f(ctx.npml)), f(2.5)))
        for arr, val in ((ctx.dx, whole), (ctx.dz, whole), (ctx.dx_half, half), (ctx.dz_half, half)):
            arr[i] = val
            arr[arr.size - 1 - i] = val
    return ctx


def late_error_ratio(pml_trace, wall_trace, reference_trace, start=350):
    """sqrt(sum (pml - ref)^2 / sum (wall - ref)^2) over the late window (:195-201)."""
    p = np.asarray(pml_trace, np.float64)[start:]
    w = np.asarray(wall_trace, np.float64)[start:]
    r = np.asarray(reference_trace, np.float64)[start:]
    wall = np.sum((w - r) ** 2)
    return float(np.sqrt(np.sum((p - r) ** 2) / wall)), wall
