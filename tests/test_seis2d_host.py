"""2-D solver host side on the CPU: the C-ABI library loads without a GPU, exports every
entry point include/seis2d_capi.h declares, and its host numerics and validation behave as
the reference's (Main_header/SolverNumerics.h, src/Seis2D/Numerics2D.inc,
CUDA_Kernels/Cuda_Check.cu:841-884, tests/SolverRegression.cpp:67-83,155-161)."""
import os
import re
import subprocess

import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import InvalidArgument, LogicError, capi2d, models2d, seis2d

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "seis2d_capi.h")


def declared_functions():
    text = open(HEADER).read()
    return set(re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(seis2d_\w+)\s*\(", text, flags=re.M))


def test_header_declarations_match_bindings():
    declared = declared_functions()
    assert len(declared) > 20
    assert declared == set(capi2d.SIGNATURES), declared ^ set(capi2d.SIGNATURES)


def test_library_exports_every_declared_symbol(solver2d_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", capi2d.LIBRARY_PATH], capture_output=True, text=True,
                         check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    assert not declared_functions() - exported
    assert solver2d_lib.seis2d_abi_version() == 1


def test_session_calls_without_session_are_lifecycle_errors(solver2d_lib):
    ctx = models2d.small_shot2d(steps=10).context
    c = ctx.to_c()
    from ctypes import byref
    assert solver2d_lib.seis2d_run_step(None, 0, byref(c), -1) == capi2d.SEIS2D_LOGIC_ERROR
    assert solver2d_lib.seis2d_update_receivers(None, None, 0) == capi2d.SEIS2D_LOGIC_ERROR
    solver2d_lib.seis2d_release(None)
    gpu = seis2d.GPUSimData()
    with pytest.raises(LogicError):
        seis2d.runGpuSimulationStep(gpu, 0, ctx, -1)
    seis2d.releaseGpuSimulation(gpu)
    seis2d.releaseGpuSimulation(gpu)


def test_stencil_weights_moments_and_courant_limits(solver2d_lib):
    # SolverRegression.cpp:67-75: sum 2 w_k (k + 1/2)^d = delta_{d,1} for d = 1, 3, 5, 7.
    w = (np.ctypeslib.as_ctypes(np.zeros(4)))
    solver2d_lib.seis2d_stencil_weights(w)
    weights = np.array(list(w))
    assert np.array_equal(weights, np.array(seis2d.kStaggeredDerivativeWeights))
    for degree in (1, 3, 5, 7):
        moment = sum(2.0 * weights[i] * (i + 0.5) ** degree for i in range(4))
        assert abs(moment - (1.0 if degree == 1 else 0.0)) < 1e-10
    magnitude = weights[0] - weights[1] + weights[2] - weights[3]
    assert seis2d.kCourantLimit2d() == np.float32(1.0 / (1.4142135623730951 * magnitude))
    assert abs(seis2d.kCourantLimit2d() - 0.550) < 1e-3
    assert np.float32(solver2d_lib.seis2d_safe_courant()) == np.float32(0.48)


def test_geometry_and_sampling_rejections(solver2d_lib):
    # SolverRegression.cpp:76-82.
    with pytest.raises(OverflowError):
        seis2d.checkedGridElementCount(100000, 100000)
    with pytest.raises(InvalidArgument):
        seis2d.validateBoundaryGeometry(96, 96, 0, True)
    with pytest.raises(InvalidArgument):
        seis2d.validateBoundaryGeometry(96, 96, 48, False)
    with pytest.raises(InvalidArgument):
        seis2d.checkedGridElementCount(8, 96)
    assert seis2d.checkedGridElementCount(440, 420) == 440 * 420
    seis2d.validateBoundaryGeometry(96, 96, 43, False)
    with pytest.raises(InvalidArgument):
        seis2d.validateBoundaryGeometry(96, 96, 44, False)
    assert seis2d.getReceiverSamplingStride(0.00024, 10000.0) == 1
    assert seis2d.getReceiverSamplingStride(0.00024, 1000.0) == 4
    with pytest.raises(InvalidArgument):
        seis2d.getReceiverSamplingStride(0.0, 1000.0)
    with pytest.raises(InvalidArgument):
        seis2d.getReceiverSamplingStride(0.001, 0.0)


def test_ricker_series_matches_the_reference_formula(solver2d_lib):
    # generateRickerWavelet (Numerics2D.inc:3-14): t = i*dt - t0 in FP32,
    # (1 - 2 pi^2 f0^2 t^2) exp(-pi^2 f0^2 t^2).
    nt, dt, f0 = 400, np.float32(0.0005), np.float32(20.0)
    t0 = np.float32(1.0) / f0
    w = seis2d.generateRickerWavelet(nt, dt, f0, t0)
    i = np.arange(nt, dtype=np.float32)
    t = (i * dt - t0).astype(np.float64)
    expected = (1 - 2 * np.pi ** 2 * 400.0 * t * t) * np.exp(-np.pi ** 2 * 400.0 * t * t)
    assert np.max(np.abs(w - expected)) < 2e-6
    assert int(np.argmax(w)) == 100 and w[100] == np.float32(1.0)
    with pytest.raises(InvalidArgument):
        seis2d.generateRickerWavelet(0, dt, f0, t0)
    with pytest.raises(InvalidArgument):
        seis2d.generateRickerWavelet(10, dt, 0.0, t0)


def test_pml_profile_and_free_surface_modulus(solver2d_lib):
    # updatePmlDampingArrays (Numerics2D.inc:36-83): d_max = 3 vp 16.12 3.5 / (2 L),
    # d = d_max ((npml - i)/npml)^2.5 at whole points and ((npml - i - 1/2)/npml)^2.5 at half points.
    ctx = models2d.two_layer_shot(10).context
    vp = np.sqrt(ctx.lambda2mu / ctx.rho).max()
    d_max = 3.0 * vp * 16.12 * 3.5 / (2.0 * 20 * 5.0)
    i = np.arange(20)
    whole = d_max * ((20 - i) / 20.0) ** 2.5
    half = d_max * ((20 - i - 0.5) / 20.0) ** 2.5
    np.testing.assert_allclose(ctx.dx[:20], whole, rtol=2e-6)
    np.testing.assert_allclose(ctx.dx[::-1][:20], whole, rtol=2e-6)
    np.testing.assert_allclose(ctx.dz_half[:20], half, rtol=2e-6)
    assert np.all(ctx.dx[20:-20] == 0) and np.all(ctx.dz[20:-20] == 0)
    # dp_flat (Numerics2D.inc:124-135): (l2m^2 - lambda^2) / l2m on the free-surface row.
    k = 20 * ctx.NX
    l2m, lam = ctx.lambda2mu[k], ctx.lambda_[k]
    assert ctx.dp_flat[0] == np.float32((l2m * l2m - lam * lam) / l2m)


def test_validation_rejections_match_the_reference(solver2d_lib):
    # SolverRegression.cpp:155-161 plus the remaining checks of validateSimulationContext.
    base = models2d.small_shot2d(steps=20).context
    seis2d.validateSimulationContext(base)
    cases = []
    c = base.copy(); c.rho = c.rho.copy(); c.rho[0] = 0.0; cases.append(c)
    c = base.copy(); c.dt = 1.0; cases.append(c)
    c = base.copy(); c.mu = c.mu.copy(); c.mu[0] = c.lambda2mu[0]; cases.append(c)
    c = base.copy(); c.flag_type = 4; cases.append(c)
    c = base.copy(); c.total_grid -= 1; cases.append(c)
    c = base.copy(); c.wavelet = c.wavelet[:-1]; cases.append(c)
    c = base.copy(); c.dx = c.dx[:-1]; cases.append(c)
    c = base.copy(); c.dp_flat = c.dp_flat[:-1]; cases.append(c)
    c = base.copy(); c.num_rcv += 1; cases.append(c)
    c = base.copy(); c.rcv_grid_idx = c.rcv_grid_idx.copy(); c.rcv_grid_idx[0] = c.total_grid; cases.append(c)
    c = base.copy(); c.dz = c.dz.copy(); c.dz[3] = -1.0; cases.append(c)
    c = base.copy(); c.lambda2mu = c.lambda2mu.copy(); c.lambda2mu[5] = np.inf; cases.append(c)
    c = base.copy(); c.nt = 0; cases.append(c)
    for bad in cases:
        with pytest.raises(InvalidArgument):
            seis2d.validateSimulationContext(bad)
    big = base.copy(); big.NX = 100000; big.NZ = 100000
    with pytest.raises(OverflowError):
        seis2d.validateSimulationContext(big)
