"""Failure handling by host-side fault injection (seis3d/seis2d_debug_fail_allocation): every
device or pinned allocation of a session's initialisation is made to fail in turn, and the
call must report a runtime error, hand back no session and leave no device memory behind
(the reference's transactional initializeGpu3D, cuda/Cuda_Seis3D.cu:533-554); a failed
receiver replacement keeps the previous receivers (:656-667).  Nothing faults on the GPU:
the failure is a refused allocation on the host side of the call."""
import ctypes

import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, capi2d, models3d, seis2d, seis3d
from seis2d_cases import make_context

pytestmark = pytest.mark.gpu

SLACK = 4 << 20   # allocation granularity of the device allocator


def free_bytes() -> int:
    from cuda.bindings import runtime as rt
    err, free, _ = rt.cudaMemGetInfo()
    assert err == rt.cudaError_t.cudaSuccess
    return int(free)


def test_3d_initialize_rolls_back_each_allocation(cuda_device):
    lib = capi.load()
    c = seis3d.validate_context3D(seis3d.default_context(nx3D=64, ny3D=48, nz3D=40, pml3D=8))
    seis3d.Session(c).release()          # the context and the kernels are loaded
    base = free_bytes()
    failures = 0
    try:
        for n in range(1, 40):
            lib.seis3d_debug_fail_allocation(n)
            h, cc = ctypes.c_void_p(), c.copy()
            status = lib.seis3d_initialize(ctypes.byref(h), ctypes.byref(cc), None)
            lib.seis3d_debug_fail_allocation(0)
            if status == capi.SEIS3D_OK:
                lib.seis3d_release(h)
                break
            failures += 1
            assert status == capi.SEIS3D_RUNTIME_ERROR and not h.value, n
            assert b"out of memory" in lib.seis3d_last_error(), n
            assert abs(free_bytes() - base) <= SLACK, n
    finally:
        lib.seis3d_debug_fail_allocation(0)
    # Fields, three CPML memories and coefficient tables, status, tensor maps, clock, staging.
    assert failures >= 11
    assert abs(free_bytes() - base) <= SLACK


def test_3d_receiver_replacement_keeps_the_old_set(cuda_device):
    lib = capi.load()
    shot = models3d.small_shot(steps=6)
    s = seis3d.Session(shot.context)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.run_steps(shot.source, 0, 6)
    before = s.sample_receivers()
    try:
        for n in (1, 2, 3):               # positions, values, pinned host copy
            lib.seis3d_debug_fail_allocation(n)
            with pytest.raises(seis3d.SolverError):
                s.set_receivers(shot.receivers[:3])
            lib.seis3d_debug_fail_allocation(0)
            assert s.receiver_count == len(shot.receivers)
            assert np.array_equal(s.sample_receivers(), before)
    finally:
        lib.seis3d_debug_fail_allocation(0)
    s.release()


def test_2d_initialize_rolls_back_each_allocation(cuda_device):
    lib = capi2d.load()
    ctx = make_context(3, free_surface=True)
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, ctx)
    seis2d.releaseGpuSimulation(gpu)
    base = free_bytes()
    failures = 0
    try:
        for n in range(1, 80):
            lib.seis2d_debug_fail_allocation(n)
            gpu = seis2d.GPUSimData()
            try:
                seis2d.initializeGpuSimulation(gpu, ctx)
            except seis3d.SolverError as e:
                failures += 1
                assert "out of memory" in str(e)
                assert not gpu._handle.value, n
                assert abs(free_bytes() - base) <= SLACK, n
                continue
            finally:
                lib.seis2d_debug_fail_allocation(0)
            seis2d.releaseGpuSimulation(gpu)
            break
    finally:
        lib.seis2d_debug_fail_allocation(0)
    # The arena of the initialisation arrays, then the receivers' index and sample buffers.
    assert failures >= 4
    assert abs(free_bytes() - base) <= SLACK
