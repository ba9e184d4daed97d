"""The bounded waits of the device code, made to run out on purpose without faulting the GPU.

3-D: every wait of the z-marching passes on a TMA stage is bounded.  seis3d_debug_stage_wait
shortens the bound to a few microseconds and makes every CTA skip the copies of one plane,
so nothing ever completes that stage: the waits give up, the CTAs record a staging stall,
drain the copies they did issue (bounded again) and exit, and the next synchronising call
reports SEIS3D_RUNTIME_ERROR.  2-D: the grid barriers of the persistent cooperative run are
bounded the same way; seis2d_debug_barrier_wait keeps one block from arriving at the first
barrier, every block gives up and the run reports its failure.

In both cases the wait that runs out is on something no one will ever complete (no copy was
issued, no arrival was made), the device keeps answering, and a fresh session afterwards
must compute a small shot correctly (checked against the CPU oracle)."""
import ctypes
import time

import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, capi2d, models2d, models3d, seis2d, seis3d

pytestmark = pytest.mark.gpu

SHORT_WAIT = 200_000   # SM cycles, ~0.1 ms at 1.9 GHz


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_3d_shot_is_correct():
    shot = models3d.small_shot(steps=40)
    s = seis3d.Session(shot.context)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.gather_begin(1, shot.steps)
    s.run_steps(shot.source, 0, shot.steps)
    gather = s.gather_fetch()
    s.release()
    o = oracle.CpuOracle(shot.context, 32)
    o.upload_model(shot.vp, shot.vs, shot.rho)
    expect = o.run_gather(shot.source, 0, shot.steps, shot.receivers, 1)
    o.close()
    return rel_l2(gather, expect)


@pytest.mark.parametrize("withheld", [0, 2, 5])
def test_3d_stage_wait_runs_out_and_reports(withheld, solver_lib, cuda_device):
    shot = models3d.small_shot(steps=4)
    s = seis3d.Session(shot.context, z_chunk=8)
    try:
        s.upload_model(shot.vp, shot.vs, shot.rho)
        s.set_receivers(shot.receivers)
        s.synchronize()
        assert solver_lib.seis3d_debug_stage_wait(s.handle, SHORT_WAIT, withheld) == capi.SEIS3D_OK
        t = time.perf_counter()
        with pytest.raises(seis3d.SolverError, match="stalled"):
            s.run_steps(shot.source, 0, 2)
            s.synchronize()
        assert time.perf_counter() - t < 10.0
        # The stall stays recorded: every later synchronising call reports it.
        with pytest.raises(seis3d.SolverError, match="stalled"):
            s.synchronize()
        assert solver_lib.seis3d_debug_stage_wait(s.handle, -1, 0) == capi.SEIS3D_INVALID_ARGUMENT
    finally:
        s.release()
    assert small_3d_shot_is_correct() < 1e-5


def test_3d_default_settings_do_not_stall(solver_lib, cuda_device):
    shot = models3d.small_shot(steps=4)
    s = seis3d.Session(shot.context)
    try:
        s.upload_model(shot.vp, shot.vs, shot.rho)
        assert solver_lib.seis3d_debug_stage_wait(s.handle, SHORT_WAIT, 1) == capi.SEIS3D_OK
        assert solver_lib.seis3d_debug_stage_wait(s.handle, 0, -1) == capi.SEIS3D_OK   # back to normal
        s.run_steps(shot.source, 0, 4)
        s.synchronize()
    finally:
        s.release()


def test_2d_grid_barrier_runs_out_and_reports(solver2d_lib, cuda_device):
    shot = models2d.small_shot2d(steps=30)
    c = shot.context
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, c)
    try:
        seis2d.setRunMode(gpu, capi2d.RUN_PERSISTENT)
        handle = seis2d._session(gpu)
        assert solver2d_lib.seis2d_debug_barrier_wait(handle, SHORT_WAIT, 0) == capi2d.SEIS2D_OK
        t = time.perf_counter()
        with pytest.raises(RuntimeError, match="grid barrier"):
            seis2d.runGpuSimulationSteps(gpu, 0, 10, c)
            seis2d.synchronize(gpu)
        assert time.perf_counter() - t < 10.0
        assert solver2d_lib.seis2d_debug_barrier_wait(handle, -5, 0) == capi2d.SEIS2D_INVALID_ARGUMENT
    finally:
        seis2d.releaseGpuSimulation(gpu)

    # A fresh session in the same mode runs correctly.
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, c)
    seis2d.setRunMode(gpu, capi2d.RUN_PERSISTENT)
    seis2d.gatherBegin(gpu, 0, 1, shot.steps)
    seis2d.runGpuSimulationSteps(gpu, 0, shot.steps, c)
    _, vz, taken = seis2d.gatherFetch(gpu, shot.steps)
    seis2d.releaseGpuSimulation(gpu)
    o = oracle.CpuOracle2D(c, 32)
    _, oz = o.run(0, shot.steps, receivers=c.rcv_grid_idx)
    o.close()
    assert taken == shot.steps
    assert rel_l2(vz[: c.num_rcv], oz) < 1e-4
