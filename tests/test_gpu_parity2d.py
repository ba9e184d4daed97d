"""Parity of the B200 2-D P-SV solver (libseis2d_b200.so through its C ABI) with the CPU oracle
and with the reference's own CUDA solver (CUDA_Kernels/Cuda_Check.cu built from source), plus
the reference's solver regression cases (tests/SolverRegression.cpp) run on the CUDA path.

Tolerances: receiver traces and wavefields within 1e-5 relative L2 of the reference CUDA
solver (same FP32 arithmetic, both built with --use_fast_math); physical totals within 1e-4
of the CPU FP32 oracle (IEEE division, no contraction: a different rounding of the same
scheme); and against the FP64 oracle an error of the order of the FP32 oracle's own (at most
ten times it, or 1e-5, and below 1e-4; the approximate division of --use_fast_math is the
difference).  Source and receiver indices are exact: a trace of the wrong cell misses these
bounds by orders of magnitude."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi2d, models2d, seis2d
from seis2d_cases import add_pml, late_error_ratio, make_context

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5    # vs the reference CUDA solver
ORACLE32_TOL = 1e-4  # vs the CPU FP32 oracle
FP64_TOL = 1e-4     # vs the CPU FP64 oracle (absolute cap)
SPLIT_PAIRS = (("vx_1", "vx_2"), ("vz_1", "vz_2"), ("sxx_1", "sxx_2"), ("szz_1", "szz_2"), ("sxz_1", "sxz_2"))


def check_accuracy(gpu_values, oracle32_values, oracle64_values):
    """GPU vs the FP64 run of the order of the FP32 oracle vs the FP64 run, capped."""
    e_gpu = rel_l2(gpu_values, oracle64_values)
    e_cpu = rel_l2(oracle32_values, oracle64_values)
    assert e_gpu < FP64_TOL and e_gpu <= max(10.0 * e_cpu, 1e-5), (e_gpu, e_cpu)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def gpu_run(ctx, steps, num_active=-1, sources=None, graph=True):
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, ctx)
    if sources is not None:
        seis2d.setActiveSources(gpu, sources)
    seis2d.gatherBegin(gpu, 0, 1, steps)
    if graph:
        seis2d.runGpuSimulationSteps(gpu, 0, steps, ctx, num_active)
    else:
        for n in range(steps):
            seis2d.runGpuSimulationStep(gpu, n, ctx, num_active)
    vx, vz, taken = seis2d.gatherFetch(gpu, steps)
    assert taken == steps
    return gpu, vx[: ctx.num_rcv], vz[: ctx.num_rcv]


def reference_available():
    return oracle.reference2d_library() is not None


def test_two_layer_shot_matches_reference_and_oracle(solver2d_lib, cuda_device):
    shot = models2d.two_layer_shot()
    c = shot.context
    gpu, vx, vz = gpu_run(c, shot.steps)
    assert np.abs(vz).max() > 0 and np.all(np.isfinite(vz))
    if reference_available():
        ref = oracle.ReferenceSolver2D(c)
        rx, rz = ref.run(0, shot.steps, nrcv=c.num_rcv)
        print("two-layer shot vs reference CUDA: vz %.3g vx %.3g (bit-equal %s)"
              % (rel_l2(vz, rz), rel_l2(vx, rx), np.array_equal(vz, rz) and np.array_equal(vx, rx)))
        assert rel_l2(vz, rz) < TRACE_TOL and rel_l2(vx, rx) < TRACE_TOL
        for a, b in SPLIT_PAIRS:
            for name in (a, b):
                assert rel_l2(seis2d.copyField(gpu, name), ref.field(capi2d.FIELD[name])) < TRACE_TOL, name
    o32 = oracle.CpuOracle2D(c, 32)
    ox, oz = o32.run(0, shot.steps, receivers=c.rcv_grid_idx)
    assert rel_l2(vz, oz) < ORACLE32_TOL and rel_l2(vx, ox) < ORACLE32_TOL
    assert rel_l2(seis2d.copyWavefieldToHost(gpu), o32.wavefield()) < ORACLE32_TOL
    o64 = oracle.CpuOracle2D(c, 64)
    dx, dz = o64.run(0, shot.steps, receivers=c.rcv_grid_idx)
    check_accuracy(vz, oz, dz)
    check_accuracy(vx, ox, dx)
    seis2d.releaseGpuSimulation(gpu)


CASES = [(1, False, capi2d.EXPLOSIVE), (2, False, capi2d.EXPLOSIVE), (3, True, capi2d.EXPLOSIVE),
         (3, False, capi2d.EXPLOSIVE), (3, True, capi2d.VERTICAL_FORCE), (3, True, capi2d.HORIZONTAL_FORCE),
         (3, True, capi2d.SHEAR), (3, True, capi2d.ROTATED_FORCE), (1, False, capi2d.ROTATED_FORCE),
         (2, False, capi2d.SHEAR), (2, False, capi2d.VERTICAL_FORCE), (2, False, capi2d.ROTATED_FORCE)]


@pytest.mark.parametrize("scheme,up,src_type", CASES)
def test_schemes_and_source_types(scheme, up, src_type, solver2d_lib, cuda_device):
    shot = models2d.small_shot2d(scheme, up, steps=300, src_type=src_type)
    c = shot.context
    gpu, vx, vz = gpu_run(c, shot.steps)
    fields = [name for pair in SPLIT_PAIRS for name in pair]
    fields += ["vx", "vz", "sigmaxx", "sigmazz", "sigmaxz"] if scheme == 2 else []
    if reference_available():
        ref = oracle.ReferenceSolver2D(c)
        rx, rz = ref.run(0, shot.steps, nrcv=c.num_rcv)
        assert rel_l2(vz, rz) < TRACE_TOL and rel_l2(vx, rx) < TRACE_TOL
        for name in fields:
            assert rel_l2(seis2d.copyField(gpu, name), ref.field(capi2d.FIELD[name])) < TRACE_TOL, name
    o = oracle.CpuOracle2D(c, 32)
    ox, oz = o.run(0, shot.steps, receivers=c.rcv_grid_idx)
    assert np.abs(oz).max() > 0
    assert rel_l2(vz, oz) < ORACLE32_TOL and rel_l2(vx, ox) < ORACLE32_TOL
    o64 = oracle.CpuOracle2D(c, 64)
    dx, dz = o64.run(0, shot.steps, receivers=c.rcv_grid_idx)
    check_accuracy(vz, oz, dz)
    check_accuracy(vx, ox, dx)
    # Physical totals of the split pairs against the FP32 oracle (a split half alone can be a
    # small difference of large terms, so its own norm is not the scale of its error).
    for a, b in SPLIT_PAIRS:
        ours = seis2d.copyField(gpu, a) + seis2d.copyField(gpu, b)
        theirs = o.field(capi2d.FIELD[a]) + o.field(capi2d.FIELD[b])
        assert rel_l2(ours, theirs) < ORACLE32_TOL, a
    seis2d.releaseGpuSimulation(gpu)


@pytest.mark.parametrize("scheme,up", [(3, True), (2, False)])
def test_graph_replay_equals_single_steps(scheme, up, solver2d_lib, cuda_device):
    shot = models2d.small_shot2d(scheme, up, steps=150)
    c = shot.context
    ga, ax, az = gpu_run(c, shot.steps, graph=True)
    gb, bx, bz = gpu_run(c, shot.steps, graph=False)
    assert np.array_equal(ax, bx) and np.array_equal(az, bz)
    for name in ("vx_1", "vz_2", "sxx_1", "szz_1", "sxz_2"):
        assert np.array_equal(seis2d.copyField(ga, name), seis2d.copyField(gb, name)), name
    # Runs split at arbitrary points continue exactly.
    gc = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gc, c)
    done = 0
    for count in (1, 63, 64, 2, 20):
        seis2d.runGpuSimulationSteps(gc, done, count, c)
        done += count
    assert np.array_equal(seis2d.copyWavefieldToHost(gc), seis2d.copyWavefieldToHost(ga))


def test_receiver_records_match_gather(solver2d_lib, cuda_device):
    shot = models2d.small_shot2d(3, True, steps=40)
    c = shot.context
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, c)
    seis2d.gatherBegin(gpu, 5, 3, 20)
    rec_vx = np.zeros(c.num_rcv * shot.steps, np.float32)
    rec_vz = np.zeros(c.num_rcv * shot.steps, np.float32)
    for n in range(shot.steps):
        seis2d.runGpuSimulationStep(gpu, n, c, -1)
        seis2d.copyReceiverRecordsFromGpu(gpu, c.num_rcv, shot.steps, n, rec_vx, rec_vz)
    vx, vz, taken = seis2d.gatherFetch(gpu, 20)
    assert taken == 12  # steps 5, 8, ..., 38
    rec_vz = rec_vz.reshape(c.num_rcv, shot.steps)
    rec_vx = rec_vx.reshape(c.num_rcv, shot.steps)
    assert np.array_equal(vz[:, :taken], rec_vz[:, 5:40:3])
    assert np.array_equal(vx[:, :taken], rec_vx[:, 5:40:3])
    assert np.all(vz[:, taken:] == 0)
    one_vx, one_vz = seis2d.recordReceiverStepOnGpu(gpu, c.num_rcv)
    assert np.array_equal(one_vz, rec_vz[:, -1])


@pytest.mark.parametrize("scheme,density,free", [(1, 1000.0, False), (2, 1000.0, False), (2, 100.0, False),
                                                 (2, 0.5, False), (3, 1000.0, True)])
def test_cubic_stress_gradient(scheme, density, free, solver2d_lib, cuda_device):
    # SolverRegression.cpp:86-111 on the CUDA path.
    ctx = make_context(scheme, free, 96, density)
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, ctx)
    z = np.arange(ctx.NZ, dtype=np.float32)
    seis2d.setField(gpu, "sigmazz" if scheme == 2 else "szz_1", np.repeat((z * z * z)[:, None], ctx.NX, axis=1))
    seis2d.runGpuSimulationStep(gpu, 0, ctx, 0)
    vz = seis2d.copyWavefieldToHost(gpu).reshape(ctx.NZ, ctx.NX)
    expected = np.float32(ctx.dt) * 3.0 * 30.5 * 30.5 / density
    assert abs(vz[30, 48] - expected) < expected * 2e-5
    if free:
        szz = seis2d.copyField(gpu, "szz_1")
        assert np.all(szz[ctx.npml, 4:-4] == 0.0)
        for layer in range(1, 5):
            assert np.array_equal(szz[ctx.npml - layer, 4:-4], -szz[ctx.npml + layer, 4:-4])


def test_disabled_free_surface_equals_split_pml(solver2d_lib, cuda_device):
    # SolverRegression.cpp:114-126.
    first, third = make_context(1), make_context(3, False)
    out = []
    for c in (first, third):
        c.src_z_idx = 12
        c.src_idx = 12 * c.NX + 48
        gpu = seis2d.GPUSimData()
        seis2d.initializeGpuSimulation(gpu, c)
        for n in range(120):
            seis2d.runGpuSimulationStep(gpu, n, c, -1)
        out.append(seis2d.copyWavefieldToHost(gpu))
    assert np.abs(out[0]).max() > 0 and np.array_equal(out[0], out[1])


def test_sources_and_resources(solver2d_lib, cuda_device):
    # SolverRegression.cpp:129-162.
    ctx = make_context(1)
    ctx.src_type = capi2d.HORIZONTAL_FORCE
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, ctx)
    seis2d.setActiveSources(gpu, [(ctx.src_idx, 0.005, 200.0, 1.0)] * 200)
    seis2d.runGpuSimulationStep(gpu, 0, ctx, 200)
    vx = seis2d.copyField(gpu, "vx_1").reshape(-1)
    expected = 200 * 1e7 * np.float32(ctx.dt) / ctx.rho[ctx.src_idx]
    assert abs(vx[ctx.src_idx] - expected) < expected * 1e-5
    with pytest.raises(seis2d.InvalidArgument):
        seis2d.runGpuSimulationStep(gpu, 0, ctx, 201)
    with pytest.raises(seis2d.InvalidArgument):
        seis2d.updateGpuReceivers(gpu, [ctx.total_grid])
    assert gpu.receiverCapacity == 1
    seis2d.writeDevice(gpu, gpu.d_rcv_grid_idx, np.array([ctx.total_grid], np.int32))
    bad_vx, bad_vz = seis2d.recordReceiverStepOnGpu(gpu, 1, np.full(1, -1.0, np.float32), np.full(1, -1.0, np.float32))
    assert bad_vx[0] == 0.0 and bad_vz[0] == 0.0
    with pytest.raises(seis2d.InvalidArgument):
        seis2d.writeDevice(gpu, gpu.d_rcv_grid_idx + 4096, np.zeros(4, np.int32))
    # The fields share one allocation; a range must still lie inside one field.
    last = gpu.d_vx_1 + 4 * (ctx.total_grid - 1)
    seis2d.writeDevice(gpu, last, vx[-1:].copy())
    with pytest.raises(seis2d.InvalidArgument):
        seis2d.writeDevice(gpu, last, np.zeros(2, np.float32))
    seis2d.updateGpuReceivers(gpu, [])
    assert gpu.receiverCapacity == 0 and gpu.d_rcv_grid_idx == 0
    with pytest.raises(seis2d.InvalidArgument):
        seis2d.recordReceiverStepOnGpu(gpu, 1)
    seis2d.releaseGpuSimulation(gpu)
    seis2d.releaseGpuSimulation(gpu)
    assert not gpu.initialized
    bad = make_context(1)
    bad.rho = bad.rho.copy()
    bad.rho[0] = 0.0
    with pytest.raises(seis2d.InvalidArgument):
        seis2d.initializeGpuSimulation(gpu, bad)
    assert not gpu.initialized


def run_trace(ctx):
    gpu, vx, vz = gpu_run(ctx, ctx.nt, graph=False)
    assert np.all(np.isfinite(vz)) and np.all(np.isfinite(vx))
    assert np.all(np.isfinite(seis2d.copyWavefieldToHost(gpu)))
    return vz[0]


@pytest.mark.parametrize("scheme,published", [(1, 0.0433824), (2, 0.0433818)])
def test_pml_late_window_ratio(scheme, published, solver2d_lib, cuda_device):
    # SolverRegression.cpp:181-205 and the published figure of its GPU build.
    ratio, wall = late_error_ratio(run_trace(add_pml(make_context(scheme))), run_trace(make_context(scheme)),
                                   run_trace(make_context(scheme, False, 288)))
    assert wall > 0 and ratio < 0.5
    assert ratio == pytest.approx(published, rel=1e-4)


def test_free_surface_finite_evolution(solver2d_lib, cuda_device):
    run_trace(make_context(3, True))


@pytest.mark.parametrize("scheme,up,src_type", [(3, True, capi2d.EXPLOSIVE), (1, False, capi2d.VERTICAL_FORCE),
                                                (2, False, capi2d.SHEAR)])
def test_advancing_multi_sources(scheme, up, src_type, solver2d_lib, cuda_device):
    # The reference time loop with multi-source mode (src/Seis2D/Workflow2D.inc:300-318):
    # every step each active source moves by dt and is dropped past 2.5 / f_peak.
    shot = models2d.small_shot2d(scheme, up, steps=120, src_type=src_type)
    c = shot.context
    fs = c.npml if (scheme == 3 and up) else 0
    sources = [((fs + 14) * c.NX + 40, 0.0, 60.0, 1.0), ((fs + 20) * c.NX + 70, -0.01, 45.0, -0.5),
               ((fs + 14) * c.NX + 40, 0.002, 80.0, 0.7), ((fs + 30) * c.NX + 90, 0.0, 150.0, 2.0)]
    gpu, vx, vz = gpu_run(c, shot.steps, num_active=len(sources), sources=sources)
    o = oracle.CpuOracle2D(c, 32)
    o.set_sources(sources)
    ox, oz = o.run(0, shot.steps, num_active=len(sources), advance=True, receivers=c.rcv_grid_idx)
    assert np.abs(oz).max() > 0
    assert rel_l2(vz, oz) < ORACLE32_TOL and rel_l2(vx, ox) < ORACLE32_TOL
    if reference_available():
        # The host loop itself, driving the reference solver.
        ref = oracle.ReferenceSolver2D(c)
        live = [list(s) for s in sources]
        rz = np.zeros_like(vz)
        for n in range(shot.steps):
            kept = []
            for s in live:
                s[1] = float(np.float32(s[1]) + np.float32(c.dt))
                if np.float32(s[1]) > np.float32(2.5) * (np.float32(1.0) / np.float32(s[2])):
                    continue
                kept.append(s)
            live = kept
            if live:
                ref.set_sources(live)
            ref.step(n, len(live))
            rz[:, n] = ref_record(ref, c)
        assert rel_l2(vz, rz) < TRACE_TOL


def ref_record(ref, c):
    import ctypes
    vx = np.zeros(c.num_rcv, np.float32)
    vz = np.zeros(c.num_rcv, np.float32)
    status = ref.lib.ref2d_record(ref.h, c.num_rcv, vx.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                  vz.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert status == 0
    return vz


def test_step_counter_and_launch_count(solver2d_lib, cuda_device):
    shot = models2d.small_shot2d(3, True, steps=10)
    gpu = seis2d.GPUSimData()
    seis2d.initializeGpuSimulation(gpu, shot.context)
    seis2d.setRunMode(gpu, capi2d.RUN_PERSISTENT)
    before = gpu.kernelLaunches
    seis2d.runGpuSimulationSteps(gpu, 0, 130, shot.context)
    # Persistent run: the run configuration and one cooperative launch.
    assert gpu.kernelLaunches - before == 2
    seis2d.setRunMode(gpu, capi2d.RUN_GRAPH)
    before = gpu.kernelLaunches
    seis2d.runGpuSimulationSteps(gpu, 130, 130, shot.context)
    # Graph replay: 2 kernels per step, one batch end per 64-step graph, one configuration.
    assert gpu.kernelLaunches - before == 130 * 2 + 3 + 1


@pytest.mark.parametrize("scheme,up,src_type", [(3, True, capi2d.EXPLOSIVE), (1, False, capi2d.ROTATED_FORCE),
                                                (2, False, capi2d.SHEAR), (3, False, capi2d.VERTICAL_FORCE)])
def test_persistent_run_equals_graph_replay(scheme, up, src_type, solver2d_lib, cuda_device):
    # The cooperative persistent kernel and the per-step kernels compute the same bits, for
    # runs split at arbitrary points, with the gather recorded by both.
    shot = models2d.small_shot2d(scheme, up, steps=150, src_type=src_type)
    c = shot.context
    runs = []
    for mode in (capi2d.RUN_PERSISTENT, capi2d.RUN_GRAPH):
        gpu = seis2d.GPUSimData()
        seis2d.initializeGpuSimulation(gpu, c)
        seis2d.setRunMode(gpu, mode)
        seis2d.gatherBegin(gpu, 0, 1, shot.steps)
        done = 0
        for count in (1, 70, 3, 76):
            seis2d.runGpuSimulationSteps(gpu, done, count, c)
            done += count
        vx, vz, taken = seis2d.gatherFetch(gpu, shot.steps)
        assert taken == shot.steps
        runs.append((vx, vz, [seis2d.copyField(gpu, n) for n in capi2d.FIELDS[:10]]))
    (ax, az, af), (bx, bz, bf) = runs
    assert np.abs(az).max() > 0
    assert np.array_equal(ax, bx) and np.array_equal(az, bz)
    for name, a, b in zip(capi2d.FIELDS[:10], af, bf):
        assert np.array_equal(a, b), name
