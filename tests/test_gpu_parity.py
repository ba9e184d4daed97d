"""Parity of the B200 solver with the CPU oracle (FP32 and FP64 restatements of the
reference scheme) and with the reference's own CUDA solver built from its source
(oracle/_ref).  Bar (north star): source/receiver indexing bit-exact, FP32 receiver traces
and wavefields within 1e-5 relative L2 of the reference implementation."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5        # relative L2, FP32 traces vs the reference implementation
FIELD_TOL = 1e-5        # relative L2, FP32 wavefields vs the reference implementation
FP64_TOL = 1e-4         # relative L2, FP32 solver vs the FP64 run of the same scheme (short runs)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    denom = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (denom if denom > 0 else 1.0)


def run_product(shot, steps=None, stride=1, graph=False, tile_y=0, z_chunk=0):
    steps = shot.steps if steps is None else steps
    s = seis3d.Session(shot.context, tile_y=tile_y, z_chunk=z_chunk)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    if graph:
        s.gather_begin(stride, steps // stride)
        s.run_steps(shot.source, 0, steps)
        gather = s.gather_fetch()
    else:
        samples = []
        for n in range(steps):
            s.run_step(shot.source, n)
            if (n + 1) % stride == 0:
                samples.append(s.sample_receivers())
        gather = np.array(samples, dtype=np.float32)
    fields = [s.field(k) for k in range(9)]
    s.release()
    return gather, fields


def run_oracle(shot, precision, steps=None, stride=1):
    steps = shot.steps if steps is None else steps
    o = oracle.CpuOracle(shot.context, precision)
    o.upload_model(shot.vp, shot.vs, shot.rho)
    gather = o.run_gather(shot.source, 0, steps, shot.receivers, stride)
    fields = [o.field(k) for k in range(9)]
    o.close()
    return gather, fields


def run_reference(shot, steps=None, stride=1):
    steps = shot.steps if steps is None else steps
    r = oracle.ReferenceSolver(shot.context)
    r.upload_model(shot.vp, shot.vs, shot.rho)
    r.set_receivers(shot.receivers)
    gather = r.run_gather(shot.source, 0, steps, stride)
    fields = [r.field(k) for k in range(9)]
    r.close()
    return gather, fields


def needs_reference():
    if oracle.reference_library() is None:
        pytest.skip("reference solver library oracle/_ref/libref3d.so not built")


CASES = {
    "free_surface_explosion": dict(free_surface=True, kind=capi.SOURCE_EXPLOSION),
    "six_face_explosion": dict(free_surface=False, kind=capi.SOURCE_EXPLOSION),
    "free_surface_force": dict(free_surface=True, kind=capi.SOURCE_FORCE),
    "six_face_force_pml12": dict(free_surface=False, kind=capi.SOURCE_FORCE, pml=12),
    "shallow_source": dict(free_surface=True, kind=capi.SOURCE_EXPLOSION, source=(20, 16, 2)),
    "ragged_tiles": dict(nx=45, ny=37, nz=33, free_surface=True, kind=capi.SOURCE_EXPLOSION),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_matches_cpu_oracle(case, cuda_device):
    shot = models3d.small_shot(steps=80, **CASES[case])
    g, f = run_product(shot)
    g32, f32 = run_oracle(shot, 32)
    g64, f64 = run_oracle(shot, 64)
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    assert rel_l2(g, g32) < TRACE_TOL
    assert rel_l2(g, g64) < FP64_TOL
    for k in range(9):
        assert rel_l2(f[k], f32[k]) < FIELD_TOL, (case, capi.FIELDS[k], rel_l2(f[k], f32[k]))
        assert rel_l2(f[k], f64[k]) < FP64_TOL, (case, capi.FIELDS[k])


def tile_census(c, planes):
    """(CTAs of the passes, CTAs whose 32 x 16 tile and z chunk touch no CPML slab), by the
    kernels' own rule: the passes run the second kind on the bodies compiled without the
    CPML code and the others on the full bodies."""
    def in_slab(v, n, top_free):
        return (not top_free and v < 4 + c.pml3D) or v >= n - 4 - c.pml3D
    total = interior = 0
    for z0 in range(4, c.gz3D - 4, planes):
        z1 = min(z0 + planes, c.gz3D - 4) - 1
        for y0 in range(4, c.gy3D - 4, 16):
            for x0 in range(4, c.gx3D - 4, 32):
                total += 1
                touches = (in_slab(x0, c.gx3D, False) or in_slab(x0 + 31, c.gx3D, False)
                           or in_slab(y0, c.gy3D, False) or in_slab(y0 + 15, c.gy3D, False)
                           or in_slab(z0, c.gz3D, c.freeSurface3D) or in_slab(z1, c.gz3D, c.freeSurface3D))
                interior += not touches
    return total, interior


INTERIOR_CASES = {
    "free_surface_explosion": dict(nx=100, ny=56, nz=60, free_surface=True, kind=capi.SOURCE_EXPLOSION),
    "six_face_force": dict(nx=100, ny=56, nz=60, free_surface=False, kind=capi.SOURCE_FORCE),
}


@pytest.mark.parametrize("case", sorted(INTERIOR_CASES))
def test_interior_and_slab_tiles_match(case, cuda_device):
    """A grid wide enough for CTAs of both kinds (the small cases above have slab CTAs only):
    traces and wavefields against the FP32 and FP64 oracle and the reference CUDA solver."""
    shot = models3d.small_shot(steps=80, **INTERIOR_CASES[case])
    s = seis3d.Session(shot.context, z_chunk=16)      # fixed, so that both kinds stay present
    planes = s.z_chunk()[1]
    s.release()
    total, interior = tile_census(shot.context, planes)
    assert 0 < interior < total, (total, interior)
    g, f = run_product(shot, z_chunk=16)
    g32, f32 = run_oracle(shot, 32)
    g64, f64 = run_oracle(shot, 64)
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    assert rel_l2(g, g32) < TRACE_TOL
    assert rel_l2(g, g64) < FP64_TOL
    for k in range(9):
        assert rel_l2(f[k], f32[k]) < FIELD_TOL, (case, capi.FIELDS[k], rel_l2(f[k], f32[k]))
        assert rel_l2(f[k], f64[k]) < FP64_TOL, (case, capi.FIELDS[k])
    if oracle.reference_library() is not None:
        gr, fr = run_reference(shot)
        assert rel_l2(g, gr) < TRACE_TOL
        for k in range(9):
            assert rel_l2(f[k], fr[k]) < FIELD_TOL, (case, capi.FIELDS[k], rel_l2(f[k], fr[k]))
    # One chunk over the whole depth: every CTA then reaches a z slab and runs the full body,
    # which must give the interior cells the same bits as the body without the CPML code.
    assert tile_census(shot.context, 1000)[1] == 0
    g1, f1 = run_product(shot, z_chunk=1000)
    assert np.array_equal(g.view(np.uint32), g1.view(np.uint32))
    for k in range(9):
        assert np.array_equal(f[k].view(np.uint32), f1[k].view(np.uint32)), capi.FIELDS[k]


@pytest.mark.parametrize("case", sorted(CASES))
def test_matches_reference_cuda_solver(case, cuda_device):
    needs_reference()
    shot = models3d.small_shot(steps=80, **CASES[case])
    g, f = run_product(shot)
    gr, fr = run_reference(shot)
    assert g.shape == gr.shape
    assert rel_l2(g, gr) < TRACE_TOL
    for k in range(9):
        assert rel_l2(f[k], fr[k]) < FIELD_TOL, (case, capi.FIELDS[k], rel_l2(f[k], fr[k]))


def test_graph_and_device_gather_equal_step_loop(cuda_device):
    shot = models3d.small_shot(steps=150, free_surface=True)
    g_loop, f_loop = run_product(shot, stride=2)
    g_graph, f_graph = run_product(shot, stride=2, graph=True)
    assert g_graph.shape == g_loop.shape == (75, len(shot.receivers), 3)
    assert np.array_equal(g_graph.view(np.uint32), g_loop.view(np.uint32))
    for k in range(9):
        assert np.array_equal(f_graph[k].view(np.uint32), f_loop[k].view(np.uint32))


@pytest.mark.parametrize("free_surface", [False, True])
@pytest.mark.parametrize("tile_y,z_chunk", [(16, 5), (0, 1), (16, 2), (0, 7), (16, 1000)])
def test_launch_shape_does_not_change_results(tile_y, z_chunk, free_surface, cuda_device):
    # With a free surface the first z chunk of each pass writes the images of its columns,
    # whatever the chunk's depth (one plane included).
    shot = models3d.small_shot(steps=40, nx=50, ny=41, nz=38, free_surface=free_surface)
    g0, f0 = run_product(shot)
    g1, f1 = run_product(shot, tile_y=tile_y, z_chunk=z_chunk)
    assert np.array_equal(g0.view(np.uint32), g1.view(np.uint32))
    for k in range(9):
        assert np.array_equal(f0[k].view(np.uint32), f1[k].view(np.uint32))


def test_reflecting_walls_match_oracle(cuda_device):
    c = seis3d.validate_context3D(seis3d.default_context(nx3D=32, ny3D=28, nz3D=30, reflecting3D=1,
                                                         modelKind3D=capi.MODEL_UNIFORM, frequency3D=30.0))
    src = seis3d.default_source(x3D=16, y3D=14, z3D=15)
    rec = [(5, 5, 5), (16, 14, 20), (30, 26, 28), (0, 0, 0)]
    s = seis3d.Session(c)
    s.set_receivers(rec)
    o = oracle.CpuOracle(c, 32)
    o.generate()
    for n in range(60):
        s.run_step(src, n)
        o.step(src, n)
    assert rel_l2(s.sample_receivers(), o.sample(rec)) < TRACE_TOL
    for k in range(9):
        assert rel_l2(s.field(k), o.field(k)) < FIELD_TOL
    s.release()


@pytest.mark.parametrize("kind", [capi.MODEL_UNIFORM, capi.MODEL_TWO_LAYER, capi.MODEL_SPHERE, capi.MODEL_THREE_LAYER,
                                  capi.MODEL_DIPPING_LAYER, capi.MODEL_LOW_VELOCITY_LAYER, capi.MODEL_FAULT,
                                  capi.MODEL_GRADIENT, capi.MODEL_SALT_DOME])
def test_procedural_materials_match_reference(kind, cuda_device):
    needs_reference()
    c = seis3d.validate_context3D(seis3d.default_context(nx3D=40, ny3D=36, nz3D=44, pml3D=8, modelKind3D=kind))
    s = seis3d.Session(c)
    r = oracle.ReferenceSolver(c)
    for k in (9, 10, 11):
        mine, ref = s.field(k), r.field(k)
        # Same FP32 device expressions: equal to rounding (nvcc may contract differently).
        assert np.allclose(mine, ref, rtol=2e-7, atol=0), k
    s.release()
    r.close()


def test_receiver_and_source_indexing_bit_exact(cuda_device):
    shot = models3d.small_shot(steps=1, nx=37, ny=29, nz=31, free_surface=True)
    c = shot.context
    s = seis3d.Session(c)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    # Receiver collocation (cuda/Cuda_Seis3D.cu:341-343) on an index-coded field.
    coded = np.arange(c.cells3D, dtype=np.float64).reshape(c.gz3D, c.gy3D, c.gx3D).astype(np.float32)
    for k in range(3):
        s.set_field(k, coded * (k + 1))
    s.set_receivers(shot.receivers)
    got = s.sample_receivers()
    for r, (x, y, z) in enumerate(shot.receivers):
        gx, gy, gz = x + c.ox3D, y + c.oy3D, z + c.oz3D
        flat = coded.ravel()
        i = (gz * c.gy3D + gy) * c.gx3D + gx
        assert got[r, 0] == np.float32(0.5) * (flat[i] + flat[i - 1])
        assert got[r, 1] == np.float32(0.5) * np.float32(2 * flat[i] + 2 * flat[i - c.gx3D])
        assert got[r, 2] == np.float32(0.5) * np.float32(3 * flat[i] + 3 * flat[i - c.gx3D * c.gy3D])
    # Explosion source touches exactly the 27 nodes around (x+ox, y+oy, z+oz) (:316-318).
    s.reset()
    s.run_step(shot.source, 0)
    sxx = s.field(3)
    nz = set(zip(*np.nonzero(sxx)))
    sx, sy, sz = shot.source.x3D + c.ox3D, shot.source.y3D + c.oy3D, shot.source.z3D + c.oz3D
    want = {(sz + dz, sy + dy, sx + dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)}
    assert nz == want
    if oracle.reference_library() is not None:
        r = oracle.ReferenceSolver(c)
        r.upload_model(shot.vp, shot.vs, shot.rho)
        r.run(shot.source, 0, 1)
        assert set(zip(*np.nonzero(r.field(3)))) == want
        r.close()
    s.release()


def test_session_lifecycle_and_validation(cuda_device):
    shot = models3d.small_shot(steps=30)
    c = shot.context
    s = seis3d.Session(c)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    with pytest.raises(seis3d.InvalidArgument):
        s.set_receivers([(c.nx3D, 0, 0)])
    with pytest.raises(seis3d.InvalidArgument):
        s.set_receivers([(1, 1, 0)] * (capi.MAX_RECEIVERS + 1))
    s.set_receivers(shot.receivers)
    with pytest.raises(seis3d.InvalidArgument):
        s.set_receivers([(-1, 0, 0)])
    assert s.views().receiverCount3D == len(shot.receivers)   # failed update kept the old set
    for bad in (dict(x3D=0), dict(x3D=c.nx3D - 1), dict(z3D=1), dict(amplitude3D=float("nan")),
                dict(direction3D=(0, float("inf"), 1))):
        src = seis3d.default_source(**{**dict(x3D=5, y3D=5, z3D=5), **bad})
        with pytest.raises(seis3d.InvalidArgument):
            s.run_step(src, 0)
    with pytest.raises(seis3d.InvalidArgument):
        s.upload_model_plane(0, np.full((c.ny3D, c.nx3D, 3), [1000.0, 900.0, 2000.0], np.float32))  # vs^2 too high
    # Reset reproduces the first run bit-for-bit.
    for n in range(30):
        s.run_step(shot.source, n)
    first = [s.field(k) for k in range(9)]
    s.reset()
    for n in range(30):
        s.run_step(shot.source, n)
    for k in range(9):
        assert np.array_equal(first[k].view(np.uint32), s.field(k).view(np.uint32))
    # Model round trip: download returns the uploaded SI materials (to FP32 rounding).
    plane = s.download_model_plane(3)
    assert np.allclose(plane[..., 0], shot.vp[3], rtol=1e-5)
    assert np.allclose(plane[..., 2], shot.rho[3], rtol=1e-6)
    probe = s.probe_material((4, 5, 6))
    assert np.allclose(probe, [shot.vp[6, 5, 4], shot.vs[6, 5, 4], shot.rho[6, 5, 4]], rtol=1e-5)
    s.release()
    s.release()
    with pytest.raises(seis3d.LogicError):
        s.run_step(shot.source, 0)


def test_non_finite_wavefield_is_reported(cuda_device):
    # A NaN planted in the stress field (host data, no GPU fault) must stop the capture the
    # way the reference does (cuda/Cuda_Seis3D.cu:243, :676-679).
    shot = models3d.small_shot(steps=2)
    c = shot.context
    s = seis3d.Session(c)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    sxx = np.zeros((c.gz3D, c.gy3D, c.gx3D), np.float32)
    sxx[c.gz3D // 2, c.gy3D // 2, c.gx3D // 2] = np.nan
    s.set_field(3, sxx)
    s.run_step(shot.source, 0)
    assert s.non_finite()
    with pytest.raises(seis3d.SolverError, match="non-finite"):
        s.sample_receivers()
    s.reset()
    assert not s.non_finite()
    s.release()


def test_cpml_refresh_on_device(cuda_device):
    # refreshCpmlCoefficients3D semantics: a session refreshed to a new frequency steps
    # bit-identically to a fresh session built at that frequency
    # (Seis3DWorkspaceRegression.cpp:244-250).
    shot = models3d.small_shot(steps=20, free_surface=False)
    c = shot.context
    c40 = c.copy()
    c40.frequency3D = 40.0
    seis3d.validate_context3D(c40)
    refreshed = seis3d.Session(c)
    refreshed.refresh_cpml(c40)
    fresh = seis3d.Session(c40)
    for s in (refreshed, fresh):
        s.upload_model(shot.vp, shot.vs, shot.rho)
        for n in range(20):
            s.run_step(shot.source, n, context=c40)
    for k in range(9):
        assert np.array_equal(refreshed.field(k).view(np.uint32), fresh.field(k).view(np.uint32))
    stale = seis3d.Session(c)
    stale.upload_model(shot.vp, shot.vs, shot.rho)
    for n in range(20):
        stale.run_step(shot.source, n)
    assert not np.array_equal(stale.field(0), fresh.field(0))
    for s in (refreshed, fresh, stale):
        s.release()


def test_receiver_cap_and_capture_cadence(cuda_device):
    """Seis3DWorkspaceRegression.cpp:541-548 and :589-594 on the device API: 301 receivers are
    refused and the previous set stays; a 64-sample capture with stride 2 records exactly 64
    three-component samples per channel in 128 steps."""
    shot = models3d.small_shot(steps=128)
    s = seis3d.Session(shot.context)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    too_many = [(1, 1, 0)] * (capi.MAX_RECEIVERS + 1)
    with pytest.raises(seis3d.InvalidArgument):
        s.set_receivers(too_many)
    assert s.receiver_count == len(shot.receivers)
    s.gather_begin(2, 64)
    s.run_steps(shot.source, 0, 128)
    g = s.gather_fetch()
    assert g.shape == (64, len(shot.receivers), 3) and np.abs(g).max() > 0
    s.release()
