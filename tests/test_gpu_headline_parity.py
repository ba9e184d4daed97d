"""Parity on the two measured 3-D workloads at full size and full length, against the
reference's own CUDA solver (cuda/Cuda_Seis3D.cu built unmodified into oracle/_ref).

* 300 x 50 x 300 reference default: 5 flat layers, free surface + 5-face CPML 20, explosion
  at (150, 25, 10), dt 0.5 ms, 2000 steps, every 2nd step recorded on 150 receivers.
* 300 x 300 x 400 size cap: vp gradient + smoothed noise, 6-face CPML 20, explosion at
  (150, 150, 100), dt 0.6 ms, 2500 steps, every step recorded on 300 receivers.

Both run with the launch shape the bench uses (z chunk tuned at initialisation).  The bar
of the FP32 path: source and receiver indexing bit-exact, the receiver gather and each of
the nine final wavefields within 1e-5 relative L2 of the reference solver.  The CPU oracle
cannot run these lengths in test time; its parity is pinned on the small cases of
test_gpu_parity.py.
"""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5        # relative L2, FP32 gather vs the reference CUDA solver
FIELD_TOL = 1e-5        # relative L2, FP32 wavefields vs the reference CUDA solver

WORKLOADS = {
    "reference_default": models3d.reference_default_shot,
    "size_cap": models3d.size_cap_shot,
}


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    denom = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (denom if denom > 0 else 1.0))


@pytest.fixture(scope="module", params=sorted(WORKLOADS))
def shot(request, cuda_device):
    if oracle.reference_library() is None:
        pytest.skip("reference solver library oracle/_ref/libref3d.so not built")
    return WORKLOADS[request.param]()


def test_headline_indexing_bit_exact(shot):
    """Receiver collocation and source footprint on the workload's own geometry."""
    c = shot.context
    coded = (np.arange(c.cells3D, dtype=np.int64) % 65521).astype(np.float32).reshape(c.gz3D, c.gy3D, c.gx3D)
    s = seis3d.Session(c)
    r = oracle.ReferenceSolver(c)
    try:
        s.upload_model(shot.vp, shot.vs, shot.rho)
        r.upload_model(shot.vp, shot.vs, shot.rho)
        for k in range(3):
            s.set_field(k, coded * np.float32(k + 1))
            r.set_field(k, coded * np.float32(k + 1))
        s.set_receivers(shot.receivers)
        r.set_receivers(shot.receivers)
        ours = s.sample_receivers()
        ref = r.sample()
        assert ours.shape == ref.shape == (len(shot.receivers), 3)
        assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))
        # One step from rest: the explosion touches the same 27 nodes in both solvers.
        for k in range(3):
            s.set_field(k, np.zeros_like(coded))
            r.set_field(k, np.zeros_like(coded))
        s.reset()
        r.reset()
        s.run_step(shot.source, 0)
        r.run(shot.source, 0, 1)
        mine = set(zip(*np.nonzero(s.field(3))))
        theirs = set(zip(*np.nonzero(r.field(3))))
        gx, gy, gz = shot.source.x3D + c.ox3D, shot.source.y3D + c.oy3D, shot.source.z3D + c.oz3D
        want = {(gz + dz, gy + dy, gx + dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)}
        assert mine == theirs == want
    finally:
        s.release()
        r.close()


def test_headline_full_run_matches_reference(shot):
    c = shot.context
    s = seis3d.Session(c, tune=True)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.gather_begin(shot.stride, shot.samples)
    s.run_steps(shot.source, 0, shot.steps)
    gather = s.gather_fetch()
    fields = [s.field(k) for k in range(9)]
    chunk = s.z_chunk()[1]
    s.release()

    r = oracle.ReferenceSolver(c)
    r.upload_model(shot.vp, shot.vs, shot.rho)
    r.set_receivers(shot.receivers)
    ref_gather = r.run_gather(shot.source, 0, shot.steps, shot.stride)
    assert gather.shape == ref_gather.shape == (shot.samples, len(shot.receivers), 3)
    assert np.all(np.isfinite(gather)) and np.abs(gather).max() > 0
    errors = {"gather": rel_l2(gather, ref_gather)}
    for k in range(9):
        errors[capi.FIELDS[k]] = rel_l2(fields[k], r.field(k))
    r.close()
    print(f"\n{shot.name}: {shot.steps} steps, z chunk {chunk}, rel-L2 vs reference CUDA solver: " +
          ", ".join(f"{k} {v:.2e}" for k, v in errors.items()))
    assert errors["gather"] < TRACE_TOL, errors
    for k in range(9):
        assert errors[capi.FIELDS[k]] < FIELD_TOL, errors
