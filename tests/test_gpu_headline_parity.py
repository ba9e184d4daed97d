"""Parity on the two measured 3-D workloads at full size and full length, against the
reference's own CUDA solver (cuda/Cuda_Seis3D.cu built unmodified into oracle/_ref).

* 300 x 50 x 300 reference default: 5 flat layers, free surface + 5-face CPML 20, explosion
  at (150, 25, 10), dt 0.5 ms, 2000 steps, every 2nd step recorded on 150 receivers.
* 300 x 300 x 400 size cap: vp gradient + smoothed noise, 6-face CPML 20, explosion at
  (150, 150, 100), dt 0.6 ms, 2500 steps, every step recorded on 300 receivers.

Both run with the launch shape the bench uses (z chunk tuned at initialisation).  The bar
of the FP32 path: source and receiver indexing bit-exact, the receiver gather within 1e-5
relative L2 of the reference solver.  The final wavefields of runs this long sit at the
floor of FP32 arithmetic: two FP32 implementations of the scheme that round differently
(the reference's compiler contracts multiply-adds as it likes) drift apart in the late,
weak coda by more than 1e-5.  Each FP32 solver is therefore measured against the FP64 run
of the same scheme on the GPU (oracle.GpuOracle64, pinned to the CPU FP64 oracle in
test_gpu_oracle64.py), and this solver must be as close to it as the reference is: its
gather and each field within 1.25 x the reference's distance to FP64.  The CPU oracle
cannot run these lengths in test time; its parity is pinned on the small cases of
test_gpu_parity.py.

The same run in the 16-bit storage mode (SEIS3D_STORAGE_BF16_CPML: CPML memories in BF16)
is measured against the same FP64 run: its gather must stay within 1e-3 relative L2.
"""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5        # relative L2, FP32 gather vs the reference CUDA solver
FP64_RATIO = 1.25       # this solver's distance to FP64 over the reference's, gather and fields
STORAGE_BAR = 1e-3      # relative L2 to FP64, gather of the BF16-CPML-memory storage mode

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
    s = seis3d.Session(c, storage=capi.STORAGE_BF16_CPML, tune=True)
    s.upload_model(shot.vp, shot.vs, shot.rho)
    s.set_receivers(shot.receivers)
    s.gather_begin(shot.stride, shot.samples)
    s.run_steps(shot.source, 0, shot.steps)
    bf16 = {"gather": s.gather_fetch()}
    for k in range(9):
        bf16[capi.FIELDS[k]] = s.field(k)
    s.release()

    g = oracle.GpuOracle64(c)
    g.upload_model(shot.vp, shot.vs, shot.rho)
    g.set_receivers(shot.receivers)
    exact_gather = g.run_gather(shot.source, 0, shot.steps, shot.stride)
    exact = {"gather": exact_gather}
    ours = {"gather": gather}
    for k in range(9):
        exact[capi.FIELDS[k]] = g.field(k)
        ours[capi.FIELDS[k]] = fields[k]
    g.close()
    del fields

    r = oracle.ReferenceSolver(c)
    r.upload_model(shot.vp, shot.vs, shot.rho)
    r.set_receivers(shot.receivers)
    ref = {"gather": r.run_gather(shot.source, 0, shot.steps, shot.stride)}
    for k in range(9):
        ref[capi.FIELDS[k]] = r.field(k)
    r.close()
    assert gather.shape == ref["gather"].shape == exact_gather.shape == (shot.samples, len(shot.receivers), 3)
    assert np.all(np.isfinite(gather)) and np.abs(gather).max() > 0
    vs_ref = {k: rel_l2(ours[k], ref[k]) for k in ours}
    ours64 = {k: rel_l2(ours[k], exact[k]) for k in ours}
    ref64 = {k: rel_l2(ref[k], exact[k]) for k in ours}
    bf64 = {k: rel_l2(bf16[k], exact[k]) for k in ours}
    print(f"\n{shot.name}: {shot.steps} steps, z chunk {chunk}")
    for k in ours:
        print(f"  {k:6s} vs reference {vs_ref[k]:.2e}   vs FP64: this solver {ours64[k]:.2e}, reference {ref64[k]:.2e}, "
              f"BF16 CPML memories {bf64[k]:.2e}")
    assert vs_ref["gather"] < TRACE_TOL, vs_ref
    for k in ours:
        assert ours64[k] <= FP64_RATIO * ref64[k], (k, ours64[k], ref64[k])
    assert bf64["gather"] < STORAGE_BAR, bf64
