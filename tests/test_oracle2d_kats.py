"""Known-answer checks of the CPU oracle of the 2-D solver, from the reference's own solver
regression (tests/SolverRegression.cpp) and its published PML figure
(docs/reviews/NUMERICAL_STABILITY_REVIEW.md:50: late-window error ratio 0.0433824 for Type 1,
0.0433818 for Type 2).  These pin the oracle before it judges the CUDA solver."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi2d, models2d
from seis2d_cases import add_pml, late_error_ratio, make_context

SZZ_1 = capi2d.FIELD["szz_1"]
SIGMAZZ = capi2d.FIELD["sigmazz"]


@pytest.mark.parametrize("scheme,density,free", [(1, 1000.0, False), (2, 1000.0, False), (2, 100.0, False),
                                                 (2, 0.5, False), (3, 1000.0, True)])
@pytest.mark.parametrize("precision", [32, 64])
def test_cubic_stress_gradient(scheme, density, free, precision):
    # SolverRegression.cpp:86-111: szz = z^3 gives vz = dt 3 (z + 1/2)^2 / rho after one step.
    ctx = make_context(scheme, free, 96, density)
    o = oracle.CpuOracle2D(ctx, precision)
    z = np.arange(ctx.NZ, dtype=np.float32)
    o.set_field(SIGMAZZ if scheme == 2 else SZZ_1, np.repeat((z * z * z)[:, None], ctx.NX, axis=1))
    o.run(0, 1, num_active=0)
    vz = o.wavefield().reshape(ctx.NZ, ctx.NX)
    expected = np.float32(ctx.dt) * 3.0 * 30.5 * 30.5 / density
    assert abs(vz[30, 48] - expected) < expected * 2e-5
    if free:
        szz = o.field(SZZ_1)
        assert np.all(szz[ctx.npml, 4:-4] == 0.0)
        for layer in range(1, 5):
            assert np.array_equal(szz[ctx.npml - layer, 4:-4], -szz[ctx.npml + layer, 4:-4])


def test_disabled_free_surface_equals_split_pml():
    # SolverRegression.cpp:114-126: Type 3 with upFlag off is bit-equal to Type 1.
    first, third = make_context(1), make_context(3, False)
    for c in (first, third):
        c.src_z_idx = 12
        c.src_idx = 12 * c.NX + 48
    a, b = oracle.CpuOracle2D(first, 32), oracle.CpuOracle2D(third, 32)
    a.run(0, 120)
    b.run(0, 120)
    assert np.abs(a.wavefield()).max() > 0
    assert np.array_equal(a.wavefield(), b.wavefield())


def test_overlapping_sources_sum():
    # SolverRegression.cpp:129-139: 200 horizontal forces on one cell add exactly.
    ctx = make_context(1)
    ctx.src_type = capi2d.HORIZONTAL_FORCE
    o = oracle.CpuOracle2D(ctx, 32)
    o.set_sources([(ctx.src_idx, 0.005, 200.0, 1.0)] * 200)
    o.run(0, 1, num_active=200)
    vx = o.field(capi2d.FIELD["vx_1"]).reshape(-1)
    expected = 200 * 1e7 * np.float32(ctx.dt) / ctx.rho[ctx.src_idx]
    assert abs(vx[ctx.src_idx] - expected) < expected * 1e-5


def trace(ctx, precision=32):
    o = oracle.CpuOracle2D(ctx, precision)
    vx, vz = o.run(0, ctx.nt, receivers=ctx.rcv_grid_idx)
    assert np.all(np.isfinite(vz)) and np.all(np.isfinite(vx))
    assert np.all(np.isfinite(o.wavefield()))
    return vz[0]


@pytest.mark.parametrize("scheme,published", [(1, 0.0433824), (2, 0.0433818)])
def test_pml_late_window_ratio(scheme, published):
    # SolverRegression.cpp:181-205: PML trace vs a 288^2 reference domain, relative to a
    # reflecting wall; the reference requires < 0.5 and publishes 0.0434 for its GPU build.
    absorbing = add_pml(make_context(scheme))
    ratio, wall = late_error_ratio(trace(absorbing), trace(make_context(scheme)), trace(make_context(scheme, False, 288)))
    assert wall > 0 and np.isfinite(ratio) and ratio < 0.5
    assert ratio == pytest.approx(published, rel=1e-4)


def test_free_surface_run_is_finite():
    trace(make_context(3, True))


@pytest.mark.parametrize("scheme,up", [(1, False), (2, False), (3, True), (3, False)])
def test_fp32_oracle_tracks_fp64(scheme, up):
    shot = models2d.small_shot2d(scheme, up, steps=300)
    c = shot.context
    r32 = oracle.CpuOracle2D(c, 32).run(0, shot.steps, receivers=c.rcv_grid_idx)
    r64 = oracle.CpuOracle2D(c, 64).run(0, shot.steps, receivers=c.rcv_grid_idx)
    for a, b in zip(r32, r64):
        assert np.abs(b).max() > 0
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 2e-5
