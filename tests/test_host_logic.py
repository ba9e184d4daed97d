"""Host-side logic that needs no GPU: defaults, validation error classes, acquisition
geometry and the synthetic model builders."""
import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d


def test_reference_defaults(solver_lib):
    c = seis3d.default_context()
    assert (c.nx3D, c.ny3D, c.nz3D, c.pml3D, c.freeSurface3D) == (300, 50, 300, 12, 1)
    assert c.spacing3D == 10.0 and c.cfl3D == pytest.approx(0.85) and c.frequency3D == 20.0
    s = seis3d.default_source()
    assert (s.x3D, s.y3D, s.z3D, s.kind3D, s.amplitude3D) == (48, 48, 24, 0, 1.0e8)
    assert list(s.direction3D) == [0.0, 0.0, 1.0]


def test_invalid_argument_is_value_error(solver_lib):
    with pytest.raises(seis3d.InvalidArgument, match="at least 16"):
        seis3d.validate_context3D(seis3d.default_context(nx3D=8))
    with pytest.raises(ValueError):
        seis3d.estimate_memory3D(seis3d.default_context(pml3D=4))


def test_storage_modes_checked_before_device_work(solver_lib):
    """16-bit wavefield storage is rejected with its reason, unknown modes too; both checks
    run before any device call (no GPU here)."""
    small = seis3d.default_context(nx3D=40, ny3D=32, nz3D=36, pml3D=8)
    for mode in (capi.STORAGE_FP16, capi.STORAGE_BF16):
        with pytest.raises(seis3d.InvalidArgument, match="SEIS3D_STORAGE_BF16_CPML"):
            seis3d.Session(small, storage=mode)
    with pytest.raises(seis3d.InvalidArgument, match="unknown storage"):
        seis3d.Session(small, storage=7)


def test_manual_dt_rules(solver_lib):
    c = seis3d.validate_context3D(seis3d.default_context(manualTimeStep3D=1, requestedDtMs3D=0.5))
    assert c.dt3D == np.float32(0.0005) and c.safeDt3D > c.dt3D
    with pytest.raises(seis3d.InvalidArgument, match="whole microseconds"):
        seis3d.validate_context3D(seis3d.default_context(manualTimeStep3D=1, requestedDtMs3D=0.5004))
    with pytest.raises(seis3d.InvalidArgument, match="CFL"):
        seis3d.validate_context3D(seis3d.default_context(manualTimeStep3D=1, requestedDtMs3D=50.0))


def test_reflecting_disables_free_surface(solver_lib):
    c = seis3d.validate_context3D(seis3d.default_context(reflecting3D=1))
    assert c.freeSurface3D == 0 and c.ox3D == 4 and c.gx3D == c.nx3D + 8


def test_default_receiver_spread():
    # Seis3DWorkspaceRegression.cpp:437-462: 150 surface channels in three 50-channel rows.
    r = models3d.fit_receivers(300, 50, 50, 3)
    assert r.shape == (150, 3) and np.all(r[:, 2] == 0)
    assert list(r[:50, 0]) == [2 + 6 * i for i in range(50)]
    assert sorted(set(r[:, 1])) == [1, 24, 47]
    r = models3d.fit_receivers(300, 300, 20, 15)
    assert r.shape == (300, 3)
    assert sorted(set(r[:, 0])) == [7 + 15 * i for i in range(20)]
    assert sorted(set(r[:, 1])) == [2 + 21 * j for j in range(15)]


def test_splitmix_is_deterministic():
    a = models3d.splitmix64_uniform(1000, 5)
    assert np.array_equal(a, models3d.splitmix64_uniform(1000, 5))
    assert a.min() >= -1 and a.max() < 1 and abs(a.mean()) < 0.1
    assert not np.array_equal(a, models3d.splitmix64_uniform(1000, 6))


def test_reference_default_shot_model(solver_lib):
    shot = models3d.reference_default_shot(steps=10)
    c = shot.context
    assert (c.gx3D, c.gy3D, c.gz3D) == (348, 98, 328)
    assert shot.active_cells == 340 * 90 * 320
    assert c.dt3D == np.float32(0.0005)
    assert sorted(np.unique(shot.vp)) == [1800, 2400, 3000, 3700, 4500]
    assert np.allclose(shot.rho, 310 * shot.vp.astype(np.float64) ** 0.25, rtol=1e-6)
    assert shot.receivers.shape == (150, 3)


def test_workspace_grid_presets_fit_the_budget(solver_lib):
    # Seis3DWorkspaceRegression.cpp:441-446: the 500x20x500 and 200x200x200 presets validate
    # and stay inside the 4 GiB session budget.
    for dims in ((500, 20, 500), (200, 200, 200)):
        c = seis3d.validate_context3D(seis3d.default_context(nx3D=dims[0], ny3D=dims[1], nz3D=dims[2]))
        assert seis3d.estimate_memory3D(c).totalBytes3D <= capi.MEMORY_LIMIT


def test_window_contexts_with_a_thin_cpml(solver_lib):
    """Survey windows with a CPML under 8 cells get the learned-boundary mode's validation (the
    reference's validator keeps 8..40 cells); the 20-cell windows are unchanged."""
    import dataclasses

    nx, ny, nz = 40, 30, 36
    vp = models3d.layered_model(nx, ny, nz, [2000, 2600])
    vp, vs, rho = models3d.elastic_from_vp(vp)
    shot = models3d.WindowShot(0, (2, 3, 0), (30, 24, 28), (15, 12, 10))
    survey = models3d.WindowSurvey("tiny", vp, vs, rho, [shot], 10.0, 20, 15.0, 0.5, 100)
    wide = survey.context(shot)
    assert (wide.pml3D, wide.gx3D, wide.gz3D) == (20, 30 + 40 + 8, 28 + 20 + 8)
    thin = dataclasses.replace(survey, pml=6).context(shot)
    assert (thin.pml3D, thin.gx3D, thin.gy3D, thin.gz3D) == (6, 30 + 12 + 8, 24 + 12 + 8, 28 + 6 + 8)
    assert thin.dt3D == wide.dt3D
    with pytest.raises(seis3d.InvalidArgument):
        seis3d.validate_context3D(thin.copy())         # the reference's rule still applies
