"""Whole-model upload (seis3d_upload_model) against the reference's per-plane path
(uploadModelPlane3D + finishModelUpload3D, cuda/Cuda_Seis3D.cu:696-717)."""
import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import models3d, seis3d

pytestmark = pytest.mark.gpu


def test_bulk_upload_equals_plane_upload(solver_lib, cuda_device):
    shot = models3d.small_shot(nx=40, ny=32, nz=36)
    a = seis3d.Session(shot.context)
    a.upload_model(shot.vp, shot.vs, shot.rho)
    b = seis3d.Session(shot.context)
    b.upload_volumes(shot.vp, shot.vs, shot.rho)
    for k in (9, 10, 11):
        assert np.array_equal(a.field(k), b.field(k)), k
    # A bad cell anywhere is rejected before any device write.
    bad = shot.vs.copy()
    bad[20, 5, 7] = shot.vp[20, 5, 7] * 1.01
    before = [b.field(k) for k in (9, 10, 11)]
    with pytest.raises(seis3d.InvalidArgument):
        b.upload_volumes(shot.vp, bad, shot.rho)
    for k, old in zip((9, 10, 11), before):
        assert np.array_equal(b.field(k), old)
    a.release()
    b.release()


def test_bulk_upload_of_many_chunks(solver_lib, cuda_device):
    """A model of several pinned chunks (69 planes of 200 x 200 cells each): bit-equal to the
    per-plane path, and a bad cell in the last chunk still leaves the session untouched."""
    nx, ny, nz = 200, 200, 220
    vp = models3d.layered_model(nx, ny, nz, [2000.0, 2700.0, 3400.0, 4100.0])
    vp = vp * (1.0 + 0.03 * models3d.splitmix64_uniform(nx * ny * nz, 5).reshape(nz, ny, nx))
    vp, vs, rho = models3d.elastic_from_vp(vp)
    c = models3d.imported_context(nx, ny, nz, 10.0, 8, True, float(vp.max()), 15.0)
    a = seis3d.Session(c)
    a.upload_model(vp, vs, rho)
    b = seis3d.Session(c)
    b.upload_volumes(vp, vs, rho)
    for k in (9, 10, 11):
        assert np.array_equal(a.field(k), b.field(k)), k
    before = [b.field(k) for k in (9, 10, 11)]
    bad = rho.copy()
    bad[nz - 3, 150, 20] = np.nan
    with pytest.raises(seis3d.InvalidArgument):
        b.upload_volumes(vp, vs, bad)
    for k, old in zip((9, 10, 11), before):
        assert np.array_equal(b.field(k), old)
    # The session still uploads and runs after the rejection.
    b.upload_volumes(vp, vs, rho)
    assert np.array_equal(b.field(10), before[1])
    a.release()
    b.release()
