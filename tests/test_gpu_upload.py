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
