"""Model files through a solver session on the GPU: importModel3D / exportModel3D
(src/Seis3D/ModelIo3D.cpp:68-102) against the plane-upload path."""
import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import files3d, seis3d
from test_files3d import small_model

pytestmark = pytest.mark.gpu


def test_import_equals_upload_and_export_round_trips(tmp_path, solver_lib, cuda_device):
    c, vp, vs, rho = small_model()
    path = tmp_path / "m.s3dm"
    files3d.write_model(path, c, vp, vs, rho)
    ctx = files3d.inspect_model(path, c)
    a = seis3d.Session(ctx)
    files3d.import_model(a, path)
    b = seis3d.Session(ctx)
    b.upload_model(vp, vs, rho)
    for k in (9, 10, 11):
        assert np.array_equal(a.field(k), b.field(k))
    out = tmp_path / "exported.s3dm"
    files3d.export_model(a, out)
    back = files3d.inspect_model(out, c)
    evp, evs, erho = files3d.read_model(out, back)
    for got, want in ((evp, vp), (evs, vs), (erho, rho)):
        np.testing.assert_allclose(got, want, rtol=2e-6)
    a.release()
    b.release()
