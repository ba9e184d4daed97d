"""The windowed-survey workload (600 x 200 x 600 smooth layered model, 64 shots on cropped
windows): deterministic, every window inside the model, every source and receiver inside its
window, and the materials of a window are the model's cells."""
import numpy as np

from cmakepro_cuda_seissim_v2_b200 import models3d


def test_window_survey_geometry():
    a = models3d.window_survey(shots=16, nx=240, ny=120, nz=200)
    b = models3d.window_survey(shots=16, nx=240, ny=120, nz=200)
    assert [q.origin for q in a.shots] == [q.origin for q in b.shots]
    assert np.array_equal(a.vp, b.vp)
    assert a.vp.min() == np.float32(1800) and a.vp.max() == np.float32(4500)
    for q in a.shots:
        assert all(0 <= o and o + w <= n for o, w, n in zip(q.origin, q.size, (240, 120, 200)))
        assert all(1 <= c < w - 1 for c, w in zip(q.source, q.size))
        assert q.source[2] == 10 and q.origin[2] == 0
        assert all(160 <= w or w == n for w, n in zip(q.size, (240, 120, 200)))
        rec = a.receivers(q)
        assert len(rec) == 150 and rec[:, 0].max() < q.size[0] and rec[:, 1].max() < q.size[1]
        vp, vs, rho = a.window(q)
        assert vp.shape == (q.size[2], q.size[1], q.size[0]) and vp.flags.c_contiguous
        x0, y0, z0 = q.origin
        assert vp[3, 4, 5] == a.vp[z0 + 3, y0 + 4, x0 + 5]
        c = a.context(q)
        assert (c.nx3D, c.ny3D, c.nz3D) == q.size and c.freeSurface3D == 1 and c.pml3D == 20
        assert abs(c.dt3D - 5e-4) < 1e-9 and c.maxVp3D == float(vp.max())
