"""The FP64 restatement of the scheme on the GPU (oracle/seis3d_oracle_gpu.cu) against the CPU
FP64 oracle, which the golden vectors pin: the same answer to FP64 rounding on small shots
with a free surface and explosion, and with six CPML faces and a force source."""
import numpy as np
import pytest

import oracle
from cmakepro_cuda_seissim_v2_b200 import capi, models3d

pytestmark = pytest.mark.gpu

TOL = 1e-11   # relative L2, FP64 vs FP64 (different operation order only)

CASES = {
    "free_surface_explosion": dict(free_surface=True, kind=capi.SOURCE_EXPLOSION),
    "six_face_force": dict(free_surface=False, kind=capi.SOURCE_FORCE),
}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("case", sorted(CASES))
def test_gpu_fp64_matches_cpu_fp64(case, cuda_device):
    shot = models3d.small_shot(steps=60, **CASES[case])
    g = oracle.GpuOracle64(shot.context)
    g.upload_model(shot.vp, shot.vs, shot.rho)
    g.set_receivers(shot.receivers)
    gather = g.run_gather(shot.source, 0, shot.steps, 1)
    fields = [g.field(k) for k in range(9)]
    g.close()
    o = oracle.CpuOracle(shot.context, 64)
    o.upload_model(shot.vp, shot.vs, shot.rho)
    expect = o.run_gather(shot.source, 0, shot.steps, shot.receivers, 1)
    assert np.abs(expect).max() > 0
    assert rel_l2(gather, expect) < TOL
    for k in range(9):
        assert rel_l2(fields[k], o.field(k)) < TOL, capi.FIELDS[k]
    o.close()
