"""The bench's reference arm builds its workload with the reference's own host code only.

The reference arm times cuda/Cuda_Seis3D.cu built unmodified (oracle/_ref/libref3d.so).  Its
context, padding and dt must come from the reference's validateContext3D
(cuda/Cuda_Seis3D.cu:433-483) and its defaults from include/Common3D.h:24-49, so the process
never maps this project's solver library.  These checks need no GPU: validation and defaults
are host code of the reference library.
"""
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(oracle.reference_library() is None, reason="oracle/_ref/libref3d.so not built")


def test_reference_api_matches_solver_contexts(solver_lib):
    from cmakepro_cuda_seissim_v2_b200 import models3d, seis3d

    api = oracle.ReferenceApi()
    ref = models3d.reference_default_shot(steps=4, api=api)
    ours = models3d.reference_default_shot(steps=4)
    assert ref.context.as_dict() == ours.context.as_dict()
    for name in ("x3D", "y3D", "z3D", "kind3D", "amplitude3D"):
        assert getattr(ref.source, name) == getattr(ours.source, name)
    assert api.default_context().as_dict() == seis3d.default_context().as_dict()
    a, b = api.default_source(), seis3d.default_source()
    assert (a.x3D, a.y3D, a.z3D, a.kind3D, a.amplitude3D, list(a.direction3D)) == \
        (b.x3D, b.y3D, b.z3D, b.kind3D, b.amplitude3D, list(b.direction3D))
    with pytest.raises(ValueError, match="at least 16"):
        api.validate_context3D(api.default_context(nx3D=8))


def test_reference_workload_maps_no_solver_library():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import oracle\n"
        "from cmakepro_cuda_seissim_v2_b200 import models3d\n"
        "shot = models3d.reference_default_shot(steps=4, api=oracle.ReferenceApi())\n"
        "assert shot.context.gx3D == 348 and shot.context.dt3D > 0\n"
        "print('\\n'.join(oracle.loaded_libraries()))\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, text=True).stdout
    mapped = [os.path.basename(p) for p in out.split()]
    assert "libref3d.so" in mapped
    assert not any(name.startswith("libseis") for name in mapped), mapped
