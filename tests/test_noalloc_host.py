"""Argument checks of seis3d_sample_receivers_noalloc that run before any device work, so
they need no GPU: a context whose offsets or sizes do not fit its padded grid would make the
collocation read below or beyond the caller's buffers, and is rejected."""
import ctypes
from ctypes import byref, c_float

import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d


def call(lib, context, receivers, pitch=None):
    dummy = (c_float * 4)()        # never dereferenced: every case fails validation first
    arr, n = seis3d.receivers_array(receivers)
    out = np.zeros((max(n, 1), 3), dtype=np.float32)
    pitch = context.gx3D if pitch is None else pitch
    return lib.seis3d_sample_receivers_noalloc(byref(context), dummy, dummy, dummy, pitch, arr, n,
                                               out.ctypes.data_as(ctypes.POINTER(c_float)), None)


@pytest.mark.parametrize("field,value", [("ox3D", 0), ("oy3D", 0), ("oz3D", 0), ("ox3D", -3), ("nx3D", 400),
                                         ("nz3D", 0), ("gy3D", 30), ("gz3D", 20)])
def test_corrupted_context_is_invalid_argument(solver_lib, field, value):
    c = models3d.imported_context(40, 32, 36, 10.0, 8, True, 3000.0, 20.0)
    bad = c.copy()
    setattr(bad, field, value)
    status = call(solver_lib, bad, [(2, 2, 0)])
    assert status == capi.SEIS3D_INVALID_ARGUMENT, field
    assert solver_lib.seis3d_noalloc_last_error()


def test_short_pitch_and_outside_receiver_are_invalid(solver_lib):
    c = models3d.imported_context(40, 32, 36, 10.0, 8, True, 3000.0, 20.0)
    assert call(solver_lib, c, [(2, 2, 0)], pitch=c.gx3D - 1) == capi.SEIS3D_INVALID_ARGUMENT
    assert call(solver_lib, c, [(c.nx3D, 2, 0)]) == capi.SEIS3D_INVALID_ARGUMENT
    assert call(solver_lib, c, [(1, 1, 0)] * (capi.NOALLOC_MAX_RECEIVERS + 1)) == capi.SEIS3D_INVALID_ARGUMENT
