"""Receiver sampling without allocation (seis3d_sample_receivers_noalloc).

For callers that cannot allocate device memory while the solver runs -- a host whose
device memory all belongs to its own pool, a loop where an allocation is not allowed, a
plugin lent another owner's wavefield buffers -- the library offers one entry point that
reads receivers from caller-owned velocity fields using only a fixed static device
scratch.  These tests call it through the C ABI and check it against the session's own
sampleReceivers3D path (seis3d_sample_receivers) on two calls in a row, with the
receiver-trace tolerance used by the other parity tests.  The file sorts last so a run
that stops at the first failure has already run every other test.
"""
import ctypes
from ctypes import byref, c_float

import numpy as np
import pytest

from cmakepro_cuda_seissim_v2_b200 import capi, models3d, seis3d

pytestmark = pytest.mark.gpu

TRACE_TOL = 1e-5  # relative L2, as for the FP32 receiver traces of the parity tests


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def sample_noalloc(lib, session, receivers):
    v = session.views()
    arr, n = seis3d.receivers_array(receivers)
    out = np.zeros((max(n, 1), 3), dtype=np.float32)
    status = lib.seis3d_sample_receivers_noalloc(byref(session.context), v.field3D[0], v.field3D[1], v.field3D[2],
                                                 v.pitch, arr, n, out.ctypes.data_as(ctypes.POINTER(c_float)),
                                                 v.stream3D)
    return status, out[:n]


def test_noalloc_sampling_matches_session_sampling(solver_lib, cuda_device):
    shot = models3d.small_shot(steps=30, free_surface=True)
    s = seis3d.Session(shot.context)
    try:
        s.upload_model(shot.vp, shot.vs, shot.rho)
        s.set_receivers(shot.receivers)
        for n in range(shot.steps):
            s.run_step(shot.source, n)
        first_ref = s.sample_receivers()
        status, first = sample_noalloc(solver_lib, s, shot.receivers)
        assert status == capi.SEIS3D_OK, solver_lib.seis3d_noalloc_last_error()
        assert np.abs(first_ref).max() > 0
        assert rel_l2(first, first_ref) < TRACE_TOL

        # Second call in a row, after one more step and with a different receiver set
        # (the scratch keeps the previous call's contents and must not leak into this one).
        s.run_step(shot.source, shot.steps)
        subset = shot.receivers[::2][:7]
        s.set_receivers(subset)
        second_ref = s.sample_receivers()
        status, second = sample_noalloc(solver_lib, s, subset)
        assert status == capi.SEIS3D_OK, solver_lib.seis3d_noalloc_last_error()
        assert second.shape == (len(subset), 3)
        assert rel_l2(second, second_ref) < TRACE_TOL
    finally:
        s.release()


def test_noalloc_sampling_rejects_oversized_and_outside_requests(solver_lib, cuda_device):
    shot = models3d.small_shot(steps=1)
    s = seis3d.Session(shot.context)
    try:
        too_many = [(1, 1, 0)] * (capi.NOALLOC_MAX_RECEIVERS + 1)
        status, _ = sample_noalloc(solver_lib, s, too_many)
        assert status == capi.SEIS3D_INVALID_ARGUMENT
        assert b"300" in solver_lib.seis3d_noalloc_last_error()
        status, _ = sample_noalloc(solver_lib, s, [(shot.context.nx3D, 0, 0)])
        assert status == capi.SEIS3D_INVALID_ARGUMENT
        status, out = sample_noalloc(solver_lib, s, [(2, 2, 0)])
        assert status == capi.SEIS3D_OK and np.all(out == 0)
    finally:
        s.release()
