"""Files of the 3-D solver over its C ABI: .s3dm models (src/Seis3D/ModelIo3D.cpp) and SEG-Y
rev1 shot gathers with their geometry CSV (src/Seis3D/Acquisition3D.cpp:40-185).

The formats are written by the library (csrc/seis3d_io.inc); this module only prepares the
arguments.  File and format errors raise :class:`SolverError` (the reference's
std::runtime_error), bad arguments :class:`InvalidArgument`.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_float, c_int

import numpy as np

from . import capi
from .seis3d import Context, InvalidArgument, Session, _check, _lib


def default_survey() -> capi.Survey:
    q = capi.Survey()
    _lib().seis3d_default_survey(byref(q))
    return q


def _planes(vp, vs, rho) -> np.ndarray:
    return np.ascontiguousarray(np.stack([vp, vs, rho], axis=-1), dtype=np.float32)


def write_model(path: str, context: Context, vp: np.ndarray, vs: np.ndarray, rho: np.ndarray) -> None:
    """A new .s3dm file holding [z][y][x] vp, vs, rho (FP32) with the context's grid header."""
    planes = _planes(vp, vs, rho)
    if planes.shape != (context.nz3D, context.ny3D, context.nx3D, 3):
        raise InvalidArgument("model arrays must be (nz, ny, nx)")
    _check(_lib().seis3d_write_model(str(path).encode(), byref(context), planes.ctypes.data_as(POINTER(c_float))))


def inspect_model(path: str, base: Context) -> Context:
    """inspectModel3D: the validated imported context of a model file."""
    c = base.copy()
    _check(_lib().seis3d_inspect_model(str(path).encode(), byref(c)))
    return c


def read_model(path: str, context: Context):
    """(vp, vs, rho) arrays [z][y][x] of an inspected model file."""
    out = np.zeros((context.nz3D, context.ny3D, context.nx3D, 3), np.float32)
    for z in range(context.nz3D):
        _check(_lib().seis3d_read_model_plane(str(path).encode(), byref(context), z,
                                              out[z].ctypes.data_as(POINTER(c_float))))
    return out[..., 0].copy(), out[..., 1].copy(), out[..., 2].copy()


def import_model(session: Session, path: str) -> None:
    _check(_lib().seis3d_import_model(session.handle, byref(session.context), str(path).encode()))


def export_model(session: Session, path: str) -> None:
    _check(_lib().seis3d_export_model(session.handle, byref(session.context), str(path).encode()))


class Gather:
    """Gather3D: the frozen geometry of one shot and its samples [sample][receiver][3]."""

    def __init__(self, context: Context, source: capi.Source, receivers, stride: int, target_samples: int,
                 shot_id: int = 1, survey: capi.Survey | None = None):
        self._receivers = np.ascontiguousarray(np.asarray(receivers, dtype=np.int32).reshape(-1, 3))
        self.record = capi.GatherRecord()
        r = self.record
        r.context3D = context
        ctypes.pointer(r.source3D)[0] = source
        r.survey3D = survey if survey is not None else default_survey()
        r.receivers3D = self._receivers.ctypes.data_as(POINTER(capi.Receiver))
        r.receiverCount3D = len(self._receivers)
        r.stride3D, r.targetSamples3D, r.shotId3D = int(stride), int(target_samples), int(shot_id)
        self._samples = np.zeros((0,), np.float32)
        _check(_lib().seis3d_freeze_gather(byref(r)))

    @property
    def sample_interval_us(self) -> int:
        return self.record.sampleIntervalUs3D

    @property
    def first_sample_time(self) -> float:
        return self.record.firstSampleTime3D

    @property
    def coordinate_scalar(self) -> int:
        return self.record.coordinateScalar3D

    def set_samples(self, samples: np.ndarray) -> None:
        s = np.ascontiguousarray(samples, dtype=np.float32)
        if s.ndim != 3 or s.shape[1:] != (len(self._receivers), 3) or s.shape[0] > self.record.targetSamples3D:
            raise InvalidArgument("samples must be [sample][receiver][3] within the target count")
        self._samples = s
        self.record.samples3D = s.ctypes.data_as(POINTER(c_float))
        self.record.sampleCount3D = s.shape[0]

    def cmp_bin(self, receiver) -> tuple[int, int]:
        p = capi.Receiver(*[int(v) for v in receiver])
        a, b = c_int(), c_int()
        _check(_lib().seis3d_cmp_bin(byref(self.record), byref(p), byref(a), byref(b)))
        return a.value, b.value

    def write_segy(self, path: str, component: int) -> None:
        _check(_lib().seis3d_write_segy_component(byref(self.record), str(path).encode(), int(component)))

    def export(self, directory: str, prefix: str) -> None:
        _check(_lib().seis3d_export_gather(byref(self.record), str(directory).encode(), str(prefix).encode()))
