"""Test oracles of the 3-D solver (TEST INFRASTRUCTURE ONLY).

* :class:`CpuOracle` drives ``_build/liboracle3d.so``, the CPU restatement of the
  reference algorithm (seis3d_oracle.cpp) in FP32 or FP64.
* :class:`ReferenceSolver` drives ``_ref/libref3d.so``, the reference's own
  cuda/Cuda_Seis3D.cu compiled unmodified (ref3d_shim.cu + Makefile); it needs a GPU to
  step and is absent when the reference tree was not available at build time.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's baseline legs use this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, byref, c_double, c_float, c_int, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle3d.so")
REFERENCE_LIB = os.path.join(HERE, "_ref", "libref3d.so")


def build(reference_root: str | None = None) -> None:
    """Run the oracle Makefile (CPU oracle always; reference shim when its tree exists)."""
    env = dict(os.environ)
    if reference_root:
        env["REFERENCE_ROOT"] = reference_root
    subprocess.run(["make", "-s", "-C", HERE], check=True, env=env)


_oracle = None
_reference = None


def oracle_library():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        from cmakepro_cuda_seissim_v2_b200.capi import Context, MemoryBudget, Receiver, Source

        lib = ctypes.CDLL(ORACLE_LIB)
        sig = {
            "oracle3d_last_error": (ctypes.c_char_p, []),
            "oracle3d_set_threads": (None, [c_int]),
            "oracle3d_max_threads": (c_int, []),
            "oracle3d_validate": (c_int, [POINTER(Context)]),
            "oracle3d_estimate_memory": (c_int, [POINTER(Context), POINTER(MemoryBudget)]),
            "oracle3d_make_coefficients": (c_int, [POINTER(Context), c_int, POINTER(c_float)]),
            "oracle3d_create": (c_void_p, [POINTER(Context), c_int]),
            "oracle3d_destroy": (None, [c_void_p]),
            "oracle3d_generate_materials": (None, [c_void_p]),
            "oracle3d_reset": (None, [c_void_p]),
            "oracle3d_upload_plane": (c_int, [c_void_p, c_int, POINTER(c_float)]),
            "oracle3d_finish_upload": (None, [c_void_p]),
            "oracle3d_step": (None, [c_void_p, POINTER(Source), c_uint64]),
            "oracle3d_run": (None, [c_void_p, POINTER(Source), c_uint64, c_int]),
            "oracle3d_run_gather": (c_int, [c_void_p, POINTER(Source), c_uint64, c_int, POINTER(Receiver), c_int,
                                            c_int, POINTER(c_double), c_int]),
            "oracle3d_sample": (None, [c_void_p, POINTER(Receiver), c_int, POINTER(c_double)]),
            "oracle3d_get_field": (None, [c_void_p, c_int, POINTER(c_double)]),
            "oracle3d_set_field": (None, [c_void_p, c_int, POINTER(c_double)]),
            "oracle3d_non_finite": (c_int, [c_void_p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _oracle = lib
    return _oracle


def reference_library():
    """The reference solver library, or None when it was not built."""
    global _reference
    if _reference is None:
        if not os.path.exists(REFERENCE_LIB):
            return None
        from cmakepro_cuda_seissim_v2_b200.capi import Context, MemoryBudget, Receiver, Source

        lib = ctypes.CDLL(REFERENCE_LIB)
        sig = {
            "ref3d_last_error": (ctypes.c_char_p, []),
            "ref3d_validate": (c_int, [POINTER(Context)]),
            "ref3d_estimate_memory": (c_int, [POINTER(Context), POINTER(MemoryBudget)]),
            "ref3d_make_coefficients": (c_int, [POINTER(Context), c_int, POINTER(c_float)]),
            "ref3d_create": (c_void_p, [POINTER(Context)]),
            "ref3d_destroy": (None, [c_void_p]),
            "ref3d_upload_plane": (c_int, [c_void_p, c_int, POINTER(c_float)]),
            "ref3d_finish_upload": (c_int, [c_void_p]),
            "ref3d_reset": (c_int, [c_void_p]),
            "ref3d_set_receivers": (c_int, [c_void_p, POINTER(Receiver), c_int]),
            "ref3d_run_steps": (c_int, [c_void_p, POINTER(Source), c_uint64, c_int]),
            "ref3d_run_gather": (c_int, [c_void_p, POINTER(Source), c_uint64, c_int, c_int, POINTER(c_float), c_int,
                                         POINTER(c_int)]),
            "ref3d_time_steps": (c_int, [c_void_p, POINTER(Source), c_uint64, c_int, POINTER(c_float)]),
            "ref3d_sample": (c_int, [c_void_p, POINTER(c_float)]),
            "ref3d_get_field": (c_int, [c_void_p, c_int, POINTER(c_float)]),
            "ref3d_set_field": (c_int, [c_void_p, c_int, POINTER(c_float)]),
            "ref3d_synchronize": (c_int, [c_void_p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _reference = lib
    return _reference


def _receivers(rec):
    from cmakepro_cuda_seissim_v2_b200.seis3d import receivers_array

    return receivers_array(rec)


class CpuOracle:
    """CPU restatement of the reference solver in FP32 (`precision=32`) or FP64."""

    def __init__(self, context, precision: int = 64, threads: int = 0):
        self.lib = oracle_library()
        self.context = context.copy()
        if self.lib.oracle3d_validate(byref(self.context)) != 0:
            raise ValueError(self.lib.oracle3d_last_error().decode())
        if threads:
            self.lib.oracle3d_set_threads(threads)
        self.h = self.lib.oracle3d_create(byref(self.context), precision)
        if not self.h:
            raise MemoryError(self.lib.oracle3d_last_error().decode())
        self.receivers = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle3d_destroy(self.h)
            self.h = None

    __del__ = close

    def generate(self):
        self.lib.oracle3d_generate_materials(self.h)

    def upload_model(self, vp, vs, rho):
        for z in range(vp.shape[0]):
            plane = np.ascontiguousarray(np.stack([vp[z], vs[z], rho[z]], axis=-1), dtype=np.float32)
            if self.lib.oracle3d_upload_plane(self.h, z, plane.ctypes.data_as(POINTER(c_float))) != 0:
                raise ValueError(self.lib.oracle3d_last_error().decode())
        self.lib.oracle3d_finish_upload(self.h)

    def reset(self):
        self.lib.oracle3d_reset(self.h)

    def step(self, source, n):
        self.lib.oracle3d_step(self.h, byref(source), int(n))

    def run(self, source, first, count):
        self.lib.oracle3d_run(self.h, byref(source), int(first), int(count))

    def run_gather(self, source, first, count, receivers, stride):
        arr, nr = _receivers(receivers)
        cap = count // stride + 1
        out = np.zeros(cap * nr * 3, dtype=np.float64)
        taken = self.lib.oracle3d_run_gather(self.h, byref(source), int(first), int(count), arr, nr, int(stride),
                                             out.ctypes.data_as(POINTER(c_double)), cap)
        return out[: taken * nr * 3].reshape(taken, nr, 3)

    def sample(self, receivers):
        arr, nr = _receivers(receivers)
        out = np.zeros(nr * 3, dtype=np.float64)
        self.lib.oracle3d_sample(self.h, arr, nr, out.ctypes.data_as(POINTER(c_double)))
        return out.reshape(nr, 3)

    def field(self, k):
        c = self.context
        out = np.zeros((c.gz3D, c.gy3D, c.gx3D), dtype=np.float64)
        self.lib.oracle3d_get_field(self.h, int(k), out.ctypes.data_as(POINTER(c_double)))
        return out

    def set_field(self, k, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.lib.oracle3d_set_field(self.h, int(k), v.ctypes.data_as(POINTER(c_double)))

    def non_finite(self) -> bool:
        return bool(self.lib.oracle3d_non_finite(self.h))


class ReferenceSolver:
    """The reference's own CUDA solver (cuda/Cuda_Seis3D.cu) driven through its API."""

    def __init__(self, context):
        self.lib = reference_library()
        if self.lib is None:
            raise FileNotFoundError(REFERENCE_LIB)
        self.context = context.copy()
        if self.lib.ref3d_validate(byref(self.context)) != 0:
            raise ValueError(self.lib.ref3d_last_error().decode())
        self.h = self.lib.ref3d_create(byref(self.context))
        if not self.h:
            raise RuntimeError(self.lib.ref3d_last_error().decode())
        self.nr = 0

    def _ok(self, status):
        if status != 0:
            raise RuntimeError(self.lib.ref3d_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref3d_destroy(self.h)
            self.h = None

    __del__ = close

    def upload_model(self, vp, vs, rho):
        for z in range(vp.shape[0]):
            plane = np.ascontiguousarray(np.stack([vp[z], vs[z], rho[z]], axis=-1), dtype=np.float32)
            self._ok(self.lib.ref3d_upload_plane(self.h, z, plane.ctypes.data_as(POINTER(c_float))))
        self._ok(self.lib.ref3d_finish_upload(self.h))

    def set_receivers(self, receivers):
        arr, nr = _receivers(receivers)
        self._ok(self.lib.ref3d_set_receivers(self.h, arr, nr))
        self.nr = nr

    def reset(self):
        self._ok(self.lib.ref3d_reset(self.h))

    def run(self, source, first, count):
        self._ok(self.lib.ref3d_run_steps(self.h, byref(source), int(first), int(count)))

    def time_steps(self, source, first, count) -> float:
        ms = c_float()
        self._ok(self.lib.ref3d_time_steps(self.h, byref(source), int(first), int(count), byref(ms)))
        return ms.value

    def run_gather(self, source, first, count, stride):
        cap = count // stride + 1
        out = np.zeros(cap * max(self.nr, 1) * 3, dtype=np.float32)
        taken = c_int()
        self._ok(self.lib.ref3d_run_gather(self.h, byref(source), int(first), int(count), int(stride),
                                           out.ctypes.data_as(POINTER(c_float)), cap, byref(taken)))
        return out[: taken.value * self.nr * 3].reshape(taken.value, self.nr, 3)

    def field(self, k):
        c = self.context
        out = np.zeros((c.gz3D, c.gy3D, c.gx3D), dtype=np.float32)
        self._ok(self.lib.ref3d_get_field(self.h, int(k), out.ctypes.data_as(POINTER(c_float))))
        return out

    def set_field(self, k, values):
        v = np.ascontiguousarray(values, dtype=np.float32)
        self._ok(self.lib.ref3d_set_field(self.h, int(k), v.ctypes.data_as(POINTER(c_float))))

    def synchronize(self):
        self._ok(self.lib.ref3d_synchronize(self.h))
