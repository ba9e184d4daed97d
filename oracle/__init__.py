"""Test oracles of the 3-D and 2-D solvers (TEST INFRASTRUCTURE ONLY).

* :class:`CpuOracle` drives ``_build/liboracle3d.so``, the CPU restatement of the
  reference algorithm (seis3d_oracle.cpp) in FP32 or FP64.
* :class:`ReferenceSolver` drives ``_ref/libref3d.so``, the reference's own
  cuda/Cuda_Seis3D.cu compiled unmodified (ref3d_shim.cu + Makefile); it needs a GPU to
  step and is absent when the reference tree was not available at build time.
* :class:`CpuOracle2D` and :class:`ReferenceSolver2D` are the same pair for the 2-D P-SV
  solver (seis2d_oracle.cpp; CUDA_Kernels/Cuda_Check.cu behind ref2d_shim.cu).
* :func:`shade_slices` / :func:`render_volume` run ``_build/libshade3d.so``, the CPU
  restatement of the reference's slice and volume shaders (seis3d_shade_oracle.cpp).

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
ORACLE2D_LIB = os.path.join(HERE, "_build", "liboracle2d.so")
REFERENCE2D_LIB = os.path.join(HERE, "_ref", "libref2d.so")
SHADE_LIB = os.path.join(HERE, "_build", "libshade3d.so")


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
            "oracle3d_set_storage": (None, [c_int, c_int]),
            "oracle3d_set_psi_storage": (None, [c_int]),
            "oracle3d_set_min_pml": (None, [c_int]),
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
            "ref3d_default_context": (None, [POINTER(Context)]),
            "ref3d_default_source": (None, [POINTER(Source)]),
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
            "ref3d_extract_views": (c_int, [c_void_p, c_void_p, POINTER(c_int), c_int, c_int, c_int, c_int,
                                            POINTER(c_float), POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _reference = lib
    return _reference


class ReferenceApi:
    """Context and source construction through the reference's own host code (its default
    member initialisers and validateContext3D), with the call surface of the solver package's
    ``default_context`` / ``default_source`` / ``validate_context3D``.  Workload builders given
    this object never load the B200 solver library, so a process that times the reference
    maps only the reference's code."""

    def __init__(self):
        self.lib = reference_library()
        if self.lib is None:
            raise RuntimeError("oracle/_ref/libref3d.so is missing")

    def default_context(self, **overrides):
        from cmakepro_cuda_seissim_v2_b200.capi import Context

        c = Context()
        self.lib.ref3d_default_context(ctypes.byref(c))
        for key, value in overrides.items():
            if not hasattr(c, key):
                raise AttributeError(key)
            setattr(c, key, value)
        return c

    def default_source(self, **overrides):
        from cmakepro_cuda_seissim_v2_b200.capi import Source

        s = Source()
        self.lib.ref3d_default_source(ctypes.byref(s))
        for key, value in overrides.items():
            if key == "direction3D":
                for a in range(3):
                    s.direction3D[a] = float(value[a])
            else:
                setattr(s, key, value)
        return s

    def validate_context3D(self, c):
        if self.lib.ref3d_validate(ctypes.byref(c)) != 0:
            raise ValueError((self.lib.ref3d_last_error() or b"").decode(errors="replace"))
        return c


GPU64_LIB = os.path.join(HERE, "_build", "liboracle3d_gpu.so")
_gpu64 = None


def gpu64_library():
    """The FP64 GPU restatement (seis3d_oracle_gpu.cu), built by the Makefile."""
    global _gpu64
    if _gpu64 is None:
        if not os.path.exists(GPU64_LIB):
            build()
        from cmakepro_cuda_seissim_v2_b200.capi import Context, Receiver, Source

        lib = ctypes.CDLL(GPU64_LIB)
        sig = {
            "oracle3d_gpu_last_error": (ctypes.c_char_p, []),
            "oracle3d_gpu_create": (c_void_p, [POINTER(Context)]),
            "oracle3d_gpu_destroy": (None, [c_void_p]),
            "oracle3d_gpu_upload_model": (c_int, [c_void_p, POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
            "oracle3d_gpu_set_receivers": (c_int, [c_void_p, POINTER(Receiver), c_int]),
            "oracle3d_gpu_run_gather": (c_int, [c_void_p, POINTER(Source), c_uint64, c_int, c_int, POINTER(c_double),
                                                c_int, POINTER(c_int)]),
            "oracle3d_gpu_get_field": (c_int, [c_void_p, c_int, POINTER(c_double)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _gpu64 = lib
    return _gpu64


class GpuOracle64:
    """The reference scheme in FP64 on the GPU (oracle role only): the yardstick of the FP32
    solvers on workloads too large for the CPU oracle."""

    def __init__(self, context):
        self.lib = gpu64_library()
        self.context = context.copy()
        self.h = self.lib.oracle3d_gpu_create(byref(self.context))
        if not self.h:
            raise RuntimeError(self.lib.oracle3d_gpu_last_error().decode())
        self.nr = 0

    def _ok(self, status):
        if status != 0:
            raise RuntimeError(self.lib.oracle3d_gpu_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle3d_gpu_destroy(self.h)
            self.h = None

    __del__ = close

    def upload_model(self, vp, vs, rho):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho)]
        self._ok(self.lib.oracle3d_gpu_upload_model(self.h, *(a.ctypes.data_as(POINTER(c_float)) for a in arrs)))

    def set_receivers(self, receivers):
        arr, nr = _receivers(receivers)
        self._ok(self.lib.oracle3d_gpu_set_receivers(self.h, arr, nr))
        self.nr = nr

    def run_gather(self, source, first, count, stride):
        cap = count // stride + 1
        out = np.zeros(cap * max(self.nr, 1) * 3, dtype=np.float64)
        taken = c_int()
        self._ok(self.lib.oracle3d_gpu_run_gather(self.h, byref(source), int(first), int(count), int(stride),
                                                  out.ctypes.data_as(POINTER(c_double)), cap, byref(taken)))
        return out[: taken.value * self.nr * 3].reshape(taken.value, self.nr, 3)

    def field(self, k):
        c = self.context
        out = np.zeros((c.gz3D, c.gy3D, c.gx3D), dtype=np.float64)
        self._ok(self.lib.oracle3d_gpu_get_field(self.h, int(k), out.ctypes.data_as(POINTER(c_double))))
        return out


def loaded_libraries() -> list[str]:
    """Shared objects mapped into this process (Linux /proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            paths = {line.split()[-1] for line in f if line.rstrip().endswith(".so") or ".so." in line}
    except OSError:
        return []
    return sorted(p for p in paths if p.startswith("/"))


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

    def sample(self):
        """sampleReceivers3D: [receiver][vx, vy, vz] of the current fields."""
        out = np.zeros((max(self.nr, 1), 3), dtype=np.float32)
        self._ok(self.lib.ref3d_sample(self.h, out.ctypes.data_as(POINTER(c_float))))
        return out[: self.nr]

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

    def extract_views(self, count, slices, component, material, volume, include_boundary=False):
        out = np.zeros(max(count, 1) * 2, np.float32)
        sl = (c_int * 3)(*[int(v) for v in slices])
        maximum, vmax = c_float(), c_float()
        rng = (c_float * 2)()
        self._ok(self.lib.ref3d_extract_views(self.h, None, sl, int(component), int(material), int(bool(volume)),
                                              int(bool(include_boundary)), out.ctypes.data_as(POINTER(c_float)),
                                              byref(maximum), rng, byref(vmax)))
        return out[: count * 2], {"maximum": maximum.value, "material_range": (rng[0], rng[1]),
                                  "velocity_maximum": vmax.value}


# ---- 2-D P-SV ----------------------------------------------------------------------------

_oracle2d = None
_reference2d = None


def oracle2d_library():
    global _oracle2d
    if _oracle2d is None:
        if not os.path.exists(ORACLE2D_LIB):
            build()
        from cmakepro_cuda_seissim_v2_b200.capi2d import Context as Context2D, Source as Source2D

        lib = ctypes.CDLL(ORACLE2D_LIB)
        P = POINTER
        sig = {
            "oracle2d_create": (c_void_p, [P(Context2D), c_int]),
            "oracle2d_destroy": (None, [c_void_p]),
            "oracle2d_set_sources": (None, [c_void_p, P(Source2D), c_int]),
            "oracle2d_get_sources": (None, [c_void_p, P(Source2D), c_int]),
            "oracle2d_run": (None, [c_void_p, c_int, c_int, P(Context2D), c_int, c_int, P(c_int), c_int, P(c_float),
                                    P(c_float)]),
            "oracle2d_field": (None, [c_void_p, c_int, P(c_float)]),
            "oracle2d_set_field": (None, [c_void_p, c_int, P(c_float)]),
            "oracle2d_record": (None, [c_void_p, P(c_int), c_int, P(c_float), P(c_float)]),
            "oracle2d_wavefield": (None, [c_void_p, P(c_float)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _oracle2d = lib
    return _oracle2d


def reference2d_library():
    """The reference 2-D solver library, or None when it was not built."""
    global _reference2d
    if _reference2d is None:
        if not os.path.exists(REFERENCE2D_LIB):
            return None
        from cmakepro_cuda_seissim_v2_b200.capi2d import Context as Context2D, Source as Source2D

        lib = ctypes.CDLL(REFERENCE2D_LIB)
        P = POINTER
        sig = {
            "ref2d_last_error": (ctypes.c_char_p, []),
            "ref2d_validate": (c_int, [P(Context2D)]),
            "ref2d_create": (c_int, [P(c_void_p), P(Context2D)]),
            "ref2d_destroy": (None, [c_void_p]),
            "ref2d_set_context": (c_int, [c_void_p, P(Context2D)]),
            "ref2d_update_receivers": (c_int, [c_void_p, P(c_int), c_int]),
            "ref2d_set_sources": (c_int, [c_void_p, P(Source2D), c_int]),
            "ref2d_step": (c_int, [c_void_p, c_int, c_int]),
            "ref2d_run": (c_int, [c_void_p, c_int, c_int, c_int, c_int, P(c_float), P(c_float)]),
            "ref2d_time_steps": (c_int, [c_void_p, c_int, c_int, P(c_float)]),
            "ref2d_record": (c_int, [c_void_p, c_int, P(c_float), P(c_float)]),
            "ref2d_wavefield": (c_int, [c_void_p, P(c_float)]),
            "ref2d_field": (c_int, [c_void_p, c_int, P(c_float)]),
            "ref2d_set_field": (c_int, [c_void_p, c_int, P(c_float)]),
            "ref2d_wavefield_texture": (c_int, [c_void_p, c_void_p, c_float, c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _reference2d = lib
    return _reference2d


def _sources2d(sources):
    from cmakepro_cuda_seissim_v2_b200.capi2d import Source as Source2D

    sources = list(sources)
    arr = (Source2D * max(len(sources), 1))(*[Source2D(int(i), float(t), float(f), float(a)) for i, t, f, a in sources])
    return arr, len(sources)


class CpuOracle2D:
    """CPU restatement of the reference 2-D solver, FP32 (`precision=32`) or FP64."""

    def __init__(self, context, precision: int = 64):
        self.lib = oracle2d_library()
        self.context = context
        self._c = context.to_c()
        self.h = self.lib.oracle2d_create(byref(self._c), int(precision))
        self.n = context.NX * context.NZ

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle2d_destroy(self.h)
            self.h = None

    __del__ = close

    def set_sources(self, sources):
        arr, n = _sources2d(sources)
        self.lib.oracle2d_set_sources(self.h, arr, n)

    def run(self, first, count, context=None, num_active=-1, advance=False, receivers=None):
        """Steps first..first+count-1; returns ([r][count] vx, vz) when receivers are given."""
        c = (context or self.context).to_c()
        if receivers is None:
            self.lib.oracle2d_run(self.h, int(first), int(count), byref(c), int(num_active), int(advance), None, 0,
                                  None, None)
            return None
        idx = np.ascontiguousarray(np.asarray(receivers, dtype=np.int32))
        vx = np.zeros((idx.size, count), np.float32)
        vz = np.zeros((idx.size, count), np.float32)
        self.lib.oracle2d_run(self.h, int(first), int(count), byref(c), int(num_active), int(advance),
                              idx.ctypes.data_as(POINTER(c_int)), idx.size, vx.ctypes.data_as(POINTER(c_float)),
                              vz.ctypes.data_as(POINTER(c_float)))
        return vx, vz

    def field(self, which: int) -> np.ndarray:
        out = np.zeros((self.context.NZ, self.context.NX), np.float32)
        self.lib.oracle2d_field(self.h, int(which), out.ctypes.data_as(POINTER(c_float)))
        return out

    def set_field(self, which: int, values):
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        self.lib.oracle2d_set_field(self.h, int(which), v.ctypes.data_as(POINTER(c_float)))

    def record(self, receivers):
        idx = np.ascontiguousarray(np.asarray(receivers, dtype=np.int32))
        vx = np.zeros(idx.size, np.float32)
        vz = np.zeros(idx.size, np.float32)
        self.lib.oracle2d_record(self.h, idx.ctypes.data_as(POINTER(c_int)), idx.size,
                                 vx.ctypes.data_as(POINTER(c_float)), vz.ctypes.data_as(POINTER(c_float)))
        return vx, vz

    def wavefield(self) -> np.ndarray:
        out = np.zeros(self.n, np.float32)
        self.lib.oracle2d_wavefield(self.h, out.ctypes.data_as(POINTER(c_float)))
        return out


class ReferenceSolver2D:
    """The reference's own 2-D CUDA solver (CUDA_Kernels/Cuda_Check.cu) through its functions."""

    def __init__(self, context):
        self.lib = reference2d_library()
        if self.lib is None:
            raise FileNotFoundError(REFERENCE2D_LIB)
        self.context = context
        self._c = context.to_c()
        h = c_void_p()
        self._ok(self.lib.ref2d_create(byref(h), byref(self._c)))
        self.h = h

    def _ok(self, status):
        if status != 0:
            raise RuntimeError(self.lib.ref2d_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref2d_destroy(self.h)
            self.h = None

    __del__ = close

    def set_context(self, context):
        self.context = context
        self._c = context.to_c()
        self._ok(self.lib.ref2d_set_context(self.h, byref(self._c)))

    def set_sources(self, sources):
        arr, n = _sources2d(sources)
        self._ok(self.lib.ref2d_set_sources(self.h, arr, n))

    def update_receivers(self, receivers):
        idx = np.ascontiguousarray(np.asarray(receivers, dtype=np.int32))
        self._ok(self.lib.ref2d_update_receivers(self.h, idx.ctypes.data_as(POINTER(c_int)), idx.size))

    def step(self, it, num_active=-1):
        self._ok(self.lib.ref2d_step(self.h, int(it), int(num_active)))

    def run(self, first, count, num_active=-1, nrcv=0):
        if nrcv <= 0:
            self._ok(self.lib.ref2d_run(self.h, int(first), int(count), int(num_active), 0, None, None))
            return None
        vx = np.zeros((nrcv, count), np.float32)
        vz = np.zeros((nrcv, count), np.float32)
        self._ok(self.lib.ref2d_run(self.h, int(first), int(count), int(num_active), int(nrcv),
                                    vx.ctypes.data_as(POINTER(c_float)), vz.ctypes.data_as(POINTER(c_float))))
        return vx, vz

    def time_steps(self, first, count) -> float:
        ms = c_float()
        self._ok(self.lib.ref2d_time_steps(self.h, int(first), int(count), byref(ms)))
        return ms.value

    def field(self, which: int) -> np.ndarray:
        out = np.zeros((self.context.NZ, self.context.NX), np.float32)
        self._ok(self.lib.ref2d_field(self.h, int(which), out.ctypes.data_as(POINTER(c_float))))
        return out

    def set_field(self, which: int, values):
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        self._ok(self.lib.ref2d_set_field(self.h, int(which), v.ctypes.data_as(POINTER(c_float))))

    def texture(self, device_rgba_ptr: int, scale: float, component: int) -> None:
        """generateWavefieldTextureOnGpu of the reference into a device buffer (synchronised)."""
        self._ok(self.lib.ref2d_wavefield_texture(self.h, c_void_p(int(device_rgba_ptr)), float(scale),
                                                  int(component)))

    def wavefield(self) -> np.ndarray:
        out = np.zeros(self.context.NX * self.context.NZ, np.float32)
        self._ok(self.lib.ref2d_wavefield(self.h, out.ctypes.data_as(POINTER(c_float))))
        return out


_shade = None


def shade_library():
    global _shade
    if _shade is None:
        if not os.path.exists(SHADE_LIB):
            build()
        from cmakepro_cuda_seissim_v2_b200.capi import Transfer, VolumeView

        lib = ctypes.CDLL(SHADE_LIB)
        lib.oracle_shade_slices.restype = None
        lib.oracle_shade_slices.argtypes = [POINTER(c_float), c_uint64, POINTER(Transfer), c_float, c_float,
                                            POINTER(c_float)]
        lib.oracle_render_volume.restype = None
        lib.oracle_render_volume.argtypes = [POINTER(c_float), c_int, c_int, c_int, POINTER(Transfer),
                                             POINTER(VolumeView), c_int, c_int, POINTER(c_float)]
        _shade = lib
    return _shade


def shade_slices(views: np.ndarray, transfer, scale: float, gain: float) -> np.ndarray:
    """Slice shader over `views` [n][2] (wave, material) -> RGBA float32 [n][4]."""
    v = np.ascontiguousarray(views, dtype=np.float32).reshape(-1, 2)
    out = np.zeros((len(v), 4), np.float32)
    shade_library().oracle_shade_slices(v.ctypes.data_as(POINTER(c_float)), len(v), byref(transfer), float(scale),
                                        float(gain), out.ctypes.data_as(POINTER(c_float)))
    return out


def render_volume(texels: np.ndarray, transfer, volume, width: int, height: int) -> np.ndarray:
    """Volume shader over `texels` [nz][ny][nx][2] -> RGBA float32 [height][width][4]."""
    t = np.ascontiguousarray(texels, dtype=np.float32)
    nz, ny, nx = t.shape[:3]
    out = np.zeros((height, width, 4), np.float32)
    shade_library().oracle_render_volume(t.ctypes.data_as(POINTER(c_float)), nx, ny, nz, byref(transfer),
                                         byref(volume), int(width), int(height), out.ctypes.data_as(POINTER(c_float)))
    return out


def to_rgba8(rgba: np.ndarray) -> np.ndarray:
    """GL_RGBA8 conversion of float colours: clamp to [0, 1], round to the nearest of 255 steps."""
    return np.rint(np.clip(np.nan_to_num(rgba, nan=0.0), 0.0, 1.0) * np.float32(255)).astype(np.uint8)
