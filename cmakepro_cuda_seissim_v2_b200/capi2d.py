"""ctypes view of the C ABI declared in include/seis2d_capi.h (the 2-D P-SV solver).

The structures mirror the header field by field; :func:`load` opens the in-tree
``libseis2d_b200.so`` built by :mod:`cmakepro_cuda_seissim_v2_b200.build` and raises if it is
missing -- there is no Python fallback for the solver.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int64, c_size_t, c_uint64, c_void_p

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "libseis2d_b200.so")

SEIS2D_OK = 0
SEIS2D_INVALID_ARGUMENT = 1
SEIS2D_LOGIC_ERROR = 2
SEIS2D_RUNTIME_ERROR = 3
SEIS2D_OVERFLOW_ERROR = 4

STENCIL_RADIUS = 4
MAX_ACTIVE_SOURCES = 200
SOURCE_INJECTION_SCALE = 1e7

SPLIT_PML, HYBRID_PML, FREE_SURFACE = 1, 2, 3
RUN_PERSISTENT, RUN_GRAPH = 0, 1
VERTICAL_FORCE, HORIZONTAL_FORCE, EXPLOSIVE, SHEAR, ROTATED_FORCE = range(5)

FIELDS = ("vx_1", "vx_2", "vz_1", "vz_2", "sxx_1", "sxx_2", "szz_1", "szz_2", "sxz_1", "sxz_2",
          "vx", "vz", "sigmaxx", "sigmazz", "sigmaxz", "rho", "mu", "lambda", "lambda2mu",
          "mu_x_flat", "lambda_x_flat", "lambda2mu_x_flat", "mu_z_flat", "rho_x_z_flat", "rho_orig_flat")
FIELD = {name: i for i, name in enumerate(FIELDS)}


class FloatView(ctypes.Structure):
    _fields_ = [("data", POINTER(c_float)), ("size", c_int64)]


class IntView(ctypes.Structure):
    _fields_ = [("data", POINTER(c_int)), ("size", c_int64)]


class Context(ctypes.Structure):
    """seis2d_context = SimulationContext (reference Main_header/Common.h:259-287) with views."""

    _fields_ = [
        ("NX", c_int), ("NZ", c_int), ("total_grid", c_int),
        ("h", c_float), ("dt", c_float),
        ("nt", c_int), ("npml", c_int), ("snap_spacenum", c_int), ("flag_type", c_int),
        ("rho", FloatView), ("mu", FloatView), ("lambda_", FloatView), ("lambda2mu", FloatView),
        ("dp_flat", FloatView),
        ("dx", FloatView), ("dx_half", FloatView), ("dz", FloatView), ("dz_half", FloatView),
        ("c1_h", c_float), ("c2_h", c_float), ("c3_h", c_float), ("c4_h", c_float),
        ("src_idx", c_int), ("src_z_idx", c_int),
        ("wavelet", FloatView),
        ("src_angle", c_float), ("src_type", c_int), ("src_amp", c_float),
        ("num_rcv", c_int), ("rcv_grid_idx", IntView),
        ("upFlag", c_int),
    ]


class Source(ctypes.Structure):
    """seis2d_source = GPUSource (reference Main_header/Common.h:251-256)."""

    _fields_ = [("idx", c_int), ("t", c_float), ("f_peak", c_float), ("amp", c_float)]


FIELD_COUNT = 25


class DeviceViews(ctypes.Structure):
    """seis2d_device_views: raw device pointers named as GPUSimData's members."""

    _fields_ = [
        ("NX", c_int), ("NZ", c_int), ("total_grid", c_int),
        ("dt", c_float), ("inv_dt", c_float),
        ("flag_type", c_int), ("npml", c_int), ("fs_idx", c_int), ("upFlag", c_int),
        ("c1_h", c_float), ("c2_h", c_float), ("c3_h", c_float), ("c4_h", c_float),
        ("field", c_void_p * FIELD_COUNT),
        ("d_dx", c_void_p), ("d_dx_half", c_void_p), ("d_dz", c_void_p), ("d_dz_half", c_void_p),
        ("d_dp_flat", c_void_p),
        ("d_wavelet", c_void_p),
        ("d_rcv_grid_idx", c_void_p),
        ("d_record_vx_step", c_void_p), ("d_record_vz_step", c_void_p),
        ("d_active_sources", c_void_p),
        ("receiverCapacity", c_int), ("reserved", c_int),
        ("stream", c_void_p),
        ("kernelLaunches", c_uint64),
    ]


P = POINTER
SIGNATURES = {
    "seis2d_last_error": (c_char_p, []),
    "seis2d_abi_version": (c_int, []),
    "seis2d_stencil_weights": (None, [P(c_double)]),
    "seis2d_courant_limit": (c_float, []),
    "seis2d_safe_courant": (c_float, []),
    "seis2d_checked_grid_element_count": (c_int, [c_int, c_int, P(c_int64)]),
    "seis2d_validate_boundary_geometry": (c_int, [c_int, c_int, c_int, c_int]),
    "seis2d_receiver_sampling_stride": (c_int, [c_double, c_double, P(c_int)]),
    "seis2d_generate_ricker": (c_int, [P(c_float), c_int, c_float, c_float, c_float]),
    "seis2d_update_pml_damping": (c_int, [P(Context), P(c_float), P(c_float), P(c_float), P(c_float)]),
    "seis2d_free_surface_modulus": (c_int, [P(Context), P(c_float)]),
    "seis2d_validate_context": (c_int, [P(Context)]),
    "seis2d_initialize": (c_int, [P(c_void_p), P(Context)]),
    "seis2d_release": (None, [c_void_p]),
    "seis2d_update_receivers": (c_int, [c_void_p, P(c_int), c_int]),
    "seis2d_set_active_sources": (c_int, [c_void_p, P(Source), c_int]),
    "seis2d_run_step": (c_int, [c_void_p, c_int, P(Context), c_int]),
    "seis2d_run_steps": (c_int, [c_void_p, c_int, c_int, P(Context), c_int]),
    "seis2d_copy_wavefield": (c_int, [c_void_p, P(c_float)]),
    "seis2d_copy_receiver_records": (c_int, [c_void_p, c_int, c_int, c_int, P(c_float), P(c_float)]),
    "seis2d_record_receiver_step": (c_int, [c_void_p, c_int, P(c_float), P(c_float)]),
    "seis2d_gather_begin": (c_int, [c_void_p, c_int, c_int, c_int]),
    "seis2d_gather_fetch": (c_int, [c_void_p, P(c_float), P(c_float), c_int, P(c_int)]),
    "seis2d_gather_end": (c_int, [c_void_p]),
    "seis2d_get_views": (c_int, [c_void_p, P(DeviceViews)]),
    "seis2d_copy_field": (c_int, [c_void_p, c_int, P(c_float)]),
    "seis2d_set_field": (c_int, [c_void_p, c_int, P(c_float)]),
    "seis2d_write_device": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "seis2d_read_device": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "seis2d_synchronize": (c_int, [c_void_p]),
    "seis2d_debug_fail_allocation": (None, [c_int]),
    "seis2d_debug_barrier_wait": (c_int, [c_void_p, ctypes.c_longlong, c_int]),
    "seis2d_wavefield_texture": (c_int, [c_void_p, c_void_p, c_float, c_int]),
    "seis2d_set_stream": (c_int, [c_void_p, c_void_p]),
    "seis2d_set_run_mode": (c_int, [c_void_p, c_int]),
    "seis2d_profile_steps": (c_int, [c_void_p, c_int, c_int, P(Context), P(c_float)]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Open libseis2d_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError(f"{LIBRARY_PATH} is missing: build it with python -m cmakepro_cuda_seissim_v2_b200.build")
        lib = ctypes.CDLL(LIBRARY_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        if lib.seis2d_abi_version() != 1:
            raise RuntimeError("libseis2d_b200.so ABI version mismatch")
        _lib = lib
    return _lib
