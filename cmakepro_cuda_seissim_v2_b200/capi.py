"""ctypes view of the C ABI declared in include/seis3d_capi.h.

The structures mirror the POD types of the header field by field; `load()` opens the
in-tree ``libseis3d_b200.so`` built by :mod:`cmakepro_cuda_seissim_v2_b200.build` and
raises if it is missing -- there is no Python fallback for the solver.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_char_p, c_float, c_int, c_int64, c_size_t, c_uint64, c_void_p

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "libseis3d_b200.so")

SEIS3D_OK = 0
SEIS3D_INVALID_ARGUMENT = 1
SEIS3D_LOGIC_ERROR = 2
SEIS3D_RUNTIME_ERROR = 3

STENCIL_RADIUS = 4
MAX_PHYSICAL_NODES = 36_000_000
MAX_RECEIVERS = 300
MAX_VOLUME_AXIS = 256          # SEIS3D_MAX_VOLUME_AXIS
MAX_VOLUME_OUTPUT = 1536       # SEIS3D_MAX_VOLUME_OUTPUT
NOALLOC_MAX_RECEIVERS = 300
BOUNDARY_PARAMETERS = 23728    # SEIS3D_BOUNDARY_PARAMETERS: FP32 parameters per face
BOUNDARY_FACES = ("x-", "x+", "y-", "y+", "z-", "z+")
MEMORY_LIMIT = 4 * 1024**3

FIELDS = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz")

(MODEL_UNIFORM, MODEL_TWO_LAYER, MODEL_SPHERE, MODEL_IMPORTED, MODEL_THREE_LAYER, MODEL_DIPPING_LAYER,
 MODEL_LOW_VELOCITY_LAYER, MODEL_FAULT, MODEL_GRADIENT, MODEL_SALT_DOME) = range(10)
SOURCE_EXPLOSION, SOURCE_FORCE = 0, 1
STORAGE_FP32, STORAGE_FP16, STORAGE_BF16, STORAGE_BF16_CPML = 0, 1, 2, 3   # enum seis3d_storage


class Context(ctypes.Structure):
    """seis3d_context = SimulationContext3D (reference include/Common3D.h:24-42)."""

    _fields_ = [
        ("nx3D", c_int), ("ny3D", c_int), ("nz3D", c_int),
        ("pml3D", c_int),
        ("freeSurface3D", c_int),
        ("reflecting3D", c_int),
        ("spacing3D", c_float), ("cfl3D", c_float), ("dt3D", c_float),
        ("manualTimeStep3D", c_int),
        ("requestedDtMs3D", c_float),
        ("safeDt3D", c_float),
        ("vp3D", c_float), ("vs3D", c_float), ("density3D", c_float),
        ("layerVp3D", c_float), ("layerVs3D", c_float), ("layerDensity3D", c_float),
        ("maxVp3D", c_float), ("frequency3D", c_float),
        ("modelKind3D", c_int),
        ("interfaceDepth3D", c_float), ("layerDip3D", c_float), ("layerThickness3D", c_float),
        ("faultThrow3D", c_float), ("anomalyRadius3D", c_float),
        ("gx3D", c_int), ("gy3D", c_int), ("gz3D", c_int), ("ox3D", c_int), ("oy3D", c_int), ("oz3D", c_int),
        ("cells3D", c_uint64),
    ]

    def copy(self) -> "Context":
        other = Context()
        ctypes.pointer(other)[0] = self
        return other

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Source(ctypes.Structure):
    """seis3d_source = Source3D (include/Common3D.h:44-49)."""

    _fields_ = [("x3D", c_int), ("y3D", c_int), ("z3D", c_int), ("kind3D", c_int),
                ("amplitude3D", c_float), ("direction3D", c_float * 3)]


class Receiver(ctypes.Structure):
    """seis3d_receiver = Receiver3D (include/Common3D.h:51)."""

    _fields_ = [("x3D", c_int), ("y3D", c_int), ("z3D", c_int)]


class MemoryBudget(ctypes.Structure):
    _fields_ = [("fieldBytes3D", c_uint64), ("cpmlBytes3D", c_uint64), ("viewBytes3D", c_uint64),
                ("totalBytes3D", c_uint64)]


class ViewLayout(ctypes.Structure):
    _fields_ = [("sliceOffset3D", c_uint64 * 3), ("sliceWidth3D", c_int * 3), ("sliceHeight3D", c_int * 3),
                ("volumeOffset3D", c_uint64), ("totalSamples3D", c_uint64),
                ("volumeX3D", c_int), ("volumeY3D", c_int), ("volumeZ3D", c_int),
                ("domainSize3D", c_int * 3), ("domainOrigin3D", c_int * 3)]


class Options(ctypes.Structure):
    _fields_ = [("storage", c_int), ("tile_y", c_int), ("z_chunk", c_int), ("compact_rows", c_int),
                ("tune", c_int), ("thin_cpml", c_int), ("reserved", c_int * 2)]


class DeviceViews(ctypes.Structure):
    _fields_ = [("field3D", c_void_p * 9), ("inverseDensity3D", c_void_p), ("lambda3D", c_void_p), ("mu3D", c_void_p),
                ("cpml3D", c_void_p * 3), ("slabCells3D", c_uint64 * 3), ("coefficients3D", c_void_p * 3),
                ("stream3D", c_void_p), ("receiverCount3D", c_int), ("storage", c_int),
                ("pitch", c_int64), ("plane", c_int64), ("field_scale", c_float * 12),
                ("allocatedBytes3D", c_uint64), ("kernelLaunches", c_uint64)]


# Exported symbols and their signatures (restype, argtypes); the symbol test checks that
# every one of them is exported by the built library and declared in the header.
class Survey(ctypes.Structure):
    """seis3d_survey = Survey3D (reference include/Seis3D_Sim.h:36-45)."""

    _fields_ = [("receiverCountX3D", c_int), ("receiverCountY3D", c_int), ("receiverOrigin3D", c_int * 3),
                ("receiverSpacing3D", c_int * 2), ("shotCountX3D", c_int), ("shotCountY3D", c_int),
                ("shotOrigin3D", c_int * 3), ("shotSpacing3D", c_int * 2), ("worldOrigin3D", c_double * 2),
                ("cmpBinSize3D", c_float * 2)]


class GatherRecord(ctypes.Structure):
    """seis3d_gather_record = Gather3D (reference include/Seis3D_Sim.h:47-57) with views."""

    _fields_ = [("context3D", Context), ("source3D", Source), ("survey3D", Survey),
                ("receivers3D", POINTER(Receiver)), ("receiverCount3D", c_int), ("samples3D", POINTER(c_float)),
                ("sampleCount3D", c_int), ("targetSamples3D", c_int), ("stride3D", c_int), ("shotId3D", c_int),
                ("sampleIntervalUs3D", c_int), ("coordinateScalar3D", c_int), ("firstSampleTime3D", c_double)]


class Transfer(ctypes.Structure):
    """seis3d_transfer: uniforms of the shared transfer function (shaders/seis3d_transfer.glsl:1-5)."""

    _fields_ = [("palette3D", (c_float * 3) * 5), ("displayMode3D", c_int), ("modelStyle3D", c_int),
                ("unsignedWave3D", c_int), ("materialRange3D", c_float * 2), ("waveOpacity3D", c_float),
                ("waveThreshold3D", c_float), ("modelOpacity3D", c_float), ("waveGamma3D", c_float),
                ("materialBrightness3D", c_float)]


class VolumeView(ctypes.Structure):
    """seis3d_volume_view: uniforms of the raymarched volume (shaders/seis3d_volume.frag:4-12)."""

    _fields_ = [("extent3D", c_float * 3), ("pan3D", c_float * 2), ("domainLow3D", c_float * 3),
                ("domainHigh3D", c_float * 3), ("physicalLow3D", c_float * 3), ("physicalHigh3D", c_float * 3),
                ("showBoundary3D", c_int), ("boundaryOpacity3D", c_float), ("yaw3D", c_float), ("pitch3D", c_float),
                ("distance3D", c_float), ("scale3D", c_float), ("gain3D", c_float), ("opacity3D", c_float),
                ("threshold3D", c_float), ("aspect3D", c_float), ("sampling3D", c_float), ("sharpness3D", c_float),
                ("volumeGain3D", c_float), ("opticalScale3D", c_float)]


class Display(ctypes.Structure):
    """seis3d_display: the workspace display settings (Seis3D_State, include/Seis3D_Sim.h:110-160)."""

    _fields_ = [("displayMode3D", c_int), ("waveStyle3D", c_int), ("modelStyle3D", c_int), ("component3D", c_int),
                ("materialRangeAuto3D", c_int), ("materialRange3D", c_float * 2),
                ("manualMaterialRange3D", c_float * 2), ("waveOpacity3D", c_float), ("waveThreshold3D", c_float),
                ("modelOpacity3D", c_float), ("waveGamma3D", c_float), ("materialBrightness3D", c_float),
                ("gain3D", c_float), ("scale3D", c_float), ("showBoundary3D", c_int), ("boundaryOpacity3D", c_float),
                ("yaw3D", c_float), ("pitch3D", c_float), ("distance3D", c_float), ("pan3D", c_float * 2),
                ("volumeOpacity3D", c_float), ("volumeThreshold3D", c_float), ("volumeSampling3D", c_float),
                ("volumeSharpness3D", c_float), ("volumeGain3D", c_float), ("volumeSizeCompensation3D", c_int),
                ("volumeRequestedWidth3D", c_int), ("volumeRequestedHeight3D", c_int)]


class BatchOptions(ctypes.Structure):
    """seis3d_batch_options (no reference counterpart)."""

    _fields_ = [("shots_per_launch", c_int), ("z_chunk", c_int), ("tune", c_int), ("reserved", c_int * 5)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("shots", c_int), ("shots_per_launch", c_int), ("z_chunk", c_int), ("tuned", c_int),
                ("candidates", c_int), ("tuned_ms_per_step", c_float), ("kernel_launches", c_uint64),
                ("stream", c_void_p)]


MAX_BATCH_SHOTS = 64

PIXELS_RGBA8 = 0
PIXELS_RGBA32F = 1

SIGNATURES = {
    "seis3d_last_error": (c_char_p, []),
    "seis3d_abi_version": (c_int, []),
    "seis3d_default_context": (None, [POINTER(Context)]),
    "seis3d_default_source": (None, [POINTER(Source)]),
    "seis3d_validate_context": (c_int, [POINTER(Context)]),
    "seis3d_estimate_memory": (c_int, [POINTER(Context), POINTER(MemoryBudget)]),
    "seis3d_make_view_layout": (c_int, [POINTER(Context), POINTER(ViewLayout)]),
    "seis3d_make_cpml_coefficients": (c_int, [POINTER(Context), c_int, POINTER(c_float), c_size_t]),
    "seis3d_initialize": (c_int, [POINTER(c_void_p), POINTER(Context), POINTER(Options)]),
    "seis3d_release": (None, [c_void_p]),
    "seis3d_reset": (c_int, [c_void_p, POINTER(Context)]),
    "seis3d_refresh_cpml": (c_int, [c_void_p, POINTER(Context)]),
    "seis3d_run_step": (c_int, [c_void_p, POINTER(Context), POINTER(Source), c_uint64]),
    "seis3d_run_steps": (c_int, [c_void_p, POINTER(Context), POINTER(Source), c_uint64, c_int]),
    "seis3d_prepare_steps": (c_int, [c_void_p, POINTER(Context), POINTER(Source)]),
    "seis3d_set_receivers": (c_int, [c_void_p, POINTER(Context), POINTER(Receiver), c_int]),
    "seis3d_sample_receivers": (c_int, [c_void_p, POINTER(Context), POINTER(POINTER(c_float))]),
    "seis3d_probe_material": (c_int, [c_void_p, POINTER(Context), POINTER(Receiver), POINTER(c_float)]),
    "seis3d_upload_model_plane": (c_int, [c_void_p, POINTER(Context), c_int, POINTER(c_float)]),
    "seis3d_finish_model_upload": (c_int, [c_void_p, POINTER(Context)]),
    "seis3d_download_model_plane": (c_int, [c_void_p, POINTER(Context), c_int, POINTER(c_float)]),
    "seis3d_gather_begin": (c_int, [c_void_p, c_int, c_int]),
    "seis3d_gather_fetch": (c_int, [c_void_p, POINTER(c_float), c_size_t, POINTER(c_int)]),
    "seis3d_gather_end": (c_int, [c_void_p]),
    "seis3d_get_views": (c_int, [c_void_p, POINTER(DeviceViews)]),
    "seis3d_get_z_chunk": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "seis3d_copy_field": (c_int, [c_void_p, c_int, c_int, POINTER(c_float)]),
    "seis3d_upload_model": (c_int, [c_void_p, POINTER(Context), POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
    "seis3d_default_survey": (None, [POINTER(Survey)]),
    "seis3d_freeze_gather": (c_int, [POINTER(GatherRecord)]),
    "seis3d_cmp_bin": (c_int, [POINTER(GatherRecord), POINTER(Receiver), POINTER(c_int), POINTER(c_int)]),
    "seis3d_write_segy_component": (c_int, [POINTER(GatherRecord), c_char_p, c_int]),
    "seis3d_export_gather": (c_int, [POINTER(GatherRecord), c_char_p, c_char_p]),
    "seis3d_inspect_model": (c_int, [c_char_p, POINTER(Context)]),
    "seis3d_read_model_plane": (c_int, [c_char_p, POINTER(Context), c_int, POINTER(c_float)]),
    "seis3d_import_model": (c_int, [c_void_p, POINTER(Context), c_char_p]),
    "seis3d_export_model": (c_int, [c_void_p, POINTER(Context), c_char_p]),
    "seis3d_write_model": (c_int, [c_char_p, POINTER(Context), POINTER(c_float)]),
    "seis3d_extract_views": (c_int, [c_void_p, POINTER(Context), c_void_p, POINTER(ViewLayout), POINTER(c_int), c_int,
                                     c_int, c_int, c_int, POINTER(c_float), POINTER(c_float), POINTER(c_float)]),
    "seis3d_default_display": (None, [POINTER(Display)]),
    "seis3d_wave_palette": (None, [c_int, POINTER(c_float)]),
    "seis3d_make_display_uniforms": (c_int, [POINTER(Context), POINTER(ViewLayout), POINTER(Display),
                                             POINTER(Transfer), POINTER(VolumeView), POINTER(c_int), POINTER(c_int)]),
    "seis3d_shade_slices": (c_int, [c_void_p, POINTER(ViewLayout), c_void_p, POINTER(Transfer), c_float, c_float, c_int,
                                    c_void_p]),
    "seis3d_render_volume": (c_int, [c_void_p, POINTER(ViewLayout), c_void_p, POINTER(Transfer), POINTER(VolumeView),
                                     c_int, c_int, c_int, c_void_p]),
    "seis3d_batch_create": (c_int, [POINTER(c_void_p), POINTER(c_void_p), c_int, POINTER(BatchOptions)]),
    "seis3d_batch_run_steps": (c_int, [c_void_p, POINTER(Source), c_uint64, c_int]),
    "seis3d_batch_synchronize": (c_int, [c_void_p]),
    "seis3d_batch_get_info": (c_int, [c_void_p, POINTER(BatchInfo)]),
    "seis3d_batch_release": (None, [c_void_p]),
    "seis3d_checkpoint_bytes": (c_int, [c_void_p, POINTER(c_uint64)]),
    "seis3d_save_checkpoint": (c_int, [c_void_p, c_void_p, c_uint64]),
    "seis3d_load_checkpoint": (c_int, [c_void_p, c_void_p, c_uint64]),
    "seis3d_write_checkpoint": (c_int, [c_void_p, c_char_p]),
    "seis3d_read_checkpoint": (c_int, [c_void_p, c_char_p]),
    "seis3d_profile_steps": (c_int, [c_void_p, POINTER(Context), POINTER(Source), c_uint64, c_int, POINTER(c_float)]),
    "seis3d_synchronize": (c_int, [c_void_p]),
    "seis3d_debug_fail_allocation": (None, [c_int]),
    "seis3d_debug_stage_wait": (c_int, [c_void_p, ctypes.c_longlong, c_int]),
    "seis3d_validate_thin_context": (c_int, [POINTER(Context)]),
    "seis3d_boundary_net_create": (c_int, [POINTER(c_void_p), c_int, c_uint64]),
    "seis3d_boundary_net_release": (None, [c_void_p]),
    "seis3d_boundary_net_get": (c_int, [c_void_p, c_int, POINTER(c_float), POINTER(c_float)]),
    "seis3d_boundary_net_set": (c_int, [c_void_p, c_int, POINTER(c_float), c_float]),
    "seis3d_boundary_dataset_create": (c_int, [POINTER(c_void_p), c_uint64]),
    "seis3d_boundary_dataset_release": (None, [c_void_p]),
    "seis3d_boundary_dataset_rows": (c_int, [c_void_p, POINTER(c_uint64)]),
    "seis3d_boundary_begin_model": (c_int, [c_void_p]),
    "seis3d_boundary_dataset_read": (c_int, [c_void_p, c_int, c_uint64, c_uint64, POINTER(c_float), POINTER(c_float),
                                             POINTER(c_float)]),
    "seis3d_boundary_collect": (c_int, [c_void_p, c_void_p, c_void_p, c_float, c_uint64]),
    "seis3d_boundary_train": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_float, c_uint64, POINTER(c_float)]),
    "seis3d_boundary_gradients": (c_int, [c_void_p, c_int, POINTER(c_float), POINTER(c_float), POINTER(c_float), c_int,
                                          POINTER(c_float), POINTER(c_float)]),
    "seis3d_boundary_attach": (c_int, [c_void_p, c_void_p, c_float]),
    "seis3d_non_finite": (c_int, [c_void_p, POINTER(c_int)]),
    "seis3d_sample_receivers_noalloc": (c_int, [POINTER(Context), c_void_p, c_void_p, c_void_p, c_int64,
                                                POINTER(Receiver), c_int, POINTER(c_float), c_void_p]),
    "seis3d_noalloc_last_error": (c_char_p, []),
}

_LIB = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Open the solver library (once).  Raises OSError when it has not been built."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    target = path or LIBRARY_PATH
    if not os.path.exists(target):
        raise OSError(f"{target} is missing: build it with `python -m cmakepro_cuda_seissim_v2_b200.build` "
                      "(the solver has no CPU fallback)")
    lib = ctypes.CDLL(target)
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if path is None:
        _LIB = lib
    return lib
