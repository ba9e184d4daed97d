"""Host-side mirror of the reference 2-D P-SV solver interface over its C ABI.

The names, argument meanings and error behaviour follow the reference:

* ``SimulationContext`` is the struct of Main_header/Common.h:259-287 (``lambda`` is spelled
  ``lambda_`` because it is a Python keyword); vectors are numpy arrays.
* ``validateSimulationContext``, ``initializeGpuSimulation``, ``releaseGpuSimulation``,
  ``updateGpuReceivers``, ``runGpuSimulationStep``, ``copyWavefieldToHost``,
  ``copyReceiverRecordsFromGpu`` and ``recordReceiverStepOnGpu`` are the functions of
  CUDA_Kernels/Cuda_Check.cuh:126-149; ``GPUSimData`` exposes the device pointers under the
  member names of Cuda_Check.cuh:68-121.
* ``checkedGridElementCount``, ``validateBoundaryGeometry``, ``getReceiverSamplingStride`` and
  the constants are Main_header/SolverNumerics.h; ``generateRickerWavelet`` and
  ``updatePmlDampingArrays`` are src/Seis2D/Numerics2D.inc.

std::invalid_argument maps to :class:`InvalidArgument` (a ValueError), std::overflow_error to
OverflowError, std::logic_error to :class:`LogicError`, CUDA failures to :class:`SolverError`.
Every solver call runs the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_float, c_int, c_int64, c_void_p

import numpy as np

from . import capi2d
from .seis3d import InvalidArgument, LogicError, SolverError

kStencilRadius = capi2d.STENCIL_RADIUS
kMaximumActiveSources = capi2d.MAX_ACTIVE_SOURCES
kSourceInjectionScale2D = np.float32(capi2d.SOURCE_INJECTION_SCALE)
kStaggeredDerivativeWeights = (1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0)
kSafeCourant2d = np.float32(0.48)


def _lib():
    return capi2d.load()


def kCourantLimit2d() -> float:
    return float(_lib().seis2d_courant_limit())


def _check(status: int) -> None:
    if status == capi2d.SEIS2D_OK:
        return
    message = (_lib().seis2d_last_error() or b"").decode(errors="replace")
    if status == capi2d.SEIS2D_INVALID_ARGUMENT:
        raise InvalidArgument(message)
    if status == capi2d.SEIS2D_OVERFLOW_ERROR:
        raise OverflowError(message)
    if status == capi2d.SEIS2D_LOGIC_ERROR:
        raise LogicError(message)
    raise SolverError(message)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _fview(a: np.ndarray) -> capi2d.FloatView:
    if a.size == 0:
        return capi2d.FloatView(None, 0)
    return capi2d.FloatView(a.ctypes.data_as(POINTER(c_float)), a.size)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_float))


class SimulationContext:
    """SimulationContext (Main_header/Common.h:259-287)."""

    _ARRAYS = ("rho", "mu", "lambda_", "lambda2mu", "dp_flat", "dx", "dx_half", "dz", "dz_half", "wavelet")

    def __init__(self, **values):
        self.NX = self.NZ = self.total_grid = 0
        self.h = self.dt = 0.0
        self.nt = self.npml = self.snap_spacenum = 0
        self.flag_type = 1
        for name in self._ARRAYS:
            setattr(self, name, np.zeros(0, dtype=np.float32))
        self.c1_h = self.c2_h = self.c3_h = self.c4_h = 0.0
        self.src_idx = self.src_z_idx = 0
        self.src_angle = 0.0
        self.src_type = 0
        self.src_amp = 1.0
        self.num_rcv = 0
        self.rcv_grid_idx = np.zeros(0, dtype=np.int32)
        self.upFlag = False
        for k, v in values.items():
            setattr(self, k, v)

    def copy(self) -> "SimulationContext":
        other = SimulationContext()
        for k, v in self.__dict__.items():
            setattr(other, k, v.copy() if isinstance(v, np.ndarray) else v)
        return other

    def to_c(self) -> capi2d.Context:
        """The C view of this context; the arrays it points at are kept on the returned object."""
        keep = {name: _f32(getattr(self, name)) for name in self._ARRAYS}
        rcv = np.ascontiguousarray(np.asarray(self.rcv_grid_idx, dtype=np.int32))
        c = capi2d.Context()
        c.NX, c.NZ, c.total_grid = int(self.NX), int(self.NZ), int(self.total_grid)
        c.h, c.dt = float(self.h), float(self.dt)
        c.nt, c.npml, c.snap_spacenum, c.flag_type = int(self.nt), int(self.npml), int(self.snap_spacenum), int(self.flag_type)
        c.rho, c.mu, c.lambda_, c.lambda2mu = (_fview(keep[n]) for n in ("rho", "mu", "lambda_", "lambda2mu"))
        c.dp_flat = _fview(keep["dp_flat"])
        c.dx, c.dx_half, c.dz, c.dz_half = (_fview(keep[n]) for n in ("dx", "dx_half", "dz", "dz_half"))
        c.c1_h, c.c2_h, c.c3_h, c.c4_h = float(self.c1_h), float(self.c2_h), float(self.c3_h), float(self.c4_h)
        c.src_idx, c.src_z_idx = int(self.src_idx), int(self.src_z_idx)
        c.wavelet = _fview(keep["wavelet"])
        c.src_angle, c.src_type, c.src_amp = float(self.src_angle), int(self.src_type), float(self.src_amp)
        c.num_rcv = int(self.num_rcv)
        c.rcv_grid_idx = (capi2d.IntView(rcv.ctypes.data_as(POINTER(c_int)), rcv.size) if rcv.size
                          else capi2d.IntView(None, 0))
        c.upFlag = int(bool(self.upFlag))
        c._keep = (keep, rcv)
        return c


class GPUSimData:
    """Handle of one device simulation; the GPUSimData members are read from the library.

    ``d_vx_1`` ... ``d_rho_orig_flat``, ``d_dx`` ..., ``d_active_sources``, ``d_rcv_grid_idx``
    are device addresses (ints, 0 when absent), valid until the next initialize/release.
    """

    def __init__(self):
        self._handle = c_void_p()

    @property
    def handle(self) -> c_void_p:
        return self._handle

    @property
    def initialized(self) -> bool:
        return bool(self._handle.value)

    def views(self) -> capi2d.DeviceViews:
        v = capi2d.DeviceViews()
        if not self.initialized:
            return v
        _check(_lib().seis2d_get_views(self._handle, byref(v)))
        return v

    def __getattr__(self, name):
        if name.startswith("d_") and name[2:] in capi2d.FIELD:
            return self.views().field[capi2d.FIELD[name[2:]]] or 0
        if name in ("d_sigmaxx", "d_sigmazz", "d_sigmaxz"):
            return self.views().field[capi2d.FIELD[name[2:]]] or 0
        if name in ("d_dx", "d_dx_half", "d_dz", "d_dz_half", "d_dp_flat", "d_wavelet", "d_rcv_grid_idx",
                    "d_record_vx_step", "d_record_vz_step", "d_active_sources", "NX", "NZ", "total_grid", "dt",
                    "inv_dt", "flag_type", "npml", "fs_idx", "upFlag", "receiverCapacity", "c1_h", "c2_h", "c3_h",
                    "c4_h", "kernelLaunches", "stream"):
            return getattr(self.views(), name) or 0
        raise AttributeError(name)

    def __del__(self):
        try:
            releaseGpuSimulation(self)
        except Exception:
            pass


# ---- SolverNumerics.h --------------------------------------------------------------------

def checkedGridElementCount(nx: int, nz: int) -> int:
    n = c_int64()
    _check(_lib().seis2d_checked_grid_element_count(int(nx), int(nz), byref(n)))
    return n.value


def validateBoundaryGeometry(nx: int, nz: int, pml_width: int, free_surface: bool) -> None:
    _check(_lib().seis2d_validate_boundary_geometry(int(nx), int(nz), int(pml_width), int(bool(free_surface))))


def getReceiverSamplingStride(time_step: float, sampling_rate_hz: float) -> int:
    s = c_int()
    _check(_lib().seis2d_receiver_sampling_stride(float(time_step), float(sampling_rate_hz), byref(s)))
    return s.value


# ---- src/Seis2D/Numerics2D.inc -------------------------------------------------------------

def generateRickerWavelet(nt: int, dt: float, f0: float, t0: float) -> np.ndarray:
    out = np.zeros(max(int(nt), 1), dtype=np.float32)
    _check(_lib().seis2d_generate_ricker(_fptr(out), int(nt), float(dt), float(f0), float(t0)))
    return out[: int(nt)]


def updatePmlDampingArrays(ctx: SimulationContext) -> None:
    dx, dxh = np.zeros(ctx.NX, np.float32), np.zeros(ctx.NX, np.float32)
    dz, dzh = np.zeros(ctx.NZ, np.float32), np.zeros(ctx.NZ, np.float32)
    c = ctx.to_c()
    _check(_lib().seis2d_update_pml_damping(byref(c), _fptr(dx), _fptr(dxh), _fptr(dz), _fptr(dzh)))
    ctx.dx, ctx.dx_half, ctx.dz, ctx.dz_half = dx, dxh, dz, dzh


def freeSurfaceModulus(ctx: SimulationContext) -> None:
    """dp_flat of setupTestContext (src/Seis2D/Numerics2D.inc:124-135)."""
    dp = np.zeros(ctx.NX, np.float32)
    c = ctx.to_c()
    _check(_lib().seis2d_free_surface_modulus(byref(c), _fptr(dp)))
    ctx.dp_flat = dp


def setGridMaterial(ctx: SimulationContext, x: int, z: int, vp: float, vs: float, rho: float) -> None:
    """setGridMaterial2D (src/Seis2D/Numerics2D.inc:159-166), FP32 arithmetic."""
    if x < 0 or x >= ctx.NX or z < 0 or z >= ctx.NZ:
        return
    k = z * ctx.NX + x
    rho, vp, vs = np.float32(rho), np.float32(vp), np.float32(vs)
    ctx.rho[k] = rho
    ctx.mu[k] = rho * vs * vs
    ctx.lambda2mu[k] = rho * vp * vp
    ctx.lambda_[k] = ctx.lambda2mu[k] - np.float32(2.0) * ctx.mu[k]


def stencil_coefficients(h: float) -> tuple[float, float, float, float]:
    """c_k_h = float(w_k) / h in FP32 (setupTestContext, src/Seis2D/Numerics2D.inc:103-106)."""
    return tuple(float(np.float32(np.float32(w) / np.float32(h))) for w in kStaggeredDerivativeWeights)


# ---- CUDA_Kernels/Cuda_Check.cuh -----------------------------------------------------------

def validateSimulationContext(ctx: SimulationContext) -> None:
    c = ctx.to_c()
    _check(_lib().seis2d_validate_context(byref(c)))


def initializeGpuSimulation(gpu: GPUSimData, ctx: SimulationContext) -> None:
    c = ctx.to_c()
    _check(_lib().seis2d_initialize(byref(gpu._handle), byref(c)))


def releaseGpuSimulation(gpu: GPUSimData) -> None:
    if gpu._handle.value:
        _lib().seis2d_release(gpu._handle)
        gpu._handle = c_void_p()


def _session(gpu: GPUSimData) -> c_void_p:
    return gpu._handle if gpu._handle.value else None


def updateGpuReceivers(gpu: GPUSimData, receiver_indices) -> None:
    idx = np.ascontiguousarray(np.asarray(receiver_indices, dtype=np.int64))
    if idx.size and (idx.min() < np.iinfo(np.int32).min or idx.max() > np.iinfo(np.int32).max):
        raise InvalidArgument("Receiver index is outside the active GPU grid")
    idx = idx.astype(np.int32)
    ptr = idx.ctypes.data_as(POINTER(c_int)) if idx.size else None
    _check(_lib().seis2d_update_receivers(_session(gpu), ptr, int(idx.size)))


def setActiveSources(gpu: GPUSimData, sources) -> None:
    """Copies GPUSource entries (idx, t, f_peak, amp) into the device array the multi-source
    injection reads (the caller side of src/Seis2D/Workflow2D.inc:314)."""
    sources = list(sources)
    arr = (capi2d.Source * max(len(sources), 1))(*[capi2d.Source(int(i), float(t), float(f), float(a))
                                                    for i, t, f, a in sources])
    _check(_lib().seis2d_set_active_sources(_session(gpu), arr, len(sources)))


def runGpuSimulationStep(gpu: GPUSimData, current_it: int, ctx: SimulationContext, num_active_sources: int) -> None:
    c = ctx.to_c()
    _check(_lib().seis2d_run_step(_session(gpu), int(current_it), byref(c), int(num_active_sources)))


def runGpuSimulationSteps(gpu: GPUSimData, first_it: int, count: int, ctx: SimulationContext,
                          num_active_sources: int = -1) -> None:
    """``count`` steps from ``first_it`` replayed from a CUDA graph (equal to ``count`` calls of
    runGpuSimulationStep; active sources advance like the reference time loop)."""
    c = ctx.to_c()
    _check(_lib().seis2d_run_steps(_session(gpu), int(first_it), int(count), byref(c), int(num_active_sources)))


def setRunMode(gpu: GPUSimData, mode: int) -> None:
    """capi2d.RUN_PERSISTENT (default) or capi2d.RUN_GRAPH for runGpuSimulationSteps."""
    _check(_lib().seis2d_set_run_mode(_session(gpu), int(mode)))


def generateWavefieldTextureOnGpu(gpu: GPUSimData, device_rgba_ptr: int, color_scale: float, component: int) -> None:
    """generateWavefieldTextureOnGpu (Cuda_Check.cu:1136-1141): NX * NZ RGBA8 pixels of the
    selected component into a device buffer (e.g. a CUDA tensor's data_ptr()), enqueued on the
    session stream."""
    _check(_lib().seis2d_wavefield_texture(_session(gpu), ctypes.c_void_p(int(device_rgba_ptr)), float(color_scale),
                                           int(component)))


def copyWavefieldToHost(gpu: GPUSimData, out: np.ndarray | None = None) -> np.ndarray:
    v = gpu.views()
    if out is None:
        out = np.zeros(max(v.total_grid, 1), dtype=np.float32)
    if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < v.total_grid:
        raise InvalidArgument("Invalid wavefield output buffer")
    _check(_lib().seis2d_copy_wavefield(_session(gpu), _fptr(out)))
    return out


def copyReceiverRecordsFromGpu(gpu: GPUSimData, num_rcv: int, nt: int, current_it: int, rec_vx: np.ndarray,
                               rec_vz: np.ndarray) -> None:
    for a in (rec_vx, rec_vz):
        if a.dtype != np.float32 or not a.flags.c_contiguous or (num_rcv > 0 and a.size < num_rcv * nt):
            raise InvalidArgument("Invalid receiver trace count, time index, or host output buffer")
    _check(_lib().seis2d_copy_receiver_records(_session(gpu), int(num_rcv), int(nt), int(current_it), _fptr(rec_vx),
                                               _fptr(rec_vz)))


def recordReceiverStepOnGpu(gpu: GPUSimData, num_rcv: int, out_vx: np.ndarray | None = None,
                            out_vz: np.ndarray | None = None):
    n = max(int(num_rcv), 1)
    out_vx = np.zeros(n, np.float32) if out_vx is None else out_vx
    out_vz = np.zeros(n, np.float32) if out_vz is None else out_vz
    for a in (out_vx, out_vz):
        if a.dtype != np.float32 or not a.flags.c_contiguous or a.size < num_rcv:
            raise InvalidArgument("Invalid receiver count or host output buffer")
    _check(_lib().seis2d_record_receiver_step(_session(gpu), int(num_rcv), _fptr(out_vx), _fptr(out_vz)))
    return out_vx, out_vz


# ---- device-resident recording and inspection -----------------------------------------------

def gatherBegin(gpu: GPUSimData, capture_start_step: int, stride: int, samples: int) -> None:
    _check(_lib().seis2d_gather_begin(_session(gpu), int(capture_start_step), int(stride), int(samples)))


def gatherFetch(gpu: GPUSimData, samples: int):
    """(vx, vz, taken): [receiver][sample] float32 traces and the samples recorded so far."""
    n = max(gpu.views().receiverCapacity, 1)
    vx = np.zeros((n, samples), np.float32)
    vz = np.zeros((n, samples), np.float32)
    taken = c_int()
    _check(_lib().seis2d_gather_fetch(_session(gpu), _fptr(vx), _fptr(vz), int(samples), byref(taken)))
    return vx, vz, taken.value


def gatherEnd(gpu: GPUSimData) -> None:
    _check(_lib().seis2d_gather_end(_session(gpu)))


def copyField(gpu: GPUSimData, name: str) -> np.ndarray:
    v = gpu.views()
    out = np.zeros((v.NZ, v.NX), np.float32)
    _check(_lib().seis2d_copy_field(_session(gpu), capi2d.FIELD[name], _fptr(out)))
    return out


def setField(gpu: GPUSimData, name: str, values) -> None:
    v = gpu.views()
    a = _f32(values).reshape(-1)
    if a.size != v.total_grid:
        raise InvalidArgument("field size must equal total_grid")
    _check(_lib().seis2d_set_field(_session(gpu), capi2d.FIELD[name], _fptr(a)))


def writeDevice(gpu: GPUSimData, device_address: int, values: np.ndarray) -> None:
    """cudaMemcpy host -> device into one of the session's own buffers."""
    a = np.ascontiguousarray(values)
    _check(_lib().seis2d_write_device(_session(gpu), c_void_p(int(device_address)), a.ctypes.data_as(c_void_p),
                                      a.nbytes))


def readDevice(gpu: GPUSimData, device_address: int, count: int, dtype=np.float32) -> np.ndarray:
    out = np.zeros(int(count), dtype=dtype)
    _check(_lib().seis2d_read_device(_session(gpu), out.ctypes.data_as(c_void_p), c_void_p(int(device_address)),
                                     out.nbytes))
    return out


def synchronize(gpu: GPUSimData) -> None:
    _check(_lib().seis2d_synchronize(_session(gpu)))


def profileSteps(gpu: GPUSimData, first_it: int, count: int, ctx: SimulationContext) -> dict:
    ms = (c_float * 3)()
    c = ctx.to_c()
    _check(_lib().seis2d_profile_steps(_session(gpu), int(first_it), int(count), byref(c), ms))
    return {"total_ms": ms[0], "stress_ms": ms[1], "velocity_ms": ms[2]}
