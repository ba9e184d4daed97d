"""Python host mirror of the SeisWave Lab ``Seis3D`` solver API on the B200 library.

Every function here calls one entry point of include/seis3d_capi.h and keeps the meaning
of the reference free function it stands for (cuda/Cuda_Seis3D.cuh:7-42); the status
codes of the C ABI come back as the exception classes the reference throws:

    std::invalid_argument -> InvalidArgument (a ValueError)
    std::logic_error      -> LogicError      (a RuntimeError)
    std::runtime_error    -> SolverError     (a RuntimeError)
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_int, c_void_p
from typing import Iterable, Sequence

import numpy as np

from . import capi
from .capi import Context, MemoryBudget, Options, Receiver, Source, ViewLayout


class InvalidArgument(ValueError):
    """std::invalid_argument of the reference (input rejected before any allocation)."""


class LogicError(RuntimeError):
    """std::logic_error of the reference (lifecycle misuse)."""


class SolverError(RuntimeError):
    """std::runtime_error of the reference (CUDA failure, VRAM budget, non-finite field)."""


def _lib():
    return capi.load()


def _check(status: int) -> None:
    if status == capi.SEIS3D_OK:
        return
    message = (_lib().seis3d_last_error() or b"").decode(errors="replace")
    if status == capi.SEIS3D_INVALID_ARGUMENT:
        raise InvalidArgument(message)
    if status == capi.SEIS3D_LOGIC_ERROR:
        raise LogicError(message)
    raise SolverError(message)


def default_context(**overrides) -> Context:
    """SimulationContext3D defaults (include/Common3D.h:24-42), then `overrides`."""
    c = Context()
    _lib().seis3d_default_context(byref(c))
    for key, value in overrides.items():
        if not hasattr(c, key):
            raise AttributeError(key)
        setattr(c, key, value)
    return c


def default_source(**overrides) -> Source:
    """Source3D defaults (include/Common3D.h:44-49), then `overrides`."""
    s = Source()
    _lib().seis3d_default_source(byref(s))
    for key, value in overrides.items():
        if key == "direction3D":
            for a in range(3):
                s.direction3D[a] = float(value[a])
        else:
            setattr(s, key, value)
    return s


def validate_context3D(c: Context) -> Context:
    """validateContext3D: derive padding, offsets and dt in place (cuda/Cuda_Seis3D.cu:433-483)."""
    _check(_lib().seis3d_validate_context(byref(c)))
    return c


def validate_thin_context3D(c: Context) -> Context:
    """validateContext3D with the learned boundary's thin CPML (4..40 cells) allowed."""
    _check(_lib().seis3d_validate_thin_context(byref(c)))
    return c


def estimate_memory3D(c: Context) -> MemoryBudget:
    """estimateMemory3D (cuda/Cuda_Seis3D.cu:504-516)."""
    b = MemoryBudget()
    _check(_lib().seis3d_estimate_memory(byref(c), byref(b)))
    return b


def make_view_layout3D(c: Context) -> ViewLayout:
    """makeViewLayout3D (cuda/Cuda_Seis3D.cu:486-501)."""
    layout = ViewLayout()
    _check(_lib().seis3d_make_view_layout(byref(c), byref(layout)))
    return layout


def make_cpml_coefficients3D(c: Context, axis: int) -> np.ndarray:
    """makeCoefficients3D (cuda/Cuda_Seis3D.cu:45-64) as float32 [2][n][3]."""
    n = (c.gx3D, c.gy3D, c.gz3D)[axis]
    out = np.zeros(n * 6, dtype=np.float32)
    _check(_lib().seis3d_make_cpml_coefficients(byref(c), axis, out.ctypes.data_as(ctypes.POINTER(c_float)), out.size))
    return out.reshape(2, n, 3)


def default_display(**overrides) -> capi.Display:
    """The workspace display defaults (Seis3D_State, include/Seis3D_Sim.h:110-160)."""
    d = capi.Display()
    _lib().seis3d_default_display(byref(d))
    for k, v in overrides.items():
        field = getattr(d, k)
        if isinstance(field, ctypes.Array):
            for i, x in enumerate(v):
                field[i] = x
        else:
            setattr(d, k, v)
    return d


def wave_palette(style: int) -> np.ndarray:
    """The five [r, g, b] stops of wave style `style` (Main_header/WavePalettes.h:9-29)."""
    out = np.zeros((5, 3), np.float32)
    _lib().seis3d_wave_palette(int(style), out.ctypes.data_as(ctypes.POINTER(c_float)))
    return out


def make_display_uniforms(c: Context, layout: ViewLayout, display: capi.Display):
    """(transfer, volume, width, height): the shader uniforms Renderer3D derives from the display
    settings (src/Seis3D/Renderer3D.cpp:148-160, 224-267)."""
    t, u, w, h = capi.Transfer(), capi.VolumeView(), c_int(), c_int()
    _check(_lib().seis3d_make_display_uniforms(byref(c), byref(layout), byref(display), byref(t), byref(u), byref(w),
                                               byref(h)))
    return t, u, w.value, h.value


def receivers_array(receivers: Iterable[Sequence[int]] | np.ndarray):
    rec = np.asarray(list(receivers) if not isinstance(receivers, np.ndarray) else receivers, dtype=np.int32)
    rec = rec.reshape(-1, 3)
    arr = (Receiver * max(1, len(rec)))()
    for k, (x, y, z) in enumerate(rec):
        arr[k].x3D, arr[k].y3D, arr[k].z3D = int(x), int(y), int(z)
    return arr, len(rec)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(c_float))


class Session:
    """One solver session on the current CUDA device (GPUSimData3D + its stream).

    Construction is initializeGpu3D (cuda/Cuda_Seis3D.cu:519-555); `release` is
    releaseGpu3D and is idempotent.  Methods take the caller's context as the reference
    functions do; it must describe the session's grid.
    """

    def __init__(self, context: Context, storage: int = capi.STORAGE_FP32, tile_y: int = 0, z_chunk: int = 0,
                 compact_rows: bool = False, tune: bool = False, thin_cpml: bool = False):
        self._handle = c_void_p()
        opts = Options()
        opts.storage, opts.tile_y, opts.z_chunk = storage, tile_y, z_chunk
        opts.compact_rows = int(bool(compact_rows))
        opts.tune = int(bool(tune))
        opts.thin_cpml = int(bool(thin_cpml))
        self.context = context.copy()
        _check(_lib().seis3d_initialize(byref(self._handle), byref(self.context), byref(opts)))
        if thin_cpml:
            validate_thin_context3D(self.context)
        else:
            validate_context3D(self.context)
        self.receiver_count = 0

    # lifecycle --------------------------------------------------------------------------
    def release(self) -> None:
        if self._handle:
            _lib().seis3d_release(self._handle)
            self._handle = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    @property
    def handle(self) -> c_void_p:
        return self._handle

    def _ctx(self, context: Context | None) -> Context:
        return self.context if context is None else context

    def reset(self, context: Context | None = None) -> None:
        """resetGpu3D (cuda/Cuda_Seis3D.cu:572-577)."""
        _check(_lib().seis3d_reset(self._handle, byref(self._ctx(context))))

    def refresh_cpml(self, context: Context) -> None:
        """refreshCpmlCoefficients3D (cuda/Cuda_Seis3D.cu:580-599)."""
        _check(_lib().seis3d_refresh_cpml(self._handle, byref(context)))
        self.context = context.copy()

    # stepping ---------------------------------------------------------------------------
    def run_step(self, source: Source, step: int, context: Context | None = None) -> None:
        """runStep3D (cuda/Cuda_Seis3D.cu:602-624)."""
        _check(_lib().seis3d_run_step(self._handle, byref(self._ctx(context)), byref(source), int(step)))

    def run_steps(self, source: Source, first: int, count: int, context: Context | None = None) -> None:
        """`count` steps from `first`, replayed from a captured CUDA graph."""
        _check(_lib().seis3d_run_steps(self._handle, byref(self._ctx(context)), byref(source), int(first), int(count)))

    def prepare_steps(self, source: Source, context: Context | None = None) -> None:
        """Capture the step graph for `source` ahead of time (no step is executed)."""
        _check(_lib().seis3d_prepare_steps(self._handle, byref(self._ctx(context)), byref(source)))

    def profile_steps(self, source: Source, first: int, count: int, context: Context | None = None) -> dict:
        """Per-pass device times (ms, summed over `count` steps run without a graph)."""
        ms = (c_float * 4)()
        _check(_lib().seis3d_profile_steps(self._handle, byref(self._ctx(context)), byref(source), int(first),
                                           int(count), ms))
        return {"velocity": ms[0], "stress": ms[1], "images_tail": ms[2], "step": ms[3]}

    # receivers ---------------------------------------------------------------------------
    def set_receivers(self, receivers, context: Context | None = None) -> None:
        """setReceivers3D (cuda/Cuda_Seis3D.cu:649-668); `receivers` is [(x, y, z)]."""
        arr, n = receivers_array(receivers)
        _check(_lib().seis3d_set_receivers(self._handle, byref(self._ctx(context)), arr, n))
        self.receiver_count = n

    def sample_receivers(self, context: Context | None = None) -> np.ndarray | None:
        """sampleReceivers3D (cuda/Cuda_Seis3D.cu:671-681): float32 [r][vx, vy, vz]."""
        ptr = ctypes.POINTER(c_float)()
        _check(_lib().seis3d_sample_receivers(self._handle, byref(self._ctx(context)), byref(ptr)))
        if not ptr:
            return None
        return np.ctypeslib.as_array(ptr, shape=(self.receiver_count * 3,)).reshape(self.receiver_count, 3).copy()

    def gather_begin(self, stride: int, target_samples: int) -> None:
        _check(_lib().seis3d_gather_begin(self._handle, int(stride), int(target_samples)))
        self._gather_target = int(target_samples)

    def gather_fetch(self) -> np.ndarray:
        """Recorded samples as float32 [sample][receiver][vx, vy, vz]."""
        count = c_int()
        cap = getattr(self, "_gather_target", 0) * max(self.receiver_count, 1) * 3
        out = np.zeros(max(cap, 1), dtype=np.float32)
        _check(_lib().seis3d_gather_fetch(self._handle, _fptr(out), out.size, byref(count)))
        n = count.value
        return out[: n * self.receiver_count * 3].reshape(n, self.receiver_count, 3)

    def gather_end(self) -> None:
        _check(_lib().seis3d_gather_end(self._handle))

    # materials ---------------------------------------------------------------------------
    def probe_material(self, point: Sequence[int], context: Context | None = None) -> np.ndarray:
        """probeMaterial3D (cuda/Cuda_Seis3D.cu:684-693): [vp, vs, rho]."""
        r = Receiver(*[int(v) for v in point])
        out = np.zeros(3, dtype=np.float32)
        _check(_lib().seis3d_probe_material(self._handle, byref(self._ctx(context)), byref(r), _fptr(out)))
        return out

    def upload_model_plane(self, z: int, values: np.ndarray, context: Context | None = None) -> None:
        """uploadModelPlane3D (cuda/Cuda_Seis3D.cu:696-711): float32 [ny][nx][3] = vp, vs, rho."""
        v = np.ascontiguousarray(values, dtype=np.float32)
        _check(_lib().seis3d_upload_model_plane(self._handle, byref(self._ctx(context)), int(z), _fptr(v)))

    def finish_model_upload(self, context: Context | None = None) -> None:
        """finishModelUpload3D (cuda/Cuda_Seis3D.cu:714-717)."""
        _check(_lib().seis3d_finish_model_upload(self._handle, byref(self._ctx(context))))

    def upload_model(self, vp: np.ndarray, vs: np.ndarray, rho: np.ndarray) -> None:
        """Stream a whole [nz][ny][nx] model plane by plane, as importModel3D does
        (src/Seis3D/ModelIo3D.cpp:68-77)."""
        for z in range(vp.shape[0]):
            plane = np.stack([vp[z], vs[z], rho[z]], axis=-1)
            self.upload_model_plane(z, plane)
        self.finish_model_upload()

    def upload_volumes(self, vp: np.ndarray, vs: np.ndarray, rho: np.ndarray) -> None:
        """The whole [nz][ny][nx] model in one call (seis3d_upload_model): same materials as
        upload_model, validated before any device write, converted on the device."""
        c = self.context
        arrays = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho)]
        for a in arrays:
            if a.shape != (c.nz3D, c.ny3D, c.nx3D):
                raise InvalidArgument("model volumes must be (nz, ny, nx)")
        _check(_lib().seis3d_upload_model(self._handle, byref(c), *[_fptr(a) for a in arrays]))

    def download_model_plane(self, z: int, context: Context | None = None) -> np.ndarray:
        """downloadModelPlane3D (cuda/Cuda_Seis3D.cu:720-733)."""
        c = self._ctx(context)
        out = np.zeros((c.ny3D, c.nx3D, 3), dtype=np.float32)
        _check(_lib().seis3d_download_model_plane(self._handle, byref(c), int(z), _fptr(out)))
        return out

    # inspection ----------------------------------------------------------------------------
    def field(self, index: int) -> np.ndarray:
        """Whole padded field in the reference layout [gz][gy][gx] (0-8 wavefields,
        9 = 1/rho, 10 = lambda, 11 = mu)."""
        c = self.context
        out = np.zeros((c.gz3D, c.gy3D, c.gx3D), dtype=np.float32)
        _check(_lib().seis3d_copy_field(self._handle, int(index), 0, _fptr(out)))
        return out

    def set_field(self, index: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32)
        c = self.context
        if v.shape != (c.gz3D, c.gy3D, c.gx3D):
            raise InvalidArgument("field shape must be (gz, gy, gx)")
        _check(_lib().seis3d_copy_field(self._handle, int(index), 1, _fptr(v)))

    def extract_views(self, output_device_ptr: int, layout: capi.ViewLayout, slices, component: int,
                      material_component: int, volume: bool, include_boundary: bool = False) -> dict:
        """extractViews3D into a device buffer of 2 floats per sample (e.g. a CUDA tensor's
        data_ptr()); returns the colour statistics."""
        c = self.context
        sl = (c_int * 3)(*[int(v) for v in slices])
        maximum, vmax = c_float(), c_float()
        rng = (c_float * 2)()
        _check(_lib().seis3d_extract_views(self._handle, byref(c), c_void_p(int(output_device_ptr)), byref(layout), sl,
                                           int(component), int(material_component), int(bool(volume)),
                                           int(bool(include_boundary)), byref(maximum), rng, byref(vmax)))
        return {"maximum": maximum.value, "material_range": (rng[0], rng[1]), "velocity_maximum": vmax.value}

    def shade_slices(self, layout: ViewLayout, views_device_ptr: int, transfer: capi.Transfer, scale: float,
                     gain: float, pixel_format: int, output_device_ptr: int) -> None:
        """The slice shader over the extracted slices: one pixel per slice sample into a device
        buffer (4 bytes RGBA8 or 16 bytes RGBA32F per pixel).  Enqueued on the session stream;
        call synchronize() before reading the pixels."""
        _check(_lib().seis3d_shade_slices(self._handle, byref(layout), c_void_p(int(views_device_ptr)), byref(transfer),
                                          float(scale), float(gain), int(pixel_format),
                                          c_void_p(int(output_device_ptr))))

    def render_volume(self, layout: ViewLayout, views_device_ptr: int, transfer: capi.Transfer,
                      volume: capi.VolumeView, width: int, height: int, pixel_format: int,
                      output_device_ptr: int) -> None:
        """The volume shader: width x height pixels (row 0 at the bottom) into a device buffer.
        Enqueued on the session stream; call synchronize() before reading the pixels."""
        _check(_lib().seis3d_render_volume(self._handle, byref(layout), c_void_p(int(views_device_ptr)),
                                           byref(transfer), byref(volume), int(width), int(height),
                                           int(pixel_format), c_void_p(int(output_device_ptr))))

    def save_checkpoint(self) -> bytes:
        """The run state (wavefields, CPML memories, step clock) as bytes."""
        n = ctypes.c_uint64()
        _check(_lib().seis3d_checkpoint_bytes(self._handle, byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(_lib().seis3d_save_checkpoint(self._handle, buf, n.value))
        return buf.raw

    def load_checkpoint(self, data: bytes) -> None:
        _check(_lib().seis3d_load_checkpoint(self._handle, data, len(data)))

    def write_checkpoint(self, path: str) -> None:
        _check(_lib().seis3d_write_checkpoint(self._handle, str(path).encode()))

    def read_checkpoint(self, path: str) -> None:
        _check(_lib().seis3d_read_checkpoint(self._handle, str(path).encode()))

    def z_chunk(self) -> tuple[int, int]:
        """(setting, planes per CTA used): the z chunk chosen at initialisation (0 = default)."""
        a, b = c_int(), c_int()
        _check(_lib().seis3d_get_z_chunk(self._handle, byref(a), byref(b)))
        return a.value, b.value

    def views(self) -> capi.DeviceViews:
        v = capi.DeviceViews()
        _check(_lib().seis3d_get_views(self._handle, byref(v)))
        return v

    def synchronize(self) -> None:
        _check(_lib().seis3d_synchronize(self._handle))

    def non_finite(self) -> bool:
        flag = c_int()
        _check(_lib().seis3d_non_finite(self._handle, byref(flag)))
        return bool(flag.value)


class BoundaryNet:
    """The learned thin boundary's networks (one MLP per CPML face) for a `pml`-cell CPML;
    see include/seis3d_capi.h for the formulation."""

    def __init__(self, pml: int, seed: int = 1):
        self._handle = c_void_p()
        self.pml = int(pml)
        _check(_lib().seis3d_boundary_net_create(byref(self._handle), self.pml, int(seed)))

    def release(self) -> None:
        if self._handle:
            _lib().seis3d_boundary_net_release(self._handle)
            self._handle = c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    @property
    def handle(self) -> c_void_p:
        return self._handle

    def parameters(self, face: int) -> tuple[np.ndarray, float]:
        out = np.zeros(capi.BOUNDARY_PARAMETERS, dtype=np.float32)
        scale = c_float()
        _check(_lib().seis3d_boundary_net_get(self._handle, int(face), _fptr(out), byref(scale)))
        return out, float(scale.value)

    def set_parameters(self, face: int, params: np.ndarray, out_scale: float) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != capi.BOUNDARY_PARAMETERS:
            raise InvalidArgument("boundary network parameters have the wrong size")
        _check(_lib().seis3d_boundary_net_set(self._handle, int(face), _fptr(p), float(out_scale)))

    def train(self, dataset: "BoundaryDataset", face: int, iterations: int, batch: int = 4096, lr: float = 1e-3,
              seed: int = 0) -> float:
        loss = c_float()
        _check(_lib().seis3d_boundary_train(self._handle, dataset.handle, int(face), int(iterations), int(batch),
                                            float(lr), int(seed), byref(loss)))
        return float(loss.value)

    def gradients(self, face: int, inputs: np.ndarray, targets: np.ndarray, weights: np.ndarray):
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        w = np.ascontiguousarray(weights, dtype=np.float32)
        rows = w.size
        grad = np.zeros(capi.BOUNDARY_PARAMETERS, dtype=np.float32)
        loss = c_float()
        _check(_lib().seis3d_boundary_gradients(self._handle, int(face), _fptr(x), _fptr(t), _fptr(w), rows, _fptr(grad),
                                                byref(loss)))
        return grad, float(loss.value)


class BoundaryDataset:
    """Device training rows of the learned boundary (inputs, targets, amplitudes per face)."""

    def __init__(self, rows_per_face: int):
        self._handle = c_void_p()
        _check(_lib().seis3d_boundary_dataset_create(byref(self._handle), int(rows_per_face)))

    def release(self) -> None:
        if self._handle:
            _lib().seis3d_boundary_dataset_release(self._handle)
            self._handle = c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    @property
    def handle(self) -> c_void_p:
        return self._handle

    def rows(self) -> list[int]:
        out = (ctypes.c_uint64 * 6)()
        _check(_lib().seis3d_boundary_dataset_rows(self._handle, out))
        return [int(v) for v in out]

    def begin_model(self) -> None:
        _check(_lib().seis3d_boundary_begin_model(self._handle))

    def read(self, face: int, first: int, count: int):
        """(inputs [count][256], targets [count][36], amplitudes [count]) of one face."""
        x = np.zeros((count, 256), dtype=np.float32)
        y = np.zeros((count, 36), dtype=np.float32)
        s = np.zeros(count, dtype=np.float32)
        _check(_lib().seis3d_boundary_dataset_read(self._handle, int(face), int(first), int(count), _fptr(x), _fptr(y),
                                                   _fptr(s)))
        return x, y, s

    def collect(self, thin: Session, wide: Session, fraction: float = 1.0, seed: int = 0) -> None:
        _check(_lib().seis3d_boundary_collect(thin.handle, wide.handle, self._handle, float(fraction), int(seed)))


def attach_boundary(session: Session, net: BoundaryNet | None, gain: float = 1.0) -> None:
    """Correct `session`'s boundary columns with `net` after every step (None detaches)."""
    _check(_lib().seis3d_boundary_attach(session.handle, net.handle if net is not None else None, float(gain)))


class Batch:
    """Shots stepped together on one device (seis3d_batch_*): every session keeps its own grid,
    model, receivers and gather; one graph replay per 64 steps runs all of them, the shots of a
    launch group as concurrent branches.  Results are bit-identical to solo runs."""

    def __init__(self, sessions: Sequence["Session"], shots_per_launch: int = 0, z_chunk: int = 0,
                 tune: bool = False):
        self._sessions = list(sessions)
        handles = (c_void_p * max(1, len(self._sessions)))(*[s._handle.value for s in self._sessions])
        opt = capi.BatchOptions(int(shots_per_launch), int(z_chunk), int(bool(tune)))
        h = c_void_p()
        _check(_lib().seis3d_batch_create(byref(h), handles, len(self._sessions), byref(opt)))
        self._handle = h

    def run_steps(self, sources: Sequence[Source], first: int, count: int) -> None:
        """Enqueue steps first .. first+count-1 of every shot (asynchronous)."""
        if len(sources) != len(self._sessions):
            raise InvalidArgument("one source per shot")
        if any(not s._handle for s in self._sessions):
            raise LogicError("a session of the batch was released")
        arr = (Source * len(sources))(*sources)
        _check(_lib().seis3d_batch_run_steps(self._handle, arr, int(first), int(count)))

    def synchronize(self) -> None:
        if any(not s._handle for s in self._sessions):
            raise LogicError("a session of the batch was released")
        _check(_lib().seis3d_batch_synchronize(self._handle))

    def info(self) -> dict:
        i = capi.BatchInfo()
        _check(_lib().seis3d_batch_get_info(self._handle, byref(i)))
        return {"shots": i.shots, "shots_per_launch": i.shots_per_launch, "z_chunk": i.z_chunk,
                "tuned": bool(i.tuned), "candidates": i.candidates, "tuned_ms_per_step": i.tuned_ms_per_step,
                "kernel_launches": i.kernel_launches, "stream": i.stream}

    def release(self) -> None:
        if self._handle is not None and self._handle.value:
            _lib().seis3d_batch_release(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
