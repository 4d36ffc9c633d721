"""Host-side mirror of gemray's GPU render backend over the C ABI.

`GpuBackend` keeps the reference's interface and semantics
(crates/gemray/src/renderer/gpu_backend.rs:102-193):

* ``GpuBackend.acquire()`` never raises: without a usable device it returns a backend
  that declines every call, exactly like ``GpuBackend::disabled()``;
* ``try_accumulate(scene, sample_offset, spp, accum)`` ADDS the traced samples
  ``[sample_offset, sample_offset + spp)`` of every pixel into ``accum`` and returns
  True, or returns False (leaving ``accum`` untouched) when the scene is declined, so
  the caller can render it on the CPU tracer instead;
* a length mismatch between ``accum`` and the frame is a caller bug: the reference
  panics (renderer/gpu/frame.rs:673-677); here it raises ``ValueError``.

`GpuFrameRenderer` mirrors renderer/gpu/frame.rs:574-647: the fallible constructor and
``accumulate`` that reports why a dispatch was declined.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import abi
from .scene import Scene


class GpuFrameError(RuntimeError):
    """A declined or failed dispatch (renderer/gpu/frame.rs:196-210)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class UnsupportedMaterial(GpuFrameError):
    pass


class UnsupportedEnvironment(GpuFrameError):
    pass


class AcquireError(GpuFrameError):
    pass


def _raise_for(lib, status: int) -> None:
    if status == abi.GR_OK:
        return
    msg = (lib.gr_last_error_string() or b"").decode(errors="replace")
    if status == abi.GR_DECLINED_MATERIAL:
        raise UnsupportedMaterial(status, msg)
    if status == abi.GR_DECLINED_ENV:
        raise UnsupportedEnvironment(status, msg)
    if status == abi.GR_NO_DEVICE:
        raise AcquireError(status, msg)
    raise GpuFrameError(status, msg)


class GpuFrameRenderer:
    """Owns one engine context (device buffers, stream); see renderer/gpu/frame.rs:566-647."""

    def __init__(self, device: int = -1, chunk_budget_bytes: int = 0, kernel: int | None = None,
                 serve_budget_bytes: int = 0):
        self._lib = abi.load_library()
        opts = abi.gr_create_opts(device=device, chunk_budget_bytes=chunk_budget_bytes,
                                  serve_budget_bytes=serve_budget_bytes)
        ctx = C.c_void_p()
        _raise_for(self._lib, self._lib.gr_create(C.byref(ctx), C.byref(opts)))
        self._ctx = ctx
        if kernel is not None:
            _raise_for(self._lib, self._lib.gr_set_kernel(self._ctx, kernel))

    @property
    def ctx(self) -> C.c_void_p:
        return self._ctx

    @property
    def lib(self):
        return self._lib

    def adapter_label(self) -> str:
        return self._lib.gr_device_label(self._ctx).decode()

    def set_kernel(self, kernel: int) -> None:
        _raise_for(self._lib, self._lib.gr_set_kernel(self._ctx, kernel))

    def accumulate(self, scene: Scene, sample_offset: int, spp: int, accum: np.ndarray) -> None:
        """Add samples [sample_offset, sample_offset+spp) of every pixel into accum (W*H, 3) f32."""
        n = scene.width * scene.height
        if accum.dtype != np.float32 or accum.size != n * 3 or not accum.flags.c_contiguous:
            raise ValueError("accumulation buffer must be a C-contiguous float32 array of width*height*3")
        st = self._lib.gr_accumulate(self._ctx, C.byref(scene.c_scene()), sample_offset, spp,
                                     accum.ctypes.data_as(C.POINTER(C.c_float)))
        _raise_for(self._lib, st)

    def accumulate_device(self, scene: Scene, sample_offset: int, spp: int, accum_device_ptr: int,
                          stream: int | None = None) -> None:
        st = self._lib.gr_accumulate_device(self._ctx, C.byref(scene.c_scene()), sample_offset, spp,
                                            C.c_void_p(accum_device_ptr), C.c_void_p(stream or 0))
        _raise_for(self._lib, st)

    def trace_samples(self, scene: Scene, first_pixel: int, n_pixels: int, sample_offset: int, spp: int) -> np.ndarray:
        out = np.empty((n_pixels * spp, 3), np.float32)
        st = self._lib.gr_trace_samples(self._ctx, C.byref(scene.c_scene()), first_pixel, n_pixels, sample_offset,
                                        spp, out.ctypes.data_as(C.POINTER(C.c_float)))
        _raise_for(self._lib, st)
        return out

    def tonemap(self, xyz: np.ndarray, scale: float) -> np.ndarray:
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        out = np.empty((xyz.shape[0], 4), np.uint8)
        st = self._lib.gr_tonemap(self._ctx, xyz.ctypes.data_as(C.POINTER(C.c_float)), scale, xyz.shape[0],
                                  out.ctypes.data_as(C.POINTER(C.c_uint8)))
        _raise_for(self._lib, st)
        return out

    def synchronize(self) -> None:
        _raise_for(self._lib, self._lib.gr_synchronize(self._ctx))

    def close(self) -> None:
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            self._lib.gr_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuBackend:
    """Drop-in for gemray's ``GpuBackend`` (renderer/gpu_backend.rs:102-193)."""

    def __init__(self, renderer: GpuFrameRenderer | None):
        self._renderer = renderer
        self._lock = threading.Lock()
        self.last_error: str | None = None

    @classmethod
    def acquire(cls, **kwargs) -> "GpuBackend":
        try:
            return cls(GpuFrameRenderer(**kwargs))
        except (GpuFrameError, abi.LibraryMissing) as e:
            b = cls(None)
            b.last_error = str(e)
            return b

    @classmethod
    def disabled(cls) -> "GpuBackend":
        return cls(None)

    @property
    def renderer(self) -> GpuFrameRenderer | None:
        return self._renderer

    def adapter_label(self) -> str | None:
        if self._renderer is None:
            return None
        with self._lock:
            return self._renderer.adapter_label()

    def try_accumulate(self, scene: Scene, sample_offset: int, spp: int, accum: np.ndarray) -> bool:
        n = scene.width * scene.height
        if accum.size != n * 3:
            raise ValueError("accumulation buffer must have one entry per pixel")
        if self._renderer is None:
            return False
        with self._lock:
            try:
                self._renderer.accumulate(scene, sample_offset, spp, accum)
                return True
            except GpuFrameError as e:
                self.last_error = str(e)
                return False
