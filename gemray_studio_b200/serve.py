"""Render-request serving over the C ABI (gr_submit / gr_poll / gr_wait / gr_cancel).

`RenderServer` keeps scenes resident on the device and accepts requests shaped like
the reference's ``RenderRequest{request_id, first_sample, samples}``
(crates/gemray-net/src/messages/render.rs:65-70): each adds samples
``[first_sample, first_sample + samples)`` of every pixel into a film of its own.
The library's worker thread admits requests by device-memory budget and advances all
running renders together, one slice per tick, in shared batched launches.  Slices
continue each pixel's running sum, so a film is bit-identical to rendering the whole
sample range alone in one call, however it was sliced and whatever else ran.  Metric
sweeps (brilliance / fire / scintillation over a list of poses) use the same request
ids and calls; they hold no film, skip admission and run on a second worker thread
beside the renders.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from .backend import GpuFrameRenderer, _raise_for
from .scene import Scene


@dataclass(frozen=True)
class RequestStatus:
    state: str            # queued / running / done / cancelled / failed
    samples_done: int
    error: int
    queued_ms: float
    latency_ms: float

    @property
    def finished(self) -> bool:
        return self.state in ("done", "cancelled", "failed")


def _status(st: abi.gr_request_status) -> RequestStatus:
    return RequestStatus(abi.REQUEST_STATES[st.state], int(st.samples_done), int(st.error), float(st.queued_ms),
                         float(st.latency_ms))


class RenderServer:
    """Resident scenes plus a request queue on one engine context."""

    def __init__(self, renderer: GpuFrameRenderer | None = None, **renderer_kw):
        self.r = renderer if renderer is not None else GpuFrameRenderer(**renderer_kw)
        self._own = renderer is None
        self.lib, self.ctx = self.r.lib, self.r.ctx
        self._shapes: dict[int, tuple[int, int]] = {}   # scene id -> (width, height)
        self._req_shape: dict[int, tuple[int, int]] = {}
        self._req_poses: dict[int, int] = {}

    # -- scenes ---------------------------------------------------------------------
    def upload(self, scene: Scene) -> int:
        sid = C.c_uint64()
        _raise_for(self.lib, self.lib.gr_scene_upload(self.ctx, C.byref(scene.c_scene()), C.byref(sid)))
        self._shapes[sid.value] = (scene.width, scene.height)
        return sid.value

    def release_scene(self, scene_id: int) -> None:
        _raise_for(self.lib, self.lib.gr_scene_release(self.ctx, scene_id))
        self._shapes.pop(scene_id, None)

    # -- requests -------------------------------------------------------------------
    def submit_render(self, scene_id: int, first_sample: int, samples: int, slice_spp: int = 0) -> int:
        """slice_spp caps the samples per pixel one tick may take (0 = no cap); the film
        never depends on it."""
        q = abi.gr_request(kind=abi.GR_REQ_RENDER, slice_spp=slice_spp, scene_id=scene_id, sample_offset=first_sample,
                           spp=samples)
        rid = C.c_uint64()
        _raise_for(self.lib, self.lib.gr_submit(self.ctx, C.byref(q), C.byref(rid)))
        self._req_shape[rid.value] = self._shapes[scene_id]
        return rid.value

    def submit_metrics(self, planes, material: abi.gr_material, poses, fp64_sums: bool = False) -> int:
        p = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
        z = np.ascontiguousarray(poses, np.float32).reshape(-1, 4)
        q = abi.gr_request(kind=abi.GR_REQ_METRICS, flags=abi.GR_METRICS_FP64_SUMS if fp64_sums else 0,
                           n_planes=p.shape[0], planes=p.ctypes.data, material=C.addressof(material),
                           poses=z.ctypes.data, n_poses=z.shape[0])
        rid = C.c_uint64()
        _raise_for(self.lib, self.lib.gr_submit(self.ctx, C.byref(q), C.byref(rid)))  # copied at submit
        self._req_poses[rid.value] = z.shape[0]
        return rid.value

    def poll(self, request_id: int) -> RequestStatus:
        st = abi.gr_request_status()
        _raise_for(self.lib, self.lib.gr_poll(self.ctx, request_id, C.byref(st)))
        return _status(st)

    def wait(self, request_id: int, timeout_ms: int = 600_000) -> RequestStatus:
        st = abi.gr_request_status()
        _raise_for(self.lib, self.lib.gr_wait(self.ctx, request_id, timeout_ms, C.byref(st)))
        return _status(st)

    def cancel(self, request_id: int) -> None:
        _raise_for(self.lib, self.lib.gr_cancel(self.ctx, request_id))

    def film(self, request_id: int) -> np.ndarray:
        w, h = self._req_shape[request_id]
        out = np.empty((w * h, 3), np.float32)
        _raise_for(self.lib, self.lib.gr_request_film(self.ctx, request_id, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def metrics(self, request_id: int) -> np.ndarray:
        n = self._req_poses[request_id]
        out = (abi.gr_metrics_out * max(n, 1))()
        _raise_for(self.lib, self.lib.gr_request_metrics(self.ctx, request_id, out))
        return np.ctypeslib.as_array(out).view(np.float32).reshape(-1, 5)[:n].copy()

    def release(self, request_id: int) -> None:
        _raise_for(self.lib, self.lib.gr_request_release(self.ctx, request_id))
        self._req_shape.pop(request_id, None)
        self._req_poses.pop(request_id, None)

    def close(self) -> None:
        if self._own:
            self.r.close()
