"""Frame-delta streaming over the C ABI (gr_stream_*).

`FrameStream` renders one request -- samples ``[first_sample, first_sample + samples)``
of a resident scene -- on a tracer thread inside the library, in sub-batches sized to
about ``target_ms`` of device time each; `take()` drains the pending delta (the FRAME
payload and its sample range), `preview()` box-downsamples the running total, and
`cancel()` stops the tracer between sub-batches.  `emit()` is the emitter half of the
worker's stream loop (apps/gemray-worker/src/stream_emit/emitter.rs:377-614): on each
cadence tick a FRAME (live-progressive mode, when a delta is pending), an optional
PREVIEW and a PROGRESS; at the end the last FRAME (or, in final-only mode, the whole
total) and DONE.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import Iterator

import numpy as np

from . import abi, radiance
from .backend import GpuFrameRenderer, _raise_for

_STATES = {abi.GR_STREAM_RUNNING: "running", abi.GR_STREAM_FINISHED: "finished",
           abi.GR_STREAM_CANCELLED: "cancelled", abi.GR_STREAM_FAILED: "failed"}


def next_batch_size(prev: int, elapsed_ms: float, target_ms: float = 100.0) -> int:
    """sizing.rs:22-30, as the library implements it (gr_next_batch_size)."""
    return int(abi.load_library().gr_next_batch_size(prev, elapsed_ms, target_ms))


@dataclass(frozen=True)
class StreamEvent:
    kind: str                 # FRAME / PREVIEW / PROGRESS / DONE
    request_id: int
    first_sample: int = 0
    samples: int = 0
    samples_done: int = 0
    payload: bytes = b""      # FRAME: radiance bytes; PREVIEW: radiance bytes of the preview
    width: int = 0
    height: int = 0
    cancelled: bool = False


class FrameStream:
    def __init__(self, renderer: GpuFrameRenderer, scene_id: int, width: int, height: int, first_sample: int,
                 samples: int, target_ms: int = 100, first_batch: int = 1, fixed_batch: int = 0):
        self._r = renderer
        self._lib = renderer.lib
        self.width, self.height = int(width), int(height)
        self.first_sample, self.samples = int(first_sample), int(samples)
        opts = abi.gr_stream_opts(target_ms=target_ms, first_batch=first_batch, fixed_batch=fixed_batch)
        sid = C.c_uint64()
        _raise_for(self._lib, self._lib.gr_stream_open(renderer.ctx, scene_id, first_sample, samples, C.byref(opts),
                                                       C.byref(sid)))
        self.id = sid.value

    def _buf(self, n: int) -> np.ndarray:
        return np.empty((n, 3), np.float32)

    def take(self) -> tuple[int, int, np.ndarray] | None:
        """PendingDelta::take: (first_sample, samples, delta film) or None."""
        out = self._buf(self.width * self.height)
        first, n = C.c_uint32(), C.c_uint32()
        _raise_for(self._lib, self._lib.gr_stream_take(self._r.ctx, self.id, C.byref(first), C.byref(n),
                                                       out.ctypes.data_as(C.POINTER(C.c_float))))
        return None if n.value == 0 else (first.value, n.value, out)

    def status(self) -> tuple[int, str]:
        done, state, err = C.c_uint32(), C.c_uint32(), C.c_int()
        _raise_for(self._lib, self._lib.gr_stream_status(self._r.ctx, self.id, C.byref(done), C.byref(state),
                                                         C.byref(err)))
        if state.value == abi.GR_STREAM_FAILED:
            _raise_for(self._lib, err.value)
        return done.value, _STATES[state.value]

    def total(self) -> np.ndarray:
        out = self._buf(self.width * self.height)
        _raise_for(self._lib, self._lib.gr_stream_total(self._r.ctx, self.id, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def preview(self, tw: int, th: int) -> np.ndarray:
        out = self._buf(max(tw, 1) * max(th, 1))
        _raise_for(self._lib, self._lib.gr_stream_preview(self._r.ctx, self.id, tw, th,
                                                          out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def cancel(self) -> None:
        _raise_for(self._lib, self._lib.gr_stream_cancel(self._r.ctx, self.id))

    def close(self) -> None:
        if self.id:
            _raise_for(self._lib, self._lib.gr_stream_close(self._r.ctx, self.id))
            self.id = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def emit(self, request_id: int, cadence_ms: float = 250.0, live: bool = True,
             preview: tuple[int, int] | None = None, should_cancel=lambda: False) -> Iterator[StreamEvent]:
        """The emitter loop: one tick per cadence while the tracer runs (emit_tick), then
        the final emission (emit_final) or, once should_cancel() turns true, a cancel and
        DONE{cancelled} with nothing further sent."""
        while True:
            deadline = time.monotonic() + cadence_ms / 1000.0
            while time.monotonic() < deadline:
                if should_cancel():
                    self.cancel()
                    yield StreamEvent("DONE", request_id, cancelled=True)
                    return
                done, state = self.status()
                if state != "running":
                    break
                time.sleep(min(0.005, max(0.0, deadline - time.monotonic())))
            done, state = self.status()
            if state != "running":
                break
            yield from self._tick(request_id, live, preview, done)
        if state == "cancelled":
            yield StreamEvent("DONE", request_id, cancelled=True)
            return
        if live:  # whatever is left un-coalesced
            d = self.take()
            if d is not None:
                yield StreamEvent("FRAME", request_id, d[0], d[1], payload=radiance.encode(d[2]),
                                  width=self.width, height=self.height)
        else:  # the whole request as one FRAME of the running total
            yield StreamEvent("FRAME", request_id, self.first_sample, self.samples,
                              payload=radiance.encode(self.total()), width=self.width, height=self.height)
        yield StreamEvent("DONE", request_id, samples_done=done)

    def _preview_event(self, request_id: int, preview: tuple[int, int], done: int) -> StreamEvent:
        tw, th = max(preview[0], 1), max(preview[1], 1)
        return StreamEvent("PREVIEW", request_id, samples_done=done, payload=radiance.encode(self.preview(tw, th)),
                           width=tw, height=th)

    def _tick(self, request_id: int, live: bool, preview: tuple[int, int] | None, done: int) -> Iterator[StreamEvent]:
        if live:
            d = self.take()
            if d is not None:
                yield StreamEvent("FRAME", request_id, d[0], d[1], payload=radiance.encode(d[2]),
                                  width=self.width, height=self.height)
        if preview is not None:
            yield self._preview_event(request_id, preview, done)
        yield StreamEvent("PROGRESS", request_id, samples_done=done)
