"""gr_stream_*: one render request streamed as FRAME deltas (apps/gemray-worker/src/
stream_emit/), through the C ABI.

* Arithmetic: with a fixed sub-batch split, every drained delta is its sub-batches'
  zero-started films copied and added in order (PendingDelta::add) and the running
  total their in-order sum from zero (tracer.rs:93-100) -- bit for bit, checked
  against sub-batches rendered one by one with gr_render_resident.
* Coverage: drained ranges are contiguous and tile the request; their sum agrees
  with one direct render of the whole range within the reference's own 1e-3
  (tests.rs:34-54, coalesced vs direct).
* Cancellation stops the tracer between sub-batches and discards the pending delta;
  the preview is the oracle's downsample_preview of the total, bit for bit; a
  streamed scene cannot be released; the emitter loop ends with DONE.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

from gemray_studio_b200 import abi, radiance, scene as S
from gemray_studio_b200.stream import FrameStream

pytestmark = pytest.mark.gpu


def _scene(w=40, h=30, material="Diamond", **kw):
    return S.Scene(width=w, height=h, planes=S.standard_round_brilliant(), material=S.builtin_material(material),
                   cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=12, **kw)


@pytest.fixture()
def resident(renderer):
    ids = []

    def upload(sc):
        sid = C.c_uint64()
        assert renderer.lib.gr_scene_upload(renderer.ctx, C.byref(sc.c_scene()), C.byref(sid)) == abi.GR_OK
        ids.append(sid.value)
        return sid.value
    yield upload
    for i in ids:
        renderer.lib.gr_scene_release(renderer.ctx, i)


def _wait(fs: FrameStream, timeout_s=60.0, drain=None):
    t0 = time.monotonic()
    while True:
        done, state = fs.status()
        if drain is not None:
            drain()
        if state != "running":
            return done, state
        assert time.monotonic() - t0 < timeout_s, "stream did not finish"
        time.sleep(0.002)


def _subbatch_films(renderer, sid, n_px, first, samples, fixed):
    import torch
    films, s = [], first
    while s < first + samples:
        n = min(fixed, first + samples - s)
        f = torch.zeros((n_px, 3), dtype=torch.float32, device="cuda")
        assert renderer.lib.gr_render_resident(renderer.ctx, sid, s, n, C.c_void_p(f.data_ptr()), None) == abi.GR_OK
        films.append((s, n, f))
        s += n
    renderer.synchronize()
    return films


def test_fixed_batches_reproduce_the_reference_fold(renderer, resident):
    import torch
    sc = _scene()
    sid = resident(sc)
    n_px = sc.width * sc.height
    first, samples, fixed = 5, 40, 3
    batches = _subbatch_films(renderer, sid, n_px, first, samples, fixed)
    with FrameStream(renderer, sid, sc.width, sc.height, first, samples, fixed_batch=fixed) as fs:
        deltas = []
        done, state = _wait(fs, drain=lambda: deltas.append(fs.take()))
        deltas.append(fs.take())
        assert state == "finished" and done == samples
        total = fs.total()
    deltas = [d for d in deltas if d is not None]
    # ranges tile the request in order
    assert deltas[0][0] == first
    for a, b in zip(deltas, deltas[1:]):
        assert b[0] == a[0] + a[1]
    assert deltas[-1][0] + deltas[-1][1] == first + samples
    # each delta: its sub-batches copied then added in order
    for f0, n, got in deltas:
        exp = None
        for s, m, film in batches:
            if f0 <= s < f0 + n:
                exp = film.clone() if exp is None else exp + film
        assert np.array_equal(got.view(np.uint32), exp.cpu().numpy().view(np.uint32)), (f0, n)
    # the running total: their in-order sum from zero
    acc = torch.zeros((n_px, 3), dtype=torch.float32, device="cuda")
    for _s, _m, film in batches:
        acc = acc + film
    assert np.array_equal(total.view(np.uint32), acc.cpu().numpy().view(np.uint32))


def test_adaptive_stream_tiles_the_request_and_matches_a_direct_render(renderer, resident):
    import torch
    sc = _scene(96, 64, material="Sapphire")
    sid = resident(sc)
    n_px = sc.width * sc.height
    with FrameStream(renderer, sid, sc.width, sc.height, 0, 96, target_ms=5) as fs:
        deltas = []
        _wait(fs, drain=lambda: deltas.append(fs.take()))
        deltas.append(fs.take())
        total = fs.total()
    deltas = [d for d in deltas if d is not None]
    assert deltas[0][0] == 0 and sum(d[1] for d in deltas) == 96
    for a, b in zip(deltas, deltas[1:]):
        assert b[0] == a[0] + a[1]
    direct = torch.zeros((n_px, 3), dtype=torch.float32, device="cuda")
    assert renderer.lib.gr_render_resident(renderer.ctx, sid, 0, 96, C.c_void_p(direct.data_ptr()), None) == abi.GR_OK
    renderer.synchronize()
    d = direct.cpu().numpy().astype(np.float64)
    summed = np.sum([x[2].astype(np.float64) for x in deltas], axis=0)
    for got in (summed, total.astype(np.float64)):
        scale = np.maximum(np.maximum(np.abs(got), np.abs(d)), 1e-6)
        assert np.max(np.abs(got - d) / scale) < 1e-3


def test_cancel_between_subbatches_discards_the_pending_delta(renderer, resident):
    sc = _scene(256, 256)
    sid = resident(sc)
    fs = FrameStream(renderer, sid, sc.width, sc.height, 0, 1 << 20, fixed_batch=16)
    try:
        t0 = time.monotonic()
        while fs.status()[0] == 0:
            assert time.monotonic() - t0 < 30
            time.sleep(0.001)
        fs.cancel()
        done, state = _wait(fs)
        assert state == "cancelled"
        assert 0 < done < (1 << 20) and done % 16 == 0
        assert fs.take() is None
    finally:
        fs.close()


def test_preview_is_the_oracle_downsample_of_the_total(renderer, resident, oracle):
    sc = _scene(40, 30)
    sid = resident(sc)
    fp = C.POINTER(C.c_float)
    with FrameStream(renderer, sid, sc.width, sc.height, 0, 24) as fs:
        _wait(fs)
        total = fs.total()
        for tw, th in [(7, 5), (40, 30), (64, 48), (1, 1), (0, 0)]:
            got = fs.preview(tw, th)
            ref = np.empty_like(got)
            oracle.gro_downsample_preview(total.ctypes.data_as(fp), sc.width, sc.height, tw, th, ref.ctypes.data_as(fp))
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (tw, th)


def test_streamed_scene_stays_resident(renderer, resident):
    sc = _scene(16, 16)
    sid = resident(sc)
    fs = FrameStream(renderer, sid, sc.width, sc.height, 0, 8)
    assert renderer.lib.gr_scene_release(renderer.ctx, sid) == abi.GR_EBUSY
    _wait(fs)
    fs.close()
    sid2 = resident(_scene(16, 16))
    with FrameStream(renderer, sid2, 16, 16, 0, 0) as fz:  # zero samples: finished at once
        assert fz.status() == (0, "finished") and fz.take() is None


@pytest.mark.parametrize("live", [True, False])
def test_emitter_loop(renderer, resident, live):
    sc = _scene(48, 32)
    sid = resident(sc)
    with FrameStream(renderer, sid, sc.width, sc.height, 3, 64, target_ms=2) as fs:
        events = list(fs.emit(request_id=7, cadence_ms=5, live=live, preview=(8, 4)))
        total = fs.total()
    assert events[-1].kind == "DONE" and not events[-1].cancelled
    assert all(e.request_id == 7 for e in events)
    frames = [e for e in events if e.kind == "FRAME"]
    if live:
        assert frames[0].first_sample == 3 and sum(f.samples for f in frames) == 64
        summed = np.sum([radiance.decode(f.payload, 48, 32).astype(np.float64) for f in frames], axis=0)
        scale = np.maximum(np.abs(total), 1e-6)
        assert np.max(np.abs(summed - total) / scale) < 1e-3
    else:
        assert len(frames) == 1 and (frames[0].first_sample, frames[0].samples) == (3, 64)
        assert frames[0].payload == radiance.encode(total)
    for e in events:
        if e.kind == "PREVIEW":
            assert (e.width, e.height) == (8, 4) and len(e.payload) == 8 * 4 * 12
