"""Serving (gr_submit / gr_poll / gr_wait / gr_cancel): continuous batching of render
requests and metric sweeps over resident scenes.

The bar: a request's film is bit-identical alone and in a mix, for any slicing, to
one gr_render_resident call over its whole sample range on a zero film (slices carry
each pixel's running sum on, Kahan compensation included); metric sweeps equal
gr_optical_metrics; cancellation stops a render between slices; admission holds
requests back until their film fits the device-memory budget and fails the ones that
never can.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import GpuFrameRenderer, abi, metrics as M, scene as S
from gemray_studio_b200.serve import RenderServer

pytestmark = pytest.mark.gpu


def _scenes():
    rng = np.random.default_rng(8)
    env = S.gaussian_blob_latlong(256, 128, seed=5)
    cam = S.camera(0.35, 0.28, 5.0, 18.0)
    return [S.Scene(width=48, height=40, planes=S.round_brilliant_57(), material=S.builtin_material("Diamond"), cam=cam,
                    max_bounces=16, env_mode=abi.GR_ENV_LATLONG, latlong=env),
            S.Scene(width=32, height=32, planes=S.emerald_cut_49(), material=S.builtin_material("Tourmaline"), cam=cam,
                    max_bounces=16, env_mode=abi.GR_ENV_STUDIO),
            S.Scene(width=24, height=30, planes=S.random_polyhedron(rng), material=S.builtin_material("Zircon"), cam=cam,
                    max_bounces=16, env_mode=abi.GR_ENV_UNIFORM, flags=abi.GR_FLAG_KAHAN_FILM)]


def _resident(srv: RenderServer, sid: int, shape, offset: int, spp: int) -> np.ndarray:
    """One gr_render_resident call over the whole sample range on a zero film."""
    import torch
    w, h = shape
    film = torch.zeros((w * h, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = srv.lib.gr_render_resident(srv.ctx, sid, offset, spp, C.c_void_p(film.data_ptr()), None)
    assert st == abi.GR_OK
    assert srv.lib.gr_synchronize(srv.ctx) == abi.GR_OK
    return film.cpu().numpy()


def test_results_identical_alone_and_in_mix(engine_lib):
    srv = RenderServer()
    try:
        scenes = _scenes()
        ids = [srv.upload(sc) for sc in scenes]
        alone = srv.submit_render(ids[0], 100, 48)  # slices sized by the library
        st = srv.wait(alone)
        assert st.state == "done" and st.samples_done == 48 and st.latency_ms > 0
        film_alone = srv.film(alone)
        # the same request again, now mixed with two renders of other scenes and a metric sweep
        poses = np.array([[0.0, 0.45 + 0.05 * k, 0.85, 0.95] for k in range(8)], np.float32)
        rids = [srv.submit_render(ids[1], 7, 40, slice_spp=8), srv.submit_render(ids[0], 100, 48, slice_spp=5),
                srv.submit_render(ids[2], 0, 33, slice_spp=16)]
        mid = srv.submit_metrics(S.standard_round_brilliant(), S.builtin_material("Diamond"), poses)
        for r in rids + [mid]:
            assert srv.wait(r).state == "done"
        mixed = srv.film(rids[1])
        assert np.array_equal(film_alone.view(np.uint32), mixed.view(np.uint32))
        assert np.array_equal(mixed.view(np.uint32), _resident(srv, ids[0], (48, 40), 100, 48).view(np.uint32))
        assert np.array_equal(srv.film(rids[0]).view(np.uint32), _resident(srv, ids[1], (32, 32), 7, 40).view(np.uint32))
        assert np.array_equal(srv.film(rids[2]).view(np.uint32), _resident(srv, ids[2], (24, 30), 0, 33).view(np.uint32))
        ref = M.evaluate_poses(srv.r, S.standard_round_brilliant(), S.builtin_material("Diamond"), poses)
        assert np.array_equal(srv.metrics(mid).view(np.uint32), ref.view(np.uint32))
        for r in [alone] + rids + [mid]:
            srv.release(r)
        with pytest.raises(Exception):
            srv.poll(alone)
    finally:
        srv.close()


def test_metric_sweeps_run_beside_a_long_render(engine_lib):
    """Metric sweeps skip render admission and run on their own worker: submitted
    behind a render of ~270 M samples they finish while it is still running, each
    bit-identical to gr_optical_metrics, and stones with more planes than any swept
    before (a larger sweep scratch) change nothing."""
    srv = RenderServer()
    try:
        sc = S.Scene(width=256, height=256, planes=S.round_brilliant_57(), material=S.builtin_material("Diamond"),
                     cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=32, env_mode=abi.GR_ENV_UNIFORM)
        sid = srv.upload(sc)
        long = srv.submit_render(sid, 0, 4096)
        rng = np.random.default_rng(21)
        stones = sorted((S.random_polyhedron(rng) for _ in range(4)), key=len)
        assert len(stones[0]) < len(stones[-1])
        mat = S.builtin_material("Spinel")
        poses = np.array([[0.1 * k, 0.45, 0.85, 0.95] for k in range(16)], np.float32)
        sweeps = [(planes, srv.submit_metrics(planes, mat, poses)) for planes in stones]
        for _planes, mid in sweeps:
            assert srv.wait(mid).state == "done"
        st = srv.poll(long)
        assert st.state in ("queued", "running") and st.samples_done < 4096
        srv.cancel(long)
        assert srv.wait(long).state == "cancelled"
        for planes, mid in sweeps:  # references after the render: they share its stream
            ref = M.evaluate_poses(srv.r, planes, mat, poses)
            assert np.array_equal(srv.metrics(mid).view(np.uint32), ref.view(np.uint32))
            srv.release(mid)
        srv.release(long)
    finally:
        srv.close()


def test_cancel_between_slices(engine_lib):
    srv = RenderServer()
    try:
        sc = _scenes()[0]
        sid = srv.upload(sc)
        rid = srv.submit_render(sid, 0, 1 << 20, slice_spp=4)
        srv.cancel(rid)
        st = srv.wait(rid)
        assert st.state == "cancelled" and st.samples_done < (1 << 20) and st.samples_done % 4 == 0
        film = srv.film(rid)   # the slices folded before the cancel
        if st.samples_done:
            assert np.array_equal(film.view(np.uint32), _resident(srv, sid, (48, 40), 0, st.samples_done).view(np.uint32))
        srv.release(rid)
    finally:
        srv.close()


def test_admission_by_memory_budget(engine_lib):
    scenes = _scenes()
    film = 48 * 40 * 12
    resident = scenes[0].planes.shape[0] * 16 + scenes[0].latlong.nbytes + scenes[1].planes.shape[0] * 16 + 16 * 8
    r = GpuFrameRenderer(serve_budget_bytes=resident + film + film // 2)  # room for exactly one film
    srv = RenderServer(r)
    try:
        ids = [srv.upload(sc) for sc in scenes[:2]]
        a = srv.submit_render(ids[0], 0, 32, slice_spp=8)
        b = srv.submit_render(ids[0], 32, 32, slice_spp=8)
        sa = srv.wait(a)
        assert sa.state == "done"
        assert srv.poll(b).state == "queued"   # a's finished film still holds the budget
        srv.release(a)
        sb = srv.wait(b)
        # b waited for a's whole run (a's latency also counts the serve loop's one-time
        # setup inside the context's first gr_submit, which b did not wait for)
        assert sb.state == "done" and sb.queued_ms >= 0.9 * (sa.latency_ms - sa.queued_ms)
        assert np.array_equal(srv.film(b).view(np.uint32), _resident(srv, ids[0], (48, 40), 32, 32).view(np.uint32))
        srv.release(b)
        big = S.Scene(width=512, height=512, planes=S.round_brilliant_57(), material=S.builtin_material("Diamond"),
                      cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=8)
        too_big = srv.submit_render(srv.upload(big), 0, 4)
        st = srv.wait(too_big)
        assert st.state == "failed" and st.error == abi.GR_EBUSY
        active = srv.submit_render(ids[0], 0, 1 << 20, slice_spp=1)
        with pytest.raises(Exception):
            srv.release(active)  # still active: GR_EBUSY
        srv.cancel(active)
        assert srv.wait(active).state == "cancelled"
    finally:
        srv.close()
        r.close()


def test_lane_renders_every_size_beside_ticks(engine_lib):
    """Renders without a slice_spp go to the render lane: requests of every size (a Kahan
    scene among them; the long render of the sweep test spans many chunks) rendered chunk by
    chunk with the single-scene kernels, interleaved by submission time plus remaining
    work; sliced renders go to the ticks beside them.  Every film is bit-identical to
    one gr_render_resident call over its range on a zero film; a lane render cancelled
    before it starts ends with no samples and a zero film."""
    srv = RenderServer()
    try:
        small = _scenes()
        rng = np.random.default_rng(4)
        big = [S.Scene(width=128, height=128, planes=S.round_brilliant_57(), material=S.builtin_material("Diamond"),
                       cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=32, env_mode=abi.GR_ENV_LATLONG,
                       latlong=S.gaussian_blob_latlong(256, 128, seed=2)),
               S.Scene(width=96, height=96, planes=S.random_polyhedron(rng), material=S.builtin_material("Zircon"),
                       cam=S.camera(0.3, 0.4, 4.0, 30.0), max_bounces=24, env_mode=abi.GR_ENV_STUDIO,
                       flags=abi.GR_FLAG_KAHAN_FILM)]
        big_ids = [srv.upload(sc) for sc in big]
        small_ids = [srv.upload(sc) for sc in small]
        jobs = [(big_ids[0], (128, 128), 5, 600), (big_ids[1], (96, 96), 0, 1000), (big_ids[0], (128, 128), 9, 200),
                (big_ids[1], (96, 96), 3, 300)]
        sizes = [w * h * spp for _, (w, h), _, spp in jobs]
        assert sizes[0] > (8 << 20) and sizes[1] > (8 << 20) and (2 << 20) < sizes[2] <= (8 << 20)
        assert (2 << 20) < sizes[3] <= (8 << 20)
        rids = [srv.submit_render(sid, off, spp) for sid, _, off, spp in jobs]
        cancelled = srv.submit_render(big_ids[0], 0, 600)
        srv.cancel(cancelled)
        shapes = [(48, 40), (32, 32), (24, 30)]
        srids = [srv.submit_render(small_ids[k], 3 * k, 24 + 8 * k) for k in range(3)]
        sliced = srv.submit_render(small_ids[0], 50, 40, slice_spp=8)
        for r in rids + srids + [sliced]:
            assert srv.wait(r).state == "done"
        st = srv.wait(cancelled)
        assert st.state == "cancelled" and st.samples_done == 0
        assert not srv.film(cancelled).any()
        for r, (sid, shape, off, spp) in zip(rids, jobs):
            assert np.array_equal(srv.film(r).view(np.uint32), _resident(srv, sid, shape, off, spp).view(np.uint32))
        for k, r in enumerate(srids):
            ref = _resident(srv, small_ids[k], shapes[k], 3 * k, 24 + 8 * k)
            assert np.array_equal(srv.film(r).view(np.uint32), ref.view(np.uint32))
        ref = _resident(srv, small_ids[0], shapes[0], 50, 40)
        assert np.array_equal(srv.film(sliced).view(np.uint32), ref.view(np.uint32))
        srv.release(sliced)
        for r in rids + srids + [cancelled]:
            srv.release(r)
    finally:
        srv.close()
