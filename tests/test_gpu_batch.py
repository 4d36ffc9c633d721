"""gr_render_batch: many resident scenes in shared launches.

Every film must be bit-identical to rendering its item alone with gr_render_resident
(same per-tuple arithmetic, same per-pixel fold order), with and without CUDA-graph
replay, across launch boundaries (a small chunk budget splits scenes between
launches) and for scenes of different plane counts, materials, environments and
frame sizes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import abi, scene as S

pytestmark = pytest.mark.gpu


def _scenes():
    rng = np.random.default_rng(4)
    env = S.gaussian_blob_latlong(256, 128, seed=2)
    cam = S.camera(0.35, 0.28, 5.0, 18.0)
    out = []
    specs = [(S.round_brilliant_57(), "Diamond", 48, 40, abi.GR_ENV_LATLONG, 0),
             (S.standard_round_brilliant(), "Sapphire", 33, 21, abi.GR_ENV_STUDIO, 0),
             (S.emerald_cut_49(), "Tourmaline", 40, 30, abi.GR_ENV_UNIFORM, 0),
             (S.random_polyhedron(rng, 17, 17), "Zircon", 24, 24, abi.GR_ENV_LATLONG, abi.GR_FLAG_KAHAN_FILM),
             (S.random_polyhedron(rng, 140, 145), "Cubic Zirconia", 30, 17, abi.GR_ENV_STUDIO, 0)]
    for planes, mat, w, h, env_mode, flags in specs:
        out.append(S.Scene(width=w, height=h, planes=planes, material=S.builtin_material(mat), cam=cam,
                           max_bounces=16, env_mode=env_mode, latlong=env, flags=flags))
    return out


@pytest.fixture()
def ctx(engine_lib):
    h = C.c_void_p()
    opts = abi.gr_create_opts(device=-1, chunk_budget_bytes=12 * 9000, serve_budget_bytes=0)
    assert engine_lib.gr_create(C.byref(h), C.byref(opts)) == abi.GR_OK
    yield h
    assert engine_lib.gr_destroy(h) == abi.GR_OK


def _upload(lib, ctx, scenes):
    ids = []
    for sc in scenes:
        sid = C.c_uint64()
        assert lib.gr_scene_upload(ctx, C.byref(sc.c_scene()), C.byref(sid)) == abi.GR_OK, lib.gr_last_error_string()
        ids.append(sid.value)
    return ids


@pytest.mark.parametrize("flags", [0, abi.GR_BATCH_GRAPH])
def test_batch_matches_scenes_rendered_alone(engine_lib, ctx, flags):
    import torch
    lib = engine_lib
    scenes = _scenes()
    ids = _upload(lib, ctx, scenes)
    spps = [24, 7, 40, 64, 3]
    alone = [torch.zeros((sc.width * sc.height, 3), dtype=torch.float32, device="cuda") for sc in scenes]
    batched = [torch.zeros_like(f) for f in alone]
    torch.cuda.synchronize()
    for rnd in range(3):  # three progressive rounds: the graph is captured once, then replayed
        items = (abi.gr_batch_item * len(scenes))()
        for i, sc in enumerate(scenes):
            off = rnd * spps[i] + 5 * i
            st = lib.gr_render_resident(ctx, ids[i], off, spps[i], C.c_void_p(alone[i].data_ptr()), None)
            assert st == abi.GR_OK, lib.gr_last_error_string()
            items[i] = abi.gr_batch_item(ids[i], batched[i].data_ptr(), off, spps[i])
        assert lib.gr_render_batch(ctx, items, len(scenes), flags, None) == abi.GR_OK, lib.gr_last_error_string()
        assert lib.gr_synchronize(ctx) == abi.GR_OK
        for i in range(len(scenes)):
            a, b = alone[i].cpu().numpy(), batched[i].cpu().numpy()
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (rnd, i)
            assert a.any()


def test_batch_edge_cases(engine_lib, ctx):
    import torch
    lib = engine_lib
    sc = _scenes()[0]
    (sid,) = _upload(lib, ctx, [sc])
    film = torch.zeros((sc.width * sc.height, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    assert lib.gr_render_batch(ctx, None, 0, 0, None) == abi.GR_OK                      # empty batch
    items = (abi.gr_batch_item * 2)(abi.gr_batch_item(sid, film.data_ptr(), 0, 0),      # spp 0 is a no-op
                                    abi.gr_batch_item(sid + 99, film.data_ptr(), 0, 4))  # unknown scene
    assert lib.gr_render_batch(ctx, items, 2, 0, None) == abi.GR_ENOTFOUND
    items[1] = abi.gr_batch_item(sid, None, 0, 4)
    assert lib.gr_render_batch(ctx, items, 2, 0, None) == abi.GR_EINVAL
    # spp larger than the whole chunk budget: one pixel per packed launch (a 12x12 frame
    # stays under the 2 M path-samples from which an item renders on its own)
    tiny = _scenes()[0]
    tiny.width = tiny.height = 12
    (tid,) = _upload(lib, ctx, [tiny])
    tfilm = torch.zeros((144, 3), dtype=torch.float32, device="cuda")
    items = (abi.gr_batch_item * 1)(abi.gr_batch_item(tid, tfilm.data_ptr(), 0, 10000))
    ref = torch.zeros_like(tfilm)
    torch.cuda.synchronize()
    assert lib.gr_render_batch(ctx, items, 1, 0, None) == abi.GR_OK
    assert lib.gr_render_resident(ctx, tid, 0, 10000, C.c_void_p(ref.data_ptr()), None) == abi.GR_OK
    assert lib.gr_synchronize(ctx) == abi.GR_OK
    assert torch.equal(tfilm, ref)
    # an item of 2 M path-samples or more renders with the single-scene kernels, beside
    # packed ones: every film is still gr_render_resident's
    small = _scenes()[1]
    (smid,) = _upload(lib, ctx, [small])
    sfilm = torch.zeros((small.width * small.height, 3), dtype=torch.float32, device="cuda")
    film.zero_()
    items = (abi.gr_batch_item * 2)(abi.gr_batch_item(sid, film.data_ptr(), 7, 1200),
                                    abi.gr_batch_item(smid, sfilm.data_ptr(), 3, 40))
    assert sc.width * sc.height * 1200 >= (2 << 20)
    ref, sref = torch.zeros_like(film), torch.zeros_like(sfilm)
    torch.cuda.synchronize()
    assert lib.gr_render_batch(ctx, items, 2, abi.GR_BATCH_GRAPH, None) == abi.GR_OK
    assert lib.gr_render_resident(ctx, sid, 7, 1200, C.c_void_p(ref.data_ptr()), None) == abi.GR_OK
    assert lib.gr_render_resident(ctx, smid, 3, 40, C.c_void_p(sref.data_ptr()), None) == abi.GR_OK
    assert lib.gr_synchronize(ctx) == abi.GR_OK
    assert torch.equal(film, ref) and torch.equal(sfilm, sref) and film.any()
