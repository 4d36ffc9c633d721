"""gr_render_resident_static (fixed device scratch, no allocation) against gr_render_resident.

Named so that it is collected last: it must pass alone and after every other test.
Two consecutive calls (sample ranges [0, spp) and [spp, 2*spp)) into the same film
must give a film bit-identical to the same two calls through gr_render_resident (same
kernels, each pixel's samples folded in the same order; only the chunking differs),
and the second call must leave the device's free memory unchanged.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import abi, scene as S
from helpers import srb_scene

pytestmark = pytest.mark.gpu


@pytest.fixture()
def ctx(engine_lib):
    h = C.c_void_p()
    assert engine_lib.gr_create(C.byref(h), None) == abi.GR_OK, engine_lib.gr_last_error_string()
    yield h
    assert engine_lib.gr_destroy(h) == abi.GR_OK


def _upload(lib, ctx, sc):
    sid = C.c_uint64()
    assert lib.gr_scene_upload(ctx, C.byref(sc.c_scene()), C.byref(sid)) == abi.GR_OK, lib.gr_last_error_string()
    return sid.value


def _two_calls(lib, ctx, fn, sid, spp, film, mem=None):
    import torch
    for k in range(2):
        st = fn(ctx, sid, k * spp, spp, C.c_void_p(film.data_ptr()), None)
        assert st == abi.GR_OK, lib.gr_last_error_string()
        assert lib.gr_synchronize(ctx) == abi.GR_OK
        if mem is not None:
            mem.append(torch.cuda.mem_get_info()[0])


@pytest.mark.parametrize("case", ["latlong_multichunk", "studio_onechunk"])
def test_static_scratch_matches_resident_on_two_calls(engine_lib, ctx, case):
    import torch
    lib = engine_lib
    if case == "latlong_multichunk":
        # 3072 px x 1024 spp: chunks of 1365 px, three per call
        sc = srb_scene("Diamond", width=64, height=48, max_bounces=16, env_mode=abi.GR_ENV_LATLONG,
                       latlong=S.gaussian_blob_latlong(256, 128, seed=3))
        spp = 1024
        assert abi.GR_STATIC_SCRATCH_TUPLES // spp < sc.width * sc.height
    else:
        sc = srb_scene("Sapphire", width=40, height=30, max_bounces=24)
        spp = 64
    sid = _upload(lib, ctx, sc)
    n = sc.width * sc.height
    seed = torch.rand((n, 3), dtype=torch.float32, generator=torch.Generator().manual_seed(5))
    ref = seed.clone().cuda()
    got = seed.clone().cuda()
    torch.cuda.synchronize()
    _two_calls(lib, ctx, lib.gr_render_resident, sid, spp, ref)
    mem = []
    _two_calls(lib, ctx, lib.gr_render_resident_static, sid, spp, got, mem)
    a = ref.cpu().numpy()
    b = got.cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert not np.array_equal(a, seed.numpy())  # the calls added light
    assert mem[0] == mem[1], mem                # the second call allocated nothing
    assert lib.gr_scene_release(ctx, sid) == abi.GR_OK


def test_static_scratch_rejects_oversize_spp(engine_lib, ctx):
    import torch
    lib = engine_lib
    sc = srb_scene("Diamond", width=4, height=4, max_bounces=4)
    sid = _upload(lib, ctx, sc)
    film = torch.ones((16, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = lib.gr_render_resident_static(ctx, sid, 0, abi.GR_STATIC_SCRATCH_TUPLES + 1, C.c_void_p(film.data_ptr()), None)
    assert st == abi.GR_EINVAL
    assert b"static scratch" in lib.gr_last_error_string()
    assert lib.gr_synchronize(ctx) == abi.GR_OK
    assert torch.equal(film.cpu(), torch.ones((16, 3)))
    # the largest accepted spp is the scratch capacity (one pixel per chunk); spp 0 is a no-op
    assert lib.gr_render_resident_static(ctx, sid, 0, 0, C.c_void_p(film.data_ptr()), None) == abi.GR_OK
    assert lib.gr_scene_release(ctx, sid) == abi.GR_OK
