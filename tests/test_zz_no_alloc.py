"""gr_render_resident_static (fixed device scratch, no allocation) against gr_render_resident.

Some callers cannot allocate device memory inside a render call: a serving loop that
commits its memory up front (a caching allocator holding the device), where a mid-frame
cudaMalloc can fail and a cudaFree would synchronise the whole device.  The static
entry point traces into a file-scope device array instead.

Named so that it is collected last: it must pass alone and after every other test.
Each case uses a fresh context and runs the static calls BEFORE any gr_render_resident
call on it, so nothing the resident path grew can hide an allocation: a one-pixel warm
call looks up the array (and loads the kernels), then the device's free memory must be
the same before the first real static call and after each of two consecutive calls
(sample ranges [0, spp) and [spp, 2*spp)).  The resident comparison runs afterwards:
the films must be bit-identical (same kernels, each pixel's samples folded in the same
order; only the chunking differs).
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


def _call(lib, ctx, fn, sid, offset, spp, film):
    st = fn(ctx, sid, offset, spp, C.c_void_p(film.data_ptr()), None)
    assert st == abi.GR_OK, lib.gr_last_error_string()
    assert lib.gr_synchronize(ctx) == abi.GR_OK


def _warm_static(lib, ctx):
    """One real static call on a 1-pixel scene: the scratch address lookup and the
    first launches of the plain trace and fold kernels happen here."""
    import torch
    tiny = srb_scene("Diamond", width=1, height=1, max_bounces=2)
    sid = _upload(lib, ctx, tiny)
    film = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    _call(lib, ctx, lib.gr_render_resident_static, sid, 0, 1, film)
    return sid, film


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
    warm_sid, warm_film = _warm_static(lib, ctx)
    sid = _upload(lib, ctx, sc)
    n = sc.width * sc.height
    seed = torch.rand((n, 3), dtype=torch.float32, generator=torch.Generator().manual_seed(5))
    got = seed.clone().cuda()
    ref = seed.clone().cuda()
    torch.cuda.synchronize()
    free = [torch.cuda.mem_get_info()[0]]
    for k in range(2):
        _call(lib, ctx, lib.gr_render_resident_static, sid, k * spp, spp, got)
        free.append(torch.cuda.mem_get_info()[0])
    assert free[0] == free[1] == free[2], free  # no call allocated device memory
    for k in range(2):
        _call(lib, ctx, lib.gr_render_resident, sid, k * spp, spp, ref)
    a = ref.cpu().numpy()
    b = got.cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert not np.array_equal(a, seed.numpy())  # the calls added light
    assert lib.gr_scene_release(ctx, sid) == abi.GR_OK
    assert lib.gr_scene_release(ctx, warm_sid) == abi.GR_OK
    del warm_film


def test_static_scratch_exact_fill(engine_lib, ctx):
    """spp = GR_STATIC_SCRATCH_TUPLES, the largest accepted: one pixel per chunk fills
    16,777,212 of the array's 16,777,216 bytes.  Two pixels, two chunks; the film is the
    resident path's bit for bit."""
    import torch
    lib = engine_lib
    spp = abi.GR_STATIC_SCRATCH_TUPLES
    sc = srb_scene("Diamond", width=2, height=1, max_bounces=3)
    warm_sid, warm_film = _warm_static(lib, ctx)
    sid = _upload(lib, ctx, sc)
    got = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
    ref = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    _call(lib, ctx, lib.gr_render_resident_static, sid, 0, spp, got)
    assert torch.cuda.mem_get_info()[0] == before
    _call(lib, ctx, lib.gr_render_resident, sid, 0, spp, ref)
    assert np.array_equal(got.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))
    assert got.sum().item() > 0
    assert lib.gr_scene_release(ctx, sid) == abi.GR_OK
    assert lib.gr_scene_release(ctx, warm_sid) == abi.GR_OK
    del warm_film


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
    # spp 0 is a no-op
    assert lib.gr_render_resident_static(ctx, sid, 0, 0, C.c_void_p(film.data_ptr()), None) == abi.GR_OK
    assert torch.equal(film.cpu(), torch.ones((16, 3)))
    assert lib.gr_scene_release(ctx, sid) == abi.GR_OK
