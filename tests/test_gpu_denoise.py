"""The device guide pass and A-Trous filter against the oracle (tests/
test_oracle_denoise.py pins the oracle to the reference's denoiser tests).

* Guide pass: bit-identical to the oracle (the same plane scan as the transport).
* A-Trous: the tap arithmetic is the reference's; only CUDA's expf (and powf for a
  non-power-of-two normal power) differs from glibc by an ULP, so the filtered images
  agree to 1e-5 relative.  The identity short-circuit at high spp is bit-exact.
* denoise_and_tonemap_frame on the device: RGBA within one 8-bit step of the oracle's
  filter followed by the oracle's tone map.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from denoise_fixtures import irregular_scene
from gemray_studio_b200 import abi, scene as S
from gemray_studio_b200.denoise import AtrousParams, GuideBuffers, denoise, generate_guide_buffers
from test_oracle_denoise import run as oracle_denoise

pytestmark = pytest.mark.gpu
fp = C.POINTER(C.c_float)
ip = C.POINTER(C.c_int32)


def _oracle_guides(oracle, sc):
    n = sc.width * sc.height
    g = GuideBuffers(np.empty(n, np.float32), np.empty((n, 3), np.float32), np.empty(n, np.int32))
    oracle.gro_guide_buffers(C.byref(sc.c_scene()), g.depth.ctypes.data_as(fp), g.normal.ctypes.data_as(fp),
                             g.facet_id.ctypes.data_as(ip))
    return g


@pytest.mark.parametrize("planes", ["srb", "rb57", "none"])
def test_guide_buffers_bit_identical(renderer, oracle, planes):
    p = {"srb": S.standard_round_brilliant(), "rb57": S.round_brilliant_57(), "none": np.zeros((0, 4), np.float32)}
    sc = S.Scene(width=97, height=61, planes=p[planes], material=S.builtin_material("Diamond"),
                 cam=S.camera(0.35, 0.28, 5.0, 18.0))
    got, ref = generate_guide_buffers(renderer, sc), _oracle_guides(oracle, sc)
    assert np.array_equal(got.facet_id, ref.facet_id)
    assert got.depth.tobytes() == ref.depth.tobytes()
    assert got.normal.tobytes() == ref.normal.tobytes()


def _close(a, b, rel=1e-5):
    return np.max(np.abs(a.astype(np.float64) - b) / np.maximum(np.abs(b), 1e-3)) <= rel


@pytest.mark.parametrize("w,h,seed", [(137, 91, 0x12345678), (113, 67, 0xABCDEF01)])
def test_atrous_matches_oracle(renderer, oracle, w, h, seed):
    color, depth, normal, facet = irregular_scene(w, h, seed)
    g = GuideBuffers(depth, normal, facet)
    for spp, params in [(1, AtrousParams()), (16, AtrousParams()), (3, AtrousParams(num_passes=8, normal_power=60.0)),
                        (0, AtrousParams(num_passes=2, sigma_depth=0.5))]:
        got = denoise(renderer, color, g, w, h, spp, params)
        ref = oracle_denoise(oracle, color, depth, normal, facet, w, h, spp,
                             (params.num_passes, params.sigma_color, params.sigma_depth, params.normal_power,
                              params.taper_reference_spp, params.taper_identity_epsilon))
        assert _close(got, ref), (spp, params)
    again = denoise(renderer, color, g, w, h, 1)
    assert again.tobytes() == denoise(renderer, color, g, w, h, 1).tobytes()  # deterministic


def test_atrous_identity_at_high_spp(renderer):
    color, depth, normal, facet = irregular_scene(40, 30, 7)
    got = denoise(renderer, color, GuideBuffers(depth, normal, facet), 40, 30, 100_000)
    assert got.tobytes() == color.tobytes()


def test_denoise_tonemap_on_device(renderer, oracle):
    import torch
    sc = S.Scene(width=96, height=64, planes=S.standard_round_brilliant(), material=S.builtin_material("Diamond"),
                 cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=12)
    count = 8
    film = np.zeros((96 * 64, 3), np.float32)
    renderer.accumulate(sc, 0, count, film)
    g = generate_guide_buffers(renderer, sc)
    dev = {k: torch.from_numpy(v).cuda() for k, v in
           {"film": film, "depth": g.depth, "normal": g.normal, "facet": g.facet_id}.items()}
    rgba = torch.zeros((96 * 64, 4), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    st = renderer.lib.gr_denoise_tonemap_device(renderer.ctx, dev["film"].data_ptr(), count, dev["depth"].data_ptr(),
                                                dev["normal"].data_ptr(), dev["facet"].data_ptr(), 96, 64, None,
                                                rgba.data_ptr(), None)
    assert st == abi.GR_OK
    renderer.synchronize()
    avg = film * np.float32(np.float32(1.0) / np.float32(count))
    ref = oracle_denoise(oracle, avg, g.depth, g.normal, g.facet_id, 96, 64, count)
    ref_rgba = np.empty((96 * 64, 4), np.uint8)
    oracle.gro_tonemap(ref.ctypes.data_as(fp), 1.0, 96 * 64, ref_rgba.ctypes.data_as(C.POINTER(C.c_uint8)))
    diff = np.abs(rgba.cpu().numpy().astype(int) - ref_rgba.astype(int))
    assert diff.max() <= 1 and np.mean(diff > 0) < 0.01
