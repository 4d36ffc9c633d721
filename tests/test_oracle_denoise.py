"""Pins the oracle's A-Trous denoiser and guide pass to the reference's own denoiser
tests (crates/gemray/tests/denoise_tests.rs, crates/gemray/src/renderer/denoise/mod.rs
tests), with their inputs and bounds; the reference holds no golden images for the
denoiser.  The device filter is compared against this oracle on the GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from denoise_fixtures import Xorshift32, irregular_scene, unit
from gemray_studio_b200 import scene as S

fp = C.POINTER(C.c_float)
ip = C.POINTER(C.c_int32)
DEFAULT = (5, 0.35, 0.1, 64.0, 4.0, 0.02)


def run(oracle, color, depth, normal, facet, w, h, spp, params=DEFAULT):
    out = np.zeros((w * h, 3), np.float32)
    c = np.ascontiguousarray(color, np.float32)
    d = np.ascontiguousarray(depth, np.float32)
    n = np.ascontiguousarray(normal, np.float32)
    f = np.ascontiguousarray(facet, np.int32)
    oracle.gro_atrous_denoise(c.ctypes.data_as(fp), d.ctypes.data_as(fp), n.ctypes.data_as(fp), f.ctypes.data_as(ip),
                              w, h, spp, *params, out.ctypes.data_as(fp))
    return out


def _flat(w, h):
    return np.ones(w * h, np.float32), np.tile(np.array([0, 0, 1], np.float32), (w * h, 1))


def test_filtering_reduces_error_against_ground_truth(oracle):
    w = h = 48
    a, b = np.array([0.6, 0.5, 0.2], np.float32), np.array([0.1, 0.3, 0.7], np.float32)
    xs = np.tile(np.arange(w), h)
    truth = np.where((xs < w // 2)[:, None], a, b).astype(np.float32)
    facet = np.where(xs < w // 2, 0, 1).astype(np.int32)
    rng = Xorshift32(12345)
    noisy = truth.copy()
    for i in range(w * h):
        nz = np.array([rng.next_signed(), rng.next_signed(), rng.next_signed()], np.float32) * np.float32(0.4)
        noisy[i] = np.maximum(noisy[i] + nz, 0)
    depth, normal = _flat(w, h)
    out = run(oracle, noisy, depth, normal, facet, w, h, 1)
    mse = lambda x: float(np.mean(np.sum((x.astype(np.float64) - truth) ** 2, axis=1)))
    assert mse(out) < 0.5 * mse(noisy)


def test_facet_edges_survive(oracle):
    w, h, split = 64, 32, 32
    xs = np.tile(np.arange(w), h)
    color = np.where((xs < split)[:, None], [0.9, 0.05, 0.05], [0.05, 0.05, 0.9]).astype(np.float32)
    facet = np.where(xs < split, 7, 42).astype(np.int32)
    depth, normal = _flat(w, h)
    out = run(oracle, color, depth, normal, facet, w, h, 1)
    y = h // 2
    l, r = y * w + split - 1, y * w + split
    assert np.linalg.norm(out[r] - out[l]) > 0.95 * np.linalg.norm(color[r] - color[l])


def test_high_sample_count_is_identity(oracle):
    rng = Xorshift32(999)
    color = np.array([[rng.next_f32(), rng.next_f32(), rng.next_f32()] for _ in range(256)], np.float32)
    facet = (np.arange(256) % 3).astype(np.int32)
    depth, normal = _flat(16, 16)
    out = run(oracle, color, depth, normal, facet, 16, 16, 100_000)
    assert out.tobytes() == color.tobytes()


def test_taper_decreases_monotonically(oracle):
    prev = oracle.gro_taper_strength(0, 4.0)
    assert abs(prev - 1.0) < 1e-6
    for spp in (1, 4, 16, 64, 256, 1024, 100_000):
        t = oracle.gro_taper_strength(spp, 4.0)
        assert 0 < t < prev
        prev = t


def test_uniform_image_is_unchanged(oracle):
    rng = Xorshift32(42)
    n = 400
    facet = np.zeros(n, np.int32)
    depth = np.zeros(n, np.float32)
    normal = np.zeros((n, 3), np.float32)
    for i in range(n):
        facet[i] = rng.next_u32() % 4
        depth[i] = rng.next_f32()
        normal[i] = unit([rng.next_signed(), rng.next_signed(), 1.0])
    const = np.array([0.37, 0.61, 0.14], np.float32)
    out = run(oracle, np.tile(const, (n, 1)), depth, normal, facet, 20, 20, 1)
    assert np.max(np.linalg.norm(out - const, axis=1)) < 1e-4


def test_degenerate_inputs(oracle):
    depth, normal = _flat(1, 1)
    one = run(oracle, np.array([[0.2, 0.3, 0.4]], np.float32), depth, normal, np.zeros(1, np.int32), 1, 1, 1)
    assert np.all(np.isfinite(one))
    run(oracle, np.zeros((0, 3), np.float32), np.zeros(0, np.float32), np.zeros((0, 3), np.float32),
        np.zeros(0, np.int32), 0, 0, 1)
    color, d, nrm, f = irregular_scene(24, 16, 5)
    for spp in (0, 1):
        assert np.all(np.isfinite(run(oracle, color, d, nrm, f, 24, 16, spp)))
    black = run(oracle, np.zeros_like(color), d, nrm, f, 24, 16, 1)
    assert np.all(black == 0)
    zero_passes = run(oracle, color, d, nrm, f, 24, 16, 1, (0,) + DEFAULT[1:])
    one_pass = run(oracle, color, d, nrm, f, 24, 16, 1, (1,) + DEFAULT[1:])
    assert zero_passes.tobytes() == one_pass.tobytes()  # num_passes clamps to [1, 8]


def test_cos_pow_matches_powf(oracle):
    for power in (1.0, 2.0, 4.0, 8.0, 16.0, 32.0, 64.0, 128.0):
        for base in (0.0, 0.1, 0.37, 0.5, 0.9, 1.0):
            fast = oracle.gro_cos_pow(base, power)
            ref = np.float32(base) ** np.float32(power)
            assert abs(fast - ref) <= abs(ref) * 1e-5 + 1e-6
    for power in (5.0, 60.0):
        for base in (0.0, 0.3, 0.7, 1.0):
            assert np.float32(oracle.gro_cos_pow(base, power)) == np.float32(np.float32(base) ** np.float32(power)) \
                or abs(oracle.gro_cos_pow(base, power) - float(np.float32(base) ** np.float32(power))) < 1e-7


def test_guide_pass_on_the_round_brilliant(oracle):
    sc = S.Scene(width=48, height=36, planes=S.standard_round_brilliant(), material=S.builtin_material("Diamond"),
                 cam=S.camera(0.35, 0.28, 5.0, 18.0))
    n = 48 * 36
    depth, normal, facet = np.empty(n, np.float32), np.empty((n, 3), np.float32), np.empty(n, np.int32)
    oracle.gro_guide_buffers(C.byref(sc.c_scene()), depth.ctypes.data_as(fp), normal.ctypes.data_as(fp),
                             facet.ctypes.data_as(ip))
    hit = facet >= 0
    assert 0.1 < hit.mean() < 0.9  # the stone covers part of the frame
    assert np.all(depth[~hit] == 1e6) and np.all(normal[~hit] == 0)
    assert np.all((depth[hit] > 0) & (depth[hit] < 10)) and np.all(facet[hit] < 74)
    assert np.allclose(np.linalg.norm(normal[hit], axis=1), 1.0, atol=1e-5)
    planes = S.standard_round_brilliant()
    assert np.array_equal(normal[hit], planes[facet[hit], :3])
