"""Pins the oracle's frosted-facet and volume-scattering paths to the reference's own
property tests for them, with the reference's sample loops, seeds and tolerances:

* crates/gemray/tests/raytracer_tests.rs:2246-2300 (all-polished finishes are
  bit-identical to no finishes), :2322-2372 (frosted girdle white furnace, tolerance
  0.9), :2411-2460 (a frosted girdle raises face-up Y by more than 1 %), :2710-2760
  (birefringent frosted girdle white furnace, tolerance 0.05);
* crates/gemray/src/optics/raytracer/scattering.rs scattering_tests (HG sampling mean
  cosine converges to g; sampled directions finite and unit; sigma_s = 0 is
  bit-identical whatever g; lossless scattering white furnace, tolerance 0.08;
  scattering changes face-up Y by more than 1 %).

The reference suite holds no golden vectors for these paths, so these properties,
together with the per-sample device-vs-oracle tests, are what pins them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from gemray_studio_b200 import abi, scene as S
from helpers import hash_draw

PLANES = S.standard_round_brilliant()
CAM = S.camera(0.35, 0.28, 5.0, 18.0)
L0 = 2.5
UNIFORM = dict(env_mode=abi.GR_ENV_UNIFORM, uniform_rgb=(L0, L0, L0))


def _girdle():
    f = np.zeros(PLANES.shape[0], np.uint32)
    f[33:49] = 1  # STANDARD_ROUND_BRILLIANT_GIRDLE_FACETS (geometry/cuts.rs:37)
    return f


def _scattering(m: abi.gr_material, sigma_s: float, g: float) -> abi.gr_material:
    m = abi.gr_material.from_buffer_copy(m)
    m.scattering_sigma_s, m.scattering_g = sigma_s, g
    return m


def _probe(oracle, sc: S.Scene, grid: int, spp: int, salt: int, max_bounces: int) -> np.ndarray:
    out = (C.c_float * 3)()
    st = oracle.gro_probe_grid(C.byref(sc.c_scene()), grid, spp, salt, max_bounces, out)
    assert st == abi.GR_OK
    return np.array(out, np.float32)


def _target(oracle) -> np.ndarray:
    t = (C.c_float * 3)()
    oracle.gro_furnace_target(L0, t)
    return np.array(t, np.float32)


def _trace(oracle, sc, origin, d, seed, max_bounces=12):
    xyz = (C.c_double * 3)()
    o3, d3 = (C.c_float * 3)(*origin), (C.c_float * 3)(*d)
    assert oracle.gro_trace_ray(C.byref(sc.c_scene()), o3, d3, seed, hash_draw(oracle, seed), max_bounces, 32, xyz,
                                None, None) == 0
    return np.array(xyz, np.float32)


def test_all_polished_finishes_bit_identical(oracle):
    d2 = np.array([0.18, -1.0, 0.07], np.float32)
    d2 = d2 / np.float32(np.sqrt(np.float32(d2 @ d2)))
    rays = [((0.0, 2.5, 0.0), (0.0, -1.0, 0.0)), ((0.0, 2.5, 0.0), tuple(float(x) for x in d2))]
    for name in ("Diamond", "Zircon", "Sapphire"):
        m = S.builtin_material(name)
        for o, d in rays:
            for seed in (1, 42, 9001):
                a = _trace(oracle, S.Scene(1, 1, PLANES, m, CAM), o, d, seed)
                b = _trace(oracle, S.Scene(1, 1, PLANES, m, CAM, finishes=np.zeros(PLANES.shape[0], np.uint32)),
                           o, d, seed)
                assert a.tobytes() == b.tobytes(), (name, seed)


def test_frosted_girdle_white_furnace(oracle):
    mean = _probe(oracle, S.Scene(12, 12, PLANES, S.custom_material(1.5, 0.0, 0.0), CAM, finishes=_girdle(),
                                  **UNIFORM), 12, 64, 0x46575230, 12)
    err = np.abs(mean - _target(oracle)) / _target(oracle)
    assert np.all(err <= 0.9), err  # the reference's bound; measured +4.9 %


def test_frosted_girdle_birefringent_white_furnace(oracle):
    mean = _probe(oracle, S.Scene(12, 12, PLANES, S.custom_material(1.5, 0.0, 0.03), CAM, finishes=_girdle(),
                                  **UNIFORM), 12, 64, 0x46524247, 12)
    err = np.abs(mean - _target(oracle)) / _target(oracle)
    assert np.all(err <= 0.05), err  # measured +1.7 %


def test_frosted_girdle_raises_face_up_y(oracle):
    d = S.builtin_material("Diamond")
    pol = _probe(oracle, S.Scene(16, 16, PLANES, d, CAM), 16, 96, 0x9A7EC6F1, 12)
    fro = _probe(oracle, S.Scene(16, 16, PLANES, d, CAM, finishes=_girdle()), 16, 96, 0x9A7EC6F1, 12)
    assert fro[1] > pol[1] and (fro[1] - pol[1]) / pol[1] > 0.01, (pol[1], fro[1])


def _unit_draws(h, salt: int, n: int) -> np.ndarray:
    """(hash_u32(i ^ salt) as f32) / 4_294_967_295.0 for i in 0..n, in f32."""
    return np.array([h(i ^ salt) for i in range(n)], np.uint32).astype(np.float32) / np.float32(4294967295.0)


def test_hg_sampling_mean_cos_converges_to_g(oracle):
    fwd = np.array([0.2, 0.6, 0.77], np.float32)
    fwd = fwd / np.float32(np.sqrt(np.float32(fwd @ fwd)))
    f3, out = (C.c_float * 3)(*fwd), (C.c_float * 3)()
    h = oracle.gro_hash_u32
    n = 400_000
    u1 = _unit_draws(h, 0x11111111, n).tolist()
    u2 = _unit_draws(h, 0x22222222, n).tolist()
    for g in (-0.7, -0.2, 0.0, 0.4, 0.85):
        s = 0.0
        for a, b in zip(u1, u2):
            oracle.gro_sample_hg(a, b, g, f3, out)
            s += out[0] * f3[0] + out[1] * f3[1] + out[2] * f3[2]
        assert abs(s / n - g) < 0.01, (g, s / n)


def test_hg_and_cosine_directions_finite_unit(oracle):
    h = oracle.gro_hash_u32
    fwd = np.array([-0.3, 0.1, 0.94], np.float32)
    fwd = fwd / np.float32(np.sqrt(np.float32(fwd @ fwd)))
    f3, out = (C.c_float * 3)(*fwd), (C.c_float * 3)()
    u1, u2 = _unit_draws(h, 0x33333333, 2000).tolist(), _unit_draws(h, 0x44444444, 2000).tolist()
    for g in (-0.999, -0.5, -1e-3, 0.0, 1e-3, 0.5, 0.999):
        for i in range(2000):
            oracle.gro_sample_hg(u1[i], u2[i], g, f3, out)
            v = np.array(out, np.float64)
            assert np.all(np.isfinite(v)) and abs(np.linalg.norm(v) - 1.0) < 1e-4, (g, i, v)
    cos_sum = 0.0
    c1, c2 = _unit_draws(h, 0x55555555, 20000).tolist(), _unit_draws(h, 0x66666666, 20000).tolist()
    for i in range(20000):
        oracle.gro_cosine_hemisphere(c1[i], c2[i], f3, out)
        v = np.array(out, np.float64)
        c = float(v @ fwd)
        assert abs(np.linalg.norm(v) - 1.0) < 1e-4 and c >= -1e-6, (i, v)
        cos_sum += c
    assert abs(cos_sum / 20000 - 2.0 / 3.0) < 0.01  # E[cos] of a cosine-weighted lobe


def test_default_off_scattering_bit_identical_whatever_g(oracle):
    ruby = S.builtin_material("Ruby")
    assert ruby.scattering_sigma_s <= 0.0
    env = dict(preset="Daylight", exposure=1.0, light_yaw=0.4, light_pitch=0.35)
    for g in (-0.6, 0.0, 0.4, 0.95):
        for salt in (0x13579BDF, 0x2468ACE0):
            a = _probe(oracle, S.Scene(6, 6, PLANES, ruby, CAM, **env), 6, 4, salt, 10)
            b = _probe(oracle, S.Scene(6, 6, PLANES, _scattering(ruby, 0.0, g), CAM, **env), 6, 4, salt, 10)
            assert a.tobytes() == b.tobytes(), g


def test_lossless_scattering_white_furnace(oracle):
    m = _scattering(S.custom_material(1.5, 0.0, 0.0), 1.2, 0.4)
    mean = _probe(oracle, S.Scene(12, 12, PLANES, m, CAM, **UNIFORM), 12, 96, 0x5CA1AB1E, 16)
    err = np.abs(mean - _target(oracle)) / _target(oracle)
    assert np.all(err <= 0.08), err  # measured -1.7 % (the polished stone at 16 bounces: -1.2 %)


def test_scattering_changes_face_up_y(oracle):
    d = S.builtin_material("Diamond")
    clear = _probe(oracle, S.Scene(14, 14, PLANES, d, CAM), 14, 96, 0x0BADF00D, 12)
    hazy = _probe(oracle, S.Scene(14, 14, PLANES, _scattering(d, 1.5, 0.3), CAM), 14, 96, 0x0BADF00D, 12)
    assert abs(hazy[1] - clear[1]) / clear[1] > 0.01, (clear[1], hazy[1])


# ---- edge rounding (optics/raytracer/intersect.rs:196-229 and its tests :312-600) ----

def _corner_planes():
    return (abi.gr_plane * 2)(abi.gr_plane((0.0, 1.0, 0.0), 0.0), abi.gr_plane((1.0, 0.0, 0.0), 0.0))


def _shade(oracle, hp, idx, hn, radius):
    out = (C.c_float * 3)()
    oracle.gro_shading_normal(_corner_planes(), 2, (C.c_float * 3)(*hp), idx, (C.c_float * 3)(*hn), radius, out)
    return np.array(out, np.float32)


def test_edge_rounding_unit_properties(oracle):
    up, right = (0.0, 1.0, 0.0), (1.0, 0.0, 0.0)
    for r in (0.0, -1.0, -0.001):  # disabled: the flat normal, unchanged
        assert _shade(oracle, (0, 0, 5), 0, up, r).tolist() == [0.0, 1.0, 0.0]
    a, b = _shade(oracle, (0, 0, 5), 0, up, 1.0), _shade(oracle, (0, 0, 5), 1, right, 1.0)
    bis = np.array([1, 1, 0], np.float32) / np.float32(np.sqrt(2))
    assert np.linalg.norm(a - b) < 1e-5 and np.linalg.norm(a - bis) < 1e-5  # continuous; the bisector at the edge
    assert _shade(oracle, (-10, 0, 5), 0, up, 1.0).tolist() == [0.0, 1.0, 0.0]  # interior stays flat
    t = np.float32(0.5)
    st = t * t * np.float32(3.0 - 2.0 * 0.5)
    exp = np.array(up, np.float32) * (1 - st) + bis * st
    exp /= np.linalg.norm(exp)
    assert np.linalg.norm(_shade(oracle, (-0.5, 0, 5), 0, up, 1.0) - exp) < 1e-5  # the smoothstep blend


def _rounded(m: abi.gr_material, radius: float) -> abi.gr_material:
    m = abi.gr_material.from_buffer_copy(m)
    m.edge_rounding_radius = radius
    return m


def test_edge_rounding_default_off_bit_identical(oracle):
    d = S.builtin_material("Diamond")
    env = dict(preset="Daylight", exposure=1.0, light_yaw=0.4, light_pitch=0.35)
    a = _probe(oracle, S.Scene(6, 6, PLANES, d, CAM, **env), 6, 4, 0x2468ACE0, 10)
    b = _probe(oracle, S.Scene(6, 6, PLANES, _rounded(d, 0.0), CAM, **env), 6, 4, 0x2468ACE0, 10)
    assert a.tobytes() == b.tobytes()


def test_edge_rounding_changes_face_up_y(oracle):
    d = S.builtin_material("Diamond")
    sharp = _probe(oracle, S.Scene(16, 16, PLANES, d, CAM), 16, 128, 0xF00DCAFE, 12)
    rounded = _probe(oracle, S.Scene(16, 16, PLANES, _rounded(d, 0.02), CAM), 16, 128, 0xF00DCAFE, 12)
    assert abs(rounded[1] - sharp[1]) / sharp[1] > 0.005, (sharp[1], rounded[1])


def test_edge_rounding_white_furnace(oracle):
    m = _rounded(S.custom_material(1.5, 0.0, 0.0), 0.03)
    mean = _probe(oracle, S.Scene(12, 12, PLANES, m, CAM, **UNIFORM), 12, 96, 0xABAD1DEA, 16)
    err = np.abs(mean - _target(oracle)) / _target(oracle)
    assert np.all(err <= 0.06), err
