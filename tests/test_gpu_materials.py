"""Frosted facet finishes, Henyey-Greenstein volume scattering
(raytracer/scattering.rs:132-602) and biaxial materials (BiaxialIndicatrix,
optics/birefringence.rs:349-839, with trichroic beta-ray absorption) on the device,
against the oracle.

Per sample the engine follows the oracle the way the polished path does: the new
arithmetic (cosine-weighted and Henyey-Greenstein directions, free-flight distances
through logf) is continuous, so most samples agree to a few ULP and a small share
flips a Fresnel, distance or roulette decision through a libm ULP.  Scene-level
properties from the reference's own tests hold on the device too: a bruted girdle
makes the face-up studio view brighter (raytracer_tests.rs:2411-2460), and a
lossless scattering medium in a uniform environment returns the environment's
radiance (the white furnace).  Every built-in material renders on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import abi, scene as S
from helpers import oracle_trace_samples

pytestmark = pytest.mark.gpu

GIRDLE = slice(33, 49)  # STANDARD_ROUND_BRILLIANT_GIRDLE_FACETS (geometry/cuts.rs:37)


def _rel(a, b):
    return np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-30)


def _girdle_finishes():
    f = np.zeros(S.standard_round_brilliant().shape[0], np.uint32)
    f[GIRDLE] = 1
    return f


def _scattering(material: abi.gr_material, sigma_s: float, g: float) -> abi.gr_material:
    m = abi.gr_material.from_buffer_copy(material)
    m.scattering_sigma_s = sigma_s
    m.scattering_g = g
    return m


def _rounded(material: abi.gr_material, radius: float) -> abi.gr_material:
    m = abi.gr_material.from_buffer_copy(material)
    m.edge_rounding_radius = radius  # shading_normal_near_edge (optics/raytracer/intersect.rs:196-229)
    return m


def _cases():
    cam = S.camera(0.35, 0.28, 5.0, 18.0)
    planes = S.standard_round_brilliant()
    env = S.gaussian_blob_latlong(256, 128, seed=4)
    return {
        "frosted Diamond studio": S.Scene(width=24, height=24, planes=planes, material=S.builtin_material("Diamond"),
                                          cam=cam, max_bounces=16, finishes=_girdle_finishes()),
        "frosted Tourmaline latlong": S.Scene(width=24, height=24, planes=planes,
                                              material=S.builtin_material("Tourmaline"), cam=cam, max_bounces=16,
                                              env_mode=abi.GR_ENV_LATLONG, latlong=env, finishes=_girdle_finishes()),
        "scattering clear": S.Scene(width=24, height=24, planes=planes,
                                    material=_scattering(S.custom_material(1.5, 0.0, 0.0), 0.8, 0.6), cam=cam,
                                    max_bounces=16, env_mode=abi.GR_ENV_STUDIO),
        "scattering tinted uniaxial": S.Scene(width=24, height=24, planes=planes,
                                              material=_scattering(S.custom_material(1.6, 0.01, 0.02, (0.3, 0.1, 0.5)),
                                                                   2.0, -0.3),
                                              cam=cam, max_bounces=16, env_mode=abi.GR_ENV_STUDIO),
        "biaxial Alexandrite studio": S.Scene(width=24, height=24, planes=planes,
                                              material=S.builtin_material("Alexandrite"), cam=cam, max_bounces=16),
        "biaxial Topaz studio": S.Scene(width=24, height=24, planes=planes, material=S.builtin_material("Topaz"),
                                        cam=cam, max_bounces=16, preset="Daylight"),
        "biaxial Tanzanite latlong": S.Scene(width=24, height=24, planes=planes,
                                             material=S.builtin_material("Tanzanite"), cam=cam, max_bounces=16,
                                             env_mode=abi.GR_ENV_LATLONG, latlong=env),
        "biaxial frosted Tanzanite": S.Scene(width=24, height=24, planes=planes,
                                             material=S.builtin_material("Tanzanite"), cam=cam, max_bounces=16,
                                             finishes=_girdle_finishes()),
        "biaxial scattering Alexandrite": S.Scene(width=24, height=24, planes=planes,
                                                  material=_scattering(S.builtin_material("Alexandrite"), 1.0, 0.5),
                                                  cam=cam, max_bounces=16),
        "rounded edges Diamond": S.Scene(width=24, height=24, planes=planes,
                                         material=_rounded(S.builtin_material("Diamond"), 0.02), cam=cam,
                                         max_bounces=16),
        "rounded edges Tourmaline latlong": S.Scene(width=24, height=24, planes=planes,
                                                    material=_rounded(S.builtin_material("Tourmaline"), 0.05),
                                                    cam=cam, max_bounces=16, env_mode=abi.GR_ENV_LATLONG,
                                                    latlong=env),
    }


@pytest.mark.parametrize("case", list(_cases()))
def test_per_sample_matches_oracle(renderer, oracle, case):
    sc = _cases()[case]
    n_pix, spp = sc.width * sc.height, 8
    gpu = renderer.trace_samples(sc, 0, n_pix, 0, spp)
    st, ref, _b, _t = oracle_trace_samples(oracle, sc, 0, n_pix, 0, spp)
    assert st == abi.GR_OK
    assert np.all(np.isfinite(gpu))
    rel = _rel(gpu, ref)
    # the polished path's bars: a lat-long lookup turns direction ULPs into radiance
    # ULPs (0.9 tight there, as for polished lat-long scenes), elsewhere 0.98 / 1 %.
    # In a scattering biaxial stone the HG directions carry CUDA's sincosf/logf ULPs
    # into the eigenvector solve, whose sensitivity grows as 1/(mode gap): more
    # samples land between 1e-5 and 1e-3 (measured 96-98 % tight), none more flip.
    tight = 0.9 if sc.env_mode == abi.GR_ENV_LATLONG else 0.98
    if sc.material.dispersion.has_biaxial_delta and sc.material.scattering_sigma_s > 0:
        tight = 0.95
    assert np.mean(rel <= 1e-5) >= tight, (case, np.mean(rel <= 1e-5))
    assert np.mean(rel > 1e-3) <= 0.01, (case, np.mean(rel > 1e-3))


def test_frosted_girdle_brightens_face_up(renderer):
    planes = S.standard_round_brilliant()
    base = dict(width=32, height=32, planes=planes, material=S.builtin_material("Diamond"),
                cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=12)
    pol = np.zeros((32 * 32, 3), np.float32)
    fro = np.zeros((32 * 32, 3), np.float32)
    renderer.accumulate(S.Scene(**base), 0, 256, pol)
    renderer.accumulate(S.Scene(finishes=_girdle_finishes(), **base), 0, 256, fro)
    yp, yf = pol[:, 1].astype(np.float64).mean(), fro[:, 1].astype(np.float64).mean()
    assert (yf - yp) / yp > 0.01, (yp, yf)


def test_scattering_white_furnace(renderer, oracle):
    l0 = 2.5
    t = (C.c_float * 3)()
    oracle.gro_furnace_target(l0, t)
    target = np.array(t, np.float64)
    for sigma_s, g in ((0.5, 0.6), (3.0, -0.2)):
        sc = S.Scene(width=48, height=48, planes=S.standard_round_brilliant(),
                     material=_scattering(S.custom_material(1.5, 0.0, 0.0), sigma_s, g),
                     cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=64, env_mode=abi.GR_ENV_UNIFORM,
                     uniform_rgb=(l0, l0, l0))
        film = np.zeros((48 * 48, 3), np.float32)
        renderer.accumulate(sc, 0, 256, film)
        mean = film.astype(np.float64).sum(0) / (48 * 48 * 256)
        assert np.all(np.abs(mean - target) / target <= 0.02), (sigma_s, mean, target)


def test_biaxial_white_furnace(renderer, oracle):
    """A lossless biaxial stone (n_gamma - n_alpha = 0.03, n_beta - n_alpha = 0.01 /
    0.02) in a uniform environment returns the environment's radiance; the oracle
    measures +0.13 % at 64 bounces."""
    l0 = 2.5
    t = (C.c_float * 3)()
    oracle.gro_furnace_target(l0, t)
    target = np.array(t, np.float64)
    for dba in (0.01, 0.02):
        m = S.custom_material(1.5, 0.0, 0.03)
        m.dispersion.has_biaxial_delta = 1
        m.dispersion.biaxial_delta_beta_alpha = dba
        sc = S.Scene(width=48, height=48, planes=S.standard_round_brilliant(), material=m,
                     cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=64, env_mode=abi.GR_ENV_UNIFORM,
                     uniform_rgb=(l0, l0, l0))
        film = np.zeros((48 * 48, 3), np.float32)
        renderer.accumulate(sc, 0, 256, film)
        mean = film.astype(np.float64).sum(0) / (48 * 48 * 256)
        assert np.all(np.abs(mean - target) / target <= 0.01), (dba, mean, target)


def test_edge_rounding_white_furnace(renderer, oracle):
    """Rounded edges (radius 0.03) on a lossless stone in a uniform environment keep the
    environment's radiance (intersect.rs edge_rounding_white_furnace_energy_conservation_holds,
    bound 0.06; the oracle measures -0.6 % at 16 bounces, the polished stone -1.2 %)."""
    l0 = 2.5
    t = (C.c_float * 3)()
    oracle.gro_furnace_target(l0, t)
    target = np.array(t, np.float64)
    sc = S.Scene(width=48, height=48, planes=S.standard_round_brilliant(),
                 material=_rounded(S.custom_material(1.5, 0.0, 0.0), 0.03), cam=S.camera(0.35, 0.28, 5.0, 18.0),
                 max_bounces=64, env_mode=abi.GR_ENV_UNIFORM, uniform_rgb=(l0, l0, l0))
    film = np.zeros((48 * 48, 3), np.float32)
    renderer.accumulate(sc, 0, 256, film)
    mean = film.astype(np.float64).sum(0) / (48 * 48 * 256)
    assert np.all(np.abs(mean - target) / target <= 0.01), (mean, target)


def test_default_off_extras_bit_identical(renderer):
    """sigma_s = 0 with any g, and an all-polished finishes array, render the bits of the
    plain scene (scattering.rs default_off_scattering_is_bit_identical_regardless_of_g,
    raytracer_tests.rs:2246)."""
    ruby = S.builtin_material("Ruby")
    base = dict(width=16, height=16, planes=S.standard_round_brilliant(), cam=S.camera(0.35, 0.28, 5.0, 18.0),
                max_bounces=10, preset="Daylight", light_yaw=0.4, light_pitch=0.35)
    ref = np.zeros((256, 3), np.float32)
    renderer.accumulate(S.Scene(material=ruby, **base), 3, 32, ref)
    variants = [S.Scene(material=_scattering(ruby, 0.0, g), **base) for g in (-0.6, 0.4, 0.95)]
    variants.append(S.Scene(material=ruby, finishes=np.zeros(S.standard_round_brilliant().shape[0], np.uint32),
                            **base))
    for sc in variants:
        film = np.zeros((256, 3), np.float32)
        renderer.accumulate(sc, 3, 32, film)
        assert film.tobytes() == ref.tobytes()


@pytest.mark.parametrize("flags", [0, abi.GR_BATCH_GRAPH])
def test_batch_with_frosted_and_scattering_scenes(engine_lib, flags):
    """Frosted and scattering scenes in shared launches with a plain one: every film is
    bit-identical to the same scene rendered alone."""
    import torch
    lib = engine_lib
    h = C.c_void_p()
    opts = abi.gr_create_opts(device=-1, chunk_budget_bytes=12 * 9000, serve_budget_bytes=0)
    assert lib.gr_create(C.byref(h), C.byref(opts)) == abi.GR_OK
    try:
        cases = _cases()
        scenes = [cases["frosted Diamond studio"], cases["scattering clear"],
                  S.Scene(width=20, height=12, planes=S.standard_round_brilliant(),
                          material=S.builtin_material("Sapphire"), cam=S.camera(0.35, 0.28, 5.0, 18.0),
                          max_bounces=16),
                  cases["scattering tinted uniaxial"], cases["biaxial Alexandrite studio"]]
        ids = []
        for sc in scenes:
            sid = C.c_uint64()
            assert lib.gr_scene_upload(h, C.byref(sc.c_scene()), C.byref(sid)) == abi.GR_OK
            ids.append(sid.value)
        spps = [12, 5, 9, 16, 7]
        alone = [torch.zeros((sc.width * sc.height, 3), dtype=torch.float32, device="cuda") for sc in scenes]
        batched = [torch.zeros_like(f) for f in alone]
        torch.cuda.synchronize()
        for rnd in range(2):
            items = (abi.gr_batch_item * len(scenes))()
            for i in range(len(scenes)):
                off = rnd * spps[i]
                assert lib.gr_render_resident(h, ids[i], off, spps[i], C.c_void_p(alone[i].data_ptr()),
                                              None) == abi.GR_OK
                items[i] = abi.gr_batch_item(ids[i], batched[i].data_ptr(), off, spps[i])
            assert lib.gr_render_batch(h, items, len(scenes), flags, None) == abi.GR_OK, lib.gr_last_error_string()
            assert lib.gr_synchronize(h) == abi.GR_OK
            for i in range(len(scenes)):
                a, b = alone[i].cpu().numpy(), batched[i].cpu().numpy()
                assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (rnd, i)
                assert a.any()
        del alone, batched
    finally:
        assert lib.gr_destroy(h) == abi.GR_OK


def test_every_builtin_material_renders(renderer):
    """No built-in material is declined (the reference's GemMaterial::gpu_supported is
    true for all of them, renderer/gpu/frame.rs:680-693); every film is finite and
    adds into the caller's buffer."""
    for name in S.BUILTIN_MATERIALS:
        sc = S.Scene(width=12, height=12, planes=S.standard_round_brilliant(), material=S.builtin_material(name),
                     cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=12)
        acc = np.full((144, 3), 1.0, np.float32)
        renderer.accumulate(sc, 0, 16, acc)
        # (a von Kries-adapted XYZ can dip below zero for saturated spectra)
        assert np.all(np.isfinite(acc)) and np.any(acc != 1.0), name
