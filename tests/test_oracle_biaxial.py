"""Pins the oracle's biaxial path (BiaxialIndicatrix, optics/birefringence.rs:349-839;
its wiring in refraction.rs:127-174,345-401,428-582,748-1011 and
raytracer/absorption.rs:175-216) to the reference's own tests for it, with their
inputs and tolerances:

* birefringence.rs biaxial_reduction_tests: wave indices reduce to the uniaxial
  formula and to the isotropic index; eigen-polarizations orthonormal and transverse;
  the eigen-equation residual below 2e-4 with continuous directions over a dense sweep
  for the three biaxial built-ins;
* crates/gemray/tests/raytracer_tests.rs:1209-1245 (every built-in renders finite and
  non-negative), :1320-1356 (tanzanite's biaxial eigenmodes differ from the uniaxial
  pair), :1550-1604 (each biaxial built-in renders measurably differently from its
  uniaxial fallback), :718-770 (alexandrite turns redder under incandescent light; the
  reference runs it on its step-cut emerald, this restatement on the round brilliant
  with the same ray, seeds and bound).

The reference suite holds no golden vectors for biaxial materials; these properties
and the per-sample device-vs-oracle tests pin the path.  The non-biaxial goldens
(tests/test_oracle_goldens.py) pin that the wiring changes nothing for the others.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from gemray_studio_b200 import abi, scene as S
from helpers import hash_draw

F3 = C.c_float * 3
F9 = C.c_float * 9
IDENTITY = F9(1, 0, 0, 0, 1, 0, 0, 0, 1)
BIAXIAL = ("Alexandrite", "Topaz", "Tanzanite")


def _unit(v) -> np.ndarray:
    v = np.asarray(v, np.float32)
    return v * (np.float32(1.0) / np.float32(np.sqrt(np.float32(v @ v))))


def _frame_for_axis(oracle, c) -> F9:
    """The (stable_orthonormal_basis(c), c) frame, via a material whose c-axis is c."""
    m = S.custom_material(1.6, 0.0, 0.01)
    m.dispersion.c_axis_and_birefringence[0:3] = [float(x) for x in c]
    m.dispersion.has_biaxial_delta = 1
    n, ax = F3(), F9()
    assert oracle.gro_material_indicatrix(C.byref(m), 589.3, n, ax) == 0
    return ax


def _wave_indices(oracle, na, nb, ng, axes, wn):
    out = (C.c_float * 2)()
    oracle.gro_biaxial_wave_indices(na, nb, ng, axes, F3(*wn), out)
    return out[0], out[1]


def _eigen(oracle, na, nb, ng, axes, wn):
    s, f = F3(), F3()
    oracle.gro_biaxial_eigen(na, nb, ng, axes, F3(*wn), s, f)
    return np.array(s, np.float64), np.array(f, np.float64)


def test_wave_indices_reduce_to_uniaxial_formula(oracle):
    n_o, n_e = 1.65, 1.72
    c = _unit([0.35, 0.82, -0.45])
    axes = _frame_for_axis(oracle, c)
    dirs = [[1, 0, 0], [0, 1, 0], [0, 0, 1], c, [0.2, 0.9, 0.1], [-0.5, 0.3, 0.8], [0.7, -0.6, 0.2],
            [0.1, 0.1, 0.99], [-0.9, -0.3, 0.2]]
    for d in dirs:
        wn = _unit(d)
        ns, nf = _wave_indices(oracle, n_o, n_o, n_e, axes, wn)
        theta = np.arccos(min(abs(float(wn @ c)), 1.0))
        n_eff = n_o * n_e / np.sqrt((n_e * np.cos(theta)) ** 2 + (n_o * np.sin(theta)) ** 2)
        assert abs(nf - min(n_o, n_eff)) < 1e-3 and abs(ns - max(n_o, n_eff)) < 1e-3, (d, ns, nf, n_eff)


def test_wave_indices_isotropic_when_all_equal(oracle):
    for d in ([1, 0, 0], [0, 1, 0], [0, 0, 1], [0.3, 0.5, 0.8]):
        ns, nf = _wave_indices(oracle, 1.9, 1.9, 1.9, IDENTITY, _unit(d))
        assert abs(ns - 1.9) < 1e-4 and abs(nf - 1.9) < 1e-4


def test_eigen_polarizations_orthonormal_and_transverse(oracle):
    for d in ([0.3, 0.5, 0.8], [0.9, 0.1, -0.2], [-0.4, 0.6, 0.5]):
        wn = _unit(d).astype(np.float64)
        ds, df = _eigen(oracle, 1.60, 1.65, 1.75, IDENTITY, _unit(d))
        assert np.all(np.isfinite(ds)) and np.all(np.isfinite(df))
        assert abs(np.linalg.norm(ds) - 1) < 1e-3 and abs(np.linalg.norm(df) - 1) < 1e-3
        assert abs(ds @ df) < 1e-2 and abs(ds @ wn) < 1e-2 and abs(df @ wn) < 1e-2


def test_eigenvectors_satisfy_eigen_equation_across_dense_sweep(oracle):
    a, b = _unit([0.4, 0.6, 0.69]), _unit([0.8, -0.3, 0.2])
    for name in BIAXIAL:
        n, ax = F3(), F9()
        assert oracle.gro_material_indicatrix(C.byref(S.builtin_material(name)), 589.3, n, ax) == 0
        na, nb, ng = n
        axes = np.array(ax, np.float64).reshape(3, 3)  # rows = principal axes
        bc = np.array([1 / na ** 2, 1 / nb ** 2, 1 / ng ** 2])
        prev = [None, None]
        for i in range(181):
            th = np.float32(i / 180.0 * np.pi)
            wn = _unit(np.cos(th) * a + np.sin(th) * b)
            local = axes @ wn.astype(np.float64)
            ns, nf = _wave_indices(oracle, na, nb, ng, ax, wn)
            ds, df = _eigen(oracle, na, nb, ng, ax, wn)
            for j, (nn, d) in enumerate(((ns, ds), (nf, df))):
                assert abs(np.linalg.norm(d) - 1) < 1e-4, (name, i)
                x = 1.0 / (nn * nn)
                dl = axes @ d
                e_dot_k = float(np.sum(local * bc * dl))
                res = dl * (x - bc) + local * e_dot_k
                assert np.linalg.norm(res) < 2e-4, (name, i, j, np.linalg.norm(res))
                if prev[j] is not None:
                    assert abs(prev[j] @ d) > 0.98, (name, i, j)
                prev[j] = d


def test_tanzanite_eigenmodes_differ_from_uniaxial_pair(oracle):
    tz = S.builtin_material("Tanzanite")
    n, ax = F3(), F9()
    assert oracle.gro_material_indicatrix(C.byref(tz), 550.0, n, ax) == 0
    wn = _unit([0.5, 0.4, 0.6])
    ba, _bb = _eigen(oracle, n[0], n[1], n[2], ax, wn)
    c = np.array(tz.dispersion.c_axis_and_birefringence[0:3], np.float64)
    ua = np.cross(wn, c)
    ua /= np.linalg.norm(ua)
    axes = np.array(ax, np.float64).reshape(3, 3)
    tensor = np.array([1.0, 1.0, 6.0])  # AbsorptionTensor3::uniaxial(1, 6, c) in the (a1, a2, c) frame

    def quad(e):
        return float(tensor @ (axes @ e) ** 2)
    assert abs(quad(ba) - quad(ua)) > 1e-3


def _ray_scene(material):
    return S.Scene(1, 1, S.standard_round_brilliant(), material, S.camera(0.35, 0.28, 5.0, 18.0))


def _trace(oracle, sc, d, seed, o=(0.0, 2.5, 0.0)):
    xyz = (C.c_double * 3)()
    assert oracle.gro_trace_ray(C.byref(sc.c_scene()), F3(*o), F3(*d), seed, hash_draw(oracle, seed), 12, 32, xyz,
                                None, None) == 0
    return np.array(xyz, np.float32)


def test_every_builtin_renders_finite_and_non_negative(oracle):
    d = _unit([0.22, -1.0, -0.13])
    for name in S.BUILTIN_MATERIALS:
        sc = _ray_scene(S.builtin_material(name))
        for seed in (1, 2, 42, 4242):
            x = _trace(oracle, sc, d, seed)
            assert np.all(np.isfinite(x)) and np.all(x >= 0), (name, seed, x)


def test_biaxial_differs_from_uniaxial_fallback(oracle):
    d = _unit([0.18, -1.0, 0.07])
    for name in BIAXIAL:
        m = S.builtin_material(name)
        fb = abi.gr_material.from_buffer_copy(m)
        fb.dispersion.has_biaxial_delta = 0
        fb.dispersion.biaxial_delta_beta_alpha = 0.0
        sb, sf = _ray_scene(m), _ray_scene(fb)
        acc_b = np.zeros(3, np.float32)
        acc_f = np.zeros(3, np.float32)
        for i in range(64):
            seed = (i * 7919 + 13) & 0xFFFFFFFF
            acc_b += _trace(oracle, sb, d, seed)
            acc_f += _trace(oracle, sf, d, seed)
        diff = np.linalg.norm(acc_b / np.float32(64) - acc_f / np.float32(64))
        assert diff > 1e-6, (name, diff)


def test_alexandrite_redder_under_incandescent(oracle):
    h = oracle.gro_hash_u32
    alex = S.builtin_material("Alexandrite")

    def chroma(preset, salt):
        sc = S.Scene(1, 1, S.standard_round_brilliant(), alex, S.camera(0.35, 0.28, 5.0, 18.0), preset=preset)
        acc = np.zeros(3, np.float32)
        for i in range(192):
            acc += _trace(oracle, sc, (0.0, -1.0, 0.0), h(salt ^ h(i ^ 0x9E3779B9)))
        acc = acc / np.float32(192)
        return acc[0] / acc.sum()
    assert chroma("Incandescent", 0xA5A50004) > chroma("Daylight", 0xA5A50003) + 0.003


def _biaxial_furnace_material(d_beta_alpha: float) -> abi.gr_material:
    """Colourless, non-dispersive, birefringent 0.03 (n_gamma - n_alpha), biaxial by
    d_beta_alpha: the furnace probe of the uniaxial furnace tests made biaxial."""
    m = S.custom_material(1.5, 0.0, 0.03)
    m.dispersion.has_biaxial_delta = 1
    m.dispersion.biaxial_delta_beta_alpha = d_beta_alpha
    return m


def test_biaxial_white_furnace(oracle):
    """A lossless biaxial stone in a uniform environment returns the environment's
    radiance (the energy check of raytracer_tests.rs:2539
    birefringent_white_furnace_energy_conservation_holds, for a biaxial indicatrix); 64 bounces leave the cap's loss under 1 %."""
    t = F3()
    oracle.gro_furnace_target(2.5, t)
    target = np.array(t, np.float64)
    for dba in (0.01, 0.02):
        sc = S.Scene(32, 32, S.standard_round_brilliant(), _biaxial_furnace_material(dba),
                     S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=64, env_mode=abi.GR_ENV_UNIFORM,
                     uniform_rgb=(2.5, 2.5, 2.5))
        out = F3()
        assert oracle.gro_probe_grid(C.byref(sc.c_scene()), 32, 64, 0x1234, 64, out) == abi.GR_OK
        err = np.abs(np.array(out, np.float64) - target) / target
        assert np.all(err < 0.01), (dba, err)
