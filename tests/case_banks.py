"""Per-function case banks: seeded inputs, scenes and ULP budgets.

The reference holds each small function its GPU port inlines to a ULP budget against
the CPU function it was translated from, with an absolute floor for values near zero
(renderer/gpu/ulp.rs:19-68 `within_tolerance`; budgets in
renderer/gpu/transport_check/*.rs, camera_check.rs:314-330,
environment_check.rs:154-168,265-275,410-421,608-620).  Each bank here carries:

* `budget`, `floor` -- the reference's budget and floor for the same function, used
  for the device against the FP32 oracle (the reference's own arithmetic);
* `budget64`, `floor64` -- the budget against the FP64 oracle.  The FP32 function
  itself carries rounding error against exact arithmetic, so this budget is the FP32
  oracle's measured error against the FP64 oracle (tests/test_oracle_case_banks.py
  holds the FP32 oracle to it on the CPU) with the same headroom for the device.

Inputs are sweeps plus a seeded random fill with the reference banks' adversarial
corners (grazing, near-critical, degenerate axes); the reference's own case lists are
not reproduced.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from gemray_studio_b200 import abi, scene as S

STOKES = np.array([[1, 0, 0, 0], [1, 1, 0, 0], [1, 0, 1, 0], [1, 0, 0, 1], [1, 0.3, -0.4, 0.2]], np.float32)


@dataclass
class Bank:
    name: str
    inputs: np.ndarray          # (n, n_in) float32
    scene: object | None        # gemray_studio_b200.scene.Scene or None
    budget: int
    floor: float
    budget64: int
    floor64: float
    fp64_rows: np.ndarray | None = None  # rows the FP64 comparison covers (None: all)


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _stokes(rng, n):
    """Physical Stokes vectors: I in (0, 2], degree of polarisation in [0, 1]."""
    i = rng.uniform(0.05, 2.0, n)
    p = rng.uniform(0.0, 1.0, n)
    d = _unit(rng, n).astype(np.float64)
    s = np.concatenate([i[:, None], (i * p)[:, None] * d], axis=1).astype(np.float32)
    return np.concatenate([s, STOKES], axis=0)


def _studio_scene(preset="RingLights", yaw=0.85, pitch=0.95):
    return S.Scene(width=8, height=8, planes=np.zeros((0, 4), np.float32), material=S.builtin_material("Diamond"),
                   cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=1, env_mode=abi.GR_ENV_STUDIO, preset=preset,
                   light_yaw=yaw, light_pitch=pitch)


def _material_scene(material, ext=None):
    return S.Scene(width=8, height=8, planes=np.zeros((0, 4), np.float32), material=material,
                   cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=1, env_mode=abi.GR_ENV_UNIFORM, ext=ext)


def _lambdas(step=0.37):
    return np.concatenate([np.arange(380.0, 780.0, step), [380.0, 780.0, 589.3, 486.1, 656.3]]).astype(np.float32)


def banks(seed: int = 7) -> list[Bank]:
    from gemray_studio_b200 import workloads as W
    rng = np.random.default_rng(seed)
    out: list[Bank] = []
    f32 = np.float32

    # camera_check.rs:314-330 (64 ULP, 1e-4): the c2 frame's camera
    n = 20000
    xy = np.stack([rng.integers(0, 1920, n), rng.integers(0, 1080, n)], axis=1).astype(f32)
    jit = rng.uniform(-0.5, 0.5, (n, 2)).astype(f32)
    corners = np.array([[0, 0, -0.5, -0.5], [1919, 1079, 0.5, 0.5], [959, 539, 0, 0], [0, 1079, 0.49, -0.49]], f32)
    cam = S.Scene(width=1920, height=1080, planes=np.zeros((0, 4), np.float32), material=S.builtin_material("Diamond"),
                  cam=S.camera(0.35, 0.28, 5.0, 18.0), max_bounces=1, env_mode=abi.GR_ENV_UNIFORM)
    out.append(Bank("camera_ray", np.concatenate([np.concatenate([xy, jit], 1), corners]), cam, 64, 1e-4, 64, 1e-4))

    lam = _lambdas()
    # environment_check.rs:154-168 (32 ULP, 1e-6)
    out.append(Bank("cmf", lam[:, None], None, 32, 1e-6, 64, 1e-6))
    # environment_check.rs:265-275 (48 ULP, 1e-5), at three lighting temperatures
    for preset in ("Incandescent", "RingLights", "Daylight"):  # 3200, 5000, 6500 K
        out.append(Bank("blackbody", lam[:, None], _studio_scene(preset), 48, 1e-5, 64, 1e-5))
    # transport_check/dispersion.rs:22-23 (24 ULP, 1e-6): Sellmeier-3, Sellmeier-1 and Cauchy materials
    for name in ("Diamond", "Sapphire", "Quartz", "Topaz", "Cubic Zirconia"):
        out.append(Bank("dispersion", lam[:, None], _material_scene(S.builtin_material(name)), 24, 1e-6, 24, 1e-6))
    em, em_ext = W.birefringent_emerald_material()
    out.append(Bank("dispersion", lam[:, None], _material_scene(em, em_ext), 24, 1e-6, 24, 1e-6))
    # transport_check/absorption_pleochroism.rs:42-43 (24 ULP, 1e-6): Gaussian bands and the tabulated extension
    for name in ("Tourmaline", "Ruby", "Emerald", "Tanzanite"):
        out.append(Bank("absorption", lam[:, None], _material_scene(S.builtin_material(name)), 24, 1e-6, 32, 1e-6))
    out.append(Bank("absorption", np.concatenate([lam, [300.0, 379.9, 780.1, 900.0]]).astype(f32)[:, None],
                    _material_scene(em, em_ext), 24, 1e-6, 4, 1e-6))
    # absorption_pleochroism.rs:178-179 (48 ULP, 1e-5): the emerald's random c-axis
    n = 8000
    st = _stokes(rng, n)[:n]
    pin = np.concatenate([st, _unit(rng, n), _unit(rng, n), rng.uniform(0.0, 2.0, (n, 2)).astype(f32)], 1)
    out.append(Bank("pleochroic", pin, _material_scene(em, em_ext), 48, 1e-5, 96, 1e-5))

    stokes = _stokes(rng, 200)
    # fresnel.rs:26-27,116-117 (16 ULP, 1e-6)
    g = np.linspace(-1.0, 1.0, 21, dtype=f32)
    rs, rp = np.meshgrid(g, g, indexing="ij")
    rr = np.stack([rs.ravel(), rp.ravel()], 1)
    rr = np.concatenate([rr, np.array([[0.9999, -0.9999], [-0.9999, 0.9999], [1e-4, -1e-4], [1, 1], [-1, -1]], f32)])
    fr = np.array([np.concatenate([a, s]) for a in rr for s in stokes[::10]], f32)
    out.append(Bank("fresnel_reflection", fr, None, 16, 1e-6, 16, 1e-6))
    rows = []
    for n1, n2 in ((1.0, 1.5), (1.0, 2.417), (2.417, 1.0), (1.64, 1.0), (1.0, 1.0)):
        for ci in np.linspace(0.02, 1.0, 25):
            s2 = (n1 / n2) ** 2 * (1 - ci * ci)
            if s2 > 1:
                continue
            ct = math.sqrt(1 - s2)
            ts = 2 * n1 * ci / (n2 * ct + n1 * ci)
            tp = 2 * n1 * ci / (n1 * ct + n2 * ci)
            for s in stokes[::20]:
                rows.append([n1, n2, ci, ct, ts, tp, *s])
    out.append(Bank("fresnel_transmission", np.asarray(rows, f32), None, 16, 1e-6, 16, 1e-6))
    # frame_and_tir.rs:43-44,126-127 (16 ULP, 1e-6); :186-187 (32, 1e-5); :306-320 (32, 2e-3)
    psi = np.concatenate([np.linspace(-math.pi, math.pi, 181), [0.0, 1e-7, -1e-7, math.pi / 2, math.pi / 4]])
    out.append(Bank("frame_rotation", np.array([[p, *s] for p in psi for s in stokes[::10]], f32), None, 16, 1e-6,
                    16, 1e-6))
    dl = np.concatenate([np.linspace(0.0, math.pi, 121), [1e-6, math.pi - 1e-6]])
    out.append(Bank("tir_retardation", np.array([[d, *s] for d in dl for s in stokes[::10]], f32), None, 16, 1e-6,
                    16, 1e-6))
    n = 20000
    sp = np.concatenate([_unit(rng, n), _unit(rng, n), _unit(rng, n)], 1)
    a = _unit(rng, 8)
    sp = np.concatenate([sp, np.concatenate([a, a, _unit(rng, 8)], 1), np.concatenate([a, -a, _unit(rng, 8)], 1)])
    out.append(Bank("signed_psi", sp.astype(f32), None, 32, 1e-5, 32, 1e-5))
    rows = []
    for n1 in (1.46, 1.54, 1.64, 1.76, 2.17, 2.417, 2.65):
        crit = math.asin(1.0 / n1)
        for th in np.concatenate([np.linspace(crit, math.pi / 2, 60), crit + np.array([-1e-3, -1e-5, 0, 1e-5, 1e-3])]):
            rows.append([n1, math.cos(th), math.sin(th)])
    out.append(Bank("tir_phase_delta", np.asarray(rows, f32), None, 32, 2e-3, 32, 2e-3))
    # eigenmodes_uniaxial.rs:31-32 (32, 1e-5); :374-375 walk-off (32, 1e-5); :526-527 per-mode index (32, 1e-6);
    # :194-195 theta_c (96, 1e-5)
    n = 10000
    k, c = _unit(rng, n), _unit(rng, n)
    par = np.concatenate([k[:8], k[:8]], 1)
    out.append(Bank("eigen_uniaxial", np.concatenate([np.concatenate([k, c], 1), par]), None, 32, 1e-5, 32, 1e-5))
    pairs = np.array([[1.640, 1.620], [1.544, 1.553], [1.768, 1.760], [2.65, 2.69], [1.658, 1.486]], f32)
    pick = pairs[rng.integers(0, len(pairs), n)]
    out.append(Bank("walk_off", np.concatenate([k, c, pick], 1), None, 32, 1e-5, 64, 1e-5))
    th = np.linspace(0.0, math.pi / 2, 91, dtype=f32)
    out.append(Bank("extraordinary_index", np.array([[a, b, t] for a, b in pairs for t in th], f32), None, 32, 1e-6,
                    32, 1e-6))
    nrm = _unit(rng, n)
    kk = _unit(rng, n)
    flip = np.sum(kk * nrm, axis=1) > 0
    kk[flip] = -kk[flip]  # the ray travels against the normal, as at a facet
    ent = (rng.uniform(size=n) < 0.5).astype(f32)
    tin = np.concatenate([kk, nrm, pick, ent[:, None]], 1)
    out.append(Bank("theta_c", tin, _material_scene(em, em_ext), 96, 1e-5, 96, 1e-5))
    # environment_check.rs:410-421 (8192, 1e-4): studio radiance over random directions
    n = 4000
    out.append(Bank("studio", np.concatenate([_unit(rng, n), rng.uniform(380, 780, (n, 1)).astype(f32)], 1),
                    _studio_scene(), 8192, 1e-4, 8192, 1e-4))
    rgb = np.concatenate([rng.uniform(0, 100, (n, 3)), rng.uniform(380, 780, (n, 1))], 1).astype(f32)
    out.append(Bank("rgb_spectral", rgb, None, 32, 1e-6, 32, 1e-6))
    # the reference polynomial exp (simd/exp_poly.rs:23-40) is the reference's own arithmetic: bit-exact;
    # against exact exp only inside its clamp range [-87.33654, 88.02875] (outside, it returns the clamp)
    xs = np.concatenate([np.linspace(-90, 90, 20001), [-87.33654, 88.02875, 0.0, -0.0, 1e-30]]).astype(f32)
    out.append(Bank("exp_poly", xs[:, None], None, 0, 0.0, 2, 0.0,
                    fp64_rows=(xs >= f32(-87.0)) & (xs <= f32(88.0))))
    # scattering.rs:179-187 (128, 2e-4): Henyey-Greenstein directions; bounce.rs:41-47 (48, 1e-5)
    n = 8000
    gg = np.array([-0.9, -0.3, 0.0, 5e-4, 0.3, 0.6, 0.9], f32)[rng.integers(0, 7, n)]
    hg = np.concatenate([rng.uniform(0, 1, (n, 2)).astype(f32), gg[:, None], _unit(rng, n)], 1)
    out.append(Bank("hg_sample", hg, None, 128, 2e-4, 128, 2e-4))
    ch = np.concatenate([rng.uniform(0, 1, (n, 2)).astype(f32), _unit(rng, n)], 1)
    out.append(Bank("cosine_hemisphere", ch, None, 48, 1e-5, 48, 1e-5))
    st = _stokes(rng, n)[:n]
    out.append(Bank("e_field", np.concatenate([st, _unit(rng, n), _unit(rng, n)], 1), None, 32, 1e-5, 64, 1e-5))
    # environment_check.rs:608-620 (4096, 1e-5): the studio white balance
    xyz = rng.uniform(0, 10, (n, 3)).astype(f32)
    out.append(Bank("von_kries", xyz, _studio_scene(), 4096, 1e-5, 4096, 1e-5))
    hero = np.concatenate([rng.uniform(0, 1, n), [0.0, 0.9999999, 0.5, 0.125]]).astype(f32)
    out.append(Bank("wavelengths", hero[:, None], None, 0, 0.0, 4, 1e-4))
    return out


def ulp(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """ULP distance of float32 arrays, zero for +0/-0, ordered across the sign
    (renderer/gpu/ulp.rs to_ordered)."""
    ia = a.astype(np.float32).view(np.int32).astype(np.int64)
    ib = b.astype(np.float32).view(np.int32).astype(np.int64)
    oa = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ob = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(oa - ob)


def over_budget(ref: np.ndarray, got: np.ndarray, budget: int, floor: float) -> np.ndarray:
    """within_tolerance negated: ULP distance above budget AND |difference| >= floor."""
    ref = ref.astype(np.float32)
    got = got.astype(np.float32)
    d = ulp(ref, got)
    bad = (d > budget) & ~(np.abs(ref.astype(np.float64) - got.astype(np.float64)) < floor)
    both_nan = np.isnan(ref) & np.isnan(got)
    return bad & ~both_nan


def oracle_bank(oracle, bank: Bank, precision: int) -> np.ndarray:
    ni, no = C.c_uint32(), C.c_uint32()
    assert oracle.gro_case_bank_arity(abi.GR_BANK[bank.name], C.byref(ni), C.byref(no)) == 0
    x = np.ascontiguousarray(bank.inputs, np.float32)
    assert x.shape[1] == ni.value, (bank.name, x.shape, ni.value)
    out = np.empty((x.shape[0], no.value), np.float64)
    sc = C.byref(bank.scene.c_scene()) if bank.scene is not None else None
    st = oracle.gro_case_bank(abi.GR_BANK[bank.name], precision, sc, x.ctypes.data_as(C.POINTER(C.c_float)),
                              x.shape[0], out.ctypes.data_as(C.POINTER(C.c_double)))
    assert st == 0
    return out


def histogram(d: np.ndarray) -> str:
    edges = [0, 1, 2, 4, 8, 16, 32, 64, 128, 512, 4096, 1 << 62]
    counts = [int(np.sum((d >= lo) & (d < hi))) for lo, hi in zip(edges[:-1], edges[1:])]
    return " ".join(f"[{lo},{hi}):{c}" for lo, hi, c in zip(edges[:-1], edges[1:], counts) if c)


def fibonacci_sphere(n: int) -> np.ndarray:
    """n well-spaced unit directions (golden-angle spiral), float32."""
    i = np.arange(n, dtype=np.float64)
    y = 1.0 - 2.0 * i / max(n - 1, 1)
    r = np.sqrt(np.maximum(1.0 - y * y, 0.0))
    th = math.pi * (3.0 - math.sqrt(5.0)) * i
    return np.stack([np.cos(th) * r, y, np.sin(th) * r], 1).astype(np.float32)


def polyhedron_rays(n_dirs: int = 1024) -> np.ndarray:
    """Ray classes of the reference's intersect_polyhedron case bank
    (renderer/gpu/polyhedron_check.rs:84-200): from outside aimed at the centre, from
    outside with a lateral offset that grazes the silhouette, from the centre outwards
    (the exit branch), and adversarial rays -- along +-Y (denominator 0 for every
    girdle plane), on the table plane, tangent to the girdle, just above / below the
    1e-7 denominator threshold, a total miss.  Rows: origin[3], dir[3]."""
    d = fibonacci_sphere(n_dirs)
    rows = [np.concatenate([d * 5.0, -d], 1)]
    pert = np.stack([d[:, 2], d[:, 0], -d[:, 1]], 1) * 0.15
    g = -d + pert
    rows.append(np.concatenate([d * 5.0, g / np.linalg.norm(g, axis=1, keepdims=True)], 1))
    rows.append(np.concatenate([np.zeros_like(d), d], 1))
    adv = [[0, 0, 0, 0, 1, 0], [0, 0, 0, 0, -1, 0], [0, 0.32, 0, 0, -1, 0], [0, 0.32, 0, 0, 1, 0],
           [1, 0, 0, 0, 0, 1], [5, 5, 5, 0.57735026, 0.57735026, 0.57735026]]
    for eps in (5e-7, 5e-8, -5e-7, -5e-8):
        v = np.array([1.0, eps, 0.0])
        v /= np.linalg.norm(v)
        adv.append([-5.0, 0.32, 0.0, *v])
    rows.append(np.asarray(adv))
    return np.concatenate(rows).astype(np.float32)
