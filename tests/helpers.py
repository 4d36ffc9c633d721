"""Shared test helpers: f32 bit utilities and standard scenes for oracle/engine parity."""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from gemray_studio_b200 import abi, scene as S


def bits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", float(x)))[0]


def ulp_distance(a: int, b: int) -> int:
    def key(u):
        return u if u < 0x80000000 else -(u & 0x7FFFFFFF)
    return abs(key(a) - key(b))


def f32_normalize(v) -> list[float]:
    v = np.asarray(v, np.float32)
    d = np.float32(np.float32(v[0] * v[0]) + np.float32(v[1] * v[1])) + np.float32(v[2] * v[2])
    r = np.float32(1.0) / np.sqrt(np.float32(d))
    return [float(x) for x in (v * r).astype(np.float32)]


def hash_draw(oracle, seed: int) -> float:
    """(hash_u32(seed) as f32) / 4294967295.0 in f32."""
    return float(np.float32(np.float32(oracle.gro_hash_u32(seed)) / np.float32(4294967295.0)))


def test_camera():
    """estimator_check's test_camera = Camera::new(0.35, 0.28, 5.0, 18.0)."""
    return S.camera(0.35, 0.28, 5.0, 18.0)


def srb_scene(material="Diamond", width=32, height=32, max_bounces=12, preset="RingLights", env_mode=abi.GR_ENV_STUDIO,
              **kw) -> S.Scene:
    return S.Scene(width=width, height=height, planes=S.standard_round_brilliant(), material=S.builtin_material(material),
                   cam=test_camera(), max_bounces=max_bounces, env_mode=env_mode, preset=preset, **kw)


def oracle_trace_samples(oracle, scene: S.Scene, first_pixel: int, n_pixels: int, offset: int, spp: int, threads=0):
    out = np.empty((n_pixels * spp, 3), np.float32)
    bounces = np.empty(n_pixels * spp, np.uint32)
    term = np.empty(n_pixels * spp, np.uint32)
    st = oracle.gro_trace_samples(C.byref(scene.c_scene()), first_pixel, n_pixels, offset, spp,
                                  out.ctypes.data_as(C.POINTER(C.c_float)),
                                  bounces.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  term.ctypes.data_as(C.POINTER(C.c_uint32)), None, threads)
    return st, out, bounces, term


def oracle_accumulate(oracle, scene: S.Scene, offset: int, spp: int, f64=False, threads=0):
    n = scene.width * scene.height
    if f64:
        acc = np.zeros((n, 3), np.float64)
        st = oracle.gro_accumulate_f64(C.byref(scene.c_scene()), offset, spp, acc.ctypes.data_as(C.POINTER(C.c_double)), threads)
    else:
        acc = np.zeros((n, 3), np.float32)
        st = oracle.gro_accumulate(C.byref(scene.c_scene()), offset, spp, acc.ctypes.data_as(C.POINTER(C.c_float)), threads)
    return st, acc


# ---- event sequences (gr_trace_events / gro_trace_events) -------------------------
TIE_EPS = 1e-4        # renderer/gpu/polyhedron_check.rs:37-43: a different facet within this t is a tie
HIT_ULP_BUDGET = 512  # polyhedron_check.rs:61: t of the same facet


def _event_arrays(n, kmax):
    return (np.empty(n, np.uint32), np.empty(n, np.uint32), np.empty((n, kmax), np.int32),
            np.empty((n, kmax), np.float32), np.empty((n, kmax), np.uint8))


def _ptrs(arrs):
    b, t, f, th, ev = arrs
    return (b.ctypes.data_as(C.POINTER(C.c_uint32)), t.ctypes.data_as(C.POINTER(C.c_uint32)),
            f.ctypes.data_as(C.POINTER(C.c_int32)), th.ctypes.data_as(C.POINTER(C.c_float)),
            ev.ctypes.data_as(C.POINTER(C.c_uint8)))


def device_events(renderer, scene: S.Scene, first_pixel: int, n_pixels: int, offset: int, spp: int, kmax: int = 64):
    arrs = _event_arrays(n_pixels * spp, kmax)
    st = renderer.lib.gr_trace_events(renderer.ctx, C.byref(scene.c_scene()), first_pixel, n_pixels, offset, spp, kmax,
                                      *_ptrs(arrs))
    assert st == abi.GR_OK, renderer.lib.gr_last_error_string()
    return arrs


def oracle_events(oracle, scene: S.Scene, first_pixel: int, n_pixels: int, offset: int, spp: int, kmax: int = 64):
    arrs = _event_arrays(n_pixels * spp, kmax)
    st = oracle.gro_trace_events(C.byref(scene.c_scene()), first_pixel, n_pixels, offset, spp, kmax, *_ptrs(arrs), 0)
    assert st == abi.GR_OK
    return arrs


def compare_sequences(dev, ora) -> dict:
    """Per-tuple comparison of two event logs (bounces, termination, facets, t, events).

    Classes: `exact` (every recorded facet and event and the ending agree); `tie` (the
    first difference is a different facet whose hit distance is within TIE_EPS of the
    oracle's -- the reference's whitelisted grazing tie); `flip` (the same facet but a
    different event, or the same sequence with a different ending: a decision at a
    threshold that libm ULPs moved); `mismatch` (anything else).  `t_ulp_max` is the
    largest ULP distance of t over the exact tuples' recorded bounces."""
    db, dt, df, dth, dev_ev = dev
    ob, ot, of, oth, oev = ora
    kmax = df.shape[1]
    n = db.shape[0]
    rec_o = np.minimum(ob + (ot == abi.GR_TERM_ROULETTE), kmax)
    rec_d = np.minimum(db + (dt == abi.GR_TERM_ROULETTE), kmax)
    idx = np.arange(kmax)[None, :]
    valid = idx < np.minimum(rec_o, rec_d)[:, None]
    fdiff = (df != of) & valid
    ediff = (dev_ev != oev) & valid
    anydiff = fdiff | ediff
    first = np.where(anydiff.any(1), anydiff.argmax(1), -1)
    ends_equal = (db == ob) & (dt == ot)
    exact = (first < 0) & ends_equal
    cls = np.full(n, "mismatch", dtype=object)
    cls[exact] = "exact"
    rows = np.nonzero(first >= 0)[0]
    j = first[rows]
    facet_diff = df[rows, j] != of[rows, j]
    close = np.abs(dth[rows, j].astype(np.float64) - oth[rows, j].astype(np.float64)) < TIE_EPS
    cls[rows[facet_diff & close]] = "tie"
    cls[rows[~facet_diff]] = "flip"
    cls[(first < 0) & ~ends_equal] = "flip"
    ia = dth.view(np.int32).astype(np.int64)
    ib = oth.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    tulp = np.where(valid & exact[:, None], np.abs(ia - ib), 0)
    out = {c: float(np.mean(cls == c)) for c in ("exact", "tie", "flip", "mismatch")}
    out["n"] = int(n)
    out["t_ulp_max"] = int(tulp.max()) if n else 0
    out["mean_bounces"] = float(ob.mean()) if n else 0.0
    return out
