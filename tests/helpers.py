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
