"""The oracle's Stokes film (the twin of gr_accumulate_stokes) on the CPU: its XYZ film is
the plain tracer's bit for bit, its I is the XYZ integral's Y (before the white balance,
which is the identity up to rounding in a uniform environment), every per-sample vector
is physical (degree of polarisation <= 1), light that never touches the stone stays
unpolarised, and the birefringent emerald polarises what it returns."""
from __future__ import annotations

import ctypes as C

import numpy as np

from gemray_studio_b200 import abi, workloads as W
from helpers import oracle_accumulate, srb_scene

FP = C.POINTER(C.c_float)


def samples(oracle, sc, first, n, spp):
    xyz = np.empty((n * spp, 3), np.float32)
    iquv = np.empty((n * spp, 4), np.float32)
    assert oracle.gro_trace_samples_stokes(C.byref(sc.c_scene()), first, n, 0, spp, xyz.ctypes.data_as(FP),
                                           iquv.ctypes.data_as(FP), 0) == abi.GR_OK
    return xyz, iquv


def test_stokes_film_xyz_is_the_plain_film(oracle):
    sc = srb_scene("Sapphire", width=24, height=16, max_bounces=16)
    n = sc.width * sc.height
    xyz = np.zeros((n, 3), np.float32)
    iquv = np.zeros((n, 4), np.float32)
    assert oracle.gro_accumulate_stokes(C.byref(sc.c_scene()), 3, 8, xyz.ctypes.data_as(FP), iquv.ctypes.data_as(FP),
                                        0) == abi.GR_OK
    st, ref = oracle_accumulate(oracle, sc, 3, 8)
    assert np.array_equal(xyz.view(np.uint32), ref.view(np.uint32))
    assert iquv[:, 0].sum() > 0


def test_stokes_i_is_y_and_vectors_are_physical(oracle):
    sc, _ = W.config_scene("c1")
    first = (sc.height // 2 - 8) * sc.width
    xyz, iquv = samples(oracle, sc, first, 16 * sc.width, 2)
    # the uniform environment's white balance is the identity, but its Bradford round trip
    # in f32 moves Y by ~1e-7 of X + Y + Z (the matrices mix the three with cancellation)
    y = xyz[:, 1].astype(np.float64)
    scale = np.abs(xyz.astype(np.float64)).sum(1)
    assert np.all(np.abs(iquv[:, 0] - y) <= 1e-6 * scale + 1e-12)
    pol = np.sqrt((iquv[:, 1:].astype(np.float64) ** 2).sum(1))
    assert np.all(pol <= iquv[:, 0] * (1 + 1e-5) + 1e-12)


def test_unpolarised_outside_the_stone_and_polarised_inside(oracle):
    sc, _ = W.config_scene("c3")
    xyz, iquv = samples(oracle, sc, (sc.height // 2) * sc.width, sc.width, 2)
    # rows through the middle of the frame: the stone's pixels carry polarisation, the
    # background's light reaches the camera directly and is unpolarised
    pol = np.sqrt((iquv[:, 1:].astype(np.float64) ** 2).sum(1))
    assert np.any(pol > 1e-3 * iquv[:, 0])
    xyz0, iquv0 = samples(oracle, sc, 0, sc.width, 2)  # the top row misses the stone
    assert np.all(iquv0[:, 1:] == 0.0) and np.all(iquv0[:, 0] > 0)
