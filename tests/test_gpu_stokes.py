"""The Stokes film on the device (gr_accumulate_stokes) against the oracle's twin.

At 1 spp a film pixel is one sample, so the device's IQUV film is compared per sample
with the FP32 oracle on a band of the c3 emerald (birefringent, dichroic, studio rig,
depth 64) and of the c2 brilliant, with the per-sample bars of the XYZ parity tests
(the largest component difference relative to I).  The XYZ film of the same call is
gr_accumulate's bit for bit, and every device vector is physical."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import abi, workloads as W
from helpers import srb_scene

pytestmark = pytest.mark.gpu
FP = C.POINTER(C.c_float)


def device_stokes(renderer, sc, offset, spp, xyz=None, iquv=None):
    n = sc.width * sc.height
    xyz = np.zeros((n, 3), np.float32) if xyz is None else xyz
    iquv = np.zeros((n, 4), np.float32) if iquv is None else iquv
    st = renderer.lib.gr_accumulate_stokes(renderer.ctx, C.byref(sc.c_scene()), offset, spp, xyz.ctypes.data_as(FP),
                                           iquv.ctypes.data_as(FP))
    assert st == abi.GR_OK, renderer.lib.gr_last_error_string()
    return xyz, iquv


@pytest.mark.parametrize("cfg,tight,loose", [("c3", 0.975, 0.02), ("c2", 0.90, 0.01)])
def test_stokes_film_matches_oracle_per_sample(renderer, oracle, cfg, tight, loose):
    """c3's bars are those of its XYZ parity test (the walk-off's ill-conditioned acos
    grows libm ULPs along depth-64 paths; tests/test_gpu_bench_scenes.py)."""
    sc, _ = W.config_scene(cfg)
    rows = 16
    xyz_d, iquv_d = device_stokes(renderer, sc, 5, 1)
    first = (sc.height // 2 - rows // 2) * sc.width
    n = rows * sc.width
    xyz_o = np.empty((n, 3), np.float32)
    iquv_o = np.empty((n, 4), np.float32)
    assert oracle.gro_trace_samples_stokes(C.byref(sc.c_scene()), first, n, 5, 1, xyz_o.ctypes.data_as(FP),
                                           iquv_o.ctypes.data_as(FP), 0) == abi.GR_OK
    dev = iquv_d[first:first + n]
    rel = np.abs(dev - iquv_o).max(1) / np.maximum(np.abs(iquv_o[:, 0]), 1e-30)
    within, bad = float(np.mean(rel <= 1e-5)), float(np.mean(rel > 1e-3))
    print(cfg, within, bad)
    assert within >= tight and bad <= loose, (within, bad)
    pol = np.sqrt((iquv_d[:, 1:].astype(np.float64) ** 2).sum(1))
    assert np.all(pol <= iquv_d[:, 0] * (1 + 1e-5) + 1e-12)
    assert np.any(pol > 1e-3 * iquv_d[:, 0])


def test_stokes_call_adds_and_keeps_the_xyz_film(renderer):
    sc = srb_scene("Tourmaline", width=32, height=24, max_bounces=24)
    n = sc.width * sc.height
    base_x = np.random.default_rng(1).uniform(0, 1, (n, 3)).astype(np.float32)
    base_s = np.random.default_rng(2).uniform(0, 1, (n, 4)).astype(np.float32)
    x, s = device_stokes(renderer, sc, 0, 16, base_x.copy(), base_s.copy())
    ref = base_x.copy()
    renderer.accumulate(sc, 0, 16, ref)
    assert np.array_equal(x.view(np.uint32), ref.view(np.uint32))
    x0, s0 = device_stokes(renderer, sc, 0, 16)
    assert np.allclose(s - base_s, s0, rtol=1e-6, atol=1e-6)
    assert s0[:, 0].sum() > 0
