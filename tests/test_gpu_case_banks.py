"""Per-function case banks on the device (gr_case_bank) against the oracle, and the
transport's convex clip (gr_intersect_rays) against intersect_polyhedron.

Each bank runs the device function the transport kernels inline over seeded sweeps
(tests/case_banks.py) and is held
  * against the FP32 oracle (the reference's own arithmetic) to the reference's budget
    and absolute floor for the same function (renderer/gpu/transport_check/*.rs,
    camera_check.rs, environment_check.rs; within_tolerance, renderer/gpu/ulp.rs), and
  * against the FP64 oracle to the FP64 budget that the FP32 oracle itself meets
    (tests/test_oracle_case_banks.py).
The ULP histogram of each comparison is printed.  The clip bank uses the reference's
rule (polyhedron_check.rs:37-61): same facet with t within 512 ULP, or a different
facet whose t is within TIE_EPS = 1e-4 (a whitelisted grazing tie).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import case_banks as CB
from gemray_studio_b200 import abi, scene as S
from helpers import HIT_ULP_BUDGET, TIE_EPS

pytestmark = pytest.mark.gpu

BANKS = CB.banks()


def device_bank(renderer, bank: CB.Bank) -> np.ndarray:
    ni, no = C.c_uint32(), C.c_uint32()
    assert renderer.lib.gr_case_bank_arity(abi.GR_BANK[bank.name], C.byref(ni), C.byref(no)) == abi.GR_OK
    x = np.ascontiguousarray(bank.inputs, np.float32)
    out = np.empty((x.shape[0], no.value), np.float32)
    sc = C.byref(bank.scene.c_scene()) if bank.scene is not None else None
    st = renderer.lib.gr_case_bank(renderer.ctx, abi.GR_BANK[bank.name], sc, x.ctypes.data_as(C.POINTER(C.c_float)),
                                   x.shape[0], out.ctypes.data_as(C.POINTER(C.c_float)))
    assert st == abi.GR_OK, renderer.lib.gr_last_error_string()
    return out


@pytest.mark.parametrize("k", range(len(BANKS)), ids=[f"{b.name}-{i}" for i, b in enumerate(BANKS)])
def test_case_bank(renderer, oracle, k):
    b = BANKS[k]
    dev = device_bank(renderer, b)
    r32 = CB.oracle_bank(oracle, b, 32).astype(np.float32)
    r64 = CB.oracle_bank(oracle, b, 64)
    d32 = CB.ulp(r32, dev)
    print(f"{b.name}: {b.inputs.shape[0]} cases, vs FP32 oracle max {int(d32.max())} ULP ({CB.histogram(d32.ravel())})")
    bad32 = CB.over_budget(r32, dev, b.budget, b.floor)
    assert not bad32.any(), (b.name, int(bad32.sum()), np.argwhere(bad32)[:5].tolist())
    rows = b.fp64_rows if b.fp64_rows is not None else slice(None)
    d64 = CB.ulp(r64[rows].astype(np.float32), dev[rows])
    print(f"{b.name}: vs FP64 oracle max {int(d64.max())} ULP ({CB.histogram(d64.ravel())})")
    bad64 = CB.over_budget(r64[rows].astype(np.float32), dev[rows], b.budget64, b.floor64)
    assert not bad64.any(), (b.name, int(bad64.sum()))


def test_exp_poly_and_wavelengths_bit_exact(renderer, oracle):
    """The reference's own polynomial exp and the hero comb are pure f32 arithmetic with
    explicit fma: bit-identical on the device."""
    for name in ("exp_poly", "wavelengths"):
        b = next(x for x in BANKS if x.name == name)
        dev = device_bank(renderer, b)
        ref = CB.oracle_bank(oracle, b, 32).astype(np.float32)
        assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32)), name


@pytest.mark.parametrize("stone", ["srb", "rb57", "em49"])
def test_polyhedron_clip_bank(renderer, oracle, stone):
    planes = {"srb": S.standard_round_brilliant, "rb57": S.round_brilliant_57, "em49": S.emerald_cut_49}[stone]()
    planes = np.ascontiguousarray(planes, np.float32)
    rays = CB.polyhedron_rays()
    n = rays.shape[0]
    fp = C.POINTER(C.c_float)
    t_d, f_d = np.empty(n, np.float32), np.empty(n, np.int32)
    st = renderer.lib.gr_intersect_rays(renderer.ctx, planes.ctypes.data, planes.shape[0], rays.ctypes.data_as(fp), n,
                                        t_d.ctypes.data_as(fp), f_d.ctypes.data_as(C.POINTER(C.c_int32)))
    assert st == abi.GR_OK
    res = {}
    for prec in (32, 64):
        t_o, f_o = np.empty(n, np.float32), np.empty(n, np.int32)
        oracle.gro_intersect_rays(planes.ctypes.data, planes.shape[0], rays.ctypes.data_as(fp), n, prec,
                                  t_o.ctypes.data_as(fp), f_o.ctypes.data_as(C.POINTER(C.c_int32)))
        res[prec] = (t_o, f_o)
    t_o, f_o = res[32]
    both_miss = (f_d < 0) & (f_o < 0)
    same = (f_d == f_o) & (f_d >= 0)
    tie = (f_d != f_o) & (f_d >= 0) & (f_o >= 0) & (np.abs(t_d - t_o) < TIE_EPS)
    assert np.all(CB.ulp(t_o[same], t_d[same]) <= HIT_ULP_BUDGET)
    mismatch = ~(both_miss | same | tie)
    print(f"{stone}: {n} rays, hits {int((f_o >= 0).sum())}, exact {int((same | both_miss).sum())}, "
          f"ties {int(tie.sum())}, t max ULP {int(CB.ulp(t_o[same], t_d[same]).max())}")
    assert not mismatch.any(), np.argwhere(mismatch)[:5].ravel().tolist()
    assert (f_o >= 0).mean() > 0.5
    # against the FP64 clip: same rule; the f32 scan's own ties are the only differences
    t64, f64 = res[64]
    same64 = (f_d == f64) & (f_d >= 0)
    tie64 = (f_d != f64) & (f_d >= 0) & (f64 >= 0) & (np.abs(t_d - t64) < TIE_EPS)
    assert not (~(((f_d < 0) & (f64 < 0)) | same64 | tie64)).any()


def test_device_code_is_sm100(renderer):
    bv, pv = C.c_uint32(), C.c_uint32()
    assert renderer.lib.gr_device_code_version(renderer.ctx, C.byref(bv), C.byref(pv)) == abi.GR_OK
    assert bv.value == 100, bv.value
