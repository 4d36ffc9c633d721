"""The FP32 oracle's per-function case banks against the FP64 oracle (CPU).

Each bank's FP64 budget (tests/case_banks.py) is the one the device is held to against
the FP64 oracle; this test shows that the reference's own FP32 arithmetic (the
oracle's FP32 instantiation) meets it, i.e. that the budget measures rounding of the
FP32 function and not a defect of the device port.  The device-side checks are in
tests/test_gpu_case_banks.py.
"""
from __future__ import annotations

import numpy as np
import pytest

import case_banks as CB

BANKS = CB.banks()


@pytest.mark.parametrize("k", range(len(BANKS)), ids=[f"{b.name}-{i}" for i, b in enumerate(BANKS)])
def test_fp32_oracle_within_fp64_budget(oracle, k):
    b = BANKS[k]
    r32 = CB.oracle_bank(oracle, b, 32)
    r64 = CB.oracle_bank(oracle, b, 64)
    rows = b.fp64_rows if b.fp64_rows is not None else slice(None)
    bad = CB.over_budget(r64[rows].astype(np.float32), r32[rows], b.budget64, b.floor64)
    assert np.all(np.isfinite(r32[rows])), b.name
    assert not bad.any(), (b.name, int(bad.sum()), CB.histogram(CB.ulp(r64[rows].astype(np.float32), r32[rows]).ravel()))


def test_bank_arities_match_header(oracle):
    import ctypes as C
    from gemray_studio_b200 import abi
    for name, i in abi.GR_BANK.items():
        ni, no = C.c_uint32(), C.c_uint32()
        assert oracle.gro_case_bank_arity(i, C.byref(ni), C.byref(no)) == 0
        assert ni.value >= 1 and no.value >= 1, name
    assert len(abi.GR_BANK) == abi.GR_BANK_COUNT


def test_exp_poly_matches_literal_formula(oracle):
    """simd/exp_poly.rs:23-40 restated in numpy float32 (fma via float64, exact for
    these products) agrees with the oracle bit for bit."""
    xs = np.linspace(-80, 80, 4001).astype(np.float32)
    got = CB.oracle_bank(oracle, CB.Bank("exp_poly", xs[:, None], None, 0, 0.0, 0, 0.0), 32)[:, 0].astype(np.float32)
    f = np.float32

    def fma(a, b, c):
        return np.float32(np.float64(a) * np.float64(b) + np.float64(c))

    c1 = np.frombuffer(np.uint32(0x3F318000).tobytes(), np.float32)[0]
    out = []
    for x in xs:
        n = np.floor(fma(x, f(1.44269504088896340736), f(0.5)))
        y = fma(n, -c1, x)
        y = fma(n, f(2.1219444e-4), y)
        z = f(y * y)
        p = f(1.9875691e-4)
        for c in (1.3981999e-3, 8.333452e-3, 4.1665796e-2, 1.6666665e-1, 5.0000003e-1):
            p = fma(p, y, f(c))
        p = f(fma(p, z, y) + f(1.0))
        out.append(f(p * np.frombuffer(np.uint32((int(n) + 127) << 23).tobytes(), np.float32)[0]))
    assert np.array_equal(np.asarray(out, np.float32).view(np.uint32), got.view(np.uint32))
