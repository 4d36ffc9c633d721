"""The oracle's material extension pinned to hand-computed values (CPU).

The step-cut emerald workload uses two material features the reference model lacks
(its uniaxial n_e is n_o + a constant Delta n, optics/materials.rs:37 /
refraction.rs:287-294, and its absorption is a sum of Gaussian bands,
optics/absorption.rs:9-33): a wavelength-dependent extraordinary index from its own
Cauchy fit and tabulated absorption coefficients, linearly interpolated.  The reference
holds no values for them ("parity unpinned"), so the oracle's restatement is pinned
here to the formulas evaluated by hand: numpy float32 in the same operation order
(bit-exact), and the same formulas in float64 (within f32 rounding).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import workloads as W


def channel(oracle, mat, ext, lam, precision=32):
    out = (C.c_double * 4)()
    st = oracle.gro_material_channel(C.byref(mat), C.byref(ext) if ext is not None else None, lam, precision, out)
    assert st == 0
    return np.array(out[:])  # n_o, n_e, alpha_o, alpha_e


def cauchy_f32(a, b, c, lam_nm):
    f = np.float32
    lum = f(lam_nm) * f(1e-3)
    l2 = f(lum * lum)
    l4 = f(l2 * l2)
    return f(f(f(a) + f(f(b) / l2)) + f(f(c) / l4))


@pytest.mark.parametrize("lam", [380.0, 450.0, 486.1, 500.0, 550.0, 589.3, 650.0, 656.3, 780.0])
def test_cauchy_extraordinary_index(oracle, lam):
    mat, ext = W.birefringent_emerald_material(lambda_dependent=True)
    n_o, n_e, _, _ = channel(oracle, mat, ext, lam)
    assert np.float32(n_o) == cauchy_f32(1.640, 0.0042, 0.0, lam)
    assert np.float32(n_e) == cauchy_f32(1.620, 0.0040, 0.0, lam)
    exact_e = 1.620 + 4000.0 / lam ** 2  # n_e = 1.620 + 4000 / lambda_nm^2
    exact_o = 1.640 + 4200.0 / lam ** 2
    assert abs(n_e - exact_e) < 4e-7 and abs(n_o - exact_o) < 4e-7
    # the FP64 oracle evaluates the same law
    n_o64, n_e64, _, _ = channel(oracle, mat, ext, lam, 64)
    assert abs(n_e64 - exact_e) < 1e-6 and abs(n_o64 - exact_o) < 1e-6


def test_constant_birefringence_variant(oracle):
    """Without the extension the emerald keeps Delta n = n_e - n_o at 589.3 nm for every
    wavelength (the reference's model)."""
    mat, ext = W.birefringent_emerald_material(lambda_dependent=False)
    d589 = (1.620 + 0.0040 / 0.5893 ** 2) - (1.640 + 0.0042 / 0.5893 ** 2)
    for lam in (400.0, 589.3, 700.0):
        n_o, n_e, _, _ = channel(oracle, mat, ext, lam)
        assert abs((n_e - n_o) - d589) < 1e-6
        assert abs(d589 - (-0.020576)) < 1e-6


def test_tabulated_absorption_knots_and_interpolation(oracle):
    mat, ext = W.birefringent_emerald_material()
    # knots (cm^-1): o 0.8 / 0.3 / 0.1 and e 0.2 / 0.6 / 1.2 at 450 / 550 / 650 nm
    for lam, ao, ae in ((450.0, 0.8, 0.2), (550.0, 0.3, 0.6), (650.0, 0.1, 1.2)):
        _, _, a_o, a_e = channel(oracle, mat, ext, lam)
        assert a_o == np.float32(ao) and a_e == np.float32(ae), lam
    # held flat outside the knots and clamped at the table ends
    for lam in (300.0, 380.0, 420.0, 450.0):
        assert channel(oracle, mat, ext, lam)[2] == np.float32(0.8)
    for lam in (650.0, 700.0, 780.0, 900.0):
        assert channel(oracle, mat, ext, lam)[3] == np.float32(1.2)
    # midway between knots: the average; between grid points: the f32 linear interpolation
    assert abs(channel(oracle, mat, ext, 500.0)[2] - 0.55) < 1e-7
    assert abs(channel(oracle, mat, ext, 600.0)[3] - 0.9) < 1e-7
    a_o_tab = np.ctypeslib.as_array(ext.alpha_o_table, (ext.n_absorption,)).copy()
    f = np.float32
    for lam in (383.7, 502.5, 611.11, 777.0):
        x = f(f(f(lam) - f(380.0)) / f(5.0))
        i = int(x)
        t = f(x - f(i))
        want = f(a_o_tab[i] + f(t * f(a_o_tab[i + 1] - a_o_tab[i])))
        assert np.float32(channel(oracle, mat, ext, lam)[2]) == want, lam
        # and against the exact piecewise-linear law through the knots (float64)
        exact = np.interp(lam, [450.0, 550.0, 650.0], [0.8, 0.3, 0.1])
        assert abs(channel(oracle, mat, ext, lam, 64)[2] - exact) < 1e-6
