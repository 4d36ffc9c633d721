"""GPU parity on the benchmarked scenes themselves: the device against the FP32 oracle
per sample (gr_trace_samples) and per film (gr_accumulate) on c1 (57-facet brilliant,
uniform white, depth 32), c2 (the same stone in the full 2048x1024 lat-long map of 12
Gaussian lights), c3 (the 49-plane step-cut emerald with the uniaxial dichroic
material, both its wavelength-dependent Delta n / tabulated-absorption extension and
the reference model's constant Delta n, studio rig, depth 64) and four C4 random stones
(the Cauchy crown glass with its absorption bands among them).  Per-sample bars are
those of tests/test_gpu_parity.py: CUDA's accurate sinf/cosf/atan2f/acosf/expf are not
glibc's, so a sample matches to a few ULP unless a libm ULP flips one of its branch
decisions; the lat-long lookup magnifies acos/atan2 ULPs through the map gradient.
The frames are cut to a band of rows through the stone (the oracle runs on the host)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gemray_studio_b200 import abi, workloads as W
from helpers import oracle_accumulate, oracle_trace_samples

pytestmark = pytest.mark.gpu

REL_TIGHT = 1e-5
REL_LOOSE = 1e-3


def _rel(a, b):
    return np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-30)


def _band(sc, rows: int):
    y0 = sc.height // 2 - rows // 2
    return y0 * sc.width, rows * sc.width


def _check(renderer, oracle, sc, first, n_pix, spp, tight, loose_bad, offset=0, vs_fp64=False):
    gpu = renderer.trace_samples(sc, first, n_pix, offset, spp)
    st, ref, _b, _t = oracle_trace_samples(oracle, sc, first, n_pix, offset, spp)
    assert st == abi.GR_OK
    assert np.all(np.isfinite(gpu))
    rel = _rel(gpu, ref)
    lit = ref.max(axis=1) > 0
    assert lit.mean() > 0.05  # the band crosses the stone or its lights
    within, bad = float(np.mean(rel <= REL_TIGHT)), float(np.mean(rel > REL_LOOSE))
    print(f"{n_pix * spp} samples: {within:.5f} within 1e-5, {bad:.5f} above 1e-3")
    assert within >= tight, within
    assert bad <= loose_bad, bad
    assert abs(gpu[:, 1].mean() - ref[:, 1].mean()) <= 0.02 * abs(ref[:, 1].mean()) + 1e-6
    if vs_fp64:
        # the same samples through the FP64 oracle: the reference's own f32 arithmetic
        # is much farther from it than the device is from the f32 reference
        r64 = np.empty_like(ref)
        assert oracle.gro_trace_samples_f64(C.byref(sc.c_scene()), first, n_pix, offset, spp,
                                            r64.ctypes.data_as(C.POINTER(C.c_float)), 0) == abi.GR_OK
        bad_ref = float(np.mean(_rel(ref, r64) > REL_LOOSE))
        print(f"  FP32 oracle vs FP64 oracle: {bad_ref:.5f} above 1e-3")
        assert bad <= 0.25 * bad_ref, (bad, bad_ref)


def test_c1_round_brilliant_uniform(renderer, oracle):
    sc, _ = W.config_scene("c1")
    _check(renderer, oracle, sc, 0, sc.width * sc.height, 4, 0.999, 0.0)


def test_c1_film_matches_oracle(renderer, oracle):
    """The full c1 frame through gr_accumulate at 8 spp: pixels whose samples all agree
    are bit-identical sums; the film's relative RMSE is at the libm-ULP level."""
    sc, _ = W.config_scene("c1")
    n = sc.width * sc.height
    acc = np.zeros((n, 3), np.float32)
    renderer.accumulate(sc, 0, 8, acc)
    st, ref = oracle_accumulate(oracle, sc, 0, 8)
    assert st == abi.GR_OK
    rel = np.sqrt(np.mean((acc - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
    assert rel < 1e-5, rel
    assert np.mean(np.all(acc.view(np.uint32) == ref.view(np.uint32), axis=1)) > 0.3


def test_c2_round_brilliant_latlong(renderer, oracle):
    sc, _ = W.config_scene("c2")
    first, n = _band(sc, 48)
    _check(renderer, oracle, sc, first, n, 2, 0.90, 0.005)


@pytest.mark.parametrize("lambda_dependent", [True, False], ids=["extension", "constant-dn"])
def test_c3_emerald_birefringent_dichroic(renderer, oracle, lambda_dependent):
    """Depth 64 through a birefringent, dichroic stone: every facet / event sequence
    matches the oracle's (tests/test_gpu_sequences.py), but the extraordinary walk-off
    takes acos of a cosine near 1 -- ill-conditioned -- so the 1-2 ULP differences of
    CUDA's acosf / atanf / sincosf against glibc's grow along the path.  Measured on
    B200: 97.9% of samples within 1e-5, 1.4% above 1e-3; the reference's own FP32
    tracer against the FP64 oracle on the same samples: 87% within 1e-5, 10% above 1e-3."""
    sc, _ = W.config_scene("c3", lambda_dependent=lambda_dependent)
    first, n = _band(sc, 64)
    _check(renderer, oracle, sc, first, n, 2, 0.975, 0.02, vs_fp64=True)


def test_c4_random_stones(renderer, oracle):
    stones = W.random_stones(64, seed=0)
    crown = [s for s in stones if s.material == "crown glass"]
    assert crown, "the C4 draw holds a crown-glass stone"
    picked = crown[:1] + [s for s in stones if s.material != "crown glass"][:3]
    for s in picked:
        sc = s.scene
        assert s.material != "crown glass" or sc.material.o_ray_band_count == 2  # absorbing bands active
        first, n = _band(sc, min(sc.height, max(4, 24576 // sc.width)))
        # lat-long maps magnify acos / atan2 ULPs through the map gradient (measured on
        # B200: 89.5-97.9% within 1e-5 across these stones, none above 1e-3)
        _check(renderer, oracle, sc, first, n, 2, 0.85, 0.01)
