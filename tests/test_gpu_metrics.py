"""Device optical metrics (gr_optical_metrics / gr_angular_profile) against the oracle
and the reference's golden metric bits (crates/gemray/tests/raytracer_tests.rs:1818-1842).

Bars: every classification count is integer work, and the ratios and the
scintillation statistics are formed from the counts with the reference's f32
operations in the reference's order, so brilliance, windowing, extinction and
scintillation are bit-exact.  Fire sums acos-derived angles: CUDA's acosf is not
glibc's, so fire is held to 1e-5 relative.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest

from gemray_studio_b200 import abi, metrics as M, scene as S

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_goldens.json").read_text())
FIRE_REL = 1e-5
EXACT = [0, 2, 3, 4]  # brilliance, scintillation, windowing, extinction


def _oracle_metrics(oracle, planes: np.ndarray, material: abi.gr_material, pose) -> np.ndarray:
    p = np.ascontiguousarray(planes, np.float32).reshape(-1, 4)
    out = (C.c_float * 5)()
    oracle.gro_metrics(p.ctypes.data_as(C.POINTER(abi.gr_plane)), p.shape[0], C.byref(material), *map(float, pose), out)
    return np.array(out, np.float32)


def _check(got: np.ndarray, ref: np.ndarray):
    assert np.array_equal(got[EXACT].view(np.uint32), ref[EXACT].view(np.uint32)), (got, ref)
    assert abs(float(got[1]) - float(ref[1])) <= FIRE_REL * abs(float(ref[1])), (got[1], ref[1])


def test_golden_pose(renderer):
    g = GOLD["metrics"]
    m = M.evaluate_gem_optical_metrics(renderer, S.standard_round_brilliant(), S.builtin_material(g["material"]),
                                       g["cam_yaw"], g["cam_pitch"], g["light_yaw"], g["light_pitch"])
    got = np.array([m.brilliance_pct, m.fire_index, m.scintillation_pct, m.windowing_pct, m.extinction_pct], np.float32)
    ref = np.array(g["bits"], np.uint32).view(np.float32)
    _check(got, ref)


@pytest.mark.parametrize("stone,material", [("srb", "Diamond"), ("srb", "Sapphire"), ("rb57", "Cubic Zirconia"),
                                            ("emerald", "Emerald"), ("rb57", "Synthetic Moissanite"), ("srb", "Tanzanite")])
def test_pose_batch_matches_oracle(renderer, oracle, stone, material):
    planes = {"srb": S.standard_round_brilliant, "rb57": S.round_brilliant_57, "emerald": S.emerald_cut_49}[stone]()
    try:
        mat = S.builtin_material(material)
    except KeyError:
        pytest.skip(f"no built-in material {material}")
    rng = np.random.default_rng(11)
    poses = np.stack([rng.uniform(-math.pi, math.pi, 12), rng.uniform(0.0, 1.4, 12),
                      rng.uniform(-math.pi, math.pi, 12), rng.uniform(0.2, 1.3, 12)], axis=1).astype(np.float32)
    got = M.evaluate_poses(renderer, planes, mat, poses)
    for i in range(len(poses)):
        _check(got[i], _oracle_metrics(oracle, planes, mat, poses[i]))


def test_angular_profile_matches_oracle(renderer, oracle):
    planes = S.standard_round_brilliant()
    mat = S.builtin_material("Diamond")
    b, e, w = M.evaluate_angular_profile_at_azimuth(renderer, planes, mat, 0.3, 0.85, 0.95)
    to_rad = np.float32(np.float32(math.pi) / np.float32(180.0))
    for i, deg in enumerate(M.PROFILE_ANGLES_DEG):
        ref = _oracle_metrics(oracle, planes, mat, (0.3, np.float32(deg) * to_rad, 0.85, 0.95))
        assert [np.float32(b[i]), np.float32(e[i]), np.float32(w[i])] == [ref[0], ref[4], ref[3]], (i, deg)
    b0, _, _ = M.evaluate_angular_profile(renderer, planes, mat, 0.85, 0.95)
    b1, _, _ = M.evaluate_angular_profile_at_azimuth(renderer, planes, mat, 0.0, 0.85, 0.95)
    assert np.array_equal(b0, b1)


def test_fp64_sums_and_placeholder(renderer):
    planes = S.standard_round_brilliant()
    mat = S.builtin_material("Diamond")
    poses = [[0.0, 0.45, 0.85, 0.95], [1.0, 0.2, -0.5, 0.7]]
    f32 = M.evaluate_poses(renderer, planes, mat, poses)
    f64 = M.evaluate_poses(renderer, planes, mat, poses, fp64_sums=True)
    assert np.array_equal(f32[:, [0, 3, 4]], f64[:, [0, 3, 4]])      # counts only
    assert np.allclose(f32, f64, rtol=1e-4)
    empty = M.evaluate_poses(renderer, np.zeros((0, 4), np.float32), mat, poses)
    assert np.array_equal(empty, np.tile(np.float32([85, 25, 75, 5, 5]), (2, 1)))
