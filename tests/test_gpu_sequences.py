"""Facet-index and event sequences, device against the FP32 oracle (gr_trace_events).

The reference checks its GPU clip case by case and whitelists a different facet when
the two hit distances agree within TIE_EPS = 1e-4 (renderer/gpu/polyhedron_check.rs:
37-61); its instrumented trace logs the path (optics/raytracer/transport.rs:512-537).
Here every tuple's whole sequence -- facet, hit distance and event (TIR / reflect /
refract) per bounce, the final bounce index and the termination -- is compared.  A
tuple is `exact`, a whitelisted `tie` at its first difference, or a `flip` (same facet,
other event, or another ending: a threshold decision that a libm ULP moved).  Bars:
isotropic clear stones, whose geometry needs no libm, agree exactly on >= 99.9% of
tuples with t within the reference's 512-ULP hit budget; absorbing / birefringent
stones (acosf / sincosf / expf in the walk-off, Stokes and roulette weights) on >= 99%.
"""
from __future__ import annotations

import numpy as np
import pytest

from gemray_studio_b200 import abi, workloads as W
from helpers import HIT_ULP_BUDGET, compare_sequences, device_events, oracle_events, srb_scene

pytestmark = pytest.mark.gpu


def _run(renderer, oracle, sc, rows, spp, kmax=64):
    y0 = sc.height // 2 - rows // 2
    first, n = y0 * sc.width, rows * sc.width
    dev = device_events(renderer, sc, first, n, 0, spp, kmax)
    ora = oracle_events(oracle, sc, first, n, 0, spp, kmax)
    stats = compare_sequences(dev, ora)
    print(sc.width, sc.height, stats)
    return stats


def test_sequences_reference_srb_diamond(renderer, oracle):
    stats = _run(renderer, oracle, srb_scene("Diamond", width=64, height=64, max_bounces=32), 64, 4)
    assert stats["exact"] >= 0.999 and stats["mismatch"] == 0.0, stats
    assert stats["t_ulp_max"] <= HIT_ULP_BUDGET


@pytest.mark.parametrize("cfg", ["c1", "c2"])
def test_sequences_round_brilliant(renderer, oracle, cfg):
    sc, _ = W.config_scene(cfg)
    stats = _run(renderer, oracle, sc, 32 if cfg == "c2" else 256, 2)
    assert stats["exact"] >= 0.999 and stats["mismatch"] == 0.0, stats
    assert stats["t_ulp_max"] <= HIT_ULP_BUDGET
    assert stats["mean_bounces"] > 0.5  # the band crosses the stone


@pytest.mark.parametrize("lambda_dependent", [True, False], ids=["extension", "constant-dn"])
def test_sequences_emerald(renderer, oracle, lambda_dependent):
    sc, _ = W.config_scene("c3", lambda_dependent=lambda_dependent)
    stats = _run(renderer, oracle, sc, 48, 2)
    assert stats["exact"] >= 0.99 and stats["mismatch"] <= 0.001, stats


@pytest.mark.parametrize("material", ["Sapphire", "Tourmaline", "Tanzanite"])
def test_sequences_builtin_materials(renderer, oracle, material):
    stats = _run(renderer, oracle, srb_scene(material, width=48, height=48, max_bounces=24), 48, 4)
    assert stats["exact"] >= 0.99 and stats["mismatch"] <= 0.001, stats


def test_sequences_random_stones(renderer, oracle):
    stones = W.random_stones(8, seed=3, side=(96, 160))
    for s in stones:
        stats = _run(renderer, oracle, s.scene, 24, 2)
        assert stats["exact"] >= 0.99 and stats["mismatch"] <= 0.001, (s.material, s.n_planes, stats)


def test_event_record_layout(renderer, oracle):
    """Unrecorded slots hold -1 / 0xFF; a zero-bounce scene ends at the cap at once."""
    sc = srb_scene("Diamond", width=8, height=8, max_bounces=0)
    b, t, f, th, ev = device_events(renderer, sc, 0, 64, 0, 2, 8)
    assert np.all(b == 0) and np.all(t == abi.GR_TERM_HIT_CAP)
    assert np.all(f == -1) and np.all(ev == abi.GR_SEQ_NONE) and np.all(th == 0.0)
    sc = srb_scene("Diamond", width=16, height=16, max_bounces=12)
    b, t, f, th, ev = device_events(renderer, sc, 0, 256, 0, 2, 4)
    rec = np.minimum(b + (t == abi.GR_TERM_ROULETTE), 4)
    for i in range(b.size):
        assert np.all(f[i, :rec[i]] >= 0) and np.all(f[i, rec[i]:] == -1)
        assert np.all(ev[i, :rec[i]] <= abi.GR_SEQ_SCATTER) and np.all(ev[i, rec[i]:] == abi.GR_SEQ_NONE)
