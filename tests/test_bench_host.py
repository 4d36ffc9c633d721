"""bench.py's host-side bookkeeping, no GPU: which transport a run used (from its launch
counts), the per-launch DRAM traffic taken from the committed captures, and the HBM
view's labelled fallback peak."""
from __future__ import annotations

import json
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parents[1]


def test_transport_resolution_from_launch_counts():
    assert bench.transport_kernel("auto", 9, 3) == "staged"    # three launches per chunk
    assert bench.transport_kernel("staged", 3, 1) == "staged"
    assert bench.transport_kernel("auto", 4, 4) == "plain"     # small launches under AUTO
    assert bench.transport_kernel("plain", 9, 9) == "plain"
    assert bench.transport_kernel("sorted", 9, 9) == "sorted"
    assert set(bench.TRANSPORT_LABELS) >= {"staged", "plain", "sorted"}


def test_traffic_scales_the_committed_per_tuple_figures():
    for kernel in ("staged", "plain"):
        per_tuple = json.loads((ROOT / "profiles" / f"k_trace_{kernel}_traffic.json").read_text())["dram_bytes_per_tuple"]
        assert bench.traffic_per_launch(2e6, kernel) == per_tuple * 2e6
    assert bench.traffic_per_launch(2e6, "sorted") is None   # no capture committed


def test_hbm_view_names_its_peak():
    v = bench.hbm_view(1e6, 10.0, "staged")
    assert v["unit"] == "GB/s" and v["peak"] > 0 and abs(v["frac"] - v["achieved"] / v["peak"]) < 1e-12
    assert "measured" in v["peak_source"] or "fallback" in v["peak_source"]
