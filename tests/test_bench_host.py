"""bench.py's host-side bookkeeping, no GPU: which transport a run used (from its launch
counts), the per-launch DRAM traffic taken from the committed captures, the HBM view's
labelled fallback peak, and where the stones' schedules come from (the committed table
or live trials)."""
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


class _FakeLib:
    """Stands in for the engine library's tuning-table loader."""

    def __init__(self, status: int, n: int = 0, error: bytes = b""):
        self.status, self.n, self.error, self.paths = status, n, error, []

    def gr_tuning_load(self, ctx, path, n_out):
        self.paths.append(path)
        n_out._obj.value = self.n
        return self.status

    def gr_last_error_string(self):
        return self.error


def test_schedule_source_names_the_committed_table_or_the_trials():
    from gemray_studio_b200 import abi
    ok = _FakeLib(abi.GR_OK, n=67)
    assert bench.load_tuning_table(ok, None).startswith("gemray_studio_b200/tuning/b200_schedules.txt (67 stones)")
    assert ok.paths == [str(bench.TUNING_TABLE).encode()]
    foreign = _FakeLib(abi.GR_EINVAL, error=b"not written for this schedule set and device")
    assert bench.load_tuning_table(foreign, None).startswith("trials (not written")
    bench._use_tuning_table = False
    try:
        off = _FakeLib(abi.GR_OK, n=67)
        assert bench.load_tuning_table(off, None) == "trials" and off.paths == []
    finally:
        bench._use_tuning_table = True
