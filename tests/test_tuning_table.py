"""The committed per-device schedule table (gemray_studio_b200/tuning/b200_schedules.txt,
written on a B200 by gemray_studio_b200/tuning_table.py): its identity line names the
current schedule set, and every entry is a stone key with one of the candidate
schedules and a positive time per M path-samples."""
from __future__ import annotations

import re
from pathlib import Path

import pytest

from gemray_studio_b200 import abi

TABLE = Path(__file__).resolve().parents[1] / "gemray_studio_b200" / "tuning" / "b200_schedules.txt"


@pytest.mark.skipif(not TABLE.exists(), reason="no committed schedule table")
def test_committed_table_names_candidate_schedules():
    lines = TABLE.read_text().splitlines()
    head = lines[0].split(" ", 2)
    assert head[0] == "gemray-schedules" and int(head[1]) == abi.GR_SCHEDULE_SET
    assert "B200" in head[2]
    candidates = {(a, b, m) for a, b in abi.SCHEDULE_CAP_PAIRS for m in abi.SCHEDULE_BLOCKS}
    keys = set()
    for line in lines[1:]:
        key, first, second, blocks, ms = line.split()
        assert re.fullmatch(r"[0-9a-f]{16}", key) and key not in keys
        keys.add(key)
        assert (int(first), int(second), int(blocks)) in candidates
        assert float(ms) > 0
    assert len(keys) >= 4  # the c1 and c2 brilliant (two environments), the c3 emerald, the c4 stones
