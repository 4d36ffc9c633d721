"""Multi-rank sharding by absolute sample range, on CPU with gloo (world size 2).

Each rank renders its slice of the sample range with the oracle standing in for the
per-GPU engine and the films are summed with one all-reduce (and, as the sharded
frame's end-to-end step does, with one reduce onto rank 0).  The result must equal,
bit for bit, the single-process composition of the same slices (each slice folded
from zero in sample order, the partial films added in rank order), and match one
render of the whole range to f32 summation accuracy.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from gemray_studio_b200.shard import sample_range


def test_sample_range_tiles_the_range():
    for world in (1, 2, 3, 8):
        for samples in (0, 1, 7, 64, 1000):
            got = [sample_range(r, world, 100, samples) for r in range(world)]
            assert sum(c for _, c in got) == samples
            nxt = 100
            for first, count in got:
                assert first == nxt
                nxt += count
    with pytest.raises(ValueError):
        sample_range(2, 2, 0, 8)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "tests")]
    import torch
    import torch.distributed as dist

    import oracle_lib
    from helpers import oracle_accumulate, srb_scene
    from gemray_studio_b200.shard import render_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        oracle = oracle_lib.lib()
        sc = srb_scene("Diamond", width=12, height=10, max_bounces=12)
        film = torch.zeros((sc.width * sc.height, 3), dtype=torch.float32)

        def render(first, count, f):
            st, acc = oracle_accumulate(oracle, sc, first, count, threads=2)
            assert st == 0
            f += torch.from_numpy(acc)

        film, rng = render_sharded(render, 5, 37, film, dst=None)
        np.save(os.path.join(out_dir, f"film{rank}.npy"), film.numpy())
        np.save(os.path.join(out_dir, f"range{rank}.npy"), np.array(rng))
        # the sharded frame's reduction onto one rank (the multi-GPU e2e step's collective)
        onto0 = torch.zeros_like(film)
        onto0, _ = render_sharded(render, 5, 37, onto0, dst=0)
        if rank == 0:
            np.save(os.path.join(out_dir, "onto0.npy"), onto0.numpy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_compose_like_one_process(oracle, tmp_path):
    import torch.multiprocessing as mp

    from helpers import oracle_accumulate, srb_scene
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    films = [np.load(tmp_path / f"film{r}.npy") for r in range(world)]
    ranges = [tuple(np.load(tmp_path / f"range{r}.npy")) for r in range(world)]
    assert ranges == [(5, 19), (24, 18)]
    assert np.array_equal(films[0].view(np.uint32), films[1].view(np.uint32))   # all-reduce: same on every rank
    sc = srb_scene("Diamond", width=12, height=10, max_bounces=12)
    parts = [oracle_accumulate(oracle, sc, f, c)[1] for f, c in ranges]
    composed = np.zeros_like(parts[0])
    for p in parts:
        composed = composed + p
    assert np.array_equal(films[0].view(np.uint32), composed.view(np.uint32))
    onto0 = np.load(tmp_path / "onto0.npy")
    assert np.array_equal(onto0.view(np.uint32), composed.view(np.uint32))   # reduce onto rank 0
    _, whole = oracle_accumulate(oracle, sc, 5, 37)
    assert np.allclose(films[0], whole, rtol=1e-5, atol=1e-6)
