"""The per-device schedule table of the benchmark stones.

Every staged schedule (stage caps x blocks per SM) gives the same films; the engine's
tuner times trial calls per stone and keeps the fastest (gr_scene_schedule).  This
script runs the tuner to its choice for every stone of the benchmark workloads -- the
c1 / c2 brilliant, the c3 emerald and the 64 random c4 stones (the c5 request stream
draws its 32 stones from the same seeded sequence, so the table covers them too) --
and writes the context's table with gr_tuning_save.  bench.py loads the committed
table (gr_tuning_load) when it was written for the same device and schedule set, so
its timed frames start from the measured choices.

    python -m gemray_studio_b200.tuning_table [--out PATH]

The table is keyed by stone (planes, finishes, material, depth, flags, environment
kind), not by view or film size.
"""
from __future__ import annotations

import argparse
import ctypes as C
from pathlib import Path

TABLE = Path(__file__).resolve().parent / "tuning" / "b200_schedules.txt"


def tune(renderer, scene, spp: int, calls: int = 12) -> tuple[int, int, int]:
    """Renders `scene` (resident) until its schedule is chosen; returns (cap1, cap2, blocks)."""
    import torch

    from . import abi
    lib, ctx = renderer.lib, renderer.ctx
    sid = C.c_uint64()
    assert lib.gr_scene_upload(ctx, C.byref(scene.c_scene()), C.byref(sid)) == abi.GR_OK, lib.gr_last_error_string()
    film = torch.zeros((scene.width * scene.height, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    c1, c2, cb = C.c_uint32(), C.c_uint32(), C.c_uint32()
    try:
        for k in range(calls):
            assert lib.gr_scene_schedule(ctx, sid.value, C.byref(c1), C.byref(c2), C.byref(cb)) == abi.GR_OK
            if c1.value:
                break
            assert lib.gr_render_resident(ctx, sid.value, k * spp, spp, C.c_void_p(film.data_ptr()), None) == abi.GR_OK
            assert lib.gr_synchronize(ctx) == abi.GR_OK
        return c1.value, c2.value, cb.value
    finally:
        del film
        torch.cuda.synchronize()
        lib.gr_scene_release(ctx, sid.value)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", type=Path, default=TABLE)
    args = ap.parse_args(argv)
    from . import GpuFrameRenderer, abi, build
    from . import workloads as W
    build.build()
    r = GpuFrameRenderer()
    try:
        for name in ("c1", "c2", "c3"):
            sc, w = W.config_scene(name)
            print(name, tune(r, sc, w["spp"]), flush=True)
        for k, st in enumerate(W.random_stones(64, seed=0, side=(128, 1024), spp=(32, 512))):
            print("c4 stone", k, st.material, st.n_planes, tune(r, st.scene, st.spp), flush=True)
        args.out.parent.mkdir(parents=True, exist_ok=True)
        assert r.lib.gr_tuning_save(r.ctx, str(args.out).encode()) == abi.GR_OK, r.lib.gr_last_error_string()
        n = C.c_uint32()
        assert r.lib.gr_tuning_count(r.ctx, C.byref(n)) == abi.GR_OK
        print(f"{n.value} stones -> {args.out}")
    finally:
        r.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
