"""Multi-GPU sharding of the transport path by absolute sample range.

Every (pixel, absolute sample) tuple is independent and films add (the reference's
partition contract: disjoint sample ranges rendered anywhere compose,
crates/gemray-net/tests/partition_correctness.rs), so N ranks --
one process per GPU -- each render a disjoint slice of [first_sample,
first_sample + samples) into a film of their own.  The only exchange is one
element-wise sum of the W*H*3 films, `reduce_films`, over torch.distributed (NCCL
over NVLink between GPUs; gloo on CPU).  Each rank's slice is folded in sample
order and the partial films are summed (for two ranks the sum is exactly
film_0 + film_1, whatever order the collective uses), which is how the reference
composes films arriving from remote workers.
"""
from __future__ import annotations


def sample_range(rank: int, world: int, first_sample: int, samples: int) -> tuple[int, int]:
    """Rank `rank`'s contiguous slice (first, count) of [first_sample, first_sample + samples):
    the first `samples % world` ranks take one sample more, so the slices tile the range
    exactly and in rank order."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(samples, world)
    count = base + (1 if rank < extra else 0)
    first = first_sample + rank * base + min(rank, extra)
    return first, count


def reduce_films(film, group=None, dst: int | None = None):
    """Sum the ranks' films element-wise.  dst=None: every rank receives the sum
    (all-reduce); else only rank `dst` (reduce).  `film` is a torch tensor (on the
    rank's GPU with NCCL, on the CPU with gloo), updated in place and returned."""
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return film
    if dst is None:
        dist.all_reduce(film, op=dist.ReduceOp.SUM, group=group)
    else:
        dist.reduce(film, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return film


def render_sharded(render_fn, first_sample: int, samples: int, film, group=None, dst: int | None = 0):
    """This rank renders its slice with render_fn(first, count, film) (which ADDs into
    `film`), then the films are summed.  Returns (film, (first, count))."""
    import torch.distributed as dist
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    first, count = sample_range(rank, world, first_sample, samples)
    if count:
        render_fn(first, count, film)
    return reduce_films(film, group, dst), (first, count)
