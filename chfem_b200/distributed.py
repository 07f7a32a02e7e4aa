"""Multi-GPU homogenization of independent samples: one process per GPU, samples sharded across
ranks with no collective on the data path (each rank solves its own images on its own GPU);
only the small results are gathered.  Launch one process per GPU (torchrun) with an initialized
torch.distributed process group -- NCCL on GPUs, gloo works too.

The reference solves one image per process run; a set of images is the natural unit to spread
over GPUs, and a single image of the workloads here fits one B200.
"""
import numpy as np


def shard_range(n, rank, world):
    """Contiguous, balanced [lo, hi) share of n units for rank (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return rank * n // world, (rank + 1) * n // world


def map_samples(fn, items, group=None):
    """Apply fn to this rank's shard of items (fn takes a list, returns a list of results of the
    same length) and return every rank's results in item order, on every rank."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    lo, hi = shard_range(len(items), rank, world)
    mine = list(fn(list(items[lo:hi]))) if hi > lo else []
    if len(mine) != hi - lo:
        raise RuntimeError(f"rank {rank}: {len(mine)} results for {hi - lo} items")
    parts = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    return [r for part in parts for r in part]


def max_over_ranks(value, group=None, device=None):
    """The largest value over the ranks (a job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def conductivity_batch(arrays, mat_props, group=None, **kw):
    """compute_conductivity_batch over all ranks' GPUs: (n, 3, 3) tensors, on every rank."""
    from .batch import compute_conductivity_batch
    props = [mat_props] * len(arrays) if isinstance(mat_props, dict) else list(mat_props)
    pairs = list(zip(arrays, props))

    def solve(chunk):
        if not chunk:
            return []
        C = compute_conductivity_batch([a for a, _ in chunk], [p for _, p in chunk], **kw)
        return [np.asarray(c) for c in C]
    return np.stack(map_samples(solve, pairs, group=group))
