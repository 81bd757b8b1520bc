"""Spreading independent solves over ranks (one process per GPU).

Matting solves of different images share nothing, so the multi-GPU form of
the batched path needs no collective on the data path: every rank takes a
bin of whole images and solves it with one batched launch.  The only
collectives are the timing reductions of the benchmark (max of the per-rank
device times, sum of the work), over whatever process group the caller set
up (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def shard_images(sizes, world: int) -> list[list[int]]:
    """Size-balanced bins: images by pixel count, largest first, each to the
    rank with the least work so far (ties to the lower rank).  Returns the
    image indices of every rank, each list in ascending index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-sizes[k][0] * sizes[k][1], k))
    load = [0] * world
    bins: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda j: (load[j], j))
        bins[r].append(k)
        load[r] += sizes[k][0] * sizes[k][1]
    return [sorted(b) for b in bins]


def _reduce(x: float, op: str) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float) -> float:
    """Largest per-rank value (the job's time is its slowest rank's)."""
    return _reduce(x, "max")


def sum_over_ranks(x: float) -> float:
    """Total over ranks (the job's work)."""
    return _reduce(x, "sum")
