"""Multi-GPU sharding of independent solves, exercised on CPU with gloo.

Images are dealt to ranks whole (no exchange on the data path); the only
collectives are the timing reductions.  Two gloo ranks check that the bins
cover every image exactly once, agree across ranks, that the max/sum
reductions give the job time and work, and that a rank which leaves without
joining a collective makes the other rank's collective fail instead of hang.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gpumatting_b200.shard import shard_images
from gpumatting_b200.synth import batch_sizes


def test_bins_cover_every_image_once_and_balance():
    sizes = batch_sizes(64, 256, 1024, seed=0)
    for world in (1, 2, 3, 4, 8):
        bins = shard_images(sizes, world)
        flat = sorted(k for b in bins for k in b)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k][0] * sizes[k][1] for k in b) for b in bins]
        biggest = max(w * h for w, h in sizes)
        assert max(loads) - min(loads) <= biggest  # greedy largest-first bound
    assert shard_images([(5, 5)], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        shard_images(sizes, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q, mode):
    import datetime

    import torch.distributed as dist

    from gpumatting_b200.shard import max_over_ranks, shard_images, sum_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        sizes = batch_sizes(64, 256, 1024, seed=0)
        mine = shard_images(sizes, world)[rank]
        if mode == "ok":
            everyone = [None] * world
            dist.all_gather_object(everyone, mine)
            t = max_over_ranks(1.5 + rank)          # per-rank "device time"
            w = sum_over_ranks(float(len(mine)))
            q.put((rank, everyone, t, w))
        else:  # rank 1 leaves before the collective; rank 0 must get an error
            if rank == 1:
                q.put((rank, "left"))
                return
            try:
                max_over_ranks(1.0)
                q.put((rank, "no error"))
            except Exception as e:  # noqa: BLE001 - any collective failure is the expected outcome
                q.put((rank, "error", type(e).__name__))
    finally:
        if mode == "ok":
            dist.destroy_process_group()


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q, mode)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda x: x[0])


def test_two_gloo_ranks_shard_and_reduce():
    out = _run("ok")
    sizes = batch_sizes(64, 256, 1024, seed=0)
    bins = shard_images(sizes, 2)
    for rank, everyone, t, w in out:
        assert everyone == bins                  # every rank derives the same bins
        assert t == 2.5                          # slowest rank's time
        assert w == 64.0                         # all images counted once


def test_rank_leaving_makes_the_collective_fail():
    out = _run("leave")
    assert out[1][1] == "left"
    assert out[0][1] == "error"
