"""The multi-rank host logic on the CPU with two gloo ranks: the bench's
maximum over ranks (the slowest rank's time is the job's), and the split of
independent point sets over ranks (contiguous, every set exactly once, point
counts within one set of an equal share)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, offsets, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from yggdrax_b200 import batch

        w, r, lr = bench._dist()
        assert (w, r, lr) == (world, rank, rank)
        got = bench._max_over_ranks([float(rank + 1), 10.0 - rank, 0.5], "cpu")
        s0, s1 = batch.shard_sets(offsets, rank, world)
        ranges = [None] * world
        dist.all_gather_object(ranges, (s0, s1))
        if rank == 0:
            out.put((got, ranges))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks(world):
    rng = np.random.default_rng(3)
    sizes = np.floor(np.exp(rng.uniform(np.log(256), np.log(65536), 300))).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, offsets, q)) for r in range(world)]
    for p in procs:
        p.start()
    got, ranges = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got == [float(world), 10.0, 0.5]
    # contiguous, complete, balanced
    assert ranges[0][0] == 0 and ranges[-1][1] == len(sizes)
    for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
        assert a1 == b0
    share = offsets[-1] / world
    for a0, a1 in ranges:
        assert abs((offsets[a1] - offsets[a0]) - share) <= sizes.max()


def test_shard_sets_single_rank_and_errors():
    from yggdrax_b200 import batch

    off = np.array([0, 5, 9, 20])
    assert batch.shard_sets(off, 0, 1) == (0, 3)
    with pytest.raises(ValueError):
        batch.shard_sets(off, 2, 2)
