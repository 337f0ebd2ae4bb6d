"""bench.py's multi-GPU host logic on CPU: two gloo ranks shard the 16
sources as replicas and reduce their timings (max) and work (sum) exactly as
the NCCL path does on GPUs."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        srcs = list(range(100, 116))
        mine = bench.shard_sources(srcs, rank, world)
        t = [1.0 + rank, 10.0 - rank]            # per-rank timed intervals
        c = [len(mine) * 1000, 7 * (rank + 1)]   # per-rank work counts
        times, counts = bench.reduce_over_ranks(t, c, "cpu", True)
        q.put((rank, mine, times, counts))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_reduction():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    shards = [o[1] for o in out]
    assert sorted(shards[0] + shards[1]) == list(range(100, 116))     # every source once
    assert not set(shards[0]) & set(shards[1])
    for _, _, times, counts in out:
        assert times == [2.0, 10.0]                                     # max over ranks
        assert counts == [16000.0, 21.0]                                # sum over ranks


def test_single_rank_and_more_ranks_than_sources():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.shard_sources([1, 2, 3], 0, 1) == [1, 2, 3]
    assert bench.shard_sources([1, 2, 3], 4, 5) == [2]
    times, counts = bench.reduce_over_ranks([1.5], [3], "cpu", False)
    assert times == [1.5] and counts == [3.0]
