"""Multi-process host logic of the benchmark on CPU (gloo, world size 2): the
C4 batch is split across ranks with no overlap, and device times combine as
the max over ranks."""
import datetime
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, REPO)
    import bench
    from bevy_eulerian_fluid_b200 import scenes
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bs = scenes.batch(96)
        shard = bench.batch_shard(len(bs.scenes), world, rank)
        shards = [None] * world
        dist.all_gather_object(shards, shard)
        cells = [None] * world
        dist.all_gather_object(cells, sum(bs.scenes[i].cells for i in shard))
        t = torch.tensor([1.0 + rank, 10.0 - rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = (shards, cells, t.tolist())
    finally:
        dist.destroy_process_group()


def test_batch_shards_and_max_over_ranks():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    shards, cells, t = res[0]
    assert res[1][0] == shards and res[1][2] == t
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(96))                     # every simulation exactly once
    assert abs(len(shards[0]) - len(shards[1])) <= 1   # balanced by count
    assert t == [2.0, 10.0]                            # max over ranks, element-wise
    from bevy_eulerian_fluid_b200 import scenes
    assert sum(cells) == scenes.batch(96).cells
