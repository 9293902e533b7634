"""Replica execution across ranks (one process per GPU): request sharding and
the whole-job timing, run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from zipgpu import replicas


def test_shard_is_a_disjoint_cover():
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = replicas.shard(10, rank, world)
        # rank r "processes" its requests in (r + 1) seconds of simulated time
        res = replicas.job_throughput(units=100.0 * len(mine), seconds=1.0 + rank, dist=dist)
        dist.barrier()
        out[rank] = (len(mine), res["units"], res["seconds"], res["value"])
    finally:
        dist.destroy_process_group()


def test_job_throughput_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    assert got[0][0] + got[1][0] == 10
    for r in range(world):
        units, seconds, value = got[r][1:]
        assert units == 1000.0  # all ranks' units
        assert seconds == 2.0   # the slowest rank's time
        assert value == 500.0


def test_single_process_needs_no_group():
    res = replicas.job_throughput(units=42.0, seconds=2.0)
    assert res == {"units": 42.0, "seconds": 2.0, "value": 21.0}
