"""The multi-GPU path is replicas: each rank processes its own share of
independent reconstructions, and the job's throughput is all ranks' units
over the slowest rank's time.  Checked with two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "nadia-coecxs_b200"))

from pynadia import replicas  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = replicas.shard(10, rank, world)
        # rank r "takes" r+1 seconds for its share of 8 reconstructions
        rate = replicas.job_rate(len(mine), rank + 1.0)
        slowest = replicas.max_over_ranks(rank + 1.0)
        total = replicas.sum_over_ranks(len(mine))
        out[rank] = (mine, rate, slowest, total)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_covers_every_item_once():
    for world in (1, 2, 3, 8):
        got = sorted(i for r in range(world) for i in replicas.shard(17, r, world))
        assert got == list(range(17))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_single_process_needs_no_group():
    assert replicas.job_rate(8, 2.0) == 4.0
    assert replicas.max_over_ranks(3.5) == 3.5


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    shares = [out[r][0] for r in range(world)]
    assert sorted(shares[0] + shares[1]) == list(range(10))
    assert not set(shares[0]) & set(shares[1])
    for r in range(world):
        mine, rate, slowest, total = out[r]
        assert slowest == 2.0
        assert total == 10
        assert rate == 10 / 2.0
