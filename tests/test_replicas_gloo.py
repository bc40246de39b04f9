"""The multi-rank bookkeeping of bench.py (replicas only: every rank steps its
own box, no collective on the data path) with two gloo ranks on the CPU: the
barrier, the max-over-ranks time and the whole-job rate."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    barrier, max_over_ranks = bench.make_collectives(world, torch.device("cpu"))
    barrier()
    ms = 10.0 + 5.0 * rank  # rank 1 is the slowest
    slowest = max_over_ranks(ms)
    out[rank] = (slowest, bench.whole_job_rate(world, 100, slowest))
    barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_whole_job_rate():
    world = 2
    port = _free_port()
    # the manager process is spawned too: a fork of this (threaded) process is unsafe
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        slowest, rate = res[rank]
        assert slowest == 15.0
        assert rate == pytest.approx(2 * 100 / 0.015)


def test_single_rank_collectives_are_identities():
    sys.path.insert(0, ROOT)
    import bench
    barrier, max_over_ranks = bench.make_collectives(1, torch.device("cpu"))
    barrier()
    assert max_over_ranks(3.5) == 3.5
    assert bench.whole_job_rate(1, 50, 100.0) == pytest.approx(500.0)
