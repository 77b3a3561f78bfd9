"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one independent replica per GPU and reports the whole job as
(units summed over ranks) / (slowest rank's time); these tests check that
aggregation with real collectives, and that the reference arm does its work
on rank 0 only.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r processed 100*(r+1) units in 1+r seconds
        rate, tmax = bench.job_rate(100.0 * (rank + 1), 1.0 + rank, world, "cpu")
        mx = bench.max_over_ranks(float(rank) - 5.0, world, "cpu")
        out.put((rank, rate, tmax, mx))
    finally:
        dist.destroy_process_group()


def test_job_rate_two_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.SimpleQueue()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    got = sorted(out.get() for _ in range(world))
    for rank, rate, tmax, mx in got:
        assert tmax == 2.0                     # the slowest rank's time, on every rank
        assert rate == pytest.approx(300.0 / 2.0)
        assert mx == -4.0


def test_single_rank_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_rate(50.0, 2.0, 1, "cpu") == (25.0, 2.0)
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5


def test_reference_arm_other_ranks_do_nothing():
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=0)
    assert bench.run_reference(args, rank=1, world=2) == 0   # returns at once, prints nothing
