"""CPU tests of the multi-rank path of bench.py with the gloo backend
(world_size 2): each rank equalizes its own cell-slots with no collective on
the data path; only the elapsed times meet, as a max over ranks."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # rank-dependent fake timings: the slowest rank decides
    got = bench.max_over_ranks([10.0 + 5.0 * rank, 1.0 + rank], world)
    rate = bench.whole_job_rate(1000, 4, world, got[0])
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (got, rate)


def test_max_over_ranks_and_whole_job_rate_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(world):
        got, rate = out[r]
        assert got == [15.0, 2.0]                      # max over both ranks
        assert rate == pytest.approx(2 * 1000 * 4 / 0.015)


def test_single_rank_is_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.0, 4.0], 1) == [3.0, 4.0]
    assert bench.whole_job_rate(100, 10, 1, 1000.0) == pytest.approx(1000.0)
