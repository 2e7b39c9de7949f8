"""CPU tests of the multi-rank path of bench.py with the gloo backend
(world_size 2): each rank equalizes its own cell-slots with no collective on
the data path; only the elapsed times meet, as a max over ranks.  The ranks'
cell-slots (bench.build_cells, on CPU tensors) come from disjoint seeds, are
valid cells, and their REs add up to the whole job's."""
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
    # each rank's work: small steps of configurations 1, 2 and 4 on CPU tensors
    import importlib

    import torch

    wl = importlib.import_module("aerial-mimo-tc-optimization_b200.workload")
    work = {}
    for cfg, slots in ((1, 3), (2, 2), (4, 3)):
        cells = bench.build_cells(wl, cfg, slots, rank, "cpu")
        seeds = bench.cell_seeds(cfg, slots, rank)
        assert len(cells) == (len(seeds) if cfg != 4 else slots)
        for c in cells:
            assert c.H.shape == (c.nSC, c.nAnt, c.nLayers) and c.Y.shape == (c.nSC, c.nSym, c.nAnt)
            assert torch.isfinite(torch.view_as_real(c.H)).all() and torch.isfinite(torch.view_as_real(c.Y)).all()
        work[cfg] = (seeds, sum(c.n_re for c in cells), float(torch.view_as_real(cells[0].Y).sum()))
    gathered = [None] * world
    dist.all_gather_object(gathered, work)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (got, rate, gathered)


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
        got, rate, gathered = out[r]
        assert got == [15.0, 2.0]                      # max over both ranks
        assert rate == pytest.approx(2 * 1000 * 4 / 0.015)
    gathered = out[0][2]
    for cfg in (1, 2, 4):
        s0, n0, y0 = gathered[0][cfg]
        s1, n1, y1 = gathered[1][cfg]
        assert not set(s0) & set(s1), cfg              # disjoint seeds: no slot is equalized twice
        assert y0 != y1, cfg                           # and the data differ
        if cfg != 4:                                   # same shapes per rank: the REs add up
            assert n0 == n1 and n0 + n1 == 2 * n0
    # the whole-job rate counts every rank's REs once (equal per-rank work)
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.whole_job_rate(gathered[0][2][1], 1, world, 1000.0) == pytest.approx(
        gathered[0][2][1] + gathered[1][2][1])


def test_single_rank_is_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.0, 4.0], 1) == [3.0, 4.0]
    assert bench.whole_job_rate(100, 10, 1, 1000.0) == pytest.approx(1000.0)
