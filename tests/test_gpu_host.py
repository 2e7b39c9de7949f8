"""GPU tests of the host-buffer entry point (aerial_pusch_eq_host): host
H / Y_rx in, host LLRs out, batches pipelined over internal streams.  The
staged launch is the same fused kernel, and a cell's results do not depend
on which cells share its launch, so outputs must equal a resident
aerial_pusch_eq_fused run bit for bit."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from test_gpu_fused import run_fused

pytestmark = pytest.mark.gpu


def host_buffers(cells, pinned=True, yeq_every=2):
    out = []
    for k, c in enumerate(cells):
        H = c.H.contiguous()
        Y = c.Y.contiguous()
        llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32)
        yeq = torch.full((c.nSC * c.nLayers * c.nSym,), float("nan"), dtype=torch.complex64) \
            if yeq_every and k % yeq_every == 0 else None
        if pinned:
            H, Y, llr = H.pin_memory(), Y.pin_memory(), llr.pin_memory()
            yeq = yeq.pin_memory() if yeq is not None else None
        out.append((H, Y, llr, yeq))
    return out


def run_host(aeq, cells, bufs, cuda, cells_per_batch=0, stream=None, tuning=None):
    descs = [aeq.host_cell_desc(H, Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=ye)
             for c, (H, Y, l, ye) in zip(cells, bufs)]
    nbytes = aeq.pusch_eq_host_workspace(descs, cells_per_batch)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
    aeq.pusch_eq_host(descs, ws, tuning if tuning is not None else aeq.make_tuning("fp16"), cells_per_batch,
                      stream)
    return ws


@pytest.mark.parametrize("cells_per_batch", [0, 1, 3])
def test_host_pipeline_matches_resident(aeq, wl, cuda, cells_per_batch):
    cells = wl.multicell(10, seed=61)
    ref = run_fused(aeq, cells, cuda, "fp16")
    bufs = host_buffers(cells)
    run_host(aeq, cells, bufs, cuda, cells_per_batch)
    torch.cuda.synchronize()
    for k, (H, Y, llr, yeq) in enumerate(bufs):
        np.testing.assert_array_equal(llr.numpy(), ref[k][0])
        if yeq is not None:
            np.testing.assert_array_equal(yeq.numpy(), ref[k][1])


def test_host_pipeline_pageable_memory(aeq, wl, cuda):
    """Pageable host buffers give the same results (the copies do not overlap)."""
    cells = [wl.config_cell(1, seed=63 + k) for k in range(4)]
    ref = run_fused(aeq, cells, cuda, "fp16")
    bufs = host_buffers(cells, pinned=False)
    run_host(aeq, cells, bufs, cuda, 1)
    torch.cuda.synchronize()
    for k, (_, _, llr, yeq) in enumerate(bufs):
        np.testing.assert_array_equal(llr.numpy(), ref[k][0])


def test_host_pipeline_orders_on_caller_stream(aeq, wl, cuda):
    """Work is enqueued behind the caller's stream and the caller's stream
    waits for all of it: synchronizing that stream alone is enough."""
    cells = [wl.config_cell(2, seed=67 + k) for k in range(5)]
    ref = run_fused(aeq, cells, cuda, "fp16")
    bufs = host_buffers(cells, yeq_every=0)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        torch.cuda._sleep(2_000_000)        # the caller's stream is busy when the call is made
        ws = run_host(aeq, cells, bufs, cuda, 1, stream=side)
    side.synchronize()
    for k, (_, _, llr, _) in enumerate(bufs):
        np.testing.assert_array_equal(llr.numpy(), ref[k][0])
    del ws


def test_host_pipeline_repeated_calls_share_streams(aeq, wl, cuda):
    cells = [wl.config_cell(1, seed=71 + k) for k in range(6)]
    ref = run_fused(aeq, cells, cuda, "bf16x3")
    for _ in range(3):
        bufs = host_buffers(cells, yeq_every=3)
        run_host(aeq, cells, bufs, cuda, 2, tuning=aeq.make_tuning("bf16x3"))
        torch.cuda.synchronize()
        for k, (_, _, llr, yeq) in enumerate(bufs):
            np.testing.assert_array_equal(llr.numpy(), ref[k][0])
            if yeq is not None:
                np.testing.assert_array_equal(yeq.numpy(), ref[k][1])


def test_host_pipeline_rejects_small_workspace(aeq, wl, cuda):
    cells = [wl.config_cell(1, seed=73)]
    bufs = host_buffers(cells)
    c = cells[0]
    H, Y, l, ye = bufs[0]
    d = [aeq.host_cell_desc(H, Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=ye)]
    need = aeq.pusch_eq_host_workspace(d)
    ws = torch.empty(need - 256, dtype=torch.uint8, device=cuda)
    with pytest.raises(aeq.AerialError):
        aeq.pusch_eq_host(d, ws)
