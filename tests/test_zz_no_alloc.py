"""The allocation-free plain chain, aerial_pusch_eq_plain_static.

Callers such as a real-time slot loop (where cudaMalloc may block or
synchronize the device) or a plugin whose host framework owns all device
memory cannot hand the plain chain a workspace.  This entry point keeps the
intermediates in the library's own static device array instead.  These tests
call it through the C ABI and require results bit-identical to the
workspace entry point (the tolerance the plain-chain tests use), on two calls
in a row with different cells, so a call cannot depend on what the previous
one left in the shared array.  This file is collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SCRATCH_LIMIT = 1008


def _run(aeq, c, cuda, static):
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
    yeq = torch.full((c.nSC * c.nLayers * c.nSym,), float("nan"), dtype=torch.complex64, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq)
    arr = (aeq.CellDesc * 1)(d)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if static:
        st = aeq.lib().aerial_pusch_eq_plain_static(arr, 1, stream)
    else:
        nbytes = aeq.lib().aerial_pusch_eq_plain_workspace(arr, 1)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
        st = aeq.lib().aerial_pusch_eq_plain(arr, 1, ctypes.c_void_p(ws.data_ptr()), nbytes, stream)
    assert st == 0, aeq.lib().aerial_error_string(st)
    torch.cuda.synchronize()
    return llr.cpu().numpy(), yeq.cpu().numpy()


def test_static_scratch_matches_workspace_entry_on_two_calls(aeq, wl, cuda):
    first = wl.config_cell(2, seed=61)       # 100 MHz cell: ~8.5 MB of intermediates
    second = wl.config_cell(1, seed=62)      # smaller cell reusing the same array
    for c in (first, second):
        ref = _run(aeq, c, cuda, static=False)
        got = _run(aeq, c, cuda, static=True)
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])


def test_static_scratch_rejects_cells_beyond_its_size(aeq, wl, cuda):
    c = wl.make_cell(nPRB=273, nAnt=128, nLayers=16, nSym=11, qam=256, snr_db=30.0, seed=63)
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    llr = torch.zeros(c.llr_numel, dtype=torch.float32, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    arr = (aeq.CellDesc * 1)(d)
    assert aeq.lib().aerial_pusch_eq_plain_workspace(arr, 1) > 16 * 1024 * 1024
    st = aeq.lib().aerial_pusch_eq_plain_static(arr, 1, None)
    assert st == SCRATCH_LIMIT
    assert b"static scratch" in aeq.lib().aerial_error_string(st)
    torch.cuda.synchronize()
    assert float(llr.abs().max()) == 0.0      # nothing ran
