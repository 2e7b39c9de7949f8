"""The allocation-free plain chain, aerial_pusch_eq_plain_static.

Callers such as a real-time slot loop (where cudaMalloc may block or
synchronize the device) or a plugin whose host framework owns all device
memory cannot hand the plain chain a workspace.  This entry point keeps the
intermediates in the library's own static device array instead.  These tests
call it through the C ABI and require results bit-identical to the
workspace entry point (the tolerance the plain-chain tests use), on two calls
in a row with different cells, so a call cannot depend on what the previous
one left in the shared array.  A caller with no allocator is also the one
most likely to pass no Y_eq buffer, so the equalized symbols then live in the
static array too; and a batch of two cells of different shapes reuses the
array within one call.  This file is collected last.
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


def _run_batch(aeq, cells, cuda, static):
    descs, llrs, keep = [], [], []
    for c in cells:
        H, Y = c.H.to(cuda), c.Y.to(cuda)
        llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        keep += [H, Y]
        llrs.append(llr)
        descs.append(aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits))
    arr = (aeq.CellDesc * len(descs))(*descs)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if static:
        st = aeq.lib().aerial_pusch_eq_plain_static(arr, len(descs), stream)
    else:
        nbytes = aeq.lib().aerial_pusch_eq_plain_workspace(arr, len(descs))
        ws = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
        st = aeq.lib().aerial_pusch_eq_plain(arr, len(descs), ctypes.c_void_p(ws.data_ptr()), nbytes, stream)
    assert st == 0, aeq.lib().aerial_error_string(st)
    torch.cuda.synchronize()
    return [l.cpu().numpy() for l in llrs]


def test_static_scratch_without_y_eq_two_cell_batch(aeq, wl, cuda):
    # two shapes in one call (the second smaller, so it reads scratch regions
    # the first one wrote), no Y_eq buffer, twice in a row
    cells = [wl.make_cell(nPRB=51, nAnt=64, nLayers=8, nSym=11, qam=256, snr_db=25.0, seed=64),
             wl.make_cell(nPRB=24, nAnt=16, nLayers=2, nSym=7, qam=4, snr_db=12.0, seed=65)]
    ref = _run_batch(aeq, cells, cuda, static=False)
    for _ in range(2):
        got = _run_batch(aeq, cells, cuda, static=True)
        for g, r in zip(got, ref):
            assert np.all(np.isfinite(g))
            np.testing.assert_array_equal(g, r)


def test_static_scratch_malformed_cell_is_an_argument_error(aeq, wl, cuda):
    # a negative layer count must not wrap into a huge size (SCRATCH_LIMIT)
    c = wl.config_cell(1, seed=66)
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    llr = torch.zeros(c.llr_numel, dtype=torch.float32, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, -4, c.nSym, c.nPamBits)
    st = aeq.lib().aerial_pusch_eq_plain_static((aeq.CellDesc * 1)(d), 1, None)
    assert st == 1001                        # AERIAL_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert float(llr.abs().max()) == 0.0


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
