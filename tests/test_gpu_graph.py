"""The fused launch replayed as a CUDA graph: identical results to the direct
launch, and re-pointing the graph at new slot buffers (same shapes) gives the
new slot's results without re-instantiation."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _descs(aeq, cells, cuda):
    bufs, descs = [], []
    for c in cells:
        H, Y = c.H.to(cuda), c.Y.to(cuda)
        llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        bufs.append((H, Y, llr))
        descs.append(aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits))
    return bufs, descs


def test_graph_replay_equals_direct_launch_and_update(aeq, wl, cuda):
    cells_a = [wl.make_cell(4, 32, 4, 11, 16, 20.0, seed=71), wl.make_cell(2, 64, 8, 11, 256, 25.0, seed=72)]
    cells_b = [wl.make_cell(4, 32, 4, 11, 16, 20.0, seed=73), wl.make_cell(2, 64, 8, 11, 256, 25.0, seed=74)]
    ref_a, da = _descs(aeq, cells_a, cuda)
    aeq.pusch_eq_fused(da)
    ref_b, db = _descs(aeq, cells_b, cuda)
    aeq.pusch_eq_fused(db)
    torch.cuda.synchronize()

    got_a, ga = _descs(aeq, cells_a, cuda)
    got_b, gb = _descs(aeq, cells_b, cuda)
    with aeq.FusedGraph(ga) as g:
        g.launch()
        g.launch()                       # replay twice: idempotent
        g.update(gb)                     # new buffers, same shapes
        g.launch()
        torch.cuda.synchronize()
    for r, o in zip(ref_a, got_a):
        np.testing.assert_array_equal(o[2].cpu().numpy(), r[2].cpu().numpy())
    for r, o in zip(ref_b, got_b):
        np.testing.assert_array_equal(o[2].cpu().numpy(), r[2].cpu().numpy())


def test_graph_update_rejects_new_shapes(aeq, wl, cuda):
    _, d1 = _descs(aeq, [wl.make_cell(2, 32, 4, 11, 16, 20.0, seed=75)], cuda)
    _, d2 = _descs(aeq, [wl.make_cell(2, 32, 8, 11, 16, 20.0, seed=76)], cuda)
    g = aeq.FusedGraph(d1)
    try:
        with pytest.raises(aeq.AerialError):
            g.update(d2)
    finally:
        g.close()


def test_graph_of_exact_tile_launch(aeq, wl, cuda):
    """All cells with 8 layers: the graph node runs the exact 8-layer kernel."""
    cells_a = [wl.make_cell(3, 64, 8, 11, 256, 25.0, seed=81), wl.make_cell(2, 24, 8, 9, 16, 20.0, seed=82)]
    cells_b = [wl.make_cell(3, 64, 8, 11, 256, 25.0, seed=83), wl.make_cell(2, 24, 8, 9, 16, 20.0, seed=84)]
    ref_a, da = _descs(aeq, cells_a, cuda)
    aeq.pusch_eq_fused(da)
    ref_b, db = _descs(aeq, cells_b, cuda)
    aeq.pusch_eq_fused(db)
    torch.cuda.synchronize()
    got_a, ga = _descs(aeq, cells_a, cuda)
    got_b, gb = _descs(aeq, cells_b, cuda)
    with aeq.FusedGraph(ga) as g:
        g.launch()
        g.update(gb)
        g.launch()
        torch.cuda.synchronize()
    for r, o in zip(ref_a + ref_b, got_a + got_b):
        np.testing.assert_array_equal(o[2].cpu().numpy(), r[2].cpu().numpy())


def test_fused_launch_captures_into_a_cuda_graph(aeq, wl, cuda):
    """aerial_pusch_eq_fused issues nothing but its kernel launch once the
    kernel is loaded, so stream capture records it; the replayed graph gives
    the direct launch's results."""
    cells = [wl.make_cell(2, 64, 8, 11, 256, 25.0, seed=91), wl.make_cell(3, 32, 4, 11, 16, 20.0, seed=92)]
    ref, dr = _descs(aeq, cells, cuda)
    t = aeq.make_tuning("fp16")
    aeq.pusch_eq_fused(dr, t)               # first call: loads the kernel and sets its limits
    torch.cuda.synchronize()
    got, dg = _descs(aeq, cells, cuda)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        aeq.pusch_eq_fused(dg, t)
    for o in got:
        o[2].fill_(float("nan"))
    graph.replay()
    torch.cuda.synchronize()
    for r, o in zip(ref, got):
        np.testing.assert_array_equal(o[2].cpu().numpy(), r[2].cpu().numpy())
    del graph
