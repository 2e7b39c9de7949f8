"""GPU tests of the dynamic group walk of the fused kernels.

A launch hands out groups of subcarriers from a counter slot in device memory
(one slot per stream, one per graph); the walk only decides which warp
equalizes which group, never the arithmetic.  Every launch must therefore
equal the static round-robin walk (AERIAL_STATIC_WALK=1) bit for bit: alone,
repeated on one stream (the counter resets itself at the end of each launch),
with fewer groups than warps, on several streams at once, as graph replays
and inside a stream-captured CUDA graph.  Output buffers are filled with NaN
before each launch, so a group that a launch skipped shows up."""
from __future__ import annotations

import contextlib
import os

import pytest
import torch

from test_gpu_fp16_io import half_pairs

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def walk(static: bool):
    old = os.environ.get("AERIAL_STATIC_WALK")
    os.environ["AERIAL_STATIC_WALK"] = "1" if static else "0"
    try:
        yield
    finally:
        if old is None:
            del os.environ["AERIAL_STATIC_WALK"]
        else:
            os.environ["AERIAL_STATIC_WALK"] = old


# (nPRB, nAnt, nLayers, nSym, qam) per cell; each batch selects one kernel family
BATCHES = {
    "unrolled_8_layers": [(6, 64, 8, 11, 256), (4, 64, 8, 11, 256), (5, 64, 8, 9, 64)],
    "unrolled_16_layers": [(3, 128, 16, 11, 256), (2, 128, 16, 11, 256)],
    "mixed_tiles": [(5, 64, 4, 11, 64), (2, 32, 8, 11, 64), (4, 64, 2, 11, 256), (3, 16, 4, 11, 16),
                    (6, 64, 8, 11, 4), (1, 16, 8, 11, 4), (2, 48, 3, 7, 16)],
    "half_uniform": [(6, 64, 8, 11, 256), (4, 64, 8, 11, 256)],
    "half_mixed": [(5, 64, 4, 11, 64), (2, 32, 8, 11, 64), (4, 64, 2, 11, 256), (3, 16, 4, 11, 16)],
}


class Batch:
    """Device inputs of a batch and one set of output buffers."""

    def __init__(self, aeq, wl, cuda, kind, seed=0, shapes=None):
        half = kind.startswith("half")
        self.aeq, self.cuda, self.half = aeq, cuda, half
        self.inputs = []
        for i, (p, a, l, s, q) in enumerate(shapes if shapes is not None else BATCHES[kind]):
            c = wl.make_cell(p, a, l, s, q, 25.0, seed=900 + 31 * i + seed)
            if half:
                self.inputs.append((c, half_pairs(c.H).to(cuda), half_pairs(c.Y).to(cuda)))
            else:
                self.inputs.append((c, c.H.to(cuda), c.Y.to(cuda)))

    def outputs(self):
        outs, descs = [], []
        for c, H, Y in self.inputs:
            n = c.nSC * c.nLayers * c.nSym
            if self.half:
                llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16, device=self.cuda)
                yeq = torch.full((n, 2), float("nan"), dtype=torch.float16, device=self.cuda)
                fmt = self.aeq.FMT_CF16
            else:
                llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=self.cuda)
                yeq = torch.full((n,), float("nan"), dtype=torch.complex64, device=self.cuda)
                fmt = self.aeq.FMT_CF32
            descs.append(self.aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                            Y_eq=yeq, fmt=fmt))
            outs.append((llr, yeq))
        return descs, outs


def same(a, b):
    return all(torch.equal(x, y) for (lx, yx), (ly, yy) in zip(a, b) for x, y in ((lx, ly), (yx, yy)))


def reference(aeq, batch, prec):
    descs, outs = batch.outputs()
    with walk(static=True):
        aeq.pusch_eq_fused(descs, aeq.make_tuning(prec))
    torch.cuda.synchronize()
    for llr, _ in outs:
        assert not torch.isnan(llr.float()).any()
    return outs


@pytest.mark.parametrize("kind,prec", [("unrolled_8_layers", "fp16"), ("unrolled_8_layers", "bf16x3"),
                                       ("unrolled_16_layers", "bf16x3"), ("unrolled_16_layers", "fp16"),
                                       ("mixed_tiles", "fp16"), ("mixed_tiles", "bf16"),
                                       ("half_uniform", "fp16"), ("half_mixed", "fp16")])
def test_dynamic_walk_equals_static_walk_repeatedly(aeq, wl, cuda, kind, prec):
    batch = Batch(aeq, wl, cuda, kind)
    ref = reference(aeq, batch, prec)
    with walk(static=False):
        for _ in range(6):                     # the same stream and slot, launch after launch
            descs, outs = batch.outputs()
            aeq.pusch_eq_fused(descs, aeq.make_tuning(prec))
            torch.cuda.synchronize()
            assert same(outs, ref)


@pytest.mark.parametrize("shape", [(1, 64, 8, 11, 256), (1, 16, 2, 3, 4), (2, 32, 4, 11, 16)])
def test_fewer_groups_than_warps(aeq, wl, cuda, shape):
    """Most warps have no group: they still count themselves done, so the
    counter resets and the next launch starts clean."""
    batch = Batch(aeq, wl, cuda, "tiny", shapes=[shape])
    ref = reference(aeq, batch, "fp16")
    with walk(static=False):
        for _ in range(4):
            descs, outs = batch.outputs()
            aeq.pusch_eq_fused(descs, aeq.make_tuning("fp16"))
            torch.cuda.synchronize()
            assert same(outs, ref)


def test_concurrent_streams_and_graph_replays(aeq, wl, cuda):
    """Launches on three streams and graph replays on a fourth, queued with no
    synchronization in between: each stream and the graph hold their own
    slots, so every launch completes every group."""
    kinds = ["unrolled_8_layers", "mixed_tiles", "unrolled_16_layers"]
    batches = [Batch(aeq, wl, cuda, k, seed=7) for k in kinds]
    refs = [reference(aeq, b, "fp16") for b in batches]
    gbatch = Batch(aeq, wl, cuda, "unrolled_8_layers", seed=11)
    gref = reference(aeq, gbatch, "fp16")
    streams = [torch.cuda.Stream() for _ in range(4)]
    results = []
    with walk(static=False):
        gdescs, gouts = gbatch.outputs()
        with aeq.FusedGraph(gdescs, aeq.make_tuning("fp16")) as graph:
            torch.cuda.synchronize()
            for _ in range(8):
                for b, st in zip(batches, streams):
                    descs, outs = b.outputs()
                    torch.cuda.synchronize()   # the NaN fill is done before the launches queue up
                    with torch.cuda.stream(st):
                        aeq.pusch_eq_fused(descs, aeq.make_tuning("fp16"))
                    results.append((outs, refs[batches.index(b)]))
                with torch.cuda.stream(streams[3]):
                    for llr, yeq in gouts:             # ordered before the replay on its stream
                        llr.fill_(float("nan"))
                        yeq.fill_(float("nan"))
                    graph.launch()
            torch.cuda.synchronize()
            assert same(gouts, gref)
    for outs, ref in results:
        assert same(outs, ref)


def test_captured_launch_takes_the_static_walk(aeq, wl, cuda):
    """A launch recorded by stream capture may be replayed anywhere: it must
    not hold a slot, and its replays equal the static walk."""
    batch = Batch(aeq, wl, cuda, "unrolled_8_layers", seed=3)
    ref = reference(aeq, batch, "fp16")
    descs, outs = batch.outputs()
    with walk(static=False):
        aeq.pusch_eq_fused(descs, aeq.make_tuning("fp16"))     # loads the kernel outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            aeq.pusch_eq_fused(descs, aeq.make_tuning("fp16"))
        for _ in range(3):
            for llr, yeq in outs:
                llr.fill_(float("nan"))
                yeq.fill_(float("nan"))
            g.replay()
            torch.cuda.synchronize()
            assert same(outs, ref)


def test_many_graphs_leave_slots_for_streams(aeq, wl, cuda):
    """Graphs reserve at most 48 of the 64 counters: with 56 graphs alive,
    the extra graphs and a direct launch on a new stream still complete
    every group."""
    batch = Batch(aeq, wl, cuda, "unrolled_8_layers", seed=5)
    ref = reference(aeq, batch, "fp16")
    with walk(static=False):
        graphs, outs = [], []
        try:
            for _ in range(56):
                descs, o = batch.outputs()
                graphs.append(aeq.FusedGraph(descs, aeq.make_tuning("fp16")))
                outs.append(o)
            for g in graphs[::5] + graphs[-3:]:
                g.launch()
            descs, direct = batch.outputs()
            st = torch.cuda.Stream()
            torch.cuda.synchronize()
            with torch.cuda.stream(st):
                aeq.pusch_eq_fused(descs, aeq.make_tuning("fp16"))
            torch.cuda.synchronize()
            for k, o in enumerate(outs):
                if k % 5 == 0 or k >= 53:
                    assert same(o, ref)
            assert same(direct, ref)
        finally:
            for g in graphs:
                g.close()
