"""GPU tests of the FP16 I/O cell format (AERIAL_FMT_CF16): H, Y_rx and Y_eq
as complex half, LLRs as __half.

On inputs that are exactly representable in half precision the FP16 I/O
kernel and the complex64 layout with FP16 operands feed identical operands to
identical tensor-core tiles and the same FP32 epilogue, so the half outputs
must equal the complex64 path's outputs rounded to half, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from test_gpu_fused import check_against_fp64

pytestmark = pytest.mark.gpu


def half_pairs(z):
    """complex64 tensor -> contiguous float16 (re, im) pairs."""
    return torch.view_as_real(z).to(torch.float16).contiguous()


def run_pair(aeq, cells, cuda, want_yeq=True):
    """The same half-representable cells through both formats."""
    d32, d16, out32, out16 = [], [], [], []
    for c in cells:
        H16, Y16 = half_pairs(c.H).to(cuda), half_pairs(c.Y).to(cuda)
        H32 = torch.view_as_complex(H16.float()).contiguous()
        Y32 = torch.view_as_complex(Y16.float()).contiguous()
        l32 = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        l16 = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16, device=cuda)
        n = c.nSC * c.nLayers * c.nSym
        y32 = torch.full((n,), float("nan"), dtype=torch.complex64, device=cuda) if want_yeq else None
        y16 = torch.full((n, 2), float("nan"), dtype=torch.float16, device=cuda) if want_yeq else None
        d32.append(aeq.cell_desc(H32, Y32, l32, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=y32))
        d16.append(aeq.cell_desc(H16, Y16, l16, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=y16,
                                 fmt=aeq.FMT_CF16))
        out32.append((H32, Y32, l32, y32))
        out16.append((H16, Y16, l16, y16))
    t = aeq.make_tuning("fp16")
    aeq.pusch_eq_fused(d32, t)
    aeq.pusch_eq_fused(d16, t)
    torch.cuda.synchronize()
    return out32, out16


@pytest.mark.parametrize("L", [4, 8, 16])
@pytest.mark.parametrize("A", [32, 64, 128])
def test_fp16_io_equals_complex64_path_rounded(aeq, wl, cuda, L, A):
    cells = [wl.make_cell(2, A, L, 11, 256, 25.0, seed=600 + A + L),
             wl.make_cell(1, A, L, 5, 16, 20.0, seed=700 + A + L),
             wl.make_cell(3, A, L, 14, 64, 25.0, seed=800 + A + L)]
    out32, out16 = run_pair(aeq, cells, cuda)
    for (_, _, l32, y32), (_, _, l16, y16) in zip(out32, out16):
        assert torch.isfinite(l16.float()).all()
        assert torch.equal(l16, l32.to(torch.float16))
        assert torch.equal(y16, torch.view_as_real(y32).to(torch.float16))


def test_fp16_io_mixed_batch_equals_complex64_path_rounded(aeq, wl, cuda):
    """Mixed batches in FP16 I/O (the configuration 4 cells: 2-, 4- and
    8-layer tiles with 16, 32 and 64 antennas, plus 48- and 256-antenna and
    16-layer cells) take the mixed-batch FP16 I/O kernel; every cell equals
    the complex64 path's result rounded to half, bit for bit."""
    cells = wl.multicell(16, seed=77)
    cells += [wl.make_cell(2, 48, 2, 11, 64, 18.0, seed=78), wl.make_cell(1, 16, 16, 9, 256, 28.0, seed=79),
              wl.make_cell(1, 256, 4, 16, 4, 12.0, seed=80)]
    for batch in (cells[:16], cells[16:], cells):
        out32, out16 = run_pair(aeq, batch, cuda)
        for (_, _, l32, y32), (_, _, l16, y16) in zip(out32, out16):
            assert torch.isfinite(l16.float()).all()
            assert torch.equal(l16, l32.to(torch.float16))
            assert torch.equal(y16, torch.view_as_real(y32).to(torch.float16))


def test_fp16_io_mixed_batch_alone_and_in_mix(aeq, wl, cuda):
    """A half-format cell's results do not depend on the batch around it."""
    cells = wl.multicell(16, seed=81)
    _, mixed = run_pair(aeq, cells, cuda)
    for i in (0, 7, 15):
        _, alone = run_pair(aeq, [cells[i]], cuda)
        assert torch.equal(alone[0][2], mixed[i][2])
        assert torch.equal(alone[0][3], mixed[i][3])


def test_fp16_io_mixed_batch_host_pipeline_and_graph(aeq, wl, cuda):
    """A mixed half-format batch through aerial_pusch_eq_host (host buffers,
    sub-batches over three streams) and as a CUDA graph replay equals the
    resident direct launch, bit for bit."""
    cells = wl.multicell(16, seed=83)
    _, ref = run_pair(aeq, cells, cuda, want_yeq=False)
    hd, hl, keep = [], [], []
    for c, (H16, Y16, _, _) in zip(cells, ref):
        hH, hY = H16.cpu().pin_memory(), Y16.cpu().pin_memory()
        l = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16).pin_memory()
        keep += [hH, hY]
        hl.append(l)
        hd.append(aeq.host_cell_desc(hH, hY, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                     fmt=aeq.FMT_CF16))
    ws = torch.empty(aeq.pusch_eq_host_workspace(hd, 5), dtype=torch.uint8, device=cuda)
    aeq.pusch_eq_host(hd, ws, aeq.make_tuning("fp16"), 5)
    torch.cuda.synchronize()
    for l, (_, _, l16, _) in zip(hl, ref):
        assert torch.equal(l, l16.cpu())
    descs, outs = [], []
    for c, (H16, Y16, _, _) in zip(cells, ref):
        l16 = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16, device=cuda)
        outs.append(l16)
        descs.append(aeq.cell_desc(H16, Y16, l16, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                   fmt=aeq.FMT_CF16))
    with aeq.FusedGraph(descs, aeq.make_tuning("fp16")) as g:
        g.launch()
        torch.cuda.synchronize()
    for o, (_, _, l16, _) in zip(outs, ref):
        assert torch.equal(o, l16)


def test_fp16_io_vs_fp64(aeq, wl, orc, cuda):
    """The headline cell in FP16 I/O against the FP64 model of its own
    (half-rounded) inputs, at the FP16 bar."""
    c = wl.config_cell(2, seed=31)
    out32, out16 = run_pair(aeq, [c], cuda)
    H16, Y16, l16, y16 = out16[0]
    hc = type(c)(**{**c.__dict__, "H": torch.view_as_complex(H16.float()).cpu(),
                    "Y": torch.view_as_complex(Y16.float()).cpu()})
    llr = l16.float().cpu().numpy()
    yeq = torch.view_as_complex(y16.float()).cpu().numpy()
    check_against_fp64(orc, hc, llr, yeq, -45.0)


def test_fp16_io_host_pipeline(aeq, wl, cuda):
    """Host half buffers through aerial_pusch_eq_host equal the resident launch."""
    cells = [wl.make_cell(2, 64, 8, 11, 256, 25.0, seed=900 + k) for k in range(5)]
    _, out16 = run_pair(aeq, cells, cuda, want_yeq=False)
    hd, hl, keep = [], [], []
    for c, (H16, Y16, _, _) in zip(cells, out16):
        hH, hY = H16.cpu().pin_memory(), Y16.cpu().pin_memory()
        l = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16).pin_memory()
        keep += [hH, hY]
        hl.append(l)
        hd.append(aeq.host_cell_desc(hH, hY, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                     fmt=aeq.FMT_CF16))
    ws = torch.empty(aeq.pusch_eq_host_workspace(hd, 2), dtype=torch.uint8, device=cuda)
    aeq.pusch_eq_host(hd, ws, aeq.make_tuning("fp16"), 2)
    torch.cuda.synchronize()
    for l, (_, _, l16, _) in zip(hl, out16):
        assert torch.equal(l, l16.cpu())


def test_fp16_io_unsupported_cases(aeq, wl, cuda):
    def desc(c, fmt=1):
        H16, Y16 = half_pairs(c.H).to(cuda), half_pairs(c.Y).to(cuda)
        l16 = torch.empty(c.llr_numel, dtype=torch.float16, device=cuda)
        return (H16, Y16, l16), aeq.cell_desc(H16, Y16, l16, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                             fmt=fmt)
    k1, d_l3 = desc(wl.make_cell(1, 32, 3, 11, 16, 20.0, seed=1))          # 3 layers: not a full tile
    k2, d_a40 = desc(wl.make_cell(1, 40, 8, 11, 16, 20.0, seed=2))         # 40 antennas: not 16k
    k3, d_ok = desc(wl.make_cell(1, 64, 8, 11, 16, 20.0, seed=3))
    for d in (d_l3, d_a40):
        with pytest.raises(aeq.AerialError):
            aeq.pusch_eq_fused([d], aeq.make_tuning("fp16"))
        with pytest.raises(aeq.AerialError):                                # also inside a mixed batch
            aeq.pusch_eq_fused([d_ok, d], aeq.make_tuning("fp16"))
    with pytest.raises(aeq.AerialError):                                    # FP16 operands only
        aeq.pusch_eq_fused([d_ok], aeq.make_tuning("bf16x3"))
    c = wl.make_cell(1, 64, 8, 11, 16, 20.0, seed=4)
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    l = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
    d32 = aeq.cell_desc(H, Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    with pytest.raises(aeq.AerialError):                                    # one format per launch
        aeq.pusch_eq_fused([d32, d_ok], aeq.make_tuning("fp16"))
    ws = torch.empty(aeq.pusch_eq_plain_workspace([d_ok]), dtype=torch.uint8, device=cuda)
    with pytest.raises(aeq.AerialError):                                    # the FP32 chain reads complex64 only
        aeq.pusch_eq_plain([d_ok], ws)


def test_fp16_io_graph_replay_and_update(aeq, wl, cuda):
    """The FP16 I/O launch as a CUDA graph: replay equals the direct launch, and
    re-pointing it at another slot's half buffers gives that slot's results."""
    def descs(cells):
        keep, ds = [], []
        for c in cells:
            H16, Y16 = half_pairs(c.H).to(cuda), half_pairs(c.Y).to(cuda)
            l16 = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16, device=cuda)
            keep.append((H16, Y16, l16))
            ds.append(aeq.cell_desc(H16, Y16, l16, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                    fmt=aeq.FMT_CF16))
        return keep, ds
    ca = [wl.make_cell(2, 64, 8, 11, 256, 25.0, seed=950 + k) for k in range(3)]
    cb = [wl.make_cell(2, 64, 8, 11, 256, 25.0, seed=960 + k) for k in range(3)]
    ref_a, da = descs(ca)
    ref_b, db = descs(cb)
    aeq.pusch_eq_fused(da, aeq.make_tuning("fp16"))
    aeq.pusch_eq_fused(db, aeq.make_tuning("fp16"))
    got_a, ga = descs(ca)
    got_b, gb = descs(cb)
    with aeq.FusedGraph(ga, aeq.make_tuning("fp16")) as g:
        g.launch()
        g.update(gb)
        g.launch()
        torch.cuda.synchronize()
    for r, o in zip(ref_a + ref_b, got_a + got_b):
        assert torch.equal(o[2], r[2])
