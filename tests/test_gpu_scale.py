"""FP16 operands at any input scale.

FP16 has 11 significant bits only between 2^-14 and 65504.  A receiver's H
and Y_rx carry whatever path-loss or ADC scale the front end gives them, so
the complex64 path normalizes each cell's operands by an exact power of two
taken from its noise variance before rounding them to FP16
(aerial_fp16_operand_scale; include/aerial_eq.h states the window).  These
tests scale H and Y_rx of configuration 1 and 2 cells by 2^k and sigma2 by
2^2k and require:
  - EVM of Y_eq against the FP64 model within 1 dB of the unit-scale run;
  - LLRs equal to the unit-scale run's, bit for bit where the normalized
    operands coincide, else within the LLR tolerance 2e-3 * max|LLR64|.
The exact unrolled kernel, the generic mixed-tile kernel (masked layers and
tail antennas), the 16-layer tile and a CUDA graph whose update crosses the
window all take the same path.  A complex-half cell stored raw at 2^-16
shows what the normalization prevents.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import evm_db

pytestmark = pytest.mark.gpu

LLR_TOL = 2e-3


def scaled(wl, c, k):
    """A copy of cell c with H, Y_rx scaled by 2^k and sigma2 by 2^2k (exact)."""
    f = float(2.0 ** k)
    return wl.Cell(**{**c.__dict__, "H": c.H * f, "Y": c.Y * f, "sigma2": c.sigma2 * f * f})


def run(aeq, cells, cuda, precision="fp16"):
    descs, outs = [], []
    for c in cells:
        H, Y = c.H.to(cuda), c.Y.to(cuda)
        llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        yeq = torch.full((c.nSC * c.nLayers * c.nSym,), float("nan"), dtype=torch.complex64, device=cuda)
        descs.append(aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq))
        outs.append((H, Y, llr, yeq))
    aeq.pusch_eq_fused(descs, aeq.make_tuning(precision))
    torch.cuda.synchronize()
    return [(o[2].cpu().numpy(), o[3].cpu().numpy()) for o in outs]


def same_operands(aeq, c, k):
    """True when the scaled cell's normalized FP16 operands equal the unit cell's."""
    s0 = aeq.fp16_operand_scale(c.sigma2)
    sk = aeq.fp16_operand_scale(c.sigma2 * 4.0 ** k)
    return sk * 2.0 ** k == s0


def compare(aeq, orc, c, k, base, got):
    y64, _, l64 = orc.chain_f64(c.H.numpy(), c.Y.numpy(), c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    (l0, y0), (lk, yk) = base, got
    assert np.all(np.isfinite(lk)) and np.all(np.isfinite(yk))
    e0, ek = evm_db(y0, y64), evm_db(yk, y64)
    assert ek <= e0 + 1.0, f"2^{k}: EVM {ek:.1f} dB against {e0:.1f} dB at unit scale"
    if same_operands(aeq, c, k):
        np.testing.assert_array_equal(lk, l0)
        np.testing.assert_array_equal(yk, y0)
    else:
        assert np.abs(lk.astype(np.float64) - l0).max() <= LLR_TOL * np.abs(l64).max()
    return ek


@pytest.mark.parametrize("cfg", [1, 2])
@pytest.mark.parametrize("k", [-12, -6, 6, 10, -40, 30])
def test_fp16_operands_any_scale(aeq, wl, orc, cuda, cfg, k):
    c = wl.config_cell(cfg, seed=71)
    base = run(aeq, [c], cuda)[0]
    got = run(aeq, [scaled(wl, c, k)], cuda)[0]
    compare(aeq, orc, c, k, base, got)


def test_fp16_scaled_mixed_batch(aeq, wl, orc, cuda):
    """Generic kernel: uneven cells (3 layers and 33 antennas take the masked
    path, 16 layers the two-tile one), each at its own scale in one launch;
    every cell equals its unit-scale self run in the same kind of batch."""
    shapes = [(4, 33, 3, 11, 64, 18.0), (2, 64, 16, 11, 256, 28.0), (3, 16, 2, 7, 4, 12.0), (2, 32, 8, 14, 16, 22.0)]
    cells = [wl.make_cell(p, a, l, s, q, snr, seed=80 + i) for i, (p, a, l, s, q, snr) in enumerate(shapes)]
    ks = [-14, 9, 0, -5]
    base = run(aeq, cells, cuda)
    got = run(aeq, [scaled(wl, c, k) for c, k in zip(cells, ks)], cuda)
    for c, k, b, g in zip(cells, ks, base, got):
        compare(aeq, orc, c, k, b, g)


def test_fp16_scaled_cfg3_tile(aeq, wl, orc, cuda):
    """The 16-layer, 128-antenna tile (configuration 3 shape, fewer PRBs)."""
    c = wl.make_cell(24, 128, 16, 11, 256, 30.0, channel="corr", seed=90)
    base = run(aeq, [c], cuda)[0]
    got = run(aeq, [scaled(wl, c, -11)], cuda)[0]
    compare(aeq, orc, c, -11, base, got)


def test_fp16_graph_update_across_window(aeq, wl, orc, cuda):
    """A graph made for unit-scale cells, updated with cells whose noise level
    needs the scaled kernel (and back), replays the direct launch's results."""
    c = wl.config_cell(2, seed=72)
    cs = scaled(wl, c, -12)
    ref_unit = run(aeq, [c], cuda)[0]
    ref_scaled = run(aeq, [cs], cuda)[0]
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    Hs, Ys = cs.H.to(cuda), cs.Y.to(cuda)
    llr = torch.zeros(c.llr_numel, dtype=torch.float32, device=cuda)
    yeq = torch.zeros(c.nSC * c.nLayers * c.nSym, dtype=torch.complex64, device=cuda)

    def desc(h, y, s2):
        return (aeq.CellDesc * 1)(aeq.cell_desc(h, y, llr, s2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits,
                                                Y_eq=yeq))
    g = ctypes.c_void_p()
    t = aeq.make_tuning("fp16")
    L = aeq.lib()
    assert L.aerial_eq_graph_create(desc(H, Y, c.sigma2), 1, ctypes.byref(t), ctypes.byref(g)) == 0
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        for h, y, s2, ref in ((Hs, Ys, cs.sigma2, ref_scaled), (H, Y, c.sigma2, ref_unit)):
            llr.zero_()
            assert L.aerial_eq_graph_update(g, desc(h, y, s2), 1) == 0
            assert L.aerial_eq_graph_launch(g, stream) == 0
            torch.cuda.synchronize()
            np.testing.assert_array_equal(llr.cpu().numpy(), ref[0])
            np.testing.assert_array_equal(yeq.cpu().numpy(), ref[1])
    finally:
        assert L.aerial_eq_graph_destroy(g) == 0


def _run_cf16(aeq, c, cuda, storage_scale, sigma2):
    """An FP16 I/O cell stored as complex half at H * storage_scale."""
    h = torch.view_as_real(c.H * storage_scale).to(torch.float16).contiguous().to(cuda)
    y = torch.view_as_real(c.Y * storage_scale).to(torch.float16).contiguous().to(cuda)
    llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16, device=cuda)
    yeq = torch.full((c.nSC * c.nLayers * c.nSym, 2), float("nan"), dtype=torch.float16, device=cuda)
    d = aeq.cell_desc(h, y, llr, sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq,
                      fmt=aeq.FMT_CF16)
    aeq.pusch_eq_fused([d], aeq.make_tuning("fp16"))
    torch.cuda.synchronize()
    yv = yeq.float().cpu().numpy()
    return llr.float().cpu().numpy(), yv[:, 0] + 1j * yv[:, 1]


def test_fp16_io_storage_scale(aeq, wl, orc, cuda):
    """Complex-half cells are read as stored.  Stored at the scale
    aerial_fp16_operand_scale gives, a cell whose front end delivered 2^-16
    of the unit-scale samples reproduces the unit-scale run bit for bit;
    stored raw it loses most of its mantissa (what the complex64 path's
    normalization prevents)."""
    c = wl.config_cell(2, seed=73)
    y64, _, _ = orc.chain_f64(c.H.numpy(), c.Y.numpy(), c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    k = -16
    s2k = c.sigma2 * 4.0 ** k
    s = aeq.fp16_operand_scale(s2k)
    base = _run_cf16(aeq, c, cuda, 1.0, c.sigma2)
    good = _run_cf16(aeq, c, cuda, 2.0 ** k * s, s2k * s * s)
    raw = _run_cf16(aeq, c, cuda, 2.0 ** k, s2k)
    assert s * 2.0 ** k == aeq.fp16_operand_scale(c.sigma2)
    np.testing.assert_array_equal(good[0], base[0])
    e_base, e_raw = evm_db(base[1], y64), evm_db(raw[1], y64)
    assert e_raw > e_base + 20.0, (e_raw, e_base)
    # the complex64 path at the same 2^-16 input scale keeps the unit-scale EVM
    l32, y32 = run(aeq, [scaled(wl, c, k)], cuda)[0]
    assert evm_db(y32, y64) <= evm_db(run(aeq, [c], cuda)[0][1], y64) + 1.0
