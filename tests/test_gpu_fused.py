"""GPU parity of the fused chain (tensor-core Gram / matched filter, FP32
Cholesky, LLR epilogue) against the FP64 model and the plain FP32 chain.

Tolerances (stated per precision):
  FP16 / BF16x3 / FP16x3 operands: EVM of Y_eq vs FP64 <= -45 dB (the target
  bar); observed margins are tighter and asserted where stated.
  LLR: max |LLR - LLR64| <= 2e-3 * max|LLR64| (relative to the LLR scale).
  Hard decisions: on full configuration 1 (20 dB) and 2 (25 dB) slots the
  number of sign flips against FP64 is asserted exactly per path, and every
  flip must sit where |LLR64| is below that path's bound (relative to
  max |LLR64|: FP16 1e-4, BF16x3 and FP16x3 1e-6, plain chain 1e-6)
  (test_hard_decisions_vs_fp64).  At 20 dB no path flips a bit.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import evm_db

pytestmark = pytest.mark.gpu


def run_fused(aeq, cells, cuda, precision="fp16", want_yeq=True, tuning=None):
    descs, outs = [], []
    for c in cells:
        H, Y = c.H.to(cuda), c.Y.to(cuda)
        llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        yeq = torch.full((c.nSC * c.nLayers * c.nSym,), float("nan"), dtype=torch.complex64, device=cuda) \
            if want_yeq else None
        descs.append(aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq))
        outs.append((H, Y, llr, yeq))
    t = tuning if tuning is not None else aeq.make_tuning(precision)
    aeq.pusch_eq_fused(descs, t)
    torch.cuda.synchronize()
    return [(o[2].cpu().numpy(), o[3].cpu().numpy() if o[3] is not None else None) for o in outs]


def oracle64(orc, c):
    return orc.chain_f64(c.H.numpy(), c.Y.numpy(), c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)


def check_against_fp64(orc, c, llr, yeq, evm_max=-45.0):
    y64, n64, l64 = oracle64(orc, c)
    assert np.all(np.isfinite(llr)), "unwritten LLRs"
    e = evm_db(yeq, y64)
    assert e <= evm_max, f"EVM {e:.1f} dB > {evm_max} dB"
    scale = np.abs(l64).max()
    err = np.abs(llr.astype(np.float64) - l64)
    assert err.max() <= 2e-3 * scale, (err.max(), scale)
    # a sign flip can only sit within the LLR error of zero
    flips = (llr < 0) != (l64 < 0)
    assert np.all(np.abs(l64[flips]) <= 2e-3 * scale)
    return e


@pytest.mark.parametrize("cfg,prec,evm_max", [(1, "fp16", -55.0), (2, "fp16", -55.0), (1, "bf16x3", -80.0),
                                               (2, "bf16x3", -80.0), (2, "bf16", -40.0), (1, "fp16x3", -100.0),
                                               (2, "fp16x3", -100.0)])
def test_fused_configs_vs_fp64(aeq, wl, orc, cuda, cfg, prec, evm_max):
    c = wl.config_cell(cfg, seed=11)
    (llr, yeq), = run_fused(aeq, [c], cuda, prec)
    if prec == "bf16":  # 8-bit mantissa operands: report, bound loosely
        y64, _, _ = oracle64(orc, c)
        assert evm_db(yeq, y64) <= evm_max
        return
    check_against_fp64(orc, c, llr, yeq, evm_max)


@pytest.mark.parametrize("prec,evm_max", [("bf16x3", -60.0), ("fp16", -45.0), ("fp16x3", -100.0)])
def test_fused_cfg3_correlated_channel(aeq, wl, orc, cuda, prec, evm_max):
    """273 PRB x 128 ant x 16 layers, rho = 0.7 correlated, SNR 30 dB."""
    c = wl.config_cell(3, seed=13)
    (llr, yeq), = run_fused(aeq, [c], cuda, prec)
    check_against_fp64(orc, c, llr, yeq, evm_max)


# Hard decisions against FP64 on full slots: (config, path) -> exact number
# of sign flips for the slot of seed 40 + config, and the path's bound on
# |LLR64| at a flip (relative to max |LLR64|: the path's LLR error).  The
# plain chain is the reference's scalar FP32 method (aerial_pusch_eq_plain).
# At 20 dB (configuration 1) every path's hard decisions equal FP64's.  At
# 25 dB the config 2 slot holds bits whose |LLR64| is a few 1e-7 of the
# maximum: below every reduced-precision path's error, so they flip; the
# plain chain's flips on the config 3 slot (tests of bench.py) show that even
# FP32 cannot decide bits at 1e-8.
FLIPS = {(1, "fp16"): 0, (2, "fp16"): 64, (1, "bf16x3"): 0, (2, "bf16x3"): 2,
         (1, "fp16x3"): 0, (2, "fp16x3"): 1, (1, "plain"): 0, (2, "plain"): 0}
FLIP_BOUND = {"fp16": 1e-4, "bf16x3": 1e-6, "fp16x3": 1e-6, "plain": 1e-6}


@pytest.mark.parametrize("cfg,path", sorted(FLIPS))
def test_hard_decisions_vs_fp64(aeq, wl, orc, cuda, cfg, path):
    c = wl.config_cell(cfg, seed=40 + cfg)
    if path == "plain":
        H, Y = c.H.to(cuda), c.Y.to(cuda)
        llr_t = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        d = aeq.cell_desc(H, Y, llr_t, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
        ws = torch.empty(aeq.pusch_eq_plain_workspace([d]), dtype=torch.uint8, device=cuda)
        aeq.pusch_eq_plain([d], ws)
        torch.cuda.synchronize()
        llr = llr_t.cpu().numpy()
    else:
        (llr, _), = run_fused(aeq, [c], cuda, path, want_yeq=False)
    _, _, l64 = oracle64(orc, c)
    assert np.all(np.isfinite(llr))
    flips = (llr < 0) != (l64 < 0)
    scale = np.abs(l64).max()
    assert int(flips.sum()) == FLIPS[(cfg, path)], f"{int(flips.sum())} flips of {flips.size}"
    assert np.all(np.abs(l64[flips]) <= FLIP_BOUND[path] * scale)


EDGE = [  # (nPRB, nAnt, nLayers, nSym, qam)
    (1, 8, 1, 1, 4),
    (1, 16, 2, 7, 16),
    (1, 32, 3, 8, 64),
    (2, 64, 4, 9, 256),
    (1, 33, 5, 14, 16),
    (1, 7, 6, 16, 4),
    (3, 128, 8, 11, 64),
    (1, 64, 12, 11, 256),
    (1, 256, 16, 16, 16),
    (5, 24, 7, 3, 256),
]


@pytest.mark.parametrize("shape", EDGE)
def test_fused_edge_shapes(aeq, wl, orc, cuda, shape):
    nPRB, A, L, S, q = shape
    c = wl.make_cell(nPRB, A, L, S, q, 25.0, seed=17)
    (llr, yeq), = run_fused(aeq, [c], cuda, "bf16x3")
    check_against_fp64(orc, c, llr, yeq, -60.0)


def test_fused_vs_plain_chain(aeq, wl, orc, cuda):
    """The fused FP16 path and the plain FP32 chain agree at the EVM bar."""
    c = wl.config_cell(2, seed=19)
    (llr, yeq), = run_fused(aeq, [c], cuda, "fp16")
    y32, _, l32 = orc.chain_f32(c.H.numpy(), c.Y.numpy(), c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    assert evm_db(yeq, y32) <= -50.0


def test_multicell_same_alone_and_in_mix(aeq, wl, cuda):
    """Per-cell results are bit-identical whether a cell runs alone or inside
    a 16-cell uneven batch (one persistent launch)."""
    cells = wl.multicell(16, seed=23)
    mixed = run_fused(aeq, cells, cuda, "fp16")
    for i in (0, 5, 15):
        alone = run_fused(aeq, [cells[i]], cuda, "fp16")[0]
        np.testing.assert_array_equal(alone[0], mixed[i][0])
        np.testing.assert_array_equal(alone[1], mixed[i][1])


@pytest.mark.parametrize("cfg,n", [(2, 3), (2, 8), (1, 5)])
def test_prb_range_split_equals_whole_cell(aeq, wl, cuda, cfg, n):
    """A cell split into PRB ranges (the same buffers at offsets, fewer PRBs)
    gives the whole cell's LLRs and Y_eq bit for bit, whether the ranges run as
    cells of one launch or as separate launches on separate streams."""
    c = wl.config_cell(cfg, seed=61)
    whole = run_fused(aeq, [c], cuda, "fp16")[0]
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    per_llr, per_y = c.llr_numel // c.nSC, c.nLayers * c.nSym
    step = -(-c.nPRB // n)
    ranges = [(p0, min(step, c.nPRB - p0)) for p0 in range(0, c.nPRB, step)]

    def descs(llr, yeq):
        return [aeq.cell_desc(H[12 * p0:], Y[12 * p0:], llr[12 * p0 * per_llr:], c.sigma2, m, c.nAnt, c.nLayers,
                              c.nSym, c.nPamBits, Y_eq=yeq[12 * p0 * per_y:]) for p0, m in ranges]
    t = aeq.make_tuning("fp16")
    llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
    yeq = torch.full((c.nSC * per_y,), float("nan"), dtype=torch.complex64, device=cuda)
    aeq.pusch_eq_fused(descs(llr, yeq), t)
    llr2, yeq2 = torch.full_like(llr, float("nan")), torch.full_like(yeq, float("nan"))
    streams = [torch.cuda.Stream() for _ in ranges]
    for d, s in zip(descs(llr2, yeq2), streams):
        aeq.pusch_eq_fused([d], t, s)
    torch.cuda.synchronize()
    for l_, y_ in ((llr, yeq), (llr2, yeq2)):
        np.testing.assert_array_equal(l_.cpu().numpy(), whole[0])
        np.testing.assert_array_equal(y_.cpu().numpy(), whole[1])


@pytest.mark.parametrize("prec", ["fp16", "bf16x3"])
def test_group_cap_does_not_change_results(aeq, wl, cuda, prec):
    """The group cap (subcarriers a warp solves together, aerial_tuning.
    sc_per_group) and the launch shape only regroup the work: every cell's
    LLRs and Y_eq are bit-identical for caps 1, 4, 8 and 32 and for the
    autotuner's choice, in an uneven batch that includes 1-, 2- and 3-layer
    tiles (masked rows) and tail antennas."""
    cells = wl.multicell(16, seed=27) + [wl.make_cell(2, 33, 1, 7, 4, 15.0, seed=28),
                                         wl.make_cell(1, 20, 3, 13, 16, 22.0, seed=29)]
    ref = run_fused(aeq, cells, cuda, prec)
    for cap in (1, 4, 32):
        got = run_fused(aeq, cells, cuda, tuning=aeq.make_tuning(prec, sc_per_group=cap))
        for a, b in zip(ref, got):
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1], b[1])
    descs, keep = [], []
    for c in cells:
        H, Y = c.H.to(cuda), c.Y.to(cuda)
        l = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
        keep += [H, Y, l]
        descs.append(aeq.cell_desc(H, Y, l, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits))
    tuned, us = aeq.autotune(descs, prec)
    assert tuned.sc_per_group in (4, 8, 32) and us > 0
    got = run_fused(aeq, cells, cuda, tuning=tuned)
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(a[0], b[0])


def test_multicell_vs_fp64(aeq, wl, orc, cuda):
    cells = wl.multicell(16, seed=29)
    res = run_fused(aeq, cells, cuda, "fp16")
    for c, (llr, yeq) in zip(cells, res):
        check_against_fp64(orc, c, llr, yeq, -45.0)


def test_fused_without_yeq_and_launch_shapes(aeq, wl, cuda):
    c = wl.config_cell(1, seed=31)
    ref = run_fused(aeq, [c], cuda, "fp16")[0][0]
    for w, k in ((2, 4), (4, 1), (4, 2), (8, 1), (3, 3), (6, 2)):
        got = run_fused(aeq, [c], cuda, "fp16", want_yeq=False,
                        tuning=aeq.make_tuning("fp16", w, k))[0][0]
        np.testing.assert_array_equal(got, ref)


def test_autotune_returns_valid_shape(aeq, wl, cuda):
    c = wl.config_cell(2, seed=37)
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    llr = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    t, us = aeq.autotune([d], "fp16")
    assert t.warps_per_cta in (2, 3, 4, 6, 8) and t.ctas_per_sm >= 1 and us > 0


def test_fused_rejects_bad_cells(aeq, wl, cuda):
    c = wl.config_cell(1, seed=41)
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    llr = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, 17, c.nSym, c.nPamBits)
    with pytest.raises(aeq.AerialError):
        aeq.pusch_eq_fused([d])
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, 17, c.nPamBits)
    with pytest.raises(aeq.AerialError):
        aeq.pusch_eq_fused([d])


def test_multicell_mixed_layer_tiles(aeq, wl, orc, cuda):
    """Cells of every layer tile (1, 2, 4, 8, 16 and padded 3, 5, 12) in one
    launch: each matches FP64 and its own single-cell run bit for bit."""
    shapes = [(2, 16, 1, 11, 4), (1, 32, 2, 11, 16), (3, 24, 3, 9, 64), (1, 16, 4, 14, 256), (2, 64, 5, 11, 16),
              (1, 64, 8, 11, 256), (1, 128, 12, 11, 64), (1, 128, 16, 11, 256)]
    cells = [wl.make_cell(p, a, l, s, q, 25.0, seed=50 + k) for k, (p, a, l, s, q) in enumerate(shapes)]
    mixed = run_fused(aeq, cells, cuda, "bf16x3")
    for k, c in enumerate(cells):
        check_against_fp64(orc, c, mixed[k][0], mixed[k][1], -60.0)
        alone = run_fused(aeq, [c], cuda, "bf16x3")[0]
        np.testing.assert_array_equal(alone[0], mixed[k][0])


# Launches whose cells all have 8 layers run the exact 8-layer kernel: antenna
# counts that leave a partial last chunk, fewer antennas than one chunk (but
# at least as many as layers), and symbol counts from 1 to 16.
TMA_SHAPES = [  # (nPRB, nAnt, nLayers, nSym, qam)
    (1, 12, 8, 1, 4),
    (1, 14, 8, 8, 16),
    (2, 8, 8, 9, 64),
    (1, 24, 8, 14, 256),
    (3, 40, 8, 16, 16),
    (2, 64, 8, 11, 256),
    (1, 128, 8, 13, 64),
    (1, 256, 8, 5, 4),
]


@pytest.mark.parametrize("shape", TMA_SHAPES)
def test_fused_exact_8_layer_shapes(aeq, wl, orc, cuda, shape):
    nPRB, A, L, S, q = shape
    c = wl.make_cell(nPRB, A, L, S, q, 25.0, seed=91)
    (llr, yeq), = run_fused(aeq, [c], cuda, "bf16x3")
    check_against_fp64(orc, c, llr, yeq, -60.0)
    if A >= 16:
        (llr, yeq), = run_fused(aeq, [c], cuda, "fp16")
        check_against_fp64(orc, c, llr, yeq, -45.0)


def test_fused_exact_8_layer_mix_alone_and_in_mix(aeq, wl, orc, cuda):
    """Several 8-layer cells of different shapes in one exact-tile launch:
    each equals its own single-cell launch bit for bit and matches FP64."""
    cells = [wl.make_cell(p, a, 8, s, q, 25.0, seed=100 + k)
             for k, (p, a, _, s, q) in enumerate(TMA_SHAPES[2:])]
    mixed = run_fused(aeq, cells, cuda, "fp16")
    for k, c in enumerate(cells):
        alone = run_fused(aeq, [c], cuda, "fp16")[0]
        np.testing.assert_array_equal(alone[0], mixed[k][0])
        check_against_fp64(orc, c, mixed[k][0], mixed[k][1], -45.0)


@pytest.mark.parametrize("L", [2, 4, 8, 16])
@pytest.mark.parametrize("A", [32, 64, 128])
def test_fused_exact_antenna_kernels(aeq, wl, orc, cuda, L, A):
    """Launches whose cells share nLayers and nAnt in {32, 64, 128} run the
    kernel with the antenna chunks unrolled; adding a cell with another
    antenna count switches the launch to the runtime-chunk kernel.  Each cell's
    results are the same bit for bit in both, and match FP64."""
    cells = [wl.make_cell(2, A, L, 11, 256, 25.0, seed=200 + A + L),
             wl.make_cell(1, A, L, 5, 16, 20.0, seed=300 + A + L),
             wl.make_cell(1, A, L, 14, 64, 25.0, seed=400 + A + L)]
    other = wl.make_cell(1, 48, L, 7, 4, 15.0, seed=500 + A + L)
    exact = run_fused(aeq, cells, cuda, "bf16x3")
    mixed = run_fused(aeq, cells + [other], cuda, "bf16x3")
    for k, c in enumerate(cells):
        np.testing.assert_array_equal(exact[k][0], mixed[k][0])
        np.testing.assert_array_equal(exact[k][1], mixed[k][1])
        check_against_fp64(orc, c, exact[k][0], exact[k][1], -60.0)


def test_tuned_shape_that_does_not_fit_is_reduced(aeq, wl, cuda):
    """A shape tuned on a light batch (2 warps x 8 CTAs) applied to a 16-layer
    cell whose warps need far more shared memory runs with the CTAs per SM
    that fit, and gives the default shape's results."""
    c = wl.make_cell(1, 128, 16, 14, 256, 30.0, seed=61)
    ref = run_fused(aeq, [c], cuda, "fp16")[0]
    got = run_fused(aeq, [c], cuda, "fp16", tuning=aeq.make_tuning("fp16", 2, 8))[0]
    np.testing.assert_array_equal(got[0], ref[0])
