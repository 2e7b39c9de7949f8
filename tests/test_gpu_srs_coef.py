"""GPU parity of the SRS filter multiply and the tensor-core coef_apply."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import cosine, evm_db

pytestmark = pytest.mark.gpu


def _d(x, dev):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


# K a multiple of 4 runs the tcgen05 kernel (rows of 16-byte multiples for TMA), the others the mma.sync kernel.
SRS_CFGS = [(24, 4, 8), (24, 2, 8), (12, 4, 12), (12, 2, 12), (8, 1, 4), (10, 2, 5), (6, 3, 3),
            (48, 4, 8), (32, 16, 4), (44, 5, 4)]   # two K atoms; six 192-column tiles, the last partial; 48 max


@pytest.mark.parametrize("K,P,F,nBlk,nAnt", [c + (66, 64) for c in SRS_CFGS] +
                         [(24, 4, 8, 5, 33), (44, 5, 4, 3, 7), (32, 16, 4, 2, 100)])   # rows not in 32s: clipped
def test_srs_filter_vs_fp64(aeq, orc, cuda, K, P, F, nBlk, nAnt):
    s, w, f = orc.ref_srs_inputs(42, nBlk * nAnt * K, K * K, P * F)
    out = torch.empty(nBlk * nAnt * K * P * 2, dtype=torch.int16, device=cuda)
    aeq.srs_filter(out, _d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda),
                   nAnt, nBlk, K, P, F)
    torch.cuda.synchronize()
    got16 = out.cpu().numpy().view(np.uint16)
    got = np.empty(got16.size, np.float32)
    orc.lib().orc_f16_to_f32(got16, got, got.size)
    ref = orc.srs_f64(s, w, f, nAnt, nBlk, K, P, F)
    g = got.view(np.complex64).astype(np.complex128)
    # FP32 sums rounded once to FP16: error <= half an FP16 ulp of each component
    tol = np.maximum(np.abs(ref.real), np.abs(ref.imag)) * 2.0 ** -11 + 2.0 ** -24
    assert np.all(np.abs(g.real - ref.real) <= tol + 1e-6 * np.abs(ref).max())
    assert np.all(np.abs(g.imag - ref.imag) <= tol + 1e-6 * np.abs(ref).max())
    # and close to the reference's FP16-arithmetic V1 (its own check is cosine, :328)
    v1 = orc.srs_v1_f16(s, w, f, nAnt, nBlk, K, P, F)
    v1f = np.empty(v1.size, np.float32)
    orc.lib().orc_f16_to_f32(v1, v1f, v1f.size)
    assert cosine(v1f.view(np.complex64), g) > 0.9999


def test_srs_many_tiles_per_cta_both_layouts(aeq, orc, cuda):
    """1000 SRS blocks x 64 antennas: each CTA of the tcgen05 kernel walks several M tiles (operand stages and
    TMEM accumulators reused across phases), for the FP16 H_est layout and the channel layout, twice."""
    K, P, F, nBlk, nAnt = 24, 4, 8, 1000, 64
    s, w, f = orc.ref_srs_inputs(21, nBlk * nAnt * K, K * K, P * F)
    args = (_d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda))
    ref = orc.srs_f64(s, w, f, nAnt, nBlk, K, P, F)
    est = torch.empty(nBlk * nAnt * K * P * 2, dtype=torch.int16, device=cuda)
    H = torch.empty(nBlk * K, nAnt, P, dtype=torch.complex64, device=cuda)
    for rep in range(2):
        est.fill_(0)
        H.fill_(0)
        aeq.srs_filter(est, *args, nAnt, nBlk, K, P, F)
        aeq.srs_to_channel(H, *args, nAnt, nBlk, K, P, F)
        torch.cuda.synchronize()
        got16 = est.cpu().numpy().view(np.uint16)
        got = np.empty(got16.size, np.float32)
        orc.lib().orc_f16_to_f32(got16, got, got.size)
        g = got.view(np.complex64).astype(np.complex128)
        tol = np.maximum(np.abs(ref.real), np.abs(ref.imag)) * 2.0 ** -11 + 2.0 ** -24
        assert np.all(np.abs(g.real - ref.real) <= tol + 1e-6 * np.abs(ref).max())
        assert np.all(np.abs(g.imag - ref.imag) <= tol + 1e-6 * np.abs(ref).max())
        ch = ref.reshape(nBlk, nAnt, K, P).transpose(0, 2, 1, 3).reshape(nBlk * K, nAnt, P)
        assert evm_db(H.cpu().numpy(), ch) < -120
    assert aeq.kernel_timeouts() == 0


@pytest.mark.parametrize("K,P,F", [(24, 4, 8), (10, 2, 5)])
def test_srs_to_channel_layout(aeq, orc, cuda, K, P, F):
    nBlk, nAnt = 66, 64
    s, w, f = orc.ref_srs_inputs(43, nBlk * nAnt * K, K * K, P * F)
    H = torch.empty(nBlk * K, nAnt, P, dtype=torch.complex64, device=cuda)
    aeq.srs_to_channel(H, _d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda),
                       nAnt, nBlk, K, P, F)
    torch.cuda.synchronize()
    ref = orc.srs_f64(s, w, f, nAnt, nBlk, K, P, F).reshape(nBlk, nAnt, K, P)
    ref = ref.transpose(0, 2, 1, 3).reshape(nBlk * K, nAnt, P)   # [sc][ant][layer]
    assert evm_db(H.cpu().numpy(), ref) < -120


@pytest.mark.parametrize("K,P,F,S,nBlk,nAnt", [(12, 4, 4, 4, 9, 48), (12, 8, 2, 4, 6, 64), (24, 4, 8, 2, 9, 48),
                                                (24, 2, 8, 4, 5, 64), (48, 4, 8, 2, 4, 64), (12, 2, 4, 1, 9, 48)])
def test_srs_to_channel_avg_vs_fp64(aeq, orc, cuda, K, P, F, S, nBlk, nAnt):
    """The channel averaged over S SRS symbols against the FP64 average of the
    per-symbol estimates.  S = 1 is srs_to_channel, bit for bit."""
    syms = [orc.ref_srs_inputs(50 + q, nBlk * nAnt * K, K * K, P * F) for q in range(S)]
    w, f = syms[0][1], syms[0][2]
    SRS = _d(np.concatenate([x[0] for x in syms]).view(np.int16), cuda)
    Wd, Fd = _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda)
    H = torch.full((nBlk * K, nAnt, P), float("nan"), dtype=torch.complex64, device=cuda)
    aeq.srs_to_channel_avg(H, SRS, S, Wd, Fd, nAnt, nBlk, K, P, F)
    torch.cuda.synchronize()
    ref = np.mean([orc.srs_f64(x[0], w, f, nAnt, nBlk, K, P, F) for x in syms], axis=0)
    ref = ref.reshape(nBlk, nAnt, K, P).transpose(0, 2, 1, 3).reshape(nBlk * K, nAnt, P)
    assert evm_db(H.cpu().numpy(), ref) < -120
    if S == 1:
        H1 = torch.empty_like(H)
        aeq.srs_to_channel(H1, SRS, Wd, Fd, nAnt, nBlk, K, P, F)
        torch.cuda.synchronize()
        assert torch.equal(H, H1)


def test_srs_to_channel_avg_envelope(aeq, orc, cuda):
    """Symbol counts other than 1, 2, 4 are invalid; shapes the tcgen05
    kernel cannot average (taps not a multiple of 4, or 4 symbols of more than
    32 taps) are unsupported, with nothing launched."""
    K, P, F, nBlk, nAnt = 10, 2, 5, 4, 32
    s, w, f = orc.ref_srs_inputs(60, 4 * nBlk * nAnt * 48, 48 * 48, 4 * 8)
    SRS, Wd, Fd = (_d(x.view(np.int16), cuda) for x in (s, w, f))
    H = torch.empty(nBlk * 48, nAnt, 4, dtype=torch.complex64, device=cuda)
    for S in (0, 3, 8):
        with pytest.raises(aeq.AerialError) as e:
            aeq.srs_to_channel_avg(H, SRS, S, Wd, Fd, nAnt, nBlk, 12, 4, 8)
        assert e.value.status == 1001
    with pytest.raises(aeq.AerialError) as e:
        aeq.srs_to_channel_avg(H, SRS, 2, Wd, Fd, nAnt, nBlk, K, P, F)
    assert e.value.status == 1002
    with pytest.raises(aeq.AerialError) as e:
        aeq.srs_to_channel_avg(H, SRS, 4, Wd, Fd, nAnt, nBlk, 48, 4, 8)
    assert e.value.status == 1002


# DMRS interpolation filter: (nPilot, nOut, ports, OCC length, antennas).  96 pilots x 4 ports over 64
# antennas is the [64 x 96] x [96 x 4] product of the reference's README.md:200.
# Pilot counts that are multiples of 4 (up to 96) run the tcgen05 kernel, the others the mma.sync kernel.
CHEST_CFGS = [(96, 96, 4, 4, 64), (48, 96, 2, 2, 64), (96, 48, 4, 2, 33), (24, 12, 1, 1, 16), (56, 40, 3, 5, 48),
              (64, 64, 2, 2, 64), (32, 20, 3, 3, 40), (45, 30, 2, 3, 40), (90, 90, 4, 2, 64), (20, 24, 4, 4, 64),
              (32, 30, 4, 2, 32), (48, 45, 4, 2, 34)]   # 4 ports, even antenna counts, ragged outputs


@pytest.mark.parametrize("nPilot,nOut,P,F,nAnt", CHEST_CFGS)
def test_chest_interp_vs_fp64(aeq, orc, cuda, nPilot, nOut, P, F, nAnt):
    nBlk = 7
    s, w, f = orc.ref_srs_inputs(11, nBlk * nAnt * nPilot, nOut * nPilot, P * F)
    H = torch.empty(nBlk * nOut, nAnt, P, dtype=torch.complex64, device=cuda)
    aeq.chest_interp(H, _d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda),
                     nAnt, nBlk, nPilot, nOut, P, F)
    torch.cuda.synchronize()
    ref = orc.chest_f64(s, w, f, nAnt, nBlk, nPilot, nOut, P, F).reshape(nBlk * nOut, nAnt, P)
    # taps split into two FP16 parts, FP32 accumulation: the error of an FP32 sum
    assert evm_db(H.cpu().numpy(), ref) < -120


@pytest.mark.parametrize("nPilot,nOut,P,F,nAnt", CHEST_CFGS)
@pytest.mark.parametrize("offset", [0, 1])
def test_chest_interp_h_equals_complex64_rounded(aeq, orc, cuda, nPilot, nOut, P, F, nAnt, offset):
    """The complex-half channel is the complex64 channel rounded once to half,
    bit for bit: the same FP32 sums on both kernels (tcgen05 and mma.sync),
    at a 16-byte aligned and at a 4-byte aligned (offset one complex) start."""
    nBlk = 7
    s, w, f = orc.ref_srs_inputs(13, nBlk * nAnt * nPilot, nOut * nPilot, P * F)
    args = (_d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda))
    H32 = torch.empty(nBlk * nOut, nAnt, P, dtype=torch.complex64, device=cuda)
    aeq.chest_interp(H32, *args, nAnt, nBlk, nPilot, nOut, P, F)
    n = nBlk * nOut * nAnt * P
    buf = torch.full((n + offset, 2), float("nan"), dtype=torch.float16, device=cuda)
    H16 = buf[offset:]
    aeq.chest_interp_h(H16, *args, nAnt, nBlk, nPilot, nOut, P, F)
    torch.cuda.synchronize()
    assert torch.equal(H16, torch.view_as_real(H32).reshape(n, 2).to(torch.float16))
    if offset:
        assert torch.isnan(buf[0]).all()                                 # nothing written before the start


def test_chest_interp_h_feeds_fp16_io_cell(aeq, wl, orc, cuda):
    """The FP16 channel straight from the pilots into an FP16 I/O cell (4
    layers = 4 ports, 64 antennas, 33 blocks x 96 subcarriers = 264 PRB): the
    LLRs equal those of the same cell built from the complex64 channel rounded
    to half."""
    nPilot, nOut, P, F, nAnt, nBlk = 96, 96, 4, 2, 64, 33
    s, w, f = orc.ref_srs_inputs(14, nBlk * nAnt * nPilot, nOut * nPilot, P * F)
    args = (_d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda))
    nSC = nBlk * nOut
    H16 = torch.empty(nSC * nAnt * P, 2, dtype=torch.float16, device=cuda)
    H32 = torch.empty(nSC, nAnt, P, dtype=torch.complex64, device=cuda)
    aeq.chest_interp_h(H16, *args, nAnt, nBlk, nPilot, nOut, P, F)
    aeq.chest_interp(H32, *args, nAnt, nBlk, nPilot, nOut, P, F)
    c = wl.make_cell(nSC // 12, nAnt, P, 11, 64, 25.0, seed=15)
    Y16 = torch.view_as_real(c.Y).to(torch.float16).contiguous().to(cuda)
    outs = []
    for H in (H16, torch.view_as_real(H32).reshape(-1, 2).to(torch.float16).contiguous()):
        llr = torch.full((c.llr_numel,), float("nan"), dtype=torch.float16, device=cuda)
        d = aeq.cell_desc(H, Y16, llr, c.sigma2, c.nPRB, nAnt, P, 11, c.nPamBits, fmt=aeq.FMT_CF16)
        aeq.pusch_eq_fused([d], aeq.make_tuning("fp16"))
        outs.append(llr)
    torch.cuda.synchronize()
    assert torch.isfinite(outs[0].float()).all()
    assert torch.equal(outs[0], outs[1])


def test_chest_interp_many_tiles_per_cta(aeq, orc, cuda):
    """200 blocks x 64 antennas: every CTA of the tcgen05 kernel walks several M tiles, so both operand stages
    and both TMEM accumulators are reused across phases."""
    nPilot, nOut, P, F, nAnt, nBlk = 96, 96, 4, 2, 64, 200
    s, w, f = orc.ref_srs_inputs(12, nBlk * nAnt * nPilot, nOut * nPilot, P * F)
    H = torch.empty(nBlk * nOut, nAnt, P, dtype=torch.complex64, device=cuda)
    args = (_d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda))
    aeq.chest_interp(H, *args, nAnt, nBlk, nPilot, nOut, P, F)
    torch.cuda.synchronize()
    first = H.clone()
    ref = orc.chest_f64(s, w, f, nAnt, nBlk, nPilot, nOut, P, F).reshape(nBlk * nOut, nAnt, P)
    assert evm_db(H.cpu().numpy(), ref) < -120
    aeq.chest_interp(H, *args, nAnt, nBlk, nPilot, nOut, P, F)        # deterministic across calls
    torch.cuda.synchronize()
    assert torch.equal(H, first)


def test_chest_interp_and_srs_to_channel_on_offset_channel_pointers(aeq, orc, cuda):
    """A channel array that starts one complex into an allocation (8-byte aligned only) takes the per-element
    stores: same values as the aligned launch, and the element before the array is left alone."""
    for nPilot, K in ((96, None), (None, 24)):
        P, F, nAnt, nBlk = 4, 2, 64, 5
        kin = nPilot or K
        nOut = nPilot or K
        s, w, f = orc.ref_srs_inputs(13, nBlk * nAnt * kin, nOut * kin, P * F)
        args = (_d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda))
        n = nBlk * nOut * nAnt * P
        base = torch.full((n + 1,), 7 + 7j, dtype=torch.complex64, device=cuda)
        ref = torch.empty(n, dtype=torch.complex64, device=cuda)
        if nPilot:
            aeq.chest_interp(base[1:], *args, nAnt, nBlk, nPilot, nOut, P, F)
            aeq.chest_interp(ref, *args, nAnt, nBlk, nPilot, nOut, P, F)
        else:
            aeq.srs_to_channel(base[1:], *args, nAnt, nBlk, K, P, F)
            aeq.srs_to_channel(ref, *args, nAnt, nBlk, K, P, F)
        torch.cuda.synchronize()
        assert torch.equal(base[1:], ref)
        assert base[0].item() == 7 + 7j


def test_tcgen05_kernel_waits_never_gave_up(aeq, orc, cuda):
    """After the filter launches of this module (tcgen05 kernel included), no bounded wait ran out."""
    nPilot, nOut, P, F, nAnt, nBlk = 96, 96, 4, 2, 64, 40
    s, w, f = orc.ref_srs_inputs(14, nBlk * nAnt * nPilot, nOut * nPilot, P * F)
    H = torch.empty(nBlk * nOut, nAnt, P, dtype=torch.complex64, device=cuda)
    aeq.chest_interp(H, _d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda),
                     nAnt, nBlk, nPilot, nOut, P, F)
    torch.cuda.synchronize()
    assert aeq.kernel_timeouts() == 0


def test_chest_interp_square_filter_equals_srs_to_channel(aeq, orc, cuda):
    K, P, F, nBlk, nAnt = 24, 4, 8, 66, 64
    s, w, f = orc.ref_srs_inputs(43, nBlk * nAnt * K, K * K, P * F)
    args = (_d(s.view(np.int16), cuda), _d(w.view(np.int16), cuda), _d(f.view(np.int16), cuda))
    H1 = torch.empty(nBlk * K, nAnt, P, dtype=torch.complex64, device=cuda)
    H2 = torch.empty_like(H1)
    aeq.srs_to_channel(H1, *args, nAnt, nBlk, K, P, F)
    aeq.chest_interp(H2, *args, nAnt, nBlk, K, K, P, F)
    torch.cuda.synchronize()
    assert torch.equal(H1, H2)


@pytest.mark.parametrize("shape", [(1584, 11, 8, 64), (288, 11, 4, 32), (48, 14, 16, 128), (12, 3, 5, 33)])
def test_coef_apply_tc_vs_v2_model(aeq, orc, cuda, shape):
    nSC, S, L, A = shape
    v = orc.ref_uniform(7, nSC * L * A * 2 + nSC * S * A * 2, 1.4)
    C = v[: nSC * L * A * 2].view(np.complex64)
    Y = v[nSC * L * A * 2:].view(np.complex64)
    O = torch.empty(nSC * L * S, dtype=torch.complex64, device=cuda)
    aeq.coef_apply_tc(_d(C, cuda), _d(Y, cuda), O, nSC, S, L, A)
    torch.cuda.synchronize()
    got = O.cpu().numpy()
    v2 = orc.coef_apply_v2_model(C, Y, nSC, S, L, A)
    v1 = orc.coef_apply_v1(C, Y, nSC, S, L, A)
    assert evm_db(got, v2) < -110          # same FP16 operands, only accumulation order differs
    assert evm_db(got, v1) < -65           # the reference's V2-vs-V1 bar is -70.3 dB at 64 ant
