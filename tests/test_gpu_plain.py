"""GPU parity of the plain FP32 chain: every stage through the C ABI must be
bit-identical to the oracle's FP32 restatement of the reference's scalar
kernels (same inputs, same operation order)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _d(x, dev):
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


SHAPES = [  # (nPRB, nAnt, nLayers, nSym)
    (2, 32, 4, 11),
    (3, 64, 8, 11),
    (1, 16, 2, 7),
    (1, 8, 1, 1),
    (2, 33, 3, 14),
    (1, 128, 16, 11),
    (1, 256, 16, 16),
    (2, 7, 5, 9),
]


@pytest.mark.parametrize("shape", SHAPES)
def test_gram_bit_exact(aeq, wl, orc, cuda, shape):
    nPRB, A, L, S = shape
    c = wl.make_cell(nPRB, A, L, S, 16, 20.0, seed=1)
    G = torch.empty(c.nSC, L, L, dtype=torch.complex64, device=cuda)
    aeq.gram(c.H.to(cuda), c.sigma2, G, c.nSC, A, L)
    torch.cuda.synchronize()
    ref = orc.gram(c.H.numpy(), c.sigma2, c.nSC, A, L)
    np.testing.assert_array_equal(G.cpu().numpy().reshape(-1), ref)


@pytest.mark.parametrize("shape", SHAPES)
def test_mmse_coef_bit_exact(aeq, wl, orc, cuda, shape):
    nPRB, A, L, S = shape
    c = wl.make_cell(nPRB, A, L, S, 16, 20.0, seed=2)
    G = orc.gram(c.H.numpy(), c.sigma2, c.nSC, A, L)
    Cd = torch.empty(c.nSC, L, A, dtype=torch.complex64, device=cuda)
    nId = torch.empty(c.nSC, L, dtype=torch.float32, device=cuda)
    aeq.mmse_coef(_d(G, cuda), c.H.to(cuda), Cd, nId, c.nSC, A, L)
    torch.cuda.synchronize()
    Cr, nIr = orc.mmse_coef(G, c.H.numpy(), c.nSC, A, L)
    np.testing.assert_array_equal(Cd.cpu().numpy().reshape(-1), Cr)
    np.testing.assert_array_equal(nId.cpu().numpy().reshape(-1), nIr)


@pytest.mark.parametrize("shape", SHAPES)
def test_coef_apply_bit_exact(aeq, orc, cuda, shape):
    nPRB, A, L, S = shape
    nSC = 12 * nPRB
    v = orc.ref_uniform(42, nSC * L * A * 2 + nSC * S * A * 2, 1.0)
    C = v[: nSC * L * A * 2].view(np.complex64)
    Y = v[nSC * L * A * 2:].view(np.complex64)
    O = torch.empty(nSC * L * S, dtype=torch.complex64, device=cuda)
    aeq.coef_apply(_d(C, cuda), _d(Y, cuda), O, nSC, S, L, A)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(O.cpu().numpy(), orc.coef_apply_v1(C, Y, nSC, S, L, A))


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_llr_f16_bit_exact(aeq, orc, cuda, n):
    N = 139392
    soft, ni = orc.ref_llr_inputs(42, N)
    out = torch.empty(N * 2 * n, dtype=torch.int16, device=cuda)
    aeq.llr(_d(soft.view(np.int16), cuda), _d(ni, cuda), out, N, n)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), orc.llr_f16io(soft, ni, n))


@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("spn", [1, 11])
def test_llr_f32_bit_exact(aeq, orc, cuda, n, spn):
    N = 1584 * 11
    rng = np.random.default_rng(n)
    soft = (rng.standard_normal(2 * N) * 0.7).astype(np.float32)
    ni = (10 ** rng.uniform(0, 3, N // spn + 1)).astype(np.float32)
    out = torch.empty(N * 2 * n, dtype=torch.float32, device=cuda)
    aeq.llr_f32(_d(soft, cuda), _d(ni, cuda), out, N, n, spn)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), orc.llr_f32(soft.view(np.complex64), ni, n, spn))


@pytest.mark.parametrize("cfg", [1, 2])
def test_plain_chain_bit_exact(aeq, wl, orc, cuda, cfg):
    """The whole plain chain (gram -> mmse_coef -> coef_apply -> llr_f32) equals
    the oracle's FP32 chain bit for bit."""
    c = wl.config_cell(cfg, seed=7)
    H, Y = c.H.to(cuda), c.Y.to(cuda)
    llr = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
    yeq = torch.empty(c.nSC * c.nLayers * c.nSym, dtype=torch.complex64, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, Y_eq=yeq)
    ws = torch.empty(aeq.pusch_eq_plain_workspace([d]), dtype=torch.uint8, device=cuda)
    aeq.pusch_eq_plain([d], ws)
    torch.cuda.synchronize()
    y32, _, l32 = orc.chain_f32(c.H.numpy(), c.Y.numpy(), c.sigma2, c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    np.testing.assert_array_equal(yeq.cpu().numpy(), y32)
    np.testing.assert_array_equal(llr.cpu().numpy(), l32)
