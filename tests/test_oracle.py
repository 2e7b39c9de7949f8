"""CPU tests: the oracle pinned against the reference's golden vectors and
recorded results, plus internal consistency of the oracle's FP32 and FP64
chains.  No GPU needed."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, cosine, evm_db, max_rel_err


def _ka():
    return json.load(open(os.path.join(GOLDEN, "known_answers.json")))


def test_pam_lut_matches_reference_literals(orc):
    """Computed D_i == the reference's c_LUT (src/llr/aerial_llr_v3.cu:42-48) in float32."""
    ref = json.load(open(os.path.join(GOLDEN, "pam_lut.json")))
    lut = np.asarray(ref["c_LUT"], np.float64)
    for n in (1, 2, 3, 4):
        d32, d64 = orc.pam_lut(n)
        off = ref["offsets"][n - 1]
        np.testing.assert_array_equal(d32, lut[off:off + n].astype(np.float32))
        np.testing.assert_allclose(d64, lut[off:off + n], rtol=2e-15)


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_llr_fp64_oracle_bit_exact_vs_reference_cpu_ref(orc, n):
    """The FP64 demapper equals the reference's cpu_ref bit for bit (after its float cast)."""
    g = np.load(os.path.join(GOLDEN, "llr_cpu_ref.npz"))
    soft = np.empty(g["soft_u16"].size, np.float32)
    orc.lib().orc_f16_to_f32(g["soft_u16"], soft, soft.size)
    mine = orc.llr_f64(soft.view(np.complex64), g["noise_inv"], n).astype(np.float32)
    np.testing.assert_array_equal(mine, g[f"llr_n{n}"])


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_llr_fp32_oracle_vs_reference_cpu_ref(orc, n):
    """FP32 restatement of llr_v1_baseline vs the FP64 cpu_ref: the reference's own
    correctness metric (cosine, maxAE; src/llr/aerial_llr_v3.cu:247-256)."""
    g = np.load(os.path.join(GOLDEN, "llr_cpu_ref.npz"))
    soft = np.empty(g["soft_u16"].size, np.float32)
    orc.lib().orc_f16_to_f32(g["soft_u16"], soft, soft.size)
    mine = orc.llr_f32(soft.view(np.complex64), g["noise_inv"], n)
    ref = g[f"llr_n{n}"].astype(np.float64)
    assert np.abs(mine - ref).max() <= 1e-6 * np.abs(ref).max() + 1e-6
    a, b = mine.astype(np.float64), ref
    assert np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.9999999
    # hard decisions identical
    assert np.array_equal(mine < 0, ref < 0)


def test_llr_f16io_is_f32_then_round(orc):
    g = np.load(os.path.join(GOLDEN, "llr_cpu_ref.npz"))
    soft = np.empty(g["soft_u16"].size, np.float32)
    orc.lib().orc_f16_to_f32(g["soft_u16"], soft, soft.size)
    o16 = orc.llr_f16io(g["soft_u16"], g["noise_inv"], 4)
    o32 = orc.llr_f32(soft.view(np.complex64), g["noise_inv"], 4)
    np.testing.assert_array_equal(o16, orc.f32_to_f16(o32))


def _coef_case(orc, ka):
    n = ka["nSC"] * ka["nLayers"] * ka["nAnt"] * 2
    m = ka["nSC"] * ka["nSym"] * ka["nAnt"] * 2
    v = orc.ref_uniform(ka["seed"], n + m, ka["scale"])
    C = v[:n].view(np.complex64)
    Y = v[n:].view(np.complex64)
    args = (ka["nSC"], ka["nSym"], ka["nLayers"], ka["nAnt"])
    return orc.coef_apply_v1(C, Y, *args), orc.coef_apply_v2_model(C, Y, *args)


def test_known_answer_coef_rigor(orc):
    """Reproduces results/coef_rigor_results.txt:5 (EVM V2 vs V1 on srand(7) data)."""
    ka = _ka()["coef_rigor"]
    v1, v2 = _coef_case(orc, ka)
    e = 10 ** (evm_db(v2, v1) / 20)
    assert round(e * 100, 4) == pytest.approx(ka["evm_pct"], abs=1e-4)
    assert round(20 * np.log10(e), 1) == ka["evm_db"]
    # max relative error is decided by one near-zero output; the tensor core's
    # internal accumulation order moves it in the 4th digit
    assert max_rel_err(v2, v1) * 100 == pytest.approx(ka["max_rel_err_pct"], abs=2e-3)


def test_known_answer_coef_wmma(orc):
    """Reproduces the README's V2-vs-V1 cosine and max-abs error on srand(42) data."""
    ka = _ka()["coef_wmma"]
    v1, v2 = _coef_case(orc, ka)
    assert round(cosine(v1, v2), 8) == pytest.approx(ka["cosine"], abs=1e-8)
    assert round(float(np.abs(v1.astype(np.complex128) - v2).max()), 6) == pytest.approx(ka["max_abs_err"], abs=1e-6)


def test_gram_restatement_consistent(orc, wl):
    """gram (M := H^H, sigma2 = 0) equals gram_scalar's restatement with an explicit M."""
    c = wl.make_cell(2, 16, 4, 3, 16, 20.0, seed=3)
    H = c.H.numpy()
    M = np.ascontiguousarray(np.conj(H).transpose(0, 2, 1))
    np.testing.assert_array_equal(orc.gram(H, 0.0, c.nSC, 16, 4), orc.gram_ref(M, H, c.nSC, 4, 16))


@pytest.mark.parametrize("cfg", [1, 2])
def test_fp32_chain_vs_fp64_model(orc, wl, cfg):
    c = wl.config_cell(cfg, seed=5)
    H, Y = c.H.numpy(), c.Y.numpy()
    args = (c.nSC, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    y32, n32, l32 = orc.chain_f32(H, Y, c.sigma2, *args)
    y64, n64, l64 = orc.chain_f64(H, Y, c.sigma2, *args)
    assert evm_db(y32, y64) < -100
    np.testing.assert_allclose(n32, n64, rtol=1e-3)
    assert np.array_equal(l32 < 0, l64 < 0) or np.mean((l32 < 0) != (l64 < 0)) < 1e-6
    # the MMSE estimate tracks the transmitted symbols at the configured SNR
    e_tx = evm_db(y64, c.x.numpy())
    assert e_tx < -c.snr_db + 3


def test_mmse_coef_unbiased(orc, wl):
    c = wl.make_cell(1, 32, 4, 2, 16, 15.0, seed=9)
    H = c.H.numpy()
    G = orc.gram(H, c.sigma2, c.nSC, 32, 4)
    C, nI = orc.mmse_coef(G, H, c.nSC, 32, 4)
    CH = np.einsum("sla,sak->slk", C.reshape(c.nSC, 4, 32).astype(np.complex128), H.astype(np.complex128))
    np.testing.assert_allclose(np.einsum("sll->sl", CH).real, 1.0, atol=1e-5)
    assert np.all(nI > 0)


@pytest.mark.parametrize("K,P,F", [(24, 4, 8), (12, 2, 12)])
def test_srs_f16_restatement_close_to_fp64(orc, K, P, F):
    nBlk, nAnt = 3, 16
    s, w, f = orc.ref_srs_inputs(42, nBlk * nAnt * K, K * K, P * F)
    o16 = orc.srs_v1_f16(s, w, f, nAnt, nBlk, K, P, F)
    o64 = orc.srs_f64(s, w, f, nAnt, nBlk, K, P, F)
    v16 = np.empty(o16.size, np.float32)
    orc.lib().orc_f16_to_f32(o16, v16, v16.size)
    assert cosine(v16.view(np.complex64), o64) > 0.9999


def test_chest_f64_square_filter_is_the_srs_filter(orc):
    """The interpolation model with nOut == nPilot is the SRS filter multiply
    (srs_filter_v1_scalar's sum, src/srs/srs_wmma_bench.cu:57-90) in the
    channel layout [blk*K + k_out][ant][port]."""
    K, P, F, nBlk, nAnt = 24, 4, 8, 3, 16
    s, w, f = orc.ref_srs_inputs(5, nBlk * nAnt * K, K * K, P * F)
    srs = orc.srs_f64(s, w, f, nAnt, nBlk, K, P, F).reshape(nBlk, nAnt, K, P).transpose(0, 2, 1, 3)
    ch = orc.chest_f64(s, w, f, nAnt, nBlk, K, K, P, F).reshape(nBlk, K, nAnt, P)
    np.testing.assert_array_equal(ch, srs)


# ---------------------------------------------------------------------------
# The oracle against the reference's OWN kernels run on a B200 (compiled
# unchanged for sm_100a): SHA-256 of the full-size outputs, regenerated here
# from the same seeds (tests/golden/make_golden.py --gpu wrote ref_gpu.json).
# ---------------------------------------------------------------------------
import hashlib  # noqa: E402
import sys  # noqa: E402

sys.path.insert(0, GOLDEN)
import make_golden as MG  # noqa: E402


def _ref_gpu():
    return json.load(open(os.path.join(GOLDEN, "ref_gpu.json")))["outputs"]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_coef_apply_v1_oracle_matches_reference_kernel_digest(orc):
    r = _ref_gpu()["coef_v1"]
    C, Y = MG.coef_inputs(r["recipe"]["seed"], r["recipe"]["nSC"], r["recipe"]["nSym"])
    o = orc.coef_apply_v1(C.view(np.complex64), Y.view(np.complex64), r["recipe"]["nSC"], r["recipe"]["nSym"], 8, 64)
    assert _sha(o.view(np.float32)) == r["sha256"]
    sl = np.load(os.path.join(GOLDEN, "ref_gpu_slices.npz"))["coef_v1"]
    np.testing.assert_array_equal(o.view(np.float32)[: sl.size], sl)


def test_coef_apply_v2_model_vs_reference_kernel(orc):
    """The FP16 model of coef_apply_v2_wmma agrees with the kernel's run to -120 dB."""
    r = _ref_gpu()["coef_v2"]
    sl = np.load(os.path.join(GOLDEN, "ref_gpu_slices.npz"))["coef_v2"]
    nsc = sl.size // (8 * 11 * 2)
    C, Y = MG.coef_inputs(r["recipe"]["seed"], r["recipe"]["nSC"], r["recipe"]["nSym"])
    o = orc.coef_apply_v2_model(C.view(np.complex64)[: nsc * 8 * 64], Y.view(np.complex64)[: nsc * 11 * 64],
                                nsc, 11, 8, 64)
    assert evm_db(o, sl.view(np.complex64)[: o.size]) < -120


def test_gram_oracle_matches_reference_kernel_digest(orc):
    r = _ref_gpu()["gram"]
    H, M = MG.gram_inputs(r["recipe"]["seed"], r["recipe"]["nSC"])
    assert _sha(orc.gram_ref(M, H, r["recipe"]["nSC"], 8, 64).view(np.float32)) == r["sha256"]
    # and the Hermitian entry point (M = H^H implied, sigma2 = 0) is the same computation
    assert _sha(orc.gram(H, 0.0, r["recipe"]["nSC"], 64, 8).view(np.float32)) == r["sha256"]


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_llr_oracle_matches_reference_kernel_digest(orc, n):
    r = _ref_gpu()[f"llr_v1_n{n}"]
    soft, ni = orc.ref_llr_inputs(r["recipe"]["seed"], r["recipe"]["N"])
    assert _sha(orc.llr_f16io(soft, ni, n)) == r["sha256"]


@pytest.mark.parametrize("K,P,F", MG.SRS_CFGS)
def test_srs_oracle_matches_reference_kernel_digest(orc, K, P, F):
    r = _ref_gpu()[f"srs_v1_K{K}_P{P}_F{F}"]
    rc = r["recipe"]
    s, w, f = MG.srs_inputs(K, P, F, rc["nBlk"], rc["nAnt"], rc["seed"])
    assert _sha(orc.srs_v1_f16(s, w, f, rc["nAnt"], rc["nBlk"], K, P, F)) == r["sha256"]
