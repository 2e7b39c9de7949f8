"""The reference's own kernels on this GPU, beside this library's equivalents.

    python tests/reference_on_b200.py            # needs a GPU and oracle/_ref/ (make -C oracle ref)

Measurement script, not a test (pytest does not collect it).  It lives with
the tests because it runs the checker libraries: the reference's .cu files
compiled unchanged for sm_100a into oracle/_ref/ by oracle/Makefile.

Shapes are the reference's own benchmark shapes:
  coef_apply      1584 subcarriers x 64 antennas x 8 layers x 11 symbols
                  (src/aerial_coef_wmma.cu:42-55, launches :400-407)
  gram_scalar     1584 subcarriers, 64 antennas, 8 layers (src/aerial_bottleneck.cu:174-179)
  llr             139,392 symbols, 256-QAM (src/llr/aerial_llr_v3.cu:258-307)
  srs filter      66 blocks x 64 antennas, K = 24, 4 ports, FOCC length 8 (src/srs/srs_wmma_bench.cu:347)
  chain           gram_scalar -> coef_apply_v2_wmma -> llr_v3 on one 1584-subcarrier cell, against
                  this library's fused launch of the same cell (Gram + MMSE solve + apply + LLR);
                  and the same over 64 cell-slots (101,376 subcarriers, inputs larger than L2)
Timing follows the reference's own method (src/aerial_coef_wmma.cu:443-462): CUDA events around each
launch on the default stream (the checker libraries' *_launch entry points do not synchronize, like this
library's calls), median of 50 after 10 warm-ups, the inputs left in place between launches (L2-warm:
every input here is smaller than the 126 MB L2).  Prints one JSON line.
"""
from __future__ import annotations

import ctypes
import importlib
import json
import os
import statistics
import sys

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
REFLIB = os.path.join(ROOT, "oracle", "_ref")
VP, CI = ctypes.c_void_p, ctypes.c_int


def ref(name):
    return ctypes.CDLL(os.path.join(REFLIB, f"libref_{name}.so"))


def timed(fn, warm=10, iters=50):
    """Median launch time in microseconds (events on the default stream around each call).  A short device
    sleep ahead of the first event keeps the GPU busy while the host enqueues the event and the launch, so the
    interval holds the kernel alone, not host-side call overhead."""
    s = torch.cuda.current_stream()
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda._sleep(200000)
        e0.record(s)
        fn()
        e1.record(s)
        torch.cuda.synchronize()
        out.append(1e3 * e0.elapsed_time(e1))
    return statistics.median(out)


def crand(shape, dev, scale=0.5):
    return torch.complex(torch.rand(shape, device=dev) - 0.5, torch.rand(shape, device=dev) - 0.5) * (2 * scale)


def main():
    aeq = importlib.import_module("aerial-mimo-tc-optimization_b200")
    wl = importlib.import_module("aerial-mimo-tc-optimization_b200.workload")
    dev = torch.device("cuda:0")
    torch.manual_seed(7)
    rows = {}
    nSC, S, L, A = 1584, 11, 8, 64

    # coef_apply: V1 scalar, V2 WMMA, V3 WMMA 4 warps (reference) vs aerial_coef_apply / aerial_coef_apply_tc
    lc = ref("coef")
    lc.ref_coef_launch.argtypes = [CI, VP, VP, VP, CI, CI]
    C, Y = crand((nSC, L, A), dev), crand((nSC, S, A), dev)
    O = torch.empty(nSC, L, S, dtype=torch.complex64, device=dev)
    p = (C.data_ptr(), Y.data_ptr(), O.data_ptr(), nSC, S)
    bytes_coef = 8 * (C.numel() + Y.numel() + O.numel())
    rows["coef_apply"] = {
        "reference_v1_scalar_us": timed(lambda: lc.ref_coef_launch(1, *p)),
        "reference_v2_wmma_us": timed(lambda: lc.ref_coef_launch(2, *p)),
        "reference_v3_wmma_us": timed(lambda: lc.ref_coef_launch(3, *p)),
        "aerial_coef_apply_us (bit-exact V1)": timed(lambda: aeq.coef_apply(C, Y, O, nSC, S, L, A)),
        "aerial_coef_apply_tc_us (V2 semantics)": timed(lambda: aeq.coef_apply_tc(C, Y, O, nSC, S, L, A)),
        "bytes": bytes_coef,
    }

    # Gram: gram_scalar (M given, no conjugate, no s2) vs aerial_gram (G = H^H H + s2 I)
    lg = ref("gram")
    lg.ref_gram_launch.argtypes = [VP, VP, VP, CI]
    H = crand((nSC, A, L), dev)
    M = H.conj().transpose(1, 2).contiguous()
    G = torch.empty(nSC, L, L, dtype=torch.complex64, device=dev)
    rows["gram"] = {
        "reference_gram_scalar_us": timed(lambda: lg.ref_gram_launch(M.data_ptr(), H.data_ptr(), G.data_ptr(), nSC)),
        "aerial_gram_us": timed(lambda: aeq.gram(H, 0.01, G, nSC, A, L)),
    }

    # LLR demapper, 256-QAM: llr_v1_baseline and llr_v3 (reference) vs aerial_llr (same FP16 I/O)
    ll = ref("llr_v3")
    ll.ref_llr_v3_launch.argtypes = [CI, VP, VP, VP, CI, CI]
    N, nb = nSC * L * S, 4
    soft = ((torch.rand(2 * N, device=dev) - 0.5) * 1.4).half()
    ni = torch.rand(N, device=dev) * 10 + 1
    lo = torch.empty(N * 2 * nb, dtype=torch.float16, device=dev)
    lp = (soft.data_ptr(), ni.data_ptr(), lo.data_ptr(), N, nb)
    rows["llr_256qam"] = {
        "reference_v1_us": timed(lambda: ll.ref_llr_v3_launch(1, *lp)),
        "reference_v3_us": timed(lambda: ll.ref_llr_v3_launch(3, *lp)),
        "aerial_llr_us (bit-exact V1)": timed(lambda: aeq.llr(soft, ni, lo, N, nb)),
    }

    # SRS filter multiply: V1 scalar FP16 and V2 WMMA (reference) vs aerial_srs_filter
    ls = ref("srs")
    ls.ref_srs_launch.argtypes = [CI, VP, VP, VP, VP, CI, CI]
    K, P, F, nBlk = 24, 4, 8, 66
    srs = ((torch.rand(nBlk * A * K * 2, device=dev) - 0.5) * 1.4).half()
    W = ((torch.rand(K * K * 2, device=dev) - 0.5) * 1.4).half()
    fo = ((torch.rand(P * F * 2, device=dev) - 0.5) * 1.4).half()
    he = torch.empty(nBlk * A * K * P * 2, dtype=torch.float16, device=dev)
    sp = (he.data_ptr(), srs.data_ptr(), W.data_ptr(), fo.data_ptr(), A, nBlk)
    rows["srs_filter"] = {
        "reference_v1_scalar_us": timed(lambda: ls.ref_srs_launch(1, *sp)),
        "reference_v2_wmma_us": timed(lambda: ls.ref_srs_launch(2, *sp)),
        "aerial_srs_filter_us": timed(lambda: aeq.srs_filter(he, srs, W, fo, A, nBlk, K, P, F)),
    }

    # one cell: the reference's unfused stages vs the fused launch
    c = wl.config_cell(2, seed=3, device=dev)
    Mc = c.H.conj().transpose(1, 2).contiguous()
    Gc = torch.empty(nSC, L, L, dtype=torch.complex64, device=dev)
    Cc = crand((nSC, L, A), dev)
    Oc = torch.empty(nSC, L, S, dtype=torch.complex64, device=dev)
    llr32 = torch.empty(c.llr_numel, dtype=torch.float32, device=dev)
    desc = aeq.cell_desc(c.H, c.Y, llr32, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    tun = aeq.make_tuning("fp16")

    def ref_chain():
        lg.ref_gram_launch(Mc.data_ptr(), c.H.data_ptr(), Gc.data_ptr(), nSC)
        lc.ref_coef_launch(2, Cc.data_ptr(), c.Y.data_ptr(), Oc.data_ptr(), nSC, S)
        ll.ref_llr_v3_launch(3, soft.data_ptr(), ni.data_ptr(), lo.data_ptr(), N, nb)

    rows["one_cell_chain"] = {
        "reference_gram_coefv2_llrv3_us (three launches, no solve)": timed(ref_chain),
        "aerial_pusch_eq_fused_us (Gram + MMSE solve + apply + LLR, one launch)":
            timed(lambda: aeq.pusch_eq_fused([desc], tun)),
    }
    # the headline scale: 64 cell-slots (101,376 subcarriers, 1.3 GB of inputs: larger than L2), the
    # reference's three stages over all of them against one fused launch of this library
    del Mc, Gc, Cc, Oc, M, H, C, Y
    torch.cuda.empty_cache()
    slots = 64
    cells = [wl.config_cell(2, seed=17 * i + 1, device=dev) for i in range(slots)]
    nS = nSC * slots
    Hs = torch.cat([x.H for x in cells])
    Ys = torch.cat([x.Y for x in cells])
    Ms = Hs.conj().transpose(1, 2).contiguous()
    Gs = torch.empty(nS, L, L, dtype=torch.complex64, device=dev)
    Cs = crand((nS, L, A), dev)
    Os = torch.empty(nS, L, S, dtype=torch.complex64, device=dev)
    Ns = nS * L * S
    soft_s = ((torch.rand(2 * Ns, device=dev) - 0.5) * 1.4).half()
    ni_s = torch.rand(Ns, device=dev) * 10 + 1
    lo_s = torch.empty(Ns * 2 * nb, dtype=torch.float16, device=dev)
    llrs = [torch.empty(x.llr_numel, dtype=torch.float32, device=dev) for x in cells]
    descs = [aeq.cell_desc(x.H, x.Y, l, x.sigma2, x.nPRB, x.nAnt, x.nLayers, x.nSym, x.nPamBits)
             for x, l in zip(cells, llrs)]

    def ref_chain_64():
        lg.ref_gram_launch(Ms.data_ptr(), Hs.data_ptr(), Gs.data_ptr(), nS)
        lc.ref_coef_launch(2, Cs.data_ptr(), Ys.data_ptr(), Os.data_ptr(), nS, S)
        ll.ref_llr_v3_launch(3, soft_s.data_ptr(), ni_s.data_ptr(), lo_s.data_ptr(), Ns, nb)

    t_ref = timed(ref_chain_64, warm=3, iters=20)
    t_fused = timed(lambda: aeq.pusch_eq_fused(descs, tun), warm=3, iters=20)
    rows["64_slot_chain"] = {
        "reference_gram_coefv2_llrv3_us (three launches, no solve)": t_ref,
        "reference_res_per_s": nS * S / (t_ref * 1e-6),
        "aerial_pusch_eq_fused_us (Gram + MMSE solve + apply + LLR, one launch)": t_fused,
        "aerial_res_per_s": nS * S / (t_fused * 1e-6),
    }
    print(json.dumps({"gpu": torch.cuda.get_device_name(0), "method": "median of 50 event-timed launches after 10 "
                      "warm-ups, inputs L2-warm (the reference's own method), the GPU kept busy across the host's "
                      "enqueue", "rows": rows}))


if __name__ == "__main__":
    main()
