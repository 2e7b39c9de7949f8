"""Generate the golden fixtures of tests/golden/ from the reference itself.

Run with AERIAL_REF naming the reference tree, after ``make -C oracle ref
REF=<that tree>``:

    python tests/golden/make_golden.py            # CPU fixtures
    python tests/golden/make_golden.py --gpu      # + outputs of the reference's
                                                  #   own kernels (needs a GPU)

CPU fixtures (no GPU needed; the reference's host code is compiled from its
sources into oracle/_ref/ by oracle/Makefile):
  llr_cpu_ref.npz     cpu_ref (src/llr/aerial_llr_v3.cu:61-79) outputs for the
                      reference's own LLR inputs (srand(42), :267-275),
                      nPamBits 1..4, first 1024 symbols
  pam_lut.json        the c_LUT initializer of src/llr/aerial_llr_v3.cu:42-48
  known_answers.json  the recorded coef_apply results (results/coef_rigor_results.txt,
                      README.md) with the data recipes that produced them
GPU fixtures (the reference's kernels compiled unchanged for sm_100a, run on
the full-size reference inputs, which the tests regenerate from the seeds):
  ref_gpu.json        SHA-256 of the outputs of coef_apply_v1_scalar / v2_wmma,
                      gram_scalar (M = H^H), llr_v1_baseline / llr_v3 (nPamBits
                      1..4) and srs_filter_v1_scalar / v2_wmma (4 configurations)
  ref_gpu_slices.npz  the first 4096 values of each of those outputs
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

REF = os.environ.get("AERIAL_REF", "")


def require_ref():
    """The reference tree the fixtures are generated from (AERIAL_REF)."""
    if not REF or not os.path.isdir(os.path.join(REF, "src")):
        sys.exit("make_golden.py: set AERIAL_REF to the reference tree (the directory holding src/ and results/)")
    return REF
REFLIB = os.path.join(ROOT, "oracle", "_ref")
VP = ctypes.c_void_p
CI = ctypes.c_int

# fixture recipes shared with the tests
LLR_N = 1024
COEF_SEED, COEF_NSC, COEF_NSYM = 7, 48, 11          # 64 ant, 8 layers fixed by the reference file
GRAM_SEED, GRAM_NSC = 11, 48
LLR_GPU_N = 4096
SRS_SEED, SRS_NBLK, SRS_NANT = 42, 6, 64
SRS_CFGS = [(24, 4, 8), (24, 2, 8), (12, 4, 12), (12, 2, 12)]


def cpu_fixtures():
    require_ref()
    lib = ctypes.CDLL(os.path.join(REFLIB, "libref_llr_v3.so"))
    lib.ref_llr_v3_cpu_ref.argtypes = [VP, VP, VP, CI, CI]
    N = 139392
    soft, ni = O.ref_llr_inputs(42, N)
    soft = soft[: 2 * LLR_N].copy()
    ni = ni[:LLR_N].copy()
    out = {"soft_u16": soft, "noise_inv": ni}
    for n in (1, 2, 3, 4):
        o = np.empty(LLR_N * 2 * n, np.float32)
        lib.ref_llr_v3_cpu_ref(soft.ctypes.data, ni.ctypes.data, o.ctypes.data, LLR_N, n)
        out[f"llr_n{n}"] = o
    np.savez_compressed(os.path.join(HERE, "llr_cpu_ref.npz"), **out)

    src = open(os.path.join(REF, "src/llr/aerial_llr_v3.cu")).read()
    m = re.search(r"__constant__ float c_LUT\[10\]\s*=\s*\{([^}]*)\}", src)
    lut = [float(v.strip().rstrip("f")) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
    json.dump({"source": "src/llr/aerial_llr_v3.cu:42-48", "c_LUT": lut, "offsets": [0, 1, 3, 6]},
              open(os.path.join(HERE, "pam_lut.json"), "w"), indent=1)

    txt = open(os.path.join(REF, "results/coef_rigor_results.txt")).read()
    evm = re.search(r"EVM\(V2 vs V1\) = ([0-9.]+)%\s+\(([-0-9.]+) dB\)\s+max_rel_err = ([0-9.]+)%", txt)
    readme = open(os.path.join(REF, "README.md")).read()
    cos = re.search(r"Cosine similarity[^0-9]*([0-9.]+)", readme)
    mae = re.search(r"Max abs error[^0-9]*([0-9.]+)", readme)
    ka = {
        "coef_rigor": {
            "source": "results/coef_rigor_results.txt:5; data src/coef_rigor.cu:101-104 (srand(7), U(-0.7,0.7), C then Y)",
            "seed": 7, "scale": 1.4, "nSC": 1584, "nLayers": 8, "nAnt": 64, "nSym": 11,
            "evm_pct": float(evm.group(1)), "evm_db": float(evm.group(2)), "max_rel_err_pct": float(evm.group(3)),
        },
        "coef_wmma": {
            "source": "README.md (V2 vs V1 correctness); data src/aerial_coef_wmma.cu:383-387 (srand(42), U(-0.5,0.5))",
            "seed": 42, "scale": 1.0, "nSC": 1584, "nLayers": 8, "nAnt": 64, "nSym": 11,
            "cosine": float(cos.group(1)) if cos else None, "max_abs_err": float(mae.group(1)) if mae else None,
        },
    }
    json.dump(ka, open(os.path.join(HERE, "known_answers.json"), "w"), indent=1)
    print("wrote CPU fixtures:", ka)


def coef_inputs(seed, nSC, nSym, L=8, A=64, scale=1.4):
    nC, nY = nSC * L * A * 2, nSC * nSym * A * 2
    v = O.ref_uniform(seed, nC + nY, scale)
    return v[:nC].copy(), v[nC:].copy()


def gram_inputs(seed, nSC, L=8, A=64):
    v = O.ref_uniform(seed, nSC * A * L * 2, 1.4)
    H = v.view(np.complex64).reshape(nSC, A, L)
    M = np.ascontiguousarray(np.conj(H).transpose(0, 2, 1))
    return np.ascontiguousarray(H), M


def srs_inputs(K, P, F, nBlk=SRS_NBLK, nAnt=SRS_NANT, seed=SRS_SEED):
    return O.ref_srs_inputs(seed, nBlk * nAnt * K, K * K, P * F)


def digest(a) -> str:
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# full-size recipes of the reference kernels' runs (shapes of the reference's main()s)
COEF_FULL = dict(seed=7, nSC=1584, nSym=11)
GRAM_FULL = dict(seed=11, nSC=1584)
LLR_FULL_N = 139392
SRS_FULL = dict(nBlk=66, nAnt=64, seed=42)


def gpu_fixtures(out_dir=HERE):
    """Run the reference's own kernels (compiled unchanged for sm_100a) on the
    full-size reference inputs; record SHA-256 digests of their outputs plus
    small value slices in ref_gpu.json / ref_gpu_slices.npz."""
    import torch

    dev = torch.device("cuda:0")

    def d(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    rec, slices = {}, {}
    coef = ctypes.CDLL(os.path.join(REFLIB, "libref_coef.so"))
    for fn in (coef.ref_coef_v1, coef.ref_coef_v2):
        fn.argtypes = [VP, VP, VP, CI, CI]
    C, Y = coef_inputs(COEF_FULL["seed"], COEF_FULL["nSC"], COEF_FULL["nSym"])
    dC, dY = d(C), d(Y)
    for name, fn in (("coef_v1", coef.ref_coef_v1), ("coef_v2", coef.ref_coef_v2)):
        o = torch.zeros(COEF_FULL["nSC"] * 8 * COEF_FULL["nSym"] * 2, dtype=torch.float32, device=dev)
        assert fn(dC.data_ptr(), dY.data_ptr(), o.data_ptr(), COEF_FULL["nSC"], COEF_FULL["nSym"]) == 0
        o = o.cpu().numpy()
        rec[name] = {"sha256": digest(o), "recipe": COEF_FULL}
        slices[name] = o[:4096]

    gram = ctypes.CDLL(os.path.join(REFLIB, "libref_gram.so"))
    gram.ref_gram.argtypes = [VP, VP, VP, CI]
    H, M = gram_inputs(GRAM_FULL["seed"], GRAM_FULL["nSC"])
    dM, dH = d(M), d(H)      # keep both alive across the call
    o = torch.zeros(GRAM_FULL["nSC"] * 64 * 2, dtype=torch.float32, device=dev)
    assert gram.ref_gram(dM.data_ptr(), dH.data_ptr(), o.data_ptr(), GRAM_FULL["nSC"]) == 0
    torch.cuda.synchronize()
    o = o.cpu().numpy()
    rec["gram"] = {"sha256": digest(o), "recipe": GRAM_FULL}
    slices["gram"] = o[:4096]

    llr = ctypes.CDLL(os.path.join(REFLIB, "libref_llr_v3.so"))
    for fn in (llr.ref_llr_v3_v1, llr.ref_llr_v3_v3):
        fn.argtypes = [VP, VP, VP, CI, CI]
    soft, ni = O.ref_llr_inputs(42, LLR_FULL_N)
    ds, dn = d(soft.view(np.int16)), d(ni)
    for n in (1, 2, 3, 4):
        for name, fn in (("v1", llr.ref_llr_v3_v1), ("v3", llr.ref_llr_v3_v3)):
            if name == "v3" and n == 1:
                continue
            o = torch.zeros(LLR_FULL_N * 2 * n, dtype=torch.int16, device=dev)
            assert fn(ds.data_ptr(), dn.data_ptr(), o.data_ptr(), LLR_FULL_N, n) == 0
            o = o.cpu().numpy().view(np.uint16)
            rec[f"llr_{name}_n{n}"] = {"sha256": digest(o), "recipe": {"seed": 42, "N": LLR_FULL_N}}
            slices[f"llr_{name}_n{n}"] = o[:4096]

    srs = ctypes.CDLL(os.path.join(REFLIB, "libref_srs.so"))
    srs.ref_srs.argtypes = [CI, VP, VP, VP, VP, CI, CI, CI, CI, CI]
    for (K, P, F) in SRS_CFGS:
        s, w, f = srs_inputs(K, P, F, SRS_FULL["nBlk"], SRS_FULL["nAnt"], SRS_FULL["seed"])
        ds_, dw, df = d(s.view(np.int16)), d(w.view(np.int16)), d(f.view(np.int16))
        for v in (1, 2):
            o = torch.zeros(SRS_FULL["nBlk"] * SRS_FULL["nAnt"] * K * P * 2, dtype=torch.int16, device=dev)
            assert srs.ref_srs(v, o.data_ptr(), ds_.data_ptr(), dw.data_ptr(), df.data_ptr(), SRS_FULL["nAnt"],
                               SRS_FULL["nBlk"], K, P, F) == 0
            o = o.cpu().numpy().view(np.uint16)
            rec[f"srs_v{v}_K{K}_P{P}_F{F}"] = {"sha256": digest(o), "recipe": dict(SRS_FULL, K=K, P=P, F=F)}
            slices[f"srs_v{v}_K{K}_P{P}_F{F}"] = o[:4096]
    props = torch.cuda.get_device_properties(dev)
    meta = {"device": props.name, "cc": f"{props.major}.{props.minor}", "nvcc": "12.9, -O3 -gencode sm_100a "
            "(LLR files with --use_fast_math, their documented build line)"}
    json.dump({"meta": meta, "outputs": rec}, open(os.path.join(out_dir, "ref_gpu.json"), "w"), indent=1)
    np.savez_compressed(os.path.join(out_dir, "ref_gpu_slices.npz"), **slices)
    print("wrote GPU fixtures to", out_dir)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true", help="also run the reference's kernels (needs a GPU)")
    ap.add_argument("--gpu-only", action="store_true")
    ap.add_argument("--out", default=HERE, help="directory for the GPU fixtures")
    a = ap.parse_args()
    if not a.gpu_only:
        cpu_fixtures()
    if a.gpu or a.gpu_only:
        os.makedirs(a.out, exist_ok=True)
        gpu_fixtures(a.out)
