"""Checker for the PUSCH equalization path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over ``oracle/liborc.so`` (built from ``oracle/aerial_oracle.c``
by ``oracle/Makefile``): a CPU restatement of the reference's scalar FP32
kernels and an FP64 model of the chain.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
import this module; the shipped library never does.

Reference functions restated (paths inside ebaenamar/aerial-mimo-tc-optimization):
  coef_apply_v1_scalar   src/aerial_coef_wmma.cu:71-104
  coef_apply_v2_wmma     src/aerial_coef_wmma.cu:146-239   (FP16 model)
  gram_scalar            src/aerial_bottleneck.cu:56-80
  llr_v1_baseline        src/llr/aerial_llr_v3.cu:84-108
  cpu_ref (FP64)         src/llr/aerial_llr_v3.cu:61-79
  srs_filter_v1_scalar   src/srs/srs_wmma_bench.cu:57-90   (FP16 arithmetic)
plus an FP64 DMRS interpolation filter (no reference kernel; README.md:200).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_L = ctypes.c_long
_I = ctypes.c_int


def lib():
    """Load (building first if needed) the oracle shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        import subprocess

        subprocess.check_call(["make", "-s", "-C", _HERE, "liborc.so"])
    L = ctypes.CDLL(_LIB_PATH)
    sig = {
        "orc_set_threads": (None, [_I]),
        "orc_get_threads": (_I, []),
        "orc_ref_uniform": (None, [ctypes.c_uint, ctypes.c_float, _f32p, _L]),
        "orc_ref_llr_inputs": (None, [ctypes.c_uint, _L, _u16p, _f32p]),
        "orc_ref_srs_inputs": (None, [ctypes.c_uint, _L, _L, _L, _u16p, _u16p, _u16p]),
        "orc_f32_to_f16": (None, [_f32p, _u16p, _L]),
        "orc_f16_to_f32": (None, [_u16p, _f32p, _L]),
        "orc_pam_lut": (None, [_I, _f32p, _f64p]),
        "orc_llr_f32": (None, [_f32p, _f32p, _f32p, _L, _I, _I]),
        "orc_llr_f16io": (None, [_u16p, _f32p, _u16p, _L, _I]),
        "orc_llr_f64": (None, [_f32p, _f32p, _f64p, _L, _I, _I]),
        "orc_coef_apply_v1": (None, [_f32p, _f32p, _f32p, _L, _I, _I, _I]),
        "orc_coef_apply_v2_model": (None, [_f32p, _f32p, _f32p, _L, _I, _I, _I]),
        "orc_gram_ref": (None, [_f32p, _f32p, _f32p, _L, _I, _I]),
        "orc_gram": (None, [_f32p, ctypes.c_float, _f32p, _L, _I, _I]),
        "orc_mmse_coef": (None, [_f32p, _f32p, _f32p, _f32p, _L, _I, _I]),
        "orc_chain_f32": (None, [_f32p, _f32p, ctypes.c_float, _L, _I, _I, _I, _I, _f32p, _f32p, _f32p]),
        "orc_chain_f64": (None, [_f32p, _f32p, ctypes.c_double, _L, _I, _I, _I, _I, _f64p, _f64p, _f64p]),
        "orc_srs_v1_f16": (None, [_u16p, _u16p, _u16p, _u16p, _I, _I, _I, _I, _I]),
        "orc_srs_f64": (None, [_u16p, _u16p, _u16p, _f64p, _I, _I, _I, _I, _I]),
        "orc_chest_f64": (None, [_u16p, _u16p, _u16p, _f64p, _I, _I, _I, _I, _I, _I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _cf(a):
    """complex64 array -> contiguous float32 view of interleaved pairs."""
    a = np.ascontiguousarray(a, dtype=np.complex64)
    return a.view(np.float32).reshape(-1)


# --- reference input generators -------------------------------------------

def ref_uniform(seed: int, n: int, scale: float = 1.0) -> np.ndarray:
    out = np.empty(n, np.float32)
    lib().orc_ref_uniform(seed, scale, out, n)
    return out


def ref_llr_inputs(seed: int, n: int):
    soft = np.empty(2 * n, np.uint16)
    ni = np.empty(n, np.float32)
    lib().orc_ref_llr_inputs(seed, n, soft, ni)
    return soft, ni


def ref_srs_inputs(seed: int, n_srs: int, n_w: int, n_focc: int):
    s = np.empty(2 * n_srs, np.uint16)
    w = np.empty(2 * n_w, np.uint16)
    f = np.empty(2 * n_focc, np.uint16)
    lib().orc_ref_srs_inputs(seed, n_srs, n_w, n_focc, s, w, f)
    return s, w, f


def f32_to_f16(x) -> np.ndarray:
    x = _c(x, np.float32).reshape(-1)
    y = np.empty(x.size, np.uint16)
    lib().orc_f32_to_f16(x, y, x.size)
    return y


def pam_lut(n: int):
    d32 = np.zeros(4, np.float32)
    d64 = np.zeros(4, np.float64)
    lib().orc_pam_lut(n, d32, d64)
    return d32[:n], d64[:n]


# --- LLR -------------------------------------------------------------------

def llr_f32(soft_c64, noise_inv, n_pam_bits: int, syms_per_noise: int = 1) -> np.ndarray:
    s = _cf(soft_c64)
    n = s.size // 2
    out = np.empty(n * 2 * n_pam_bits, np.float32)
    lib().orc_llr_f32(s, _c(noise_inv, np.float32).reshape(-1), out, n, n_pam_bits, syms_per_noise)
    return out


def llr_f16io(soft_u16, noise_inv, n_pam_bits: int) -> np.ndarray:
    s = _c(soft_u16, np.uint16).reshape(-1)
    n = s.size // 2
    out = np.empty(n * 2 * n_pam_bits, np.uint16)
    lib().orc_llr_f16io(s, _c(noise_inv, np.float32).reshape(-1), out, n, n_pam_bits)
    return out


def llr_f64(soft_c64, noise_inv, n_pam_bits: int, syms_per_noise: int = 1) -> np.ndarray:
    s = _cf(soft_c64)
    n = s.size // 2
    out = np.empty(n * 2 * n_pam_bits, np.float64)
    lib().orc_llr_f64(s, _c(noise_inv, np.float32).reshape(-1), out, n, n_pam_bits, syms_per_noise)
    return out


# --- coef_apply / gram / solve ----------------------------------------------

def coef_apply_v1(C, Y, n_sc, n_sym, L, A) -> np.ndarray:
    out = np.empty(n_sc * L * n_sym * 2, np.float32)
    lib().orc_coef_apply_v1(_cf(C), _cf(Y), out, n_sc, n_sym, L, A)
    return out.view(np.complex64)


def coef_apply_v2_model(C, Y, n_sc, n_sym, L, A) -> np.ndarray:
    out = np.empty(n_sc * L * n_sym * 2, np.float32)
    lib().orc_coef_apply_v2_model(_cf(C), _cf(Y), out, n_sc, n_sym, L, A)
    return out.view(np.complex64)


def gram_ref(M, H, n_sc, L, A) -> np.ndarray:
    out = np.empty(n_sc * L * L * 2, np.float32)
    lib().orc_gram_ref(_cf(M), _cf(H), out, n_sc, L, A)
    return out.view(np.complex64)


def gram(H, sigma2, n_sc, A, L) -> np.ndarray:
    out = np.empty(n_sc * L * L * 2, np.float32)
    lib().orc_gram(_cf(H), float(sigma2), out, n_sc, A, L)
    return out.view(np.complex64)


def mmse_coef(G, H, n_sc, A, L):
    C = np.empty(n_sc * L * A * 2, np.float32)
    nI = np.empty(n_sc * L, np.float32)
    lib().orc_mmse_coef(_cf(G), _cf(H), C, nI, n_sc, A, L)
    return C.view(np.complex64), nI


def chain_f32(H, Y, sigma2, n_sc, A, L, n_sym, n_pam_bits, want_llr=True):
    yeq = np.empty(n_sc * L * n_sym * 2, np.float32)
    nI = np.empty(n_sc * L, np.float32)
    llr = np.empty(n_sc * L * n_sym * 2 * n_pam_bits if want_llr else 1, np.float32)
    lib().orc_chain_f32(_cf(H), _cf(Y), float(sigma2), n_sc, A, L, n_sym, n_pam_bits, yeq, nI,
                        llr if want_llr else np.empty(0, np.float32))
    return yeq.view(np.complex64), nI, (llr if want_llr else None)


def chain_f64(H, Y, sigma2, n_sc, A, L, n_sym, n_pam_bits):
    yeq = np.empty(n_sc * L * n_sym * 2, np.float64)
    nI = np.empty(n_sc * L, np.float64)
    llr = np.empty(n_sc * L * n_sym * 2 * n_pam_bits, np.float64)
    lib().orc_chain_f64(_cf(H), _cf(Y), float(sigma2), n_sc, A, L, n_sym, n_pam_bits, yeq, nI, llr)
    return yeq.view(np.complex128), nI, llr


# --- SRS -------------------------------------------------------------------

def srs_v1_f16(srs_u16, w_u16, focc_u16, n_ant, n_blocks, K, P, F) -> np.ndarray:
    out = np.empty(2 * n_blocks * n_ant * K * P, np.uint16)
    lib().orc_srs_v1_f16(_c(srs_u16, np.uint16), _c(w_u16, np.uint16), _c(focc_u16, np.uint16), out,
                         n_ant, n_blocks, K, P, F)
    return out


def srs_f64(srs_u16, w_u16, focc_u16, n_ant, n_blocks, K, P, F) -> np.ndarray:
    out = np.empty(2 * n_blocks * n_ant * K * P, np.float64)
    lib().orc_srs_f64(_c(srs_u16, np.uint16), _c(w_u16, np.uint16), _c(focc_u16, np.uint16), out,
                      n_ant, n_blocks, K, P, F)
    return out.view(np.complex128)


def chest_f64(yp_u16, wf_u16, occ_u16, n_ant, n_blocks, n_pilot, n_out, P, F) -> np.ndarray:
    """FP64 DMRS interpolation filter in the channel layout [blk*n_out + o][ant][p] (no reference kernel)."""
    out = np.empty(2 * n_blocks * n_out * n_ant * P, np.float64)
    lib().orc_chest_f64(_c(yp_u16, np.uint16), _c(wf_u16, np.uint16), _c(occ_u16, np.uint16), out,
                        n_ant, n_blocks, n_pilot, n_out, P, F)
    return out.view(np.complex128)
