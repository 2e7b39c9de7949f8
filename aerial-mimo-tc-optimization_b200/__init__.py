"""B200-native PUSCH receiver equalization path (host-side mirror of the C ABI).

The shared library ``libaerial_eq.so`` (built from ``csrc/`` for sm_100a by the
``Makefile`` in this directory) holds every kernel; this module only binds its
C ABI (``include/aerial_eq.h``) with ctypes and passes torch CUDA tensors'
device pointers and the current stream.  There is no CPU fallback: if the
library is missing or a call fails, an exception is raised.

Function names and argument order mirror the reference's kernel entries
(ebaenamar/aerial-mimo-tc-optimization):

  coef_apply(C, Y_rx, Y_eq, nSC, nSym, ...)   coef_apply_v1_scalar, src/aerial_coef_wmma.cu:71-75
  coef_apply_tc(...)                          coef_apply_v2_wmma,   src/aerial_coef_wmma.cu:146-150
  gram(H, sigma2, G, nSC, ...)                gram_scalar,          src/aerial_bottleneck.cu:56-60
  llr(softEst, noiseInv, llrOut, N, nPamBits) llr_v1_baseline,      src/llr/aerial_llr_v3.cu:84-86
  srs_filter(H_est, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen)
                                              srs_filter_v1_scalar, src/srs/srs_wmma_bench.cu:57-63
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaerial_eq.so")

AERIAL_OK = 0
PREC_FP16, PREC_BF16, PREC_BF16X3, PREC_FP32, PREC_FP16X3 = 0, 1, 2, 3, 4
PREC_NAMES = {"fp16": PREC_FP16, "bf16": PREC_BF16, "bf16x3": PREC_BF16X3, "fp32": PREC_FP32,
              "fp16x3": PREC_FP16X3}
FMT_CF32, FMT_CF16 = 0, 1          # cell storage formats (aerial_cell_desc.format)
MAX_CELLS = 64
MAX_PRB = 524288            # AERIAL_MAX_PRB: PRBs per cell descriptor


class AerialError(RuntimeError):
    """A non-zero status from the C ABI (the reference would exit(1) here)."""

    def __init__(self, status: int, where: str):
        self.status = status
        msg = _lib_handle().aerial_error_string(status).decode() if _LIB is not None else str(status)
        super().__init__(f"{where}: status {status}: {msg}")


class CellDesc(ctypes.Structure):
    """``aerial_cell_desc``: one cell-slot of the fused chain."""

    _fields_ = [
        ("H", ctypes.c_void_p),
        ("Y_rx", ctypes.c_void_p),
        ("llr", ctypes.c_void_p),
        ("Y_eq", ctypes.c_void_p),
        ("sigma2", ctypes.c_float),
        ("nPRB", ctypes.c_int),
        ("nAnt", ctypes.c_int),
        ("nLayers", ctypes.c_int),
        ("nSym", ctypes.c_int),
        ("nPamBits", ctypes.c_int),
        ("format", ctypes.c_int),
    ]


class Tuning(ctypes.Structure):
    """``aerial_tuning``: operand precision and launch shape (0 = default)."""

    _fields_ = [
        ("precision", ctypes.c_int),
        ("warps_per_cta", ctypes.c_int),
        ("ctas_per_sm", ctypes.c_int),
        ("sc_per_group", ctypes.c_int),
    ]


class ServerConfig(ctypes.Structure):
    """``aerial_server_config``."""

    _fields_ = [
        ("memory_budget_bytes", ctypes.c_int64),
        ("streams", ctypes.c_int),
        ("max_batch", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("mode", ctypes.c_int),
        ("queue_capacity", ctypes.c_int),
        ("start_paused", ctypes.c_int),
        ("deadline_us", ctypes.c_float),
        ("batch_window_us", ctypes.c_float),
        ("min_batch", ctypes.c_int),
    ]


class ServerCompletion(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_uint64), ("cell_id", ctypes.c_int), ("status", ctypes.c_int),
                ("latency_us", ctypes.c_float)]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("slots_done", ctypes.c_long),
        ("p50_us", ctypes.c_float), ("p99_us", ctypes.c_float), ("max_us", ctypes.c_float),
        ("mean_us", ctypes.c_float),
        ("queue_p99_us", ctypes.c_float),
        ("service_p99_us", ctypes.c_float),
        ("deadline_misses", ctypes.c_long),
        ("res_done", ctypes.c_long),
        ("span_s", ctypes.c_double),
        ("res_per_s", ctypes.c_double),
        ("batches", ctypes.c_long),
        ("mean_batch", ctypes.c_float),
        ("srs_updates", ctypes.c_long),
        ("budget_used_bytes", ctypes.c_int64),
        ("pending", ctypes.c_long),
        ("submit_lag_p99_us", ctypes.c_float),
        ("submit_lag_max_us", ctypes.c_float),
        ("dispatch_gap_max_us", ctypes.c_float),
        ("launch_call_max_us", ctypes.c_float),
        ("misses_late_submit", ctypes.c_long),
    ]


SERVER_FUSED, SERVER_PLAIN = 0, 1

_LIB = None

# exported symbol -> (restype, argtypes)
_P, _I, _F, _Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
SIGNATURES = {
    "aerial_error_string": (ctypes.c_char_p, [_I]),
    "aerial_version": (_I, []),
    "aerial_prepare": (_I, []),
    "aerial_coef_apply": (_I, [_P, _P, _P, _I, _I, _I, _I, _P]),
    "aerial_coef_apply_tc": (_I, [_P, _P, _P, _I, _I, _I, _I, _P]),
    "aerial_gram": (_I, [_P, _F, _P, _I, _I, _I, _P]),
    "aerial_mmse_coef": (_I, [_P, _P, _P, _P, _I, _I, _I, _P]),
    "aerial_llr": (_I, [_P, _P, _P, _I, _I, _P]),
    "aerial_llr_f32": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "aerial_srs_filter": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P]),
    "aerial_srs_to_channel": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P]),
    "aerial_chest_interp": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "aerial_srs_to_channel_avg": (_I, [_P, _P, _I, _P, _P, _I, _I, _I, _I, _I, _P]),
    "aerial_chest_interp_h": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "aerial_kernel_timeouts": (_I, [ctypes.POINTER(ctypes.c_uint)]),
    "aerial_fp16_operand_scale": (_F, [_F]),
    "aerial_pusch_eq_fused": (_I, [ctypes.POINTER(CellDesc), _I, ctypes.POINTER(Tuning), _P]),
    "aerial_pusch_eq_plain_workspace": (_Z, [ctypes.POINTER(CellDesc), _I]),
    "aerial_pusch_eq_plain": (_I, [ctypes.POINTER(CellDesc), _I, _P, _Z, _P]),
    "aerial_autotune": (_I, [ctypes.POINTER(CellDesc), _I, ctypes.POINTER(Tuning), ctypes.POINTER(_F), _P]),
    "aerial_pusch_eq_plain_static": (_I, [ctypes.POINTER(CellDesc), _I, _P]),
    "aerial_pusch_eq_host_workspace": (_I, [ctypes.POINTER(CellDesc), _I, _I, ctypes.POINTER(_Z)]),
    "aerial_pusch_eq_host": (_I, [ctypes.POINTER(CellDesc), _I, ctypes.POINTER(Tuning), _I, _P, _Z, _P]),
    "aerial_eq_graph_create": (_I, [ctypes.POINTER(CellDesc), _I, ctypes.POINTER(Tuning), ctypes.POINTER(_P)]),
    "aerial_eq_graph_update": (_I, [_P, ctypes.POINTER(CellDesc), _I]),
    "aerial_eq_graph_launch": (_I, [_P, _P]),
    "aerial_eq_graph_destroy": (_I, [_P]),
    "aerial_server_create": (_I, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]),
    "aerial_server_destroy": (_I, [_P]),
    "aerial_server_add_cell": (_I, [_P, _I, _I, _I, _I, _I, _F, ctypes.POINTER(_I)]),
    "aerial_server_set_channel": (_I, [_P, _I, _P, _F]),
    "aerial_server_srs_update": (_I, [_P, _I, _P, _P, _P, _I, _I, ctypes.POINTER(ctypes.c_uint64)]),
    "aerial_server_srs_update_n": (_I, [_P, _I, _P, _I, _P, _P, _I, _I, ctypes.POINTER(ctypes.c_uint64)]),
    "aerial_server_submit": (_I, [_P, _I, _P, _P, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]),
    "aerial_server_poll": (_I, [_P, ctypes.POINTER(ServerCompletion), _I, ctypes.POINTER(_I)]),
    "aerial_server_wait": (_I, [_P, ctypes.c_uint64, _I]),
    "aerial_server_drain": (_I, [_P, _I]),
    "aerial_server_pause": (_I, [_P, _I]),
    "aerial_server_stats": (_I, [_P, ctypes.POINTER(ServerStats)]),
    "aerial_server_reset_stats": (_I, [_P]),
    "aerial_server_inject_alloc_failure": (_I, [_P, _I]),
}


def _lib_handle():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                f"(make -C {_HERE}); there is no CPU fallback")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def lib():
    """The loaded ``libaerial_eq.so`` (ctypes handle)."""
    return _lib_handle()


def fp16_operand_scale(sigma2: float) -> float:
    """The power-of-two scale the FP16 path applies to a complex64 cell's H and
    Y_rx for noise variance sigma2 (1 where raw FP16 operands are safe)."""
    return float(lib().aerial_fp16_operand_scale(float(sigma2)))


def prepare():
    """Load every kernel of the library on the current device (avoids first-launch stalls)."""
    _check(lib().aerial_prepare(), "prepare")


def _check(status: int, where: str) -> None:
    if status != AERIAL_OK:
        raise AerialError(status, where)


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor (device memory)")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


# ---------------------------------------------------------------------------
# per-stage entry points (reference kernel names)
# ---------------------------------------------------------------------------

def coef_apply(C, Y_rx, Y_eq, nSC, nSym, nLayers, nAnt, stream=None):
    """Y_eq[sc][l][s] = sum_a C[sc][l][a] Y_rx[sc][s][a] (FP32, bit-exact V1)."""
    _check(lib().aerial_coef_apply(_ptr(C), _ptr(Y_rx), _ptr(Y_eq), nSC, nSym, nLayers, nAnt, _stream(stream)),
           "coef_apply")


def coef_apply_tc(C, Y_rx, Y_eq, nSC, nSym, nLayers, nAnt, stream=None):
    """coef_apply on the tensor cores (FP16 operands, FP32 accumulation)."""
    _check(lib().aerial_coef_apply_tc(_ptr(C), _ptr(Y_rx), _ptr(Y_eq), nSC, nSym, nLayers, nAnt,
                                      _stream(stream)), "coef_apply_tc")


def gram(H, sigma2, G, nSC, nAnt, nLayers, stream=None):
    """G[sc] = H[sc]^H H[sc] + sigma2 I (FP32)."""
    _check(lib().aerial_gram(_ptr(H), float(sigma2), _ptr(G), nSC, nAnt, nLayers, _stream(stream)), "gram")


def mmse_coef(G, H, C, noiseInv, nSC, nAnt, nLayers, stream=None):
    """C = diag(1/mu) G^-1 H^H and noiseInv = mu/(1-mu) per (sc, layer) (FP32 Cholesky)."""
    _check(lib().aerial_mmse_coef(_ptr(G), _ptr(H), _ptr(C), _ptr(noiseInv), nSC, nAnt, nLayers,
                                  _stream(stream)), "mmse_coef")


def llr(softEst, noiseInv, llrOut, N, nPamBits, stream=None):
    """Max-log PAM LLRs, FP16 in / FP16 out (the reference's I/O, bit-exact)."""
    _check(lib().aerial_llr(_ptr(softEst), _ptr(noiseInv), _ptr(llrOut), N, nPamBits, _stream(stream)), "llr")


def llr_f32(softEst, noiseInv, llrOut, N, nPamBits, nSymPerNoise=1, stream=None):
    """Max-log PAM LLRs, complex64 in / float32 out; noiseInv[idx // nSymPerNoise]."""
    _check(lib().aerial_llr_f32(_ptr(softEst), _ptr(noiseInv), _ptr(llrOut), N, nPamBits, nSymPerNoise,
                                _stream(stream)), "llr_f32")


def srs_filter(H_est, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, stream=None):
    """H_est[blk][ant][k_out][p] = sum_k W[k_out][k] FOCC[p][k%F] SRS[blk][ant][k] (FP16 I/O, FP32 sums)."""
    _check(lib().aerial_srs_filter(_ptr(H_est), _ptr(SRS), _ptr(W), _ptr(FOCC), nAnt, nBlocks, K, nPorts, foccLen,
                                   _stream(stream)), "srs_filter")


def srs_to_channel(H, SRS, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, stream=None):
    """SRS filter multiply written as the PUSCH channel H[blk*K+k_out][ant][port] (complex64)."""
    _check(lib().aerial_srs_to_channel(_ptr(H), _ptr(SRS), _ptr(W), _ptr(FOCC), nAnt, nBlocks, K, nPorts, foccLen,
                                       _stream(stream)), "srs_to_channel")


def srs_to_channel_avg(H, SRS, nSrsSym, W, FOCC, nAnt, nBlocks, K, nPorts, foccLen, stream=None):
    """srs_to_channel averaged over nSrsSym (1, 2 or 4) consecutive SRS symbols in SRS."""
    _check(lib().aerial_srs_to_channel_avg(_ptr(H), _ptr(SRS), int(nSrsSym), _ptr(W), _ptr(FOCC), nAnt, nBlocks, K,
                                           nPorts, foccLen, _stream(stream)), "srs_to_channel_avg")


def kernel_timeouts() -> int:
    """Bounded waits of the tcgen05 kernels that gave up on the current device (0 in correct operation)."""
    n = ctypes.c_uint(0)
    _check(lib().aerial_kernel_timeouts(ctypes.byref(n)), "kernel_timeouts")
    return int(n.value)


def chest_interp(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen, stream=None):
    """DMRS frequency-interpolation filter written as the PUSCH channel H[blk*nOut+o][ant][port] (complex64)."""
    _check(lib().aerial_chest_interp(_ptr(H), _ptr(Yp), _ptr(Wf), _ptr(OCC), nAnt, nBlocks, nPilot, nOut, nPorts,
                                     occLen, _stream(stream)), "chest_interp")


def chest_interp_h(H, Yp, Wf, OCC, nAnt, nBlocks, nPilot, nOut, nPorts, occLen, stream=None):
    """The same filter written as complex half (float16 (re, im) pairs): the H of an FMT_CF16 cell."""
    _check(lib().aerial_chest_interp_h(_ptr(H), _ptr(Yp), _ptr(Wf), _ptr(OCC), nAnt, nBlocks, nPilot, nOut, nPorts,
                                       occLen, _stream(stream)), "chest_interp_h")


# ---------------------------------------------------------------------------
# fused chain
# ---------------------------------------------------------------------------

def cell_desc(H, Y_rx, llr_out, sigma2, nPRB, nAnt, nLayers, nSym, nPamBits, Y_eq=None, fmt=FMT_CF32) -> CellDesc:
    """One cell-slot on device tensors.  fmt=FMT_CF16: H, Y_rx, Y_eq are complex
    half stored as (re, im) float16 pairs and the LLRs float16."""
    d = CellDesc()
    d.H = _ptr(H).value
    d.Y_rx = _ptr(Y_rx).value
    d.llr = _ptr(llr_out).value
    d.Y_eq = _ptr(Y_eq).value if Y_eq is not None else None
    d.sigma2 = float(sigma2)
    d.nPRB, d.nAnt, d.nLayers, d.nSym, d.nPamBits = int(nPRB), int(nAnt), int(nLayers), int(nSym), int(nPamBits)
    d.format = int(fmt)
    return d


def _cells_array(cells):
    n = len(cells)
    if n < 1 or n > MAX_CELLS:
        raise ValueError(f"1..{MAX_CELLS} cells per launch, got {n}")
    arr = (CellDesc * n)(*cells)
    return arr, n


def make_tuning(precision=PREC_FP16, warps_per_cta=0, ctas_per_sm=0, sc_per_group=0) -> Tuning:
    """Operand precision, launch shape and group cap (0 = default for each)."""
    if isinstance(precision, str):
        precision = PREC_NAMES[precision]
    return Tuning(int(precision), int(warps_per_cta), int(ctas_per_sm), int(sc_per_group))


def pusch_eq_fused(cells, tuning: Tuning | None = None, stream=None):
    """Fused Gram -> Cholesky MMSE -> apply -> LLR over all cells in one launch."""
    arr, n = _cells_array(cells)
    tp = ctypes.pointer(tuning) if tuning is not None else None
    _check(lib().aerial_pusch_eq_fused(arr, n, tp, _stream(stream)), "pusch_eq_fused")


def pusch_eq_plain_workspace(cells) -> int:
    arr, n = _cells_array(cells)
    return int(lib().aerial_pusch_eq_plain_workspace(arr, n))


def pusch_eq_plain(cells, workspace, stream=None):
    """The plain FP32 chain (gram, mmse_coef, coef_apply, llr_f32 per cell)."""
    arr, n = _cells_array(cells)
    _check(lib().aerial_pusch_eq_plain(arr, n, _ptr(workspace), workspace.numel() * workspace.element_size(),
                                       _stream(stream)), "pusch_eq_plain")


def pusch_eq_plain_static(cells, stream=None):
    """The plain FP32 chain without a workspace argument, for callers that cannot
    allocate device memory: intermediates live in the library's static 16 MiB
    device array (shared by all calls; calls overlapping on the GPU race)."""
    arr, n = _cells_array(cells)
    _check(lib().aerial_pusch_eq_plain_static(arr, n, _stream(stream)), "pusch_eq_plain_static")


def _host_ptr(t):
    if t is None:
        return None
    if t.is_cuda:
        raise ValueError("expected a host tensor (pinned for overlapped copies)")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def host_cell_desc(H, Y_rx, llr_out, sigma2, nPRB, nAnt, nLayers, nSym, nPamBits, Y_eq=None, fmt=FMT_CF32) -> CellDesc:
    """A cell whose buffers are host tensors, for pusch_eq_host."""
    d = CellDesc()
    d.H = _host_ptr(H).value
    d.Y_rx = _host_ptr(Y_rx).value
    d.llr = _host_ptr(llr_out).value
    d.Y_eq = _host_ptr(Y_eq).value if Y_eq is not None else None
    d.sigma2 = float(sigma2)
    d.nPRB, d.nAnt, d.nLayers, d.nSym, d.nPamBits = int(nPRB), int(nAnt), int(nLayers), int(nSym), int(nPamBits)
    d.format = int(fmt)
    return d


def pusch_eq_host_workspace(cells, cells_per_batch=0) -> int:
    """Device bytes that pusch_eq_host needs to stage these host cells."""
    arr = (CellDesc * len(cells))(*cells)
    b = _Z(0)
    _check(lib().aerial_pusch_eq_host_workspace(arr, len(cells), int(cells_per_batch), ctypes.byref(b)),
           "pusch_eq_host_workspace")
    return int(b.value)


def pusch_eq_host(cells, workspace, tuning: Tuning | None = None, cells_per_batch=0, stream=None):
    """The fused chain on host buffers (host_cell_desc cells): copies in,
    equalizes and copies the LLRs back, batches overlapped over three streams.
    Asynchronous on `stream`: synchronize it before reading the outputs."""
    arr = (CellDesc * len(cells))(*cells)
    tp = ctypes.pointer(tuning) if tuning is not None else None
    _check(lib().aerial_pusch_eq_host(arr, len(cells), tp, int(cells_per_batch), _ptr(workspace),
                                      workspace.numel() * workspace.element_size(), _stream(stream)),
           "pusch_eq_host")


def autotune(cells, precision=PREC_FP16, stream=None):
    """Pick the fastest group cap and launch shape for these cells; returns (Tuning, microseconds)."""
    arr, n = _cells_array(cells)
    t = make_tuning(precision)
    us = ctypes.c_float(0.0)
    _check(lib().aerial_autotune(arr, n, ctypes.pointer(t), ctypes.pointer(us), _stream(stream)), "autotune")
    return t, float(us.value)


class FusedGraph:
    """The fused launch for a fixed set of cell shapes as an executable CUDA graph.

    ``update(cells)`` re-points it at new buffers (same shapes); ``launch()``
    replays it.  Call ``close()`` (or use as a context manager) to free it."""

    def __init__(self, cells, tuning: Tuning | None = None):
        arr, n = _cells_array(cells)
        h = ctypes.c_void_p()
        tp = ctypes.pointer(tuning) if tuning is not None else None
        _check(lib().aerial_eq_graph_create(arr, n, tp, ctypes.byref(h)), "eq_graph_create")
        self._h = h

    def update(self, cells):
        arr, n = _cells_array(cells)
        _check(lib().aerial_eq_graph_update(self._h, arr, n), "eq_graph_update")

    def launch(self, stream=None):
        _check(lib().aerial_eq_graph_launch(self._h, _stream(stream)), "eq_graph_launch")

    def close(self):
        if self._h:
            _check(lib().aerial_eq_graph_destroy(self._h), "eq_graph_destroy")
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """The slot-serving loop (continuous batching into fused launches).

    Cells are registered with ``add_cell`` and keep their channel resident;
    ``submit`` queues one slot (device tensors in / out) and returns its id;
    completions come back through ``poll`` / ``wait`` / ``drain``; ``stats``
    reports p50/p99 latency, deadline misses and REs/s."""

    def __init__(self, memory_budget_bytes=16 << 30, streams=3, max_batch=64, precision=PREC_FP16,
                 mode=SERVER_FUSED, queue_capacity=0, start_paused=False, deadline_us=500.0,
                 batch_window_us=0.0, min_batch=0):
        if isinstance(precision, str):
            precision = PREC_NAMES[precision]
        cfg = ServerConfig(int(memory_budget_bytes), int(streams), int(max_batch), int(precision), int(mode),
                           int(queue_capacity), int(bool(start_paused)), float(deadline_us),
                           float(batch_window_us), int(min_batch))
        h = ctypes.c_void_p()
        _check(lib().aerial_server_create(ctypes.byref(cfg), ctypes.byref(h)), "server_create")
        self._h = h

    def add_cell(self, nPRB, nAnt, nLayers, nSym, nPamBits, sigma2) -> int:
        cid = ctypes.c_int()
        _check(lib().aerial_server_add_cell(self._h, nPRB, nAnt, nLayers, nSym, nPamBits, float(sigma2),
                                            ctypes.byref(cid)), "server_add_cell")
        return cid.value

    def set_channel(self, cell, H, sigma2):
        _check(lib().aerial_server_set_channel(self._h, cell, ctypes.c_void_p(H.data_ptr()), float(sigma2)),
               "server_set_channel")

    def srs_update(self, cell, SRS, W, FOCC, K, foccLen, n_symbols=1) -> int:
        """Queue an SRS update of the cell's resident channel; n_symbols (1, 2
        or 4) consecutive SRS symbols in SRS are averaged."""
        rid = ctypes.c_uint64()
        _check(lib().aerial_server_srs_update_n(self._h, cell, _ptr(SRS), int(n_symbols), _ptr(W), _ptr(FOCC), K,
                                                foccLen, ctypes.byref(rid)), "server_srs_update")
        return rid.value

    def submit(self, cell, Y, llr_out, arrival_ns=0) -> int:
        rid = ctypes.c_uint64()
        _check(lib().aerial_server_submit(self._h, cell, _ptr(Y), _ptr(llr_out), int(arrival_ns),
                                          ctypes.byref(rid)), "server_submit")
        return rid.value

    def submit_status(self, cell, Y, llr_out, arrival_ns=0) -> int:
        """submit() returning the raw status instead of raising."""
        rid = ctypes.c_uint64()
        return lib().aerial_server_submit(self._h, cell, _ptr(Y), _ptr(llr_out), int(arrival_ns), ctypes.byref(rid))

    def poll(self, max_out=4096):
        buf = (ServerCompletion * max_out)()
        n = ctypes.c_int()
        _check(lib().aerial_server_poll(self._h, buf, max_out, ctypes.byref(n)), "server_poll")
        return [(buf[i].request_id, buf[i].cell_id, buf[i].status, buf[i].latency_us) for i in range(n.value)]

    def wait(self, request_id, timeout_ms=10000) -> int:
        return lib().aerial_server_wait(self._h, request_id, int(timeout_ms))

    def drain(self, timeout_ms=60000):
        _check(lib().aerial_server_drain(self._h, int(timeout_ms)), "server_drain")

    def pause(self, paused=True):
        _check(lib().aerial_server_pause(self._h, int(bool(paused))), "server_pause")

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().aerial_server_stats(self._h, ctypes.byref(st)), "server_stats")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def reset_stats(self):
        _check(lib().aerial_server_reset_stats(self._h), "server_reset_stats")

    def inject_alloc_failure(self, nth):
        """Fault injection for tests: the nth device allocation from now on fails (0 disarms)."""
        _check(lib().aerial_server_inject_alloc_failure(self._h, int(nth)), "server_inject_alloc_failure")

    def close(self):
        if self._h:
            _check(lib().aerial_server_destroy(self._h), "server_destroy")
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
