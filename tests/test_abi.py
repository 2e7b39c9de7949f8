"""CPU tests of the C-ABI boundary: the library loads and exports every symbol
declared in include/aerial_eq.h; no kernel is launched."""
from __future__ import annotations

import ctypes
import os
import re

from conftest import ROOT, load_pkg


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "aerial_eq.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aerial_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("aerial_coef_apply", "aerial_gram", "aerial_mmse_coef", "aerial_llr", "aerial_llr_f32",
              "aerial_srs_filter", "aerial_pusch_eq_fused", "aerial_pusch_eq_plain"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    pkg = load_pkg()
    lib = ctypes.CDLL(pkg.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    pkg = load_pkg()
    assert set(declared_symbols()) <= set(pkg.SIGNATURES)
    pkg.lib()  # binds all signatures (raises if a symbol is absent)


def test_error_strings_and_version_without_gpu():
    pkg = load_pkg()
    lib = pkg.lib()
    assert lib.aerial_version() >= 10000
    assert b"invalid" in lib.aerial_error_string(1001)
    assert lib.aerial_error_string(0) == b"ok"


def test_invalid_arguments_rejected_before_any_launch():
    """Null pointers and out-of-envelope shapes return a status, never exit()."""
    pkg = load_pkg()
    lib = pkg.lib()
    assert lib.aerial_coef_apply(None, None, None, 10, 11, 8, 64, None) == 1001
    assert lib.aerial_gram(None, 0.1, None, 10, 64, 8, None) == 1001
    assert lib.aerial_llr(None, None, None, 10, 4, None) == 1001
    fake = ctypes.c_void_p(0x100000)
    assert lib.aerial_llr(fake, fake, fake, 10, 5, None) == 1001       # nPamBits > 4
    assert lib.aerial_coef_apply(fake, fake, fake, 10, 17, 8, 64, None) == 1001   # nSym > 16
    assert lib.aerial_coef_apply(fake, fake, fake, 10, 11, 17, 64, None) == 1001  # nLayers > 16
    assert lib.aerial_srs_filter(fake, fake, fake, fake, 64, 66, 49, 4, 8, None) == 1001   # K > 48
    assert lib.aerial_chest_interp(fake, fake, fake, fake, 64, 34, 97, 96, 4, 4, None) == 1001  # nPilot > 96
    assert lib.aerial_chest_interp(fake, fake, fake, fake, 64, 34, 96, 0, 4, 4, None) == 1001   # nOut < 1
    assert lib.aerial_chest_interp(None, fake, fake, fake, 64, 34, 96, 96, 4, 4, None) == 1001
    assert lib.aerial_chest_interp_h(fake, fake, fake, fake, 64, 34, 97, 96, 4, 4, None) == 1001
    assert lib.aerial_chest_interp_h(None, fake, fake, fake, 64, 34, 96, 96, 4, 4, None) == 1001
    assert lib.aerial_srs_to_channel_avg(fake, fake, 3, fake, fake, 64, 66, 12, 4, 4, None) == 1001
    assert lib.aerial_srs_to_channel_avg(None, fake, 4, fake, fake, 64, 66, 12, 4, 4, None) == 1001
    assert lib.aerial_server_srs_update_n(None, 0, fake, 4, fake, fake, 12, 4, None) == 1001
    assert lib.aerial_kernel_timeouts(None) == 1001
    cells = (pkg.CellDesc * 1)()
    assert lib.aerial_pusch_eq_fused(cells, 1, None, None) == 1001     # null buffers
    assert lib.aerial_pusch_eq_fused(cells, 0, None, None) == 1001
    assert lib.aerial_pusch_eq_fused(cells, 65, None, None) == 1001


def test_server_rejects_bad_config_without_gpu():
    """Host-side argument checks of the serving loop (no device needed)."""
    pkg = load_pkg()
    lib = pkg.lib()
    h = ctypes.c_void_p()
    assert lib.aerial_server_create(None, ctypes.byref(h)) == 1001
    cfg = pkg.ServerConfig(0, 2, 64, 0, 0, 0, 0, 500.0, 0.0, 0)   # zero budget
    assert lib.aerial_server_create(ctypes.byref(cfg), ctypes.byref(h)) == 1001
    cfg = pkg.ServerConfig(1 << 30, 0, 64, 0, 0, 0, 0, 500.0, 0.0, 0)   # no stream
    assert lib.aerial_server_create(ctypes.byref(cfg), ctypes.byref(h)) == 1001
    assert lib.aerial_server_destroy(None) == 1001
    assert lib.aerial_server_inject_alloc_failure(None, 1) == 1001
    n = ctypes.c_int()
    assert lib.aerial_server_poll(None, None, 0, ctypes.byref(n)) == 1001


def test_host_pipeline_workspace_and_checks_without_gpu():
    """Workspace sizing and argument checks of aerial_pusch_eq_host run on the
    host: three slots of the largest batch, every buffer 256-byte aligned."""
    pkg = load_pkg()
    lib = pkg.lib()
    fake = 0x100000
    def desc(nPRB, nAnt, nLayers, nSym, nPam, yeq=False):
        return pkg.CellDesc(fake, fake, fake, fake if yeq else None, 0.1, nPRB, nAnt, nLayers, nSym, nPam)
    al = lambda v: (v + 255) // 256 * 256
    def foot(p, a, l, s, n, yeq=False):
        sc = 12 * p
        return al(sc * a * l * 8) + al(sc * s * a * 8) + al(sc * l * s * 2 * n * 4) + (al(sc * l * s * 8) if yeq else 0)
    cells = [desc(132, 64, 8, 11, 4), desc(24, 32, 4, 11, 2, True), desc(273, 128, 16, 11, 4),
             desc(51, 16, 2, 14, 1), desc(106, 64, 4, 11, 3)]
    arr = (pkg.CellDesc * 5)(*cells)
    b = ctypes.c_size_t(0)
    assert lib.aerial_pusch_eq_host_workspace(arr, 5, 2, ctypes.byref(b)) == 0
    f = [foot(132, 64, 8, 11, 4), foot(24, 32, 4, 11, 2, True), foot(273, 128, 16, 11, 4), foot(51, 16, 2, 14, 1),
         foot(106, 64, 4, 11, 3)]
    assert b.value == 3 * max(f[0] + f[1], f[2] + f[3], f[4])
    assert lib.aerial_pusch_eq_host_workspace(arr, 1, 0, ctypes.byref(b)) == 0
    assert b.value == f[0]                      # one batch, one slot
    assert lib.aerial_pusch_eq_host_workspace(arr, 5, -1, ctypes.byref(b)) == 1001
    assert lib.aerial_pusch_eq_host_workspace(None, 5, 0, ctypes.byref(b)) == 1001
    bad = (pkg.CellDesc * 1)(desc(132, 64, 17, 11, 4))
    assert lib.aerial_pusch_eq_host_workspace(bad, 1, 0, ctypes.byref(b)) == 1001
    wide = (pkg.CellDesc * 1)(desc(pkg.MAX_PRB + 1, 16, 2, 11, 4))   # beyond AERIAL_MAX_PRB
    assert lib.aerial_pusch_eq_host_workspace(wide, 1, 0, ctypes.byref(b)) == 1001
    wide[0].nPRB = pkg.MAX_PRB
    assert lib.aerial_pusch_eq_host_workspace(wide, 1, 0, ctypes.byref(b)) == 0
    ws = ctypes.c_void_p(0x200000)
    assert lib.aerial_pusch_eq_host(arr, 5, None, 2, ws, 1024, None) == 1001         # workspace too small
    assert lib.aerial_pusch_eq_host(arr, 5, None, 2, ctypes.c_void_p(0x200010), 1 << 40, None) == 1001  # misaligned
    assert lib.aerial_pusch_eq_host(bad, 1, None, 0, ws, 1 << 40, None) == 1001


def test_fp16_operand_scale_window():
    """The host-side FP16 operand scale: 1 inside the window the header
    states, else an exact power of two putting s^2 sigma2 in [2^-10, 2^-8)."""
    import math
    pkg = load_pkg()
    for s2 in (2.0 ** -16, 0.001, 0.01, 1.0, 2.0 ** 7 * 0.999, 0.0, float("inf"), float("nan")):
        assert pkg.fp16_operand_scale(s2) == 1.0
    for s2 in (2.0 ** -16 * 0.999, 1e-9, 1e-20, 2.0 ** 7, 1e6, 1e20):
        s = pkg.fp16_operand_scale(s2)
        e = math.log2(s)
        assert s != 1.0 and e == int(e)
        v = ctypes.c_float(s2).value * s * s          # the float32 sigma2 the kernel sees
        assert 2.0 ** -10 <= v < 2.0 ** -8, (s2, s, v)
