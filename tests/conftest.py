"""Shared fixtures for the equalization-path tests.

Markers: ``gpu`` -- needs a CUDA device (parity tests through the C ABI).
Tests without the marker run on CPU only (oracle vs golden vectors, host
logic, and that the C-ABI library loads and exports every declared symbol).
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

PKG_NAME = "aerial-mimo-tc-optimization_b200"
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_pkg():
    return importlib.import_module(PKG_NAME)


def load_workload():
    return importlib.import_module(PKG_NAME + ".workload")


@pytest.fixture(scope="session")
def aeq():
    return load_pkg()


@pytest.fixture(scope="session")
def wl():
    return load_workload()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


# ---------------------------------------------------------------------------
# metrics (the reference's host checks, src/aerial_coef_wmma.cu:340-354 and
# src/coef_rigor.cu:132-138, in numpy)
# ---------------------------------------------------------------------------

def evm_db(test, ref) -> float:
    t = np.asarray(test, np.complex128).reshape(-1)
    r = np.asarray(ref, np.complex128).reshape(-1)
    num = float(np.sum(np.abs(t - r) ** 2))
    den = float(np.sum(np.abs(r) ** 2))
    return 10.0 * np.log10(max(num, 1e-300) / den)


def cosine(a, b) -> float:
    a = np.asarray(a, np.complex128).reshape(-1)
    b = np.asarray(b, np.complex128).reshape(-1)
    dot = float(np.sum(a.real * b.real + a.imag * b.imag))
    return dot / (np.sqrt(np.sum(np.abs(a) ** 2)) * np.sqrt(np.sum(np.abs(b) ** 2)) + 1e-30)


def max_rel_err(test, ref) -> float:
    t = np.asarray(test, np.complex128).reshape(-1)
    r = np.asarray(ref, np.complex128).reshape(-1)
    e2 = np.abs(t - r) ** 2
    r2 = np.abs(r) ** 2
    rel = np.where(r2 > 1e-9, np.sqrt(e2 / np.where(r2 > 0, r2, 1.0)), 0.0)
    return float(rel.max())
