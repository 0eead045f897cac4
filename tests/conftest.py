"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
CPU.  The oracle (oracle/) is imported here only as the checker."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reffn():
    """The reference's own scalar kernels built for the host (oracle/_ref)."""
    from oracle.oracle import RefFunctions
    if not RefFunctions.available():
        from oracle import build_ref
        ref = build_ref.reference_tree()
        if ref:
            build_ref.build(ref)
    if not RefFunctions.available():
        pytest.skip("reference functions not built (reference tree absent)")
    return RefFunctions()


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rel_linf(a, b):
    """max|a-b| / max|b| per field (leading axis = field)."""
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for i in range(a.shape[0]):
        den = np.max(np.abs(b[i]))
        out.append(np.max(np.abs(a[i] - b[i])) / (den if den > 0 else 1.0))
    return np.array(out)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for i in range(a.shape[0]):
        den = np.linalg.norm(b[i])
        out.append(np.linalg.norm(a[i] - b[i]) / (den if den > 0 else 1.0))
    return np.array(out)
