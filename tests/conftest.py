"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and call the B200 library through
its C ABI; the rest run on CPU (oracle pinning, golden vectors, host logic,
library symbol table).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_port():
    from oracle import oracle
    return oracle.get("port")


@pytest.fixture(scope="session")
def oracle_ref():
    from oracle import oracle
    if not oracle.ref_available():
        pytest.skip("compiled reference not available")
    return oracle.get("ref")


@pytest.fixture(scope="session")
def lib():
    from yoricktrtt_b200 import _lib
    return _lib.load()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
