"""Test configuration: the `gpu` marker and shared fixtures.

CPU tests (``-m "not gpu"``) cover the oracle against independent references
and its committed fixtures, the library's host-side tables, and the C ABI's
exported symbols.  GPU tests (``-m gpu``) compare the CUDA library, called
through its C ABI, with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def chylib():
    """The product library, built in-tree if missing."""
    from chymera_uo_b200 import build as b
    if not os.path.exists(b.LIB):
        b.build()
    import chymera_uo_b200 as chy
    return chy


@pytest.fixture(scope="session")
def ora():
    from oracle import oracle as O
    O.build()
    return O
