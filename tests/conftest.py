"""Shared pytest setup.

Markers: ``gpu`` tests need a B200 and the built libspk.so; everything else
runs on a CPU-only machine (oracle, fixtures, host logic, ABI exports).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "spades-rs_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and libspk.so")


@pytest.fixture(scope="session")
def ora():
    from oracle import ora as _ora
    _ora.build()
    return _ora


@pytest.fixture(scope="session")
def spk_lib():
    """libspk.so, built in-tree if it is missing (nvcc cross-compiles without a GPU)."""
    import spk
    from spk import _lib
    if not os.path.exists(_lib.lib_path()):
        _lib.build()
    return spk
