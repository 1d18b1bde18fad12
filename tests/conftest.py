"""Shared pytest setup: import paths, the `gpu` marker, and the oracle library build."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "physicssimulation-agony_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
LIB_DIR = os.path.join(PKG, "ag2d")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and the built CUDA library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oraapi
    oraapi.build()
    return oraapi.lib()
