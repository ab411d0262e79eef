"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The engine package lives in ``webgpu-fluid-sim_b200/`` (a name with hyphens),
so it is loaded through importlib.  The oracle (``oracle/``) is the checker.
"""
from __future__ import annotations

import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs the CUDA engine")


def load_engine():
    return importlib.import_module("webgpu-fluid-sim_b200")


@pytest.fixture(scope="session")
def bh():
    pkg = load_engine()
    pkg.load()  # fails loudly when libbh_b200.so is missing
    return pkg


@pytest.fixture(scope="session")
def orc():
    import oracle  # noqa: WPS433  (oracle/oracle.py)
    oracle.load()
    return oracle
