"""Shared test setup: markers, import paths, library/oracle fixtures.

`-m "not gpu"` tests run anywhere (CPU): oracle pins against the golden
fixtures and the compiled reference, host logic, and that libmrt.so loads and
exports what include/mrt.h declares. `-m gpu` tests call the CUDA path
through the C-ABI and compare with the oracle.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
PKG = REPO / "42-minirt_b200"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO))

GOLDEN = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls libmrt.so")
    config.addinivalue_line("markers", "slow: longer CPU-only oracle runs")


@pytest.fixture(scope="session")
def mrt():
    import mrt as m
    return m


@pytest.fixture(scope="session")
def scenes():
    import scenes as s
    return s


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


@pytest.fixture(scope="session")
def has_reference():
    import oracle as o
    return o.REF_LIB.exists()


def golden(name: str):
    return np.load(GOLDEN / name, allow_pickle=False)
