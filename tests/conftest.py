"""Pytest configuration: the `gpu` marker and shared builders/helpers.

`-m "not gpu"` runs here without a GPU (oracle pins, host logic, ABI
surface); `-m gpu` runs the CUDA parity tests through the C ABI.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle_lib():
    """The oracle library, built on demand (test infrastructure)."""
    from oracle import build as ob
    ob.build_oracle()
    from oracle import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def product_lib_path():
    from heliocubed_b200 import _native
    if not os.path.exists(_native.LIB_PATH):
        from heliocubed_b200 import build
        build.build()
    return _native.LIB_PATH


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def rel_err_components(a: np.ndarray, b: np.ndarray, comp_axis: int = 1) -> np.ndarray:
    """Per-component normwise relative error max|a-b| / max|b|."""
    a = np.moveaxis(np.asarray(a), comp_axis, 0).reshape(8, -1)
    b = np.moveaxis(np.asarray(b), comp_axis, 0).reshape(8, -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return np.abs(a - b).max(axis=1) / scale
