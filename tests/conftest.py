"""Shared test set-up: import paths, the ``gpu`` marker, and the seeded cases."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for path in (ROOT / "ad-tlert_b200", ROOT / "tests" / "golden", ROOT):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA GPU (B200 kernels of libadtlert_b200)")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="requires a CUDA GPU")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def assert_close(actual, expected, tol, what=""):
    """Max-norm relative comparison (the reference's own test metric): sums with cancellation
    are accurate relative to their largest term."""

    import numpy as np

    actual, expected = np.asarray(actual, dtype=float), np.asarray(expected, dtype=float)
    assert actual.shape == expected.shape, f"{what}: shape {actual.shape} != {expected.shape}"
    error = np.abs(actual - expected).max() / max(np.abs(expected).max(), 1e-300)
    assert error < tol, f"{what}: relative max-norm error {error:.2e} >= {tol:.0e}"
    return error
