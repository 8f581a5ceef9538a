"""Shared test set-up: the `gpu` marker, library builds and small helpers."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def lq():
    """The product package with its CUDA library built in-tree."""
    import loquat_b200
    from loquat_b200 import build

    if not loquat_b200.lib_path().exists():
        build.build()
    loquat_b200.lib()
    return loquat_b200


@pytest.fixture(scope="session")
def orc():
    """The test-only FP64 oracle."""
    import oracle

    if not oracle.LIB.exists():
        oracle.build(ref=False)
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


def rel_l2(a, b, axis=None) -> float:
    """||a - b|| / ||b|| (0 when both are zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    num = np.linalg.norm((a - b).ravel())
    den = np.linalg.norm(b.ravel())
    if den == 0.0:
        return float(num)
    return float(num / den)
