"""Shared pytest configuration: the ``gpu`` marker and fixture loading."""

from __future__ import annotations

import sys
from functools import lru_cache
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@lru_cache(maxsize=None)
def golden(name: str):
    """Load ``tests/golden/<name>.npz`` (frozen reference outputs)."""
    return np.load(GOLDEN / f"{name}.npz")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def device():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch

    return torch.device("cuda:0")
