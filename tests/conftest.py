"""Shared pytest configuration: the ``gpu`` marker and repository paths."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")
    config.addinivalue_line("markers", "slow: long-running CPU check")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return {
        "planes": np.load(GOLDEN / "ocl_planes.npz"),
        "farfield": np.load(GOLDEN / "ocl_farfield.npz"),
        "numpy": np.load(GOLDEN / "numpy_ref.npz"),
    }
