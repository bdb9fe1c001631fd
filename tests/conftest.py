"""Shared fixtures. ``-m gpu`` tests need a CUDA device and the in-tree library;
everything else runs on the CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


@pytest.fixture(scope="session")
def engine():
    """One device context for the session; fails loudly without a GPU."""
    from swiftimpute_b200.engine import Engine
    eng = Engine(0)
    yield eng
    eng.close()


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
