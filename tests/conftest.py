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


def r2_masked(got, want, codes) -> float:
    """Squared Pearson correlation of two dosage arrays over the masked (untyped)
    cells, where imputation happens; typed cells reproduce the call in both."""
    m = np.asarray(codes) == 3
    x, y = np.asarray(got, np.float64)[m], np.asarray(want, np.float64)[m]
    if x.size < 2 or x.std() == 0 or y.std() == 0:
        return 1.0 if np.array_equal(x, y) else 0.0
    return float(np.corrcoef(x, y)[0, 1] ** 2)


def report(name: str, **values) -> None:
    """Record measured parity figures of a test in $SI_REPORT_DIR/parity.json (when set)."""
    import json
    import os
    d = os.environ.get("SI_REPORT_DIR")
    if not d:
        return
    path = Path(d) / "parity.json"
    data = json.loads(path.read_text()) if path.exists() else {}
    data[name] = {k: (float(v) if isinstance(v, (np.floating, float)) else v) for k, v in values.items()}
    path.write_text(json.dumps(data, indent=1, sort_keys=True))
