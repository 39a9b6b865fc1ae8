"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: large problem sizes")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from bfam_b200 import build
    build.build_product()
    build.build_oracle()
    yield


def relerr(a, b):
    """per-field relative L2 error of a against b (arrays [field][n])."""
    import numpy as np
    a = np.asarray(a).reshape(a.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    den = np.sqrt((b ** 2).sum(axis=1))
    num = np.sqrt(((a - b) ** 2).sum(axis=1))
    scale = max(den.max(), 1e-300)
    # a field that is identically (or nearly) zero is measured against the
    # largest field's norm
    return num / np.where(den > 1e-8 * scale, den, scale)
