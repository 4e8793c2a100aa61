"""Shared fixtures and markers.  GPU tests are marked ``gpu``; everything else runs on CPU."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
SEED = 20261014


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture
def rng() -> np.random.Generator:
    return np.random.default_rng(SEED)


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def check(name, expected, actual, rtol=None, atol=None, per_vector=False):
    """Assert |actual - expected| <= atol + rtol |expected| elementwise (exact when neither
    tolerance is given); per_vector measures 3-vectors by their length."""
    if rtol is None and atol is None:
        ok = bool(np.all(np.asarray(expected) == np.asarray(actual)))
        assert ok, f"{name}: not equal"
        return
    e = np.asarray(expected, np.float64)
    a = np.asarray(actual, np.float64)
    assert e.shape == a.shape or e.size == 1, f"{name}: shape {e.shape} vs {a.shape}"
    if per_vector:
        err = np.linalg.norm(a - e, axis=-1)
        size = np.linalg.norm(np.broadcast_to(e, a.shape), axis=-1)
    else:
        err = np.abs(a - e)
        size = np.abs(np.broadcast_to(e, a.shape))
    limit = (atol or 0.0) + (rtol or 0.0) * size
    bad = ~(err <= limit)
    assert not np.any(bad), (
        f"{name}: {int(bad.sum())} of {bad.size} outside tolerance; worst err "
        f"{float(np.max(err - limit)):.3g} beyond limit"
    )
