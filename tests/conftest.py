import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_oracle():
    import pyoracle
    if not os.path.exists(pyoracle.ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    import pyoracle
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def reference():
    import pyoracle
    if not os.path.exists(pyoracle.REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    return pyoracle.Reference()


@pytest.fixture(scope="session")
def fixtures():
    return dict(np.load(os.path.join(GOLDEN, "reference_fixtures.npz")))


@pytest.fixture(scope="session")
def ref_maps():
    return dict(np.load(os.path.join(GOLDEN, "ref_maps.npz")))


@pytest.fixture(scope="session")
def fields32(ref_maps):
    return tuple(ref_maps[f"fields32/{k}"] for k in ("bx", "by", "bz", "ne"))


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if b.size else 0.0
    d = np.abs(a - b).max() if b.size else 0.0
    if s == 0.0:
        return d
    return d / s


def point_err(a, b, floor=1e-3):
    """max |a - b| / |b| over the pixels where |b| > floor * max |b|: the
    pointwise relative error of a map away from its zero crossings (Q and U
    oscillate through zero, where a relative error means nothing)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if b.size == 0:
        return 0.0
    s = np.abs(b).max()
    if s == 0.0:
        return np.abs(a - b).max()
    sel = np.abs(b) > floor * s
    return float((np.abs(a - b)[sel] / np.abs(b[sel])).max())
