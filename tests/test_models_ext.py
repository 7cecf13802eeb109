"""Breg_jaffe (ring and bar), Breg_jf12 and TEreg_ymw16 on the device against
full maps computed by the reference integrator itself with the template's
parameters (tests/golden/ref_models_ext.npz, made by make_golden.py)."""
import ctypes as C
import os

import numpy as np
import pytest

import cases
from conftest import rel_err
from hammurabix_b200 import abi
from hammurabix_b200 import integrator as I

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("jaffe_ring_ymw16", "jaffe_bar_expdisk", "jf12_ymw16", "spiral_ymw16")
TOL64 = {"dm": 1e-10, "fd": 1e-10, "is": 1e-9, "qs": 1e-9, "us": 1e-9}
TOL32 = 1e-5


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "ref_models_ext.npz"))


def _models(golden, name):
    raw = golden[f"{name}/models"].tobytes()
    assert len(raw) == C.sizeof(abi.Models)
    return abi.Models.from_buffer_copy(raw)


def test_fixture_holds_every_case_and_model_block(golden):
    for name in NAMES:
        m = _models(golden, name)
        assert m.cre in (abi.HXG_CRE_ANA, abi.HXG_CRE_UNIF)
        for k in ("dm", "fd", "is", "qs", "us"):
            a = golden[f"{name}/pass0/{k}"]
            assert np.isfinite(a).all() and np.abs(a).max() > 0, (name, k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_gpu_models_ext_match_reference(golden, name, precision):
    m = _models(golden, name)
    o = cases.obs_models_ext()[0]
    with I.Integrator(precision) as integ:
        integ.set_models(m)
        got = integ.write_grid(o)
    for k, v in got.items():
        if v is None:
            continue
        e = rel_err(v, golden[f"{name}/pass0/{k}"])
        tol = TOL64[k] if precision == "fp64" else TOL32
        assert e <= tol, (name, precision, k, e)
