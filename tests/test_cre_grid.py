"""CRE-grid synchrotron emissivity (integrator.cc:282-330, 351-400;
CREfield::read_grid_num, cre.cc:144-199).

The reference evaluates F(x) and G(x) with GSL (gsl_sf_synchrotron_1/2),
which is not part of the reference tree and not installed here; its parity
is unpinned at that boundary.  The library's tables are checked against
scipy (Bessel K by Amos' algorithm, quadrature for F), and the full maps
against the reference integrator compiled with the oracle's own F and G
(oracle/shim/shim.cc, from the same integral definitions)."""
import os

import numpy as np
import pytest

import cases
from conftest import rel_err
from hammurabix_b200 import abi, units as U, workloads as W
from hammurabix_b200 import integrator as I

HERE = os.path.dirname(os.path.abspath(__file__))


def test_synchrotron_tables_match_scipy():
    special = pytest.importorskip("scipy.special")
    integrate = pytest.importorskip("scipy.integrate")
    xs = np.array([1e-9, 1e-6, 1e-3, 0.05, 0.29, 1.0, 3.0, 10.0, 30.0, 80.0])
    F = I.synchrotron(1, xs)
    G = I.synchrotron(2, xs)
    for x, f, g in zip(xs, F, G):
        # F = x Int_x^inf K_5/3 over [x, x+60] in u = ln t (the tail beyond
        # is below e^-60 of the value)
        u1 = np.log(x + 60.)
        fi = integrate.quad(lambda u: special.kv(5. / 3., np.exp(u)) * np.exp(u), np.log(x), u1,
                            epsabs=0, epsrel=1e-13, limit=2000)[0] * x
        gi = x * special.kv(2. / 3., x)
        assert abs(f / fi - 1.) < 1e-9, (x, f, fi)
        assert abs(g / gi - 1.) < 1e-9, (x, g, gi)
    assert np.all(I.synchrotron(1, np.array([0., -1.])) == 0.)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("fp32c", 1e-5)])
def test_gpu_cre_grid_matches_reference(precision, tol):
    golden = np.load(os.path.join(HERE, "golden", "ref_cre_grid.npz"))
    passes, m, grids = cases.case_cre_grid()
    with I.Integrator(precision) as integ:
        integ.set_models(m)
        for field, (desc, comps) in grids.items():
            integ.upload_grid(field, desc, comps)
        for i, o in enumerate(passes):
            got = integ.write_grid(o)
            for k, v in got.items():
                if v is None:
                    continue
                ref = golden[f"cre_grid/pass{i}/{k}"]
                t = 1e-10 if (precision == "fp64" and k in ("dm", "fd")) else tol
                assert rel_err(v, ref) <= t, (precision, i, k, rel_err(v, ref))
                assert np.abs(ref).max() > 0
