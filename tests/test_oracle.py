"""CPU tests: the oracle (oracle/hxo.c) against the reference's own unit-test
fixtures and against outputs of the reference integrator itself.

Mirrors hammurabiX's tests/unit_tests: hamdis_tests.cc (pointing,
accumulate, interpolation), hamsk_tests.cc (mask duplicate),
integrator_tests.cc (shell geometry, LOS versor/projections/IPA) and
grid_tests.cc (trilinear read of a linear field).
"""
import os

import numpy as np
import pytest

import cases
from conftest import GOLDEN, rel_err
from hammurabix_b200 import abi, units as U, workloads as W
from hammurabix_b200.param import Param


@pytest.mark.parametrize("nside", [2, 4, 8, 16, 32])
def test_pointing_vs_healpy(oracle, fixtures, nside):
    """hamdis_tests.cc:156-232: RING pix2ang vs healpy to 1e-10."""
    th, ph = oracle.pix2ang(nside)
    ref = fixtures[f"pointing_nside{nside}"]
    assert np.abs(th - ref[:, 0]).max() < 1e-10
    assert np.abs(ph - ref[:, 1]).max() < 1e-10


def test_accumulate_constant_maps(oracle):
    """hamdis_tests.cc:297-318."""
    m = np.zeros(192)
    m = oracle.accumulate(4, m, 4, np.ones(192))
    assert np.all(m == 1.0)
    m = oracle.accumulate(4, m, 2, np.full(48, 2.0))
    assert np.all(m == 3.0)
    m = oracle.accumulate(4, m, 8, np.full(768, 2.0))
    assert np.all(m == 5.0)


def test_interpolation_fixture(oracle, fixtures):
    """hamdis_tests.cc:320-370: up/down-grade of a random Nside-4 map."""
    base = fixtures["random_map_nside4"]
    low = oracle.accumulate(2, np.zeros(48), 4, base)
    high = oracle.accumulate(8, np.zeros(768), 4, base)
    assert np.abs(low - fixtures["random_map_nside2"]).max() < 1e-10
    assert np.abs(high - fixtures["random_map_nside8"]).max() < 1e-10


def test_mask_duplicate_fixture(oracle, fixtures):
    """hamsk_tests.cc:33-55: mask downgrade 8->2 and upgrade 8->64."""
    m8 = fixtures["mask_map_nside8"]
    assert np.array_equal(oracle.mask_duplicate(8, m8, 2), fixtures["mask_map_nside2"])
    assert np.array_equal(oracle.mask_duplicate(8, m8, 64), fixtures["mask_map_nside64"])
    zero = np.zeros(192)
    assert np.all(oracle.mask_duplicate(4, zero, 2) == 0)
    assert np.all(oracle.mask_duplicate(4, zero, 8) == 0)


def test_shell_geometry_auto(oracle):
    """integrator_tests.cc:28-81 with reference/int_tests_01.xml."""
    par = Param(os.path.join(GOLDEN, "int_tests_01.xml"))
    assert par.sync_freqs == [23.0 * U.GHz, 1.4 * U.GHz]
    assert par.nside_shell == [32, 64, 128]
    o = par.obs_pass(0)
    ds, dd, st = oracle.shell_ref(o, 0)
    assert st == 333
    assert ds == 5 * U.kpc
    assert abs(dd - (10 * U.kpc) / 333) < 1e-10 * U.kpc
    ds, dd, st = oracle.shell_ref(o, 2)
    assert st == 666
    assert ds == 40 * U.kpc / 2 + 5 * U.kpc
    assert abs(dd - (20 * U.kpc) / 666) < 1e-10 * U.kpc


def test_shell_geometry_manual(oracle):
    """integrator_tests.cc:82-139 with reference/int_tests_02.xml."""
    par = Param(os.path.join(GOLDEN, "int_tests_02.xml"))
    assert par.nside_shell == [32, 16, 8]
    o = par.obs_pass(0)
    expect = [(100, 0., 3.), (600, 0.1 * 30, 18.), (300, 0.7 * 30, 9.)]
    for s, (steps, dstart_kpc, span_kpc) in enumerate(expect):
        ds, dd, st = oracle.shell_ref(o, s)
        assert st == steps
        assert abs(ds - dstart_kpc * U.kpc) <= 1e-12 * U.kpc
        assert abs(dd - span_kpc * U.kpc / steps) < 1e-10 * U.kpc


def test_shell_geometry_vs_reference(oracle, reference):
    par = Param(os.path.join(GOLDEN, "int_tests_01.xml"))
    o = par.obs_pass(0)
    for s in range(3):
        ds, dd, st = oracle.shell_ref(o, s)
        rds, rdd, rst, dist = reference.shell_ref(o, s)
        assert (ds, dd, st) == (rds, rdd, rst)
        assert np.array_equal(dist, ds + (np.arange(st) + 0.5) * dd)


def test_los_known_answers(oracle):
    """integrator_tests.cc:143-209."""
    theta = np.array([0., 90. * U.rad, 90. * U.rad])
    phi = np.array([0., 180. * U.rad, 270. * U.rad])
    b = np.tile([1., 0., 0.], (3, 1))
    ver, par, per, ipa = oracle.los_geometry(theta, phi, b)
    assert np.abs(ver - [[0, 0, 1], [-1, 0, 0], [0, -1, 0]]).max() < 1e-10
    assert np.abs(par - [0., -1., 0.]).max() < 1e-10
    assert np.abs(per - [1., 0., 1.]).max() < 1e-10
    assert abs(ipa[0] + 90. * U.rad) < 1e-10
    assert abs(ipa[2] - 180. * U.rad) < 1e-10


def _linear_grid():
    """grid_tests.cc:24-96 fill functions on the 10 x 8 x 29 unit box."""
    d = abi.GridDesc()
    d.nx, d.ny, d.nz = 10, 8, 29
    d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max = 0., 1., 0., 1., 0., 1.
    i, j, k = np.meshgrid(np.arange(10), np.arange(8), np.arange(29), indexing="ij")
    x = i * 1.0 / 9 + 0.
    y = j * 1.0 / 7 + 0.
    z = k * 1.0 / 28 + 0.
    return d, x.reshape(-1), y.reshape(-1), z.reshape(-1)


def test_trilinear_linear_field(oracle):
    """grid_tests.cc:137-260: a linear field is reproduced exactly."""
    d, x, y, z = _linear_grid()
    rng = np.random.Generator(np.random.PCG64(3))
    pos = rng.random((64, 3))
    b = oracle.read_grid(d, [x, y, z], pos)
    assert np.abs(b - pos).max() < 1e-10
    te = oracle.read_grid(d, [x + y + z], pos)
    assert np.abs(te - pos.sum(1)).max() < 1e-10
    # zero on and outside the box surface (breg.cc:34-54)
    out = oracle.read_grid(d, [x, y, z], np.array([[0., .5, .5], [1., .5, .5], [.5, .5, 1.2]]))
    assert np.all(out == 0)


def _compare_case(oracle, ref_maps, key, passes, m, grids, mask, tol=1e-13):
    for i, o in enumerate(passes):
        kw = {} if mask is None else dict(mask_nside=mask[0], mask=mask[1])
        got = oracle.write_grid(o, m, grids, **kw)
        for k, v in got.items():
            if v is None:
                continue
            ref = ref_maps[f"{key}/pass{i}/{k}"]
            assert rel_err(v, ref) <= tol, (key, i, k, rel_err(v, ref))


def test_oracle_vs_reference_config1(oracle, ref_maps):
    _compare_case(oracle, ref_maps, "config1", *cases.case_config1())


def test_oracle_vs_reference_grids(oracle, ref_maps, fields32):
    _compare_case(oracle, ref_maps, "grid_small", *cases.case_grid_small(fields32))
    _compare_case(oracle, ref_maps, "grid_lowfreq", *cases.case_grid_lowfreq(fields32))


def test_oracle_vs_reference_mask(oracle, ref_maps):
    _compare_case(oracle, ref_maps, "mask", *cases.case_mask())


def test_oracle_vs_reference_models(oracle, ref_maps):
    for name, passes, m in cases.case_models():
        _compare_case(oracle, ref_maps, f"model_{name}", passes, m, None, None)


def test_oracle_vs_reference_live(oracle, reference):
    """Two grid geometries, DM only, against the reference run live."""
    passes, m, g, mask = cases.case_dm_only()
    got = oracle.write_grid(passes[0], m, g)
    ref, _ = reference.write_grid(passes[0], m, g)
    assert rel_err(got["dm"], ref["dm"]) <= 1e-13
    assert np.abs(ref["dm"]).max() > 0


def test_emissivity_vs_reference(oracle, reference):
    """sync_emissivity_t/_p (integrator.cc:282-420), analytic branch."""
    m = W.spiral_models()
    rng = np.random.Generator(np.random.PCG64(4))
    pos = (rng.random((16, 3)) - 0.5) * np.array([30., 30., 4.]) * U.kpc
    bper = rng.random(16) * 5e-6
    obs = [v * U.kpc for v in W.OBSERVER_KPC]
    for beta in (0.0, 0.07):
        m.cre_ana.beta = beta
        jt, jp = oracle.sync_emissivity(m, obs, 1.4 * U.GHz, pos, bper)
        rt, rp = reference.sync_emissivity(m, obs, 1.4 * U.GHz, pos, bper)
        assert rel_err(jt, rt) < 1e-14 and rel_err(jp, rp) < 1e-14


def test_temp_convert_vs_reference(oracle, reference):
    for f in (0.408, 1.4, 23.0, 30.0):
        assert oracle.temp_convert(1.234, f * U.GHz) == reference.temp_convert(1.234, f * U.GHz)
