"""GPU parity tests: the sm_100a kernels, called through the C ABI, against
the reference's own fixtures, outputs of the reference integrator
(tests/golden/ref_maps.npz) and the CPU oracle.

Tolerances (max |gpu - ref| / max |ref| per map):
  FP64 form:  DM and FD <= 1e-10 (the reference's FP64 integrator);
              I, Q, U   <= 1e-9
  FP32C form: every map <= 1e-5 against the FP64 oracle.
"""
import numpy as np
import pytest

import cases
from conftest import rel_err
from hammurabix_b200 import _lib, abi, units as U, workloads as W
from hammurabix_b200 import integrator as I

pytestmark = pytest.mark.gpu

TOL64 = {"dm": 1e-10, "fd": 1e-10, "is": 1e-9, "qs": 1e-9, "us": 1e-9}
TOL32 = 1e-5
# FP32-compensated form on the strong-rotation stress case (0.408 GHz, 0.05 kpc
# steps: ~600 samples through thousands of radians of Faraday rotation).  The
# FP32 trilinear interpolation of the gridded n_e and B rounds each sample by
# ~1 ulp at random; the running Faraday phase random-walks that into
# ~1e-5 of Q/U.  On 0.01-kpc steps (five times the samples, a fifth of the
# phase per sample) the same form stays below TOL32.
TOL32_STRONG = 3e-5


def _run_gpu(precision, passes, m, grids, mask):
    outs = []
    with I.Integrator(precision) as integ:
        integ.set_models(m)
        for field, (desc, comps) in (grids or {}).items():
            integ.upload_grid(field, desc, comps)
        if mask is not None:
            integ.set_mask(mask[0], mask[1])
        for o in passes:
            outs.append(integ.write_grid(o))
    return outs


def _check_vs_golden(ref_maps, key, passes, m, grids, mask):
    outs = _run_gpu("fp64", passes, m, grids, mask)
    for i, got in enumerate(outs):
        for k, v in got.items():
            if v is None:
                continue
            ref = ref_maps[f"{key}/pass{i}/{k}"]
            e = rel_err(v, ref)
            assert e <= TOL64[k], (key, i, k, e)
            assert np.abs(ref).max() > 0 or k == "fd", (key, k)


# ---- device known-answer helpers ------------------------------------------

@pytest.mark.parametrize("nside", [2, 4, 8, 16, 32])
def test_gpu_pointing_vs_healpy(fixtures, nside):
    th, ph = I.pix2ang(nside)
    ref = fixtures[f"pointing_nside{nside}"]
    assert np.abs(th - ref[:, 0]).max() < 1e-10
    assert np.abs(ph - ref[:, 1]).max() < 1e-10


def test_gpu_accumulate_and_interpolate(fixtures):
    m = I.accumulate(4, np.zeros(192), 4, np.ones(192))
    m = I.accumulate(4, m, 2, np.full(48, 2.0))
    m = I.accumulate(4, m, 8, np.full(768, 2.0))
    assert np.all(m == 5.0)
    base = fixtures["random_map_nside4"]
    assert np.abs(I.accumulate(2, np.zeros(48), 4, base)
                  - fixtures["random_map_nside2"]).max() < 1e-10
    assert np.abs(I.accumulate(8, np.zeros(768), 4, base)
                  - fixtures["random_map_nside8"]).max() < 1e-10


def test_gpu_interpolate_vs_oracle(oracle):
    rng = np.random.Generator(np.random.PCG64(1))
    m = rng.random(abi.npix(16))
    th = rng.random(1000) * np.pi
    ph = rng.random(1000) * 2 * np.pi
    assert np.abs(I.interpolate(16, m, th, ph) - oracle.interpolate(16, m, th, ph)).max() < 1e-13


def test_gpu_los_geometry(oracle):
    theta = np.array([0., 90. * U.rad, 90. * U.rad])
    phi = np.array([0., 180. * U.rad, 270. * U.rad])
    b = np.tile([1., 0., 0.], (3, 1))
    ver, par, per, c2, s2 = I.los_geometry(theta, phi, b)
    assert np.abs(ver - [[0, 0, 1], [-1, 0, 0], [0, -1, 0]]).max() < 1e-10
    assert np.abs(par - [0., -1., 0.]).max() < 1e-10
    assert np.abs(per - [1., 0., 1.]).max() < 1e-10
    rng = np.random.Generator(np.random.PCG64(2))
    th = rng.random(500) * np.pi
    ph = rng.random(500) * 2 * np.pi
    bb = rng.standard_normal((500, 3))
    ver, par, per, c2, s2 = I.los_geometry(th, ph, bb)
    over, opar, oper, oipa = oracle.los_geometry(th, ph, bb)
    assert np.abs(ver - over).max() < 1e-14
    assert np.abs(par - opar).max() < 1e-13
    assert np.abs(per - oper).max() < 1e-13
    assert np.abs(c2 - np.cos(2 * oipa)).max() < 1e-12
    assert np.abs(s2 - np.sin(2 * oipa)).max() < 1e-12


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-6)])
def test_gpu_trilinear_linear_field(precision, tol):
    """grid_tests.cc:137-260 on the device grid sampler."""
    d = abi.GridDesc()
    d.nx, d.ny, d.nz = 10, 8, 29
    d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max = (
        -1. * U.kpc, 1. * U.kpc, -1. * U.kpc, 1. * U.kpc, -1. * U.kpc, 1. * U.kpc)
    i, j, k = np.meshgrid(np.arange(10), np.arange(8), np.arange(29), indexing="ij")
    x = (i * 2.0 / 9 - 1.).reshape(-1) * 1e-6
    y = (j * 2.0 / 7 - 1.).reshape(-1) * 1e-6
    z = (k * 2.0 / 28 - 1.).reshape(-1) * 1e-6
    m = W.spiral_models()
    m.breg = abi.HXG_BREG_NONE
    m.brnd = abi.HXG_BRND_GRID
    m.tereg = abi.HXG_TEREG_GRID
    rng = np.random.Generator(np.random.PCG64(3))
    pos = (rng.random((64, 3)) * 2 - 1) * U.kpc
    with I.Integrator(precision) as integ:
        integ.set_models(m)
        integ.upload_grid(abi.HXG_FIELD_BRND, d, [x, y, z])
        integ.upload_grid(abi.HXG_FIELD_TEREG, d, [(x + y + z) * 1e6])
        b = integ.read_grid(abi.HXG_FIELD_BRND, pos)
        te = integ.read_grid(abi.HXG_FIELD_TEREG, pos)
    assert np.abs(b - pos / U.kpc * 1e-6).max() < tol * 1e-6
    assert np.abs(te - pos.sum(1) / U.kpc).max() < tol * 3


# ---- full maps: FP64 form vs the reference ----------------------------------

def test_gpu_fp64_config1(ref_maps):
    _check_vs_golden(ref_maps, "config1", *cases.case_config1())


def test_gpu_fp64_grids(ref_maps, fields32):
    _check_vs_golden(ref_maps, "grid_small", *cases.case_grid_small(fields32))
    _check_vs_golden(ref_maps, "grid_lowfreq", *cases.case_grid_lowfreq(fields32))


def test_gpu_fp64_mask(ref_maps):
    _check_vs_golden(ref_maps, "mask", *cases.case_mask())


def test_gpu_fp64_models(ref_maps):
    for name, passes, m in cases.case_models():
        _check_vs_golden(ref_maps, f"model_{name}", passes, m, None, None)


def test_gpu_fp64_two_geometries_vs_oracle(oracle):
    passes, m, g, mask = cases.case_dm_only()
    got = _run_gpu("fp64", passes, m, g, mask)[0]
    ref = oracle.write_grid(passes[0], m, g)
    assert rel_err(got["dm"], ref["dm"]) <= 1e-10


# ---- FP32-compensated form vs the FP64 oracle ---------------------------------

def _check_fp32c(oracle, passes, m, grids, mask, tol=TOL32):
    outs = _run_gpu("fp32c", passes, m, grids, mask)
    errs = {}
    for o, got in zip(passes, outs):
        kw = {} if mask is None else dict(mask_nside=mask[0], mask=mask[1])
        ref = oracle.write_grid(o, m, grids, **kw)
        for k, v in got.items():
            if v is None:
                continue
            errs[k] = max(errs.get(k, 0.0), rel_err(v, ref[k]))
    for k, e in errs.items():
        assert e <= tol, (k, e, errs)
    return errs


def test_gpu_fp32c_config1(oracle):
    _check_fp32c(oracle, *cases.case_config1())


def test_gpu_fp32c_grids(oracle, fields32):
    _check_fp32c(oracle, *cases.case_grid_small(fields32))
    _check_fp32c(oracle, *cases.case_grid_lowfreq(fields32), tol=TOL32_STRONG)


def test_gpu_fp32c_vs_fp64_config3_steps():
    """Config-3 sampling (0.01 kpc steps to 30 kpc, 0.408 / 1.4 / 30 GHz) at
    Nside 8-64 on a 128^3 random grid: FP32-compensated vs the FP64 form."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    bx, by, bz, ne = W.random_grids_torch(128, 3, 4, device=dev)
    f64 = [t.double().reshape(-1).contiguous() for t in (bx, by, bz, ne)]
    passes = W.config_grid([8, 16, 32, 64], 30.0, 0.01, [0.408, 1.4, 30.0])
    res = {}
    for prec in ("fp64", "fp32c"):
        with I.Integrator(prec) as integ:
            integ.set_models(W.grid_models())
            integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(128), f64[:3])
            integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(128), f64[3:])
            res[prec] = [integ.write_grid(o) for o in passes]
    for a, b in zip(res["fp32c"], res["fp64"]):
        for k, v in a.items():
            if v is not None:
                assert rel_err(v, b[k]) <= TOL32, (k, rel_err(v, b[k]))


def test_gpu_fp32c_models_and_mask(oracle):
    for name, passes, m in cases.case_models():
        _check_fp32c(oracle, passes, m, None, None)
    _check_fp32c(oracle, *cases.case_mask())


# ---- edge cases and error behaviour -----------------------------------------

def test_gpu_fully_masked_is_zero():
    passes, m, g, mask = cases.case_mask()
    zero = (mask[0], np.zeros_like(mask[1]))
    out = _run_gpu("fp64", passes[:1], m, None, zero)[0]
    for k, v in out.items():
        if v is not None:
            assert np.all(v == 0), k


def test_gpu_shell_outside_galaxy_is_zero():
    """All samples beyond gc_r_max (integrator.cc:179-182) contribute nothing."""
    o = W.make_obs([8], 60.0, 0.5, freq_ghz=1.4, r_min_kpc=40.0)
    out = _run_gpu("fp64", [o], W.spiral_models(), None, None)[0]
    for k, v in out.items():
        if v is not None:
            assert np.all(v == 0), k


def test_gpu_errors():
    with I.Integrator("fp64") as integ:
        o, m = W.config1()
        with pytest.raises(_lib.HxgError) as e:
            integ.write_grid(o)               # models not set
        assert e.value.status == abi.HXG_ERR_STATE
        integ.set_models(W.grid_models())
        with pytest.raises(_lib.HxgError) as e:
            integ.write_grid(o)               # grid slot never uploaded
        assert e.value.status == abi.HXG_ERR_STATE
        bad = abi.Models.from_buffer_copy(m)
        bad.breg = 99
        with pytest.raises(_lib.HxgError) as e:
            integ.set_models(bad)
        assert e.value.status == abi.HXG_ERR_UNSUPPORTED
        integ.set_models(m)
        o2 = abi.Obs.from_buffer_copy(o)
        o2.nside_shell[0] = 33
        with pytest.raises(_lib.HxgError) as e:
            integ.write_grid(o2)
        assert e.value.status == abi.HXG_ERR_INVALID
        nocre = abi.Models.from_buffer_copy(m)
        nocre.cre = abi.HXG_CRE_NONE
        integ.set_models(nocre)
        with pytest.raises(_lib.HxgError) as e:
            integ.write_grid(o)
        assert e.value.status == abi.HXG_ERR_INVALID
