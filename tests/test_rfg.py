"""Random-field generators (hxg_generate_brnd_es / hxg_generate_ternd_dft).

Parity: the reference's own Brnd_es / TErnd_dft code, compiled from its
sources with the shim's cell-indexed Philox deviates and direct-sum DFT
(oracle/shim), produced tests/golden/ref_rfg.npz; the numpy restatement
(oracle/rfg.py) and the device generators must both reproduce it.  FFT
rounding differs between the three (FFTW-style direct sums, numpy's pocketfft,
cuFFT), so the bar is 1e-12 of the field's maximum, not bit equality.

Statistics (device, 48^3 - 64^3 grids): the divergence-free projection holds
to rounding off the Nyquist planes, the n_e variance is normalised to rms^2, the spectral slope of
n_e is a0 - 2, B is isotropic for rho = 1 and elongated along the regular
field for rho != 1, and the total B variance is the reference's ~2 rms^2
(its sqrt(3) and sqrt(2) factors, brnd_es.cc:69-73, 250-256).
"""
import os

import numpy as np
import pytest

import cases
from conftest import GOLDEN, rel_err
from hammurabix_b200 import abi, units as U

RFG_TOL = 1e-12


@pytest.fixture(scope="session")
def ref_rfg():
    return dict(np.load(os.path.join(GOLDEN, "ref_rfg.npz")))


def _rfg():
    import rfg
    return rfg


def _case_table(ref_rfg):
    """cases with the models block of each B case taken from the fixture."""
    out = []
    for name, kind, desc, p, seed, m, grids in cases.case_rfg(abi.BregJf12()):
        if kind == "brnd":
            m = abi.Models.from_buffer_copy(ref_rfg[f"{name}/models"].tobytes())
        out.append((name, kind, desc, p, seed, m, grids))
    return out


# ---- CPU ------------------------------------------------------------------

def test_philox_known_answers():
    """Philox4x32-10 against the Random123 known-answer vectors."""
    rfg = _rfg()
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in kat:
        got = rfg.philox4x32_10([np.array([c], dtype=np.uint64) for c in ctr], key)
        assert tuple(int(g[0]) for g in got) == want


def test_cell_deviates_are_standard_normal():
    g = _rfg().cell_gauss(2024, np.arange(200000)).reshape(-1)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1.0) < 0.01
    assert abs(np.mean(g ** 4) - 3.0) < 0.05


def test_oracle_generators_match_reference_golden(oracle, ref_rfg):
    """The numpy restatement against the reference's generator code (JF12 is
    skipped: the C oracle has no JF12 model; the device test covers it)."""
    rfg = _rfg()
    for name, kind, desc, p, seed, m, grids in _case_table(ref_rfg):
        if kind == "ternd":
            te = rfg.ternd_dft(desc, p, cases.RFG_OBSERVER, seed)
            assert rel_err(te, ref_rfg[f"{name}/te"]) <= RFG_TOL, name
            continue
        if m.breg == abi.HXG_BREG_JF12:
            continue
        if m.breg == abi.HXG_BREG_GRID:
            gd, gb = grids[abi.HXG_FIELD_BREG]
            breg_at = lambda x, y, z: oracle.read_grid(gd, gb, np.stack([x, y, z], -1))
        else:
            breg_at = lambda x, y, z: oracle.breg_field(m, cases.RFG_OBSERVER,
                                                        np.stack([x, y, z], -1))
        b = rfg.brnd_es(desc, p, cases.RFG_OBSERVER, seed, breg_at)
        for c, a in zip(("bx", "by", "bz"), b):
            assert rel_err(a, ref_rfg[f"{name}/{c}"]) <= RFG_TOL, (name, c)


def test_reference_build_reproduces_golden(reference, ref_rfg):
    """The committed fixture is what the reference build gives (runs only
    where oracle/_ref exists)."""
    tab = cases.case_rfg(abi.BregJf12())
    for name, kind, desc, p, seed, m, grids in tab:
        if kind == "ternd":
            te = reference.generate_ternd_dft(cases.RFG_OBSERVER, desc, p, seed)
            assert rel_err(te, ref_rfg[f"{name}/te"]) <= 1e-14, name
        elif m.breg != abi.HXG_BREG_JF12:
            b = reference.generate_brnd_es(m, grids, cases.RFG_OBSERVER, desc, p, seed)
            for c, a in zip(("bx", "by", "bz"), b):
                assert rel_err(a, ref_rfg[f"{name}/{c}"]) <= 1e-14, (name, c)


def _divergence(bx, by, bz, desc):
    """max |k . B(k)| / (max |k| max |B(k)|) over the grid's FFT modes, k as
    the generators define it (ternd_dft.cc:60-62).  Modes on the Nyquist
    plane of an even axis are left out: there the reference pairs k with a
    mirror mode whose k is not -k (brnd_es.cc:215-245, the Nyquist index is
    its own mirror but its k keeps the negative sign), so its projection
    leaves k . B non-zero by construction."""
    rfg = _rfg()
    kx, ky, kz = rfg._kgrid(desc)
    B = [np.fft.fftn(a) for a in (bx, by, bz)]
    kb = kx * B[0] + ky * B[1] + kz * B[2]
    keep = np.ones(kb.shape, dtype=bool)
    for ax, n in enumerate(kb.shape):
        if n % 2 == 0:
            idx = [slice(None)] * 3
            idx[ax] = n // 2
            keep[tuple(idx)] = False
    kb = np.where(keep, kb, 0.0)
    kmax = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2).max()
    bmax = np.sqrt(sum(np.abs(c) ** 2 for c in B)).max()
    return np.abs(kb).max() / (kmax * bmax)


def test_reference_fields_are_divergence_free(ref_rfg):
    for name, kind, desc, p, seed, m, grids in cases.case_rfg(abi.BregJf12()):
        if kind == "brnd":
            b = [ref_rfg[f"{name}/{c}"] for c in ("bx", "by", "bz")]
            assert _divergence(*b, desc) < 1e-12, name


# ---- GPU ------------------------------------------------------------------

def _integrator(precision="fp64"):
    from hammurabix_b200 import integrator as I
    return I.Integrator(precision)


def _generate(integ, kind, desc, p, seed, m, grids, observer=cases.RFG_OBSERVER):
    if kind == "ternd":
        integ.generate_ternd_dft(desc, p, observer, seed)
        return integ.download_grid(abi.HXG_FIELD_TERND, desc)[0]
    integ.set_models(m)
    for field, (gd, comps) in (grids or {}).items():
        integ.upload_grid(field, gd, comps)
    integ.generate_brnd_es(desc, p, observer, seed)
    return integ.download_grid(abi.HXG_FIELD_BRND, desc)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_device_generators_match_reference_golden(ref_rfg, precision):
    with _integrator(precision) as integ:
        for name, kind, desc, p, seed, m, grids in _case_table(ref_rfg):
            got = _generate(integ, kind, desc, p, seed, m, grids)
            if kind == "ternd":
                assert rel_err(got, ref_rfg[f"{name}/te"]) <= RFG_TOL, name
            else:
                for c, a in zip(("bx", "by", "bz"), got):
                    assert rel_err(a, ref_rfg[f"{name}/{c}"]) <= RFG_TOL, (name, c)


@pytest.mark.gpu
def test_device_generators_are_deterministic_in_the_seed():
    name, kind, desc, p, seed, m, grids = cases.case_rfg()[2]
    with _integrator() as integ:
        a = _generate(integ, kind, desc, p, seed, m, grids)
        b = _generate(integ, kind, desc, p, seed, m, grids)
        c = _generate(integ, kind, desc, p, seed + 1, m, grids)
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, y)
        assert rel_err(x, z) > 0.1


@pytest.mark.gpu
def test_generated_slots_feed_the_integrator(oracle):
    """write_grid over generated BRND / TERND slots equals the oracle's
    write_grid over the downloaded grids."""
    from hammurabix_b200 import workloads as W
    tab = cases.case_rfg()
    _, _, dt, pt, st, _, _ = tab[0]
    _, _, db, pb, sb, m, _ = tab[2]
    m = abi.Models.from_buffer_copy(m)
    m.brnd, m.ternd = abi.HXG_BRND_GRID, abi.HXG_TERND_GRID
    pt = abi.TerndDft.from_buffer_copy(pt)
    pt.rms = 0.01
    o = W.make_obs([8, 16], 18.0, 0.1, freq_ghz=1.4)
    o.observer[:] = list(cases.RFG_OBSERVER)
    with _integrator() as integ:
        integ.set_models(m)
        te = _generate(integ, "ternd", dt, pt, st, m, None)
        b = _generate(integ, "brnd", db, pb, sb, m, None)
        got = integ.write_grid(o)
    grids = {abi.HXG_FIELD_BRND: (db, [a.reshape(-1) for a in b]),
             abi.HXG_FIELD_TERND: (dt, [te.reshape(-1)])}
    want = oracle.write_grid(o, m, grids)
    for k in ("dm", "fd", "is", "qs", "us"):
        assert rel_err(got[k], want[k]) <= 1e-10, k


@pytest.mark.gpu
def test_export_grid_file_round_trip(tmp_path):
    """export_grid_file writes the reference's layout (bx, by, bz per voxel);
    loading it back gives the same slot."""
    name, kind, desc, p, seed, m, grids = cases.case_rfg()[3]
    path = str(tmp_path / "brnd.bin")
    with _integrator() as integ:
        b = _generate(integ, kind, desc, p, seed, m, grids)
        integ.export_grid_file(abi.HXG_FIELD_BRND, path)
        raw = np.fromfile(path, dtype=np.float64)
        assert np.array_equal(raw, np.stack([a.reshape(-1) for a in b], -1).reshape(-1))
        with _integrator() as other:
            other.upload_grid_file(abi.HXG_FIELD_BRND, desc, path)
            back = other.download_grid(abi.HXG_FIELD_BRND, desc)
        for x, y in zip(b, back):
            assert np.array_equal(x, y)
        _, kind, dt, pt, st, _, _ = cases.case_rfg()[0]
        te = _generate(integ, "ternd", dt, pt, st, None, None)
        integ.export_grid_file(abi.HXG_FIELD_TERND, path)
        assert np.array_equal(np.fromfile(path, dtype=np.float64), te.reshape(-1))


@pytest.mark.gpu
def test_generator_argument_errors():
    from hammurabix_b200 import _lib
    name, kind, desc, p, seed, m, grids = cases.case_rfg()[4]   # BREG-grid case
    with _integrator() as integ:
        with pytest.raises(_lib.HxgError) as e:
            integ.generate_brnd_es(desc, p, cases.RFG_OBSERVER, seed)
        assert e.value.status == abi.HXG_ERR_STATE            # models not set
        integ.set_models(m)
        with pytest.raises(_lib.HxgError) as e:
            integ.generate_brnd_es(desc, p, cases.RFG_OBSERVER, seed)
        assert e.value.status == abi.HXG_ERR_STATE            # BREG grid missing
        bad = abi.BrndEs.from_buffer_copy(p)
        bad.rho = 0.0
        with pytest.raises(_lib.HxgError) as e:
            integ.generate_brnd_es(desc, bad, cases.RFG_OBSERVER, seed)
        assert e.value.status == abi.HXG_ERR_INVALID
        pt = cases.rfg_dft(k0=1e3)                             # no power on the grid
        with pytest.raises(_lib.HxgError) as e:
            integ.generate_ternd_dft(desc, pt, cases.RFG_OBSERVER, 3)
        assert e.value.status == abi.HXG_ERR_INVALID


def _flat_box(n):
    return cases._rfg_desc((n, n, n), (-20., 20., -20., 20., -20., 20.))


@pytest.mark.gpu
def test_ternd_statistics():
    """Variance normalisation (flat per-shell spectrum, a0 = 0) and the
    spectral slope a0 - 2 (steep spectrum), profile switched off."""
    n = 64
    d = _flat_box(n)
    origin = (0.0, 0.0, 0.0)
    with _integrator() as integ:
        pt = cases.rfg_dft(rms=1.0, k0=0.05, a0=0.0, r0_kpc=1e9, z0_kpc=1e9)
        integ.generate_ternd_dft(d, pt, origin, 3)
        te = integ.download_grid(abi.HXG_FIELD_TERND, d)[0]
        assert abs(np.var(te) - 1.0) < 0.03
        assert abs(np.mean(te)) < 1e-8
        a0 = -11.0 / 3.0
        pt = cases.rfg_dft(rms=1.0, k0=0.05, a0=a0, r0_kpc=1e9, z0_kpc=1e9)
        integ.generate_ternd_dft(d, pt, origin, 4)
        te = integ.download_grid(abi.HXG_FIELD_TERND, d)[0]
    kx, ky, kz = _rfg()._kgrid(d)
    k = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2).reshape(-1)
    P = (np.abs(np.fft.fftn(te)) ** 2).reshape(-1)
    edges = np.geomspace(0.08, 0.6, 9)
    kc, pc = [], []
    for lo, hi in zip(edges[:-1], edges[1:]):
        s = (k >= lo) & (k < hi)
        kc.append(np.exp(np.mean(np.log(k[s]))))
        pc.append(np.mean(P[s]))
    slope = np.polyfit(np.log(kc), np.log(pc), 1)[0]
    assert abs(slope - (a0 - 2.0)) < 0.15, slope


@pytest.mark.gpu
def test_brnd_statistics():
    """Divergence-free to rounding; isotropic for rho = 1, elongated along
    the regular field (uniform, along x) for rho = 3 and flattened for
    rho = 1/3; total variance ~2 rms^2 (the reference's normalisation)."""
    n = 48
    d = _flat_box(n)
    m = abi.Models()
    m.breg = abi.HXG_BREG_CART
    m.cart.bx = 1e-6
    origin = (0.0, 0.0, 0.0)
    var = {}
    with _integrator() as integ:
        integ.set_models(m)
        for rho in (1.0, 3.0, 1.0 / 3.0):
            p = cases.rfg_es(rho=rho, r0_kpc=1e9, z0_kpc=1e9)
            integ.generate_brnd_es(d, p, origin, 11)
            b = integ.download_grid(abi.HXG_FIELD_BRND, d)
            assert _divergence(*b, d) < 1e-11, rho
            var[rho] = [np.var(a) / p.rms ** 2 for a in b]
    v1 = var[1.0]
    assert max(v1) / min(v1) < 1.1, v1
    assert abs(sum(v1) - 2.0) < 0.15, v1
    v3 = var[3.0]
    assert v3[0] / v3[1] > 4 and v3[0] / v3[2] > 4, v3
    v13 = var[1.0 / 3.0]
    assert v13[1] / v13[0] > 3 and v13[2] / v13[0] > 3, v13
