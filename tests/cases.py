"""Small parity cases shared by the golden-fixture generator and the tests.

Each case returns (list of Obs passes, Models, grids dict or None,
(mask_nside, mask) or None).  Sizes are chosen so that the CPU oracle runs
each case in about a second.
"""
import numpy as np

from hammurabix_b200 import abi, workloads as W
from hammurabix_b200 import units as U


def _grid_fields(n, seeds):
    bx, by, bz, ne = W.random_grids(n, *seeds)
    return bx, by, bz, ne


def case_config1():
    """The analytic config-1 workload itself (Nside 32, 512 steps)."""
    obs, m = W.config1()
    return [obs], m, None, None


def case_grid_small(fields=None):
    """Config-2 shape, scaled down: 32^3 grids, Nside 4/8/16, 30 kpc, two
    frequencies in the reference's Pipeline order."""
    bx, by, bz, ne = fields if fields is not None else _grid_fields(32, (1, 2))
    passes = W.config_grid([4, 8, 16], 30.0, 0.1, [1.4, 23.0])
    return passes, W.grid_models(), W.grids_dict(32, bx, by, bz, ne), None


def case_grid_lowfreq(fields=None):
    """Strong Faraday rotation: 0.408 GHz, Nside 8/16/32 output at 32,
    3 shells to 30 kpc."""
    bx, by, bz, ne = fields if fields is not None else _grid_fields(32, (1, 2))
    passes = W.config_grid([8, 16, 32], 30.0, 0.05, [0.408])
    return passes, W.grid_models(), W.grids_dict(32, bx, by, bz, ne), None


def case_mask(fields=None):
    """A HEALPix mask at Nside 8 applied to Nside 4/8/16 shells."""
    passes = W.config_grid([4, 8, 16], 20.0, 0.1, [23.0])
    rng = np.random.Generator(np.random.PCG64(11))
    mask = (rng.random(abi.npix(8)) > 0.3).astype(np.float64)
    for o in passes:
        o.do_mask = 1
    m = W.spiral_models()
    return passes, m, None, (8, mask)


def case_models():
    """One pass per analytic model of the reference (LSA, unif, cart, helix;
    TEreg_unif; CRE_unif), Nside 8, 2 shells, DM + FD + sync 1.4 GHz."""
    out = []
    base = W.make_obs([8, 16], 20.0, 0.05, freq_ghz=1.4, nside_out=16)
    def mk(breg, tereg, cre):
        m = W.spiral_models()
        m.breg = breg
        m.lsa.b0 = 3.0 * U.muGauss
        m.lsa.psi0 = 27.0 * U.rad
        m.lsa.psi1 = 0.9 * U.rad
        m.lsa.chi0 = 25.0 * U.rad
        m.unif.bp = 2.0 * U.muGauss
        m.unif.bv = 0.5 * U.muGauss
        m.unif.l0 = 70.0 * U.rad
        m.cart.bx = 1.0 * U.muGauss
        m.cart.by = -0.5 * U.muGauss
        m.cart.bz = 0.2 * U.muGauss
        m.helix.bx = 1.0 * U.muGauss
        m.helix.by = 1.0 * U.muGauss
        m.helix.bz = 0.3 * U.muGauss
        m.helix.r_min = 3.0 * U.kpc
        m.helix.r_max = 9.0 * U.kpc
        m.tereg = tereg
        m.te_unif.n0 = 0.01
        m.te_unif.r0 = 3.0 * U.kpc
        m.cre = cre
        m.cre_unif.alpha = 3.0
        m.cre_unif.r0 = 3.0 * U.kpc
        m.cre_unif.E0 = 20.6 * U.GeV
        m.cre_unif.j0 = 0.0217
        return m
    combos = [
        ("lsa", abi.HXG_BREG_LSA, abi.HXG_TEREG_EXPDISK, abi.HXG_CRE_ANA),
        ("unif", abi.HXG_BREG_UNIF, abi.HXG_TEREG_UNIF, abi.HXG_CRE_UNIF),
        ("cart", abi.HXG_BREG_CART, abi.HXG_TEREG_EXPDISK, abi.HXG_CRE_UNIF),
        ("helix", abi.HXG_BREG_HELIX, abi.HXG_TEREG_EXPDISK, abi.HXG_CRE_ANA),
        ("cre_vary", abi.HXG_BREG_SPIRAL, abi.HXG_TEREG_EXPDISK, abi.HXG_CRE_ANA),
    ]
    for name, b, t, c in combos:
        m = mk(b, t, c)
        if name == "cre_vary":
            m.cre_ana.beta = 0.05
            m.cre_ana.theta = 0.1
        out.append((name, [base], m))
    return out


def obs_models_ext():
    """Pass of the large-model cases: 3 shells (Nside 8/16/32) to 20 kpc at
    0.05 kpc, DM + FD + sync at 1.4 GHz, output Nside 32."""
    return [W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=1.4)]


def case_models_ext(blocks):
    """Breg_jaffe with its molecular ring and with its elliptical bar, and
    Breg_jf12, each with TEreg_ymw16 or the exponential disk; `blocks` holds
    the jaffe / jf12 / ymw16 parameter blocks (the reference template's
    values; the fixtures store the full model block of every case)."""
    out = []
    def mk(breg, tereg, cre):
        m = W.spiral_models()
        m.breg, m.tereg, m.cre = breg, tereg, cre
        m.jaffe = blocks["jaffe"]
        m.jf12 = blocks["jf12"]
        m.ymw16 = blocks["ymw16"]
        m.cre_unif.alpha = 3.0
        m.cre_unif.r0 = 3.0 * U.kpc
        m.cre_unif.E0 = 20.6 * U.GeV
        m.cre_unif.j0 = 0.0217
        return m
    m = mk(abi.HXG_BREG_JAFFE, abi.HXG_TEREG_YMW16, abi.HXG_CRE_ANA)
    m.jaffe.ring, m.jaffe.bar = 1, 0
    out.append(("jaffe_ring_ymw16", m))
    m = mk(abi.HXG_BREG_JAFFE, abi.HXG_TEREG_EXPDISK, abi.HXG_CRE_ANA)
    m.jaffe.ring, m.jaffe.bar = 0, 1
    out.append(("jaffe_bar_expdisk", m))
    out.append(("jf12_ymw16", mk(abi.HXG_BREG_JF12, abi.HXG_TEREG_YMW16, abi.HXG_CRE_UNIF)))
    out.append(("spiral_ymw16", mk(abi.HXG_BREG_SPIRAL, abi.HXG_TEREG_YMW16, abi.HXG_CRE_ANA)))
    return out


def case_dm_only():
    """DM-only pass (no FD, no sync) with two grid geometries."""
    o = W.make_obs([8, 16], 25.0, 0.05, freq_ghz=None, do_fd=False)
    bx, by, bz, ne = _grid_fields(24, (5, 6))
    g = W.grids_dict(24, bx, by, bz, ne)
    # a second n_e grid on a different box, read as Grid_ternd
    d2 = W.grid_desc(16, (-15.0, 15.0, -15.0, 15.0, -3.0, 3.0))
    rng = np.random.Generator(np.random.PCG64(9))
    ne2 = (0.01 * rng.random(16 ** 3)).astype(np.float32).astype(np.float64)
    g[abi.HXG_FIELD_TERND] = (d2, [ne2])
    m = W.grid_models()
    m.ternd = abi.HXG_TERND_GRID
    return [o], m, g, None


def case_cre_grid():
    """Power-law CRE flux on a 9 x 9 x 5 box grid with 8 energies from 2 to
    200 GeV: flux(E, pos) = 1e-2 (E / 10 GeV)^-3 exp(-r/8 kpc) sech^2(z/1 kpc)
    (GeV m^2 s sr)^-1, with the analytic spiral B and exponential n_e."""
    nx, ny, nz, nE = 9, 9, 5, 8
    d = abi.GridDesc()
    d.nx, d.ny, d.nz, d.nE = nx, ny, nz, nE
    d.x_min, d.x_max = -20. * U.kpc, 20. * U.kpc
    d.y_min, d.y_max = -20. * U.kpc, 20. * U.kpc
    d.z_min, d.z_max = -4. * U.kpc, 4. * U.kpc
    d.E_min = 2. * U.GeV
    d.E_max = 200. * U.GeV
    d.E_fact = np.log(d.E_max / d.E_min) / (nE - 1)
    x = np.linspace(-20, 20, nx)[:, None, None, None]
    y = np.linspace(-20, 20, ny)[None, :, None, None]
    z = np.linspace(-4, 4, nz)[None, None, :, None]
    E = (d.E_min * np.exp(np.arange(nE) * d.E_fact) / U.GeV)[None, None, None, :]
    r = np.sqrt(x * x + y * y)
    flux = 1e-2 * (E / 10.) ** -3 * np.exp(-r / 8.) / np.cosh(z) ** 2
    m = W.spiral_models()
    m.cre = abi.HXG_CRE_GRID
    passes = [W.make_obs([8, 16], 20.0, 0.05, freq_ghz=f) for f in (1.4, 0.408)]
    return passes, m, {abi.HXG_FIELD_CRE: (d, [np.ascontiguousarray(flux.reshape(-1))])}


# ---- random-field generators --------------------------------------------

RFG_OBSERVER = (-8.3 * U.kpc, 0.0, 0.006 * U.kpc)


def _rfg_desc(n, box_kpc):
    d = abi.GridDesc()
    d.nx, d.ny, d.nz = n
    d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max = (v * U.kpc for v in box_kpc)
    return d


def rfg_es(rms_muG=0.8, k0=10.0, k1=0.1, a0=1.7, a1=0.0, rho=1.0, r0_kpc=8.0, z0_kpc=1.0):
    """Brnd_es parameters; defaults are templates/params_template.xml:239-249."""
    p = abi.BrndEs()
    p.rms, p.k0, p.k1, p.a0, p.a1, p.rho = rms_muG * U.muGauss, k0, k1, a0, a1, rho
    p.r0, p.z0 = r0_kpc * U.kpc, z0_kpc * U.kpc
    return p


def rfg_dft(rms=1.0, k0=2.0, a0=-1.7, r0_kpc=8.0, z0_kpc=1.0):
    """TErnd_dft parameters; defaults are templates/params_template.xml:399-406."""
    p = abi.TerndDft()
    p.rms, p.k0, p.a0, p.r0, p.z0 = rms, k0, a0, r0_kpc * U.kpc, z0_kpc * U.kpc
    return p


def case_rfg(jf12_block=None):
    """Generator cases: (name, kind, desc, params, seed, models, grids).
    Boxes of a few tens of kpc give k = i / L below the template's k0 of
    the n_e spectrum, so those cases lower k0 to keep power on the grid.
    The B cases cover an analytic field everywhere non-zero (LSA), one that
    is zero outside 3-20 kpc (the spiral: unscaled vertices), a BREG grid
    on a smaller box (zero outside it), and JF12 when its block is given;
    the sizes mix odd and even axes (Nyquist planes)."""
    A = (-20., 20., -18., 18., -4., 4.)
    out = []
    out.append(("ternd_a", "ternd", _rfg_desc((12, 10, 9), A), rfg_dft(k0=0.06), 12345,
                None, None))
    out.append(("ternd_even", "ternd", _rfg_desc((8, 8, 8), (-2., 2., -2., 2., -1., 1.)),
                rfg_dft(rms=0.5, a0=-11. / 3., k0=0.3), 5, None, None))
    m = W.spiral_models()
    m.breg = abi.HXG_BREG_LSA
    m.lsa.b0, m.lsa.psi0, m.lsa.psi1, m.lsa.chi0 = 2e-6, 27 * U.rad, 0.9 * U.rad, 25 * U.rad
    out.append(("brnd_lsa", "brnd", _rfg_desc((12, 10, 9), A), rfg_es(rho=3.0), 777, m, None))
    out.append(("brnd_spiral", "brnd", _rfg_desc((10, 12, 8), (-25., 25., -25., 25., -3., 3.)),
                rfg_es(rho=0.5, a1=-0.4), 31, W.spiral_models(), None))
    gd = _rfg_desc((9, 9, 7), (-15., 15., -14., 14., -2., 2.))
    rng = np.random.Generator(np.random.PCG64(17))
    gb = [rng.normal(0., 1e-6, 9 * 9 * 7) for _ in range(3)]
    m = W.spiral_models()
    m.breg = abi.HXG_BREG_GRID
    out.append(("brnd_grid", "brnd", _rfg_desc((10, 8, 12), A), rfg_es(rho=2.0), 99, m,
                {abi.HXG_FIELD_BREG: (gd, gb)}))
    if jf12_block is not None:
        m = W.spiral_models()
        m.breg = abi.HXG_BREG_JF12
        m.jf12 = jf12_block
        out.append(("brnd_jf12", "brnd", _rfg_desc((11, 10, 8), A), rfg_es(rho=3.0), 4242, m,
                    None))
    return out
