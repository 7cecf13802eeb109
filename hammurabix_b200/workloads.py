"""Synthetic workloads for the line-of-sight integrator.

Each workload is a set of hxg ABI structs (Obs per frequency pass, Models)
plus seeded synthetic field grids.  The geometry follows hammurabiX's
parameter template (templates/params_template.xml:26-134): observer at
(-8.3, 0, 0.006) kpc, galacto-centric limits |pos| <= 20 kpc and
|z| <= 10 kpc, auto shells from oc_r_min = 0 (Param::obs_param,
source/param/param.cc:91-108), field box 40 x 40 x 10 kpc.

Field grids are synthetic stand-ins for hammurabiX's random-field outputs:
 - B_rnd: per component a Gaussian random field with power spectrum
   P(k) ~ k^-11/3 on the FFT lattice, zero mean, rms 1 muG over the box;
 - n_e: lognormal 0.03 * exp(sigma*g - sigma^2/2) cm^-3, sigma = 0.5, g a
   unit-variance Gaussian random field with the same spectrum.
Grids are generated in FP32 and handed to every consumer as FP64 copies of
those FP32 values, so the FP64 and FP32 forms see identical field values.
"""
import math

import numpy as np

from . import abi
from . import units as U

OBSERVER_KPC = (-8.3, 0.0, 0.006)
BOX_KPC = (-20.0, 20.0, -20.0, 20.0, -5.0, 5.0)


def spiral_models(b0_muG=6.0, pitch_deg=-30.0, rb_kpc=8.0, hb_kpc=1.0, n0=0.03,
                  rn_kpc=20.0, hn_kpc=1.0, cre_j0=0.0217):
    """Analytic models of the config-1 workload: exponential-disk log-spiral B,
    exponential n_e disk, CRE_ana (alpha 3, r0 5 kpc, z0 1 kpc, E0 20.6 GeV,
    j0 0.0217 as in templates/params_template.xml:417-427)."""
    m = abi.Models()
    m.breg = abi.HXG_BREG_SPIRAL
    m.spiral.b0 = b0_muG * U.muGauss
    m.spiral.pitch = pitch_deg * U.rad
    m.spiral.r_scale = rb_kpc * U.kpc
    m.spiral.h_scale = hb_kpc * U.kpc
    m.brnd = abi.HXG_BRND_NONE
    m.tereg = abi.HXG_TEREG_EXPDISK
    m.te_exp.n0 = n0
    m.te_exp.r_scale = rn_kpc * U.kpc
    m.te_exp.h_scale = hn_kpc * U.kpc
    m.ternd = abi.HXG_TERND_NONE
    m.cre = abi.HXG_CRE_ANA
    m.cre_ana.alpha = 3.0
    m.cre_ana.beta = 0.0
    m.cre_ana.theta = 0.0
    m.cre_ana.r0 = 5.0 * U.kpc
    m.cre_ana.z0 = 1.0 * U.kpc
    m.cre_ana.E0 = 20.6 * U.GeV
    m.cre_ana.j0 = cre_j0
    return m


def make_obs(nside_shells, r_max_kpc, res_kpc, freq_ghz=None, do_dm=True, do_fd=True,
             nside_out=None, r_min_kpc=0.0, observer_kpc=OBSERVER_KPC):
    """Obs for an auto-layer shell set (Param::obs_param, param.cc:91-108):
    nside_shell as given, radii r_min + (r_max - r_min) * 0.5^(N-1-s)."""
    o = abi.Obs()
    for i in range(3):
        o.observer[i] = U.kpc * observer_kpc[i]
    o.gc_r_min = 0.0 * U.kpc
    o.gc_r_max = 20.0 * U.kpc
    o.gc_z_min = -10.0 * U.kpc
    o.gc_z_max = 10.0 * U.kpc
    o.oc_r_res = res_kpc * U.kpc
    n = len(nside_shells)
    o.total_shell = n
    for i, ns in enumerate(nside_shells):
        o.nside_shell[i] = ns
    rmin, rmax = r_min_kpc * U.kpc, r_max_kpc * U.kpc
    o.radii_shell[0] = rmin
    for i in range(n):
        o.radii_shell[i + 1] = (rmax - rmin) * math.pow(0.5, n - i - 1) + rmin
    nout = nside_out or max(nside_shells)
    o.do_dm = int(do_dm)
    o.do_fd = int(do_fd)
    o.nside_dm = nout if do_dm else 0
    o.nside_fd = nout if do_fd else 0
    o.do_sync = int(freq_ghz is not None)
    o.nside_sync = nout if freq_ghz is not None else 0
    o.sync_freq = (freq_ghz or 0.0) * U.GHz
    o.do_mask = 0
    return o


def frequency_passes(obs_template, freqs_ghz):
    """The Pipeline::assemble_obs loop (source/pipeline/pipeline.cc:165-190):
    frequencies are taken from the back of the <sync> list; only the first
    pass keeps DM and FD (later passes run with do_dm = do_fd = false)."""
    passes = []
    for i, f in enumerate(reversed(freqs_ghz)):
        o = abi.Obs.from_buffer_copy(obs_template)
        o.do_sync = 1
        o.sync_freq = f * U.GHz
        if o.nside_sync == 0:
            o.nside_sync = max(o.nside_shell[: o.total_shell])
        if i > 0:
            o.do_dm = 0
            o.do_fd = 0
        passes.append(o)
    return passes


def grid_desc(n, box_kpc=BOX_KPC):
    g = abi.GridDesc()
    g.nx = g.ny = g.nz = n
    g.x_min, g.x_max, g.y_min, g.y_max, g.z_min, g.z_max = (v * U.kpc for v in box_kpc)
    return g


def _spectrum_filter(n, slope=-11.0 / 3.0):
    k = np.fft.fftfreq(n) * n
    kr = np.fft.rfftfreq(n) * n
    kk = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2)
    with np.errstate(divide="ignore"):
        amp = np.where(kk > 0, kk ** (slope / 2.0), 0.0)
    return amp


def gaussian_field(n, seed, slope=-11.0 / 3.0):
    """Unit-variance, zero-mean Gaussian random field on an n^3 lattice with
    power spectrum ~ k^slope (numpy PCG64, seeded), FP32."""
    rng = np.random.Generator(np.random.PCG64(seed))
    white = rng.standard_normal((n, n, n))
    f = np.fft.rfftn(white) * _spectrum_filter(n, slope)
    g = np.fft.irfftn(f, s=(n, n, n), axes=(0, 1, 2))
    g -= g.mean()
    g /= g.std()
    return g.astype(np.float32)


def random_grids(n, seed_b, seed_n, brms_muG=1.0, ne_mean=0.03, sigma_ln=0.5):
    """(bx, by, bz, ne) FP32 arrays (CGS) of the synthetic random fields."""
    comps = []
    for c in range(3):
        g = gaussian_field(n, seed_b * 16 + c)
        comps.append(g)
    b = np.stack(comps)
    b *= np.float32(brms_muG * U.muGauss / np.sqrt((b.astype(np.float64) ** 2).sum(0).mean()))
    g = gaussian_field(n, seed_n * 16 + 3).astype(np.float64)
    ne = (ne_mean * np.exp(sigma_ln * g - 0.5 * sigma_ln ** 2)).astype(np.float32)
    return b[0], b[1], b[2], ne


def random_grids_torch(n, seed_b, seed_n, device="cpu", brms_muG=1.0, ne_mean=0.03,
                       sigma_ln=0.5, slope=-11.0 / 3.0):
    """Large-grid variant of random_grids() built with torch FFTs (seeded
    torch.Generator); returns FP32 tensors (bx, by, bz, ne) in CGS."""
    import torch

    k = torch.fft.fftfreq(n, device=device, dtype=torch.float32) * n
    kr = torch.fft.rfftfreq(n, device=device, dtype=torch.float32) * n
    kk = torch.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2)
    amp = torch.where(kk > 0, kk.clamp_min(1e-30) ** (slope / 2.0), torch.zeros_like(kk))
    del kk

    def grf(seed):
        g = torch.Generator(device=device).manual_seed(int(seed))
        x = torch.randn((n, n, n), generator=g, device=device, dtype=torch.float32)
        f = torch.fft.rfftn(x)
        del x
        f *= amp
        x = torch.fft.irfftn(f, s=(n, n, n))
        del f
        x -= x.mean()
        x /= x.std()
        return x

    b = [grf(seed_b * 16 + c) for c in range(3)]
    rms = torch.sqrt(sum((c.double() ** 2).mean() for c in b))
    scale = float(brms_muG * U.muGauss / rms)
    b = [(c * scale).float() for c in b]
    g = grf(seed_n * 16 + 3).double()
    ne = (ne_mean * torch.exp(sigma_ln * g - 0.5 * sigma_ln ** 2)).float()
    return b[0], b[1], b[2], ne


def grid_models(base=None):
    """Models of the grid workloads: analytic spiral B_reg, B_rnd from the
    random grid, n_e from the lognormal grid (read as Grid_tereg), CRE_ana."""
    m = abi.Models.from_buffer_copy(base or spiral_models())
    m.brnd = abi.HXG_BRND_GRID
    m.tereg = abi.HXG_TEREG_GRID
    m.ternd = abi.HXG_TERND_NONE
    return m


def grids_dict(n, bx, by, bz, ne):
    """dict field -> (GridDesc, [FP64 SoA arrays]) in the Grid_* layout
    (x-major, z fastest: toolkit::index3d, include/toolkit.h:29-34)."""
    d = grid_desc(n)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return {
        abi.HXG_FIELD_BRND: (d, [f64(bx), f64(by), f64(bz)]),
        abi.HXG_FIELD_TEREG: (d, [f64(ne)]),
    }


# ---- the named workloads --------------------------------------------------

def config1():
    """Analytic only: Nside 32, 1 shell, r in [0, 20] kpc in 512 steps, DM, FD
    and sync at 23 GHz (6.29 M samples)."""
    obs = make_obs([32], 20.0, 20.0 / 512.0, freq_ghz=23.0)
    return obs, spiral_models()


def config_grid(nside_shells, r_max_kpc, res_kpc, freqs_ghz):
    """Grid workload geometry: returns the per-frequency Obs passes."""
    tmpl = make_obs(nside_shells, r_max_kpc, res_kpc, freq_ghz=freqs_ghz[-1])
    return frequency_passes(tmpl, freqs_ghz)


CONFIG2 = dict(nside_shells=[64, 128, 256], r_max_kpc=30.0, res_kpc=0.01,
               freqs_ghz=[1.4, 23.0], grid_n=256, seeds=(1, 2))
CONFIG3 = dict(nside_shells=[128, 256, 512, 1024], r_max_kpc=30.0, res_kpc=0.01,
               freqs_ghz=[0.408, 1.4, 30.0], grid_n=512, seeds=(3, 4))


def samples_of(obs):
    """Number of LOS samples (reference loop iterations) of one pass:
    sum over shells of Npix * step."""
    tot = 0
    for s in range(obs.total_shell):
        ds = obs.radii_shell[s]
        de = obs.radii_shell[s + 1]
        dd = obs.oc_r_res
        step = int(math.floor(de / dd - ds / dd))
        tot += abi.npix(obs.nside_shell[s]) * step
    return tot


# ---- samples that pass the cuts ----------------------------------------------

def ring_directions(nside, start, stop):
    """Unit vectors (x, y, z) of RING pixels [start, stop) of an Nside map:
    the HEALPix pixel centres (Gorski et al. 2005, ApJ 622, 759, eqs. 4-9),
    as Hampix::fillpoint computes them (include/hamdis.h:302-356)."""
    p = np.arange(start, stop, dtype=np.int64)
    n = int(nside)
    npix, ncap = 12 * n * n, 2 * n * (n - 1)
    z = np.empty(p.shape)
    phi = np.empty(p.shape)
    north = p < ncap
    south = p >= npix - ncap
    eq = ~(north | south)
    if north.any():
        q = p[north]
        ir = np.floor(0.5 * (1.0 + np.sqrt(1.0 + 2.0 * q))).astype(np.int64)
        iphi = q + 1 - 2 * ir * (ir - 1)
        z[north] = 1.0 - ir * ir / (3.0 * n * n)
        phi[north] = (iphi - 0.5) * (0.5 * math.pi / ir)
    if eq.any():
        q = p[eq] - ncap
        ir = q // (4 * n) + n
        iphi = q % (4 * n) + 1
        fodd = 0.5 * (1 + ((ir + n) & 1))
        z[eq] = (2 * n - ir) * (2.0 / (3.0 * n))
        phi[eq] = (iphi - fodd) * (0.5 * math.pi / n)
    if south.any():
        q = npix - p[south]
        ir = np.floor(0.5 * (1.0 + np.sqrt(2.0 * q - 1.0))).astype(np.int64)
        iphi = 4 * ir + 1 - (q - 2 * ir * (ir - 1))
        z[south] = -1.0 + ir * ir / (3.0 * n * n)
        phi[south] = (iphi - 0.5) * (0.5 * math.pi / ir)
    s = np.sqrt(np.maximum(0.0, (1.0 - z) * (1.0 + z)))
    return s * np.cos(phi), s * np.sin(phi), z


def _count_in(ds, dd, step, a, b):
    """Number of sample indices i in [0, step) with ds + (i + 1/2) dd in
    [a, b] (elementwise; empty where a > b)."""
    lo = np.ceil((a - ds) / dd - 0.5)
    hi = np.floor((b - ds) / dd - 0.5)
    lo = np.clip(lo, 0, step)
    hi = np.clip(hi, -1, step - 1)
    return np.maximum(hi - lo + 1, 0).astype(np.int64)


def valid_samples(obs, chunk=1 << 20):
    """Per shell, the number of LOS samples that pass the galacto-centric
    cuts gc_r_min <= |pos| <= gc_r_max and gc_z_min <= z <= gc_z_max
    (integrator.cc:176-185): the samples whose fields are read and summed,
    as opposed to the reference's loop count (samples_of).  Exact up to
    samples within rounding of a cut boundary."""
    o = np.array([obs.observer[i] for i in range(3)])
    oo = float(o @ o)
    out = []
    for s in range(obs.total_shell):
        d0, d1, res = obs.radii_shell[s], obs.radii_shell[s + 1], obs.oc_r_res
        step = int(math.floor(d1 / res - d0 / res))      # assemble_shell_ref
        dd = (d1 - d0) / step
        nside = obs.nside_shell[s]
        total = 0
        for a in range(0, abi.npix(nside), chunk):
            ux, uy, uz = ring_directions(nside, a, min(a + chunk, abi.npix(nside)))
            ou = o[0] * ux + o[1] * uy + o[2] * uz
            # |o + u d|^2 = d^2 + 2 (o.u) d + |o|^2 between r_min^2 and r_max^2
            def roots(r):
                disc = ou * ou - (oo - r * r)
                sq = np.sqrt(np.maximum(disc, 0.0))
                return -ou - sq, -ou + sq, disc >= 0.0
            olo, ohi, _ = roots(obs.gc_r_max)
            # z = o_z + u_z d in [z_min, z_max]
            with np.errstate(divide="ignore", invalid="ignore"):
                za = (obs.gc_z_min - o[2]) / uz
                zb = (obs.gc_z_max - o[2]) / uz
            zlo = np.where(uz != 0.0, np.minimum(za, zb), -np.inf)
            zhi = np.where(uz != 0.0, np.maximum(za, zb), np.inf)
            inside_z = (o[2] >= obs.gc_z_min) & (o[2] <= obs.gc_z_max)
            zlo = np.where((uz == 0.0) & ~inside_z, np.inf, zlo)
            lo, hi = np.maximum(olo, zlo), np.minimum(ohi, zhi)
            n_out = _count_in(d0, dd, step, lo, hi)
            if obs.gc_r_min > 0.0:
                ilo, ihi, hit = roots(obs.gc_r_min)
                # strictly inside the inner sphere: excluded
                ilo, ihi = np.maximum(ilo, lo), np.minimum(ihi, hi)
                n_in = _count_in(d0, dd, step, np.nextafter(ilo, np.inf),
                                 np.nextafter(ihi, -np.inf))
                n_out = n_out - np.where(hit, n_in, 0)
            total += int(n_out.sum())
        out.append(total)
    return out
