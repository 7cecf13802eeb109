"""Random-field generators restated in numpy.

TEST INFRASTRUCTURE ONLY: the checker for the device generators
(hxg_generate_brnd_es / hxg_generate_ternd_dft).  Nothing in the
hammurabix_b200 product imports it.

Restates, step by step and in the reference's in-place complex packing:
  TErnd_dft::write_grid  (source/field/te/ternd_dft.cc:35-128)
  Brnd_es::write_grid    (source/field/b/brnd_es.cc:76-308)
with numpy FFTs (FFTW_BACKWARD = unnormalised inverse) and the cell-indexed
Gaussian deviates of the device generators: Philox4x32-10 (Salmon, Moraes,
Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011) keyed by
the seed, counter {cell, cell >> 32, block, 0x52464721}, two 53-bit uniforms
per 64 output bits, Box-Muller.  The same deviates drive the reference build
in oracle/_ref through the shim's cell-stream mode, which pins this
restatement to the reference's own generator code.
"""
import numpy as np

KPC = 3.0856775806e21  # cm (include/hamunits.h)
PI = 3.14159265358979323846264338327950288
_TAG = 0x52464721
_M0, _M1 = 0xD2511F53, 0xCD9E8D57
_W0, _W1 = 0x9E3779B9, 0xBB67AE85
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c, key):
    """c: four uint64 arrays holding 32-bit words; key: (k0, k1) ints."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) for x in c)
    k0, k1 = int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF
    for _ in range(10):
        p0 = np.uint64(_M0) * c0
        p1 = np.uint64(_M1) * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK32
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
        k0 = (k0 + _W0) & 0xFFFFFFFF
        k1 = (k1 + _W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


def cell_gauss(seed, cells):
    """Four standard normals per k-space cell index: shape (len(cells), 4)."""
    cells = np.asarray(cells, dtype=np.uint64)
    key = (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u = []
    for b in range(2):
        w = philox4x32_10((cells & _MASK32, cells >> np.uint64(32),
                           np.full_like(cells, b), np.full_like(cells, _TAG)), key)
        for q in range(2):
            v = (w[2 * q] << np.uint64(21)) ^ (w[2 * q + 1] >> np.uint64(11))
            v &= np.uint64((1 << 53) - 1)
            u.append((v.astype(np.float64) + 0.5) * 2.0 ** -53)
    out = np.empty((len(cells), 4))
    for q in range(2):
        r = np.sqrt(-2.0 * np.log(u[2 * q]))
        a = 2.0 * PI * u[2 * q + 1]
        out[:, 2 * q] = r * np.cos(a)
        out[:, 2 * q + 1] = r * np.sin(a)
    return out


def _kaxis(n, L):
    """k of FFT index i in 1/kpc, wrapped for the upper half
    (ternd_dft.cc:60-62, brnd_es.cc:106-108)."""
    i = np.arange(n, dtype=np.float64)
    k = KPC * i / L
    k[np.arange(n) >= (n + 1) // 2] -= KPC * n / L
    return k


def _box(desc):
    n = (int(desc.nx), int(desc.ny), int(desc.nz))
    lo = (desc.x_min, desc.y_min, desc.z_min)
    L = (desc.x_max - desc.x_min, desc.y_max - desc.y_min, desc.z_max - desc.z_min)
    return n, lo, L


def _kgrid(desc):
    n, _, L = _box(desc)
    kx, ky, kz = (_kaxis(n[a], L[a]) for a in range(3))
    return np.meshgrid(kx, ky, kz, indexing="ij")


def vertices(desc):
    """Vertex positions i*L/(n-1) + min (ternd_dft.cc:105-113)."""
    n, lo, L = _box(desc)
    ax = [np.arange(n[a]) * L[a] / (n[a] - 1) + lo[a] for a in range(3)]
    return np.meshgrid(*ax, indexing="ij")


def _profile(x, y, z, observer, r0, z0):
    """spatial_profile (ternd_dft.cc:26-33, brnd_es.cc:53-59)."""
    r_cyl = np.sqrt(x * x + y * y) - abs(observer[0])
    zz = np.abs(z) - abs(observer[2])
    return np.exp(-r_cyl / r0) * np.exp(-zz / z0)


def _sym(a):
    """a[-k]: index 0 maps to itself, i to n - i on every axis."""
    return np.roll(a[::-1, ::-1, ::-1], 1, axis=(0, 1, 2))


def _var_first_doubles(c):
    """toolkit::variance over the first c.size doubles of the interleaved
    (Re, Im) array (include/toolkit.h:70-78)."""
    d = np.ascontiguousarray(c).reshape(-1).view(np.float64)[: c.size]
    return np.mean((d - np.mean(d)) ** 2)


def ternd_dft(desc, p, observer, seed):
    """TErnd_dft::write_grid; returns te as an (nx, ny, nz) array."""
    n, _, _ = _box(desc)
    N = n[0] * n[1] * n[2]
    kx, ky, kz = _kgrid(desc)
    ks = np.sqrt(kx * kx + ky * ky + kz * kz).reshape(-1)
    dk3 = KPC ** 3 / np.prod(_box(desc)[2])
    spec = np.zeros(N)
    nz = ks >= p.k0  # spectrum(): 0 below k0 (ternd_dft.cc:17-24)
    spec[nz] = p.rms * (ks[nz] / p.k0) ** p.a0 / (4 * PI * ks[nz] ** 2)
    sigma = np.sqrt(spec * dk3)
    g = cell_gauss(seed, np.arange(N))
    c = sigma * g[:, 0] + 1j * sigma * g[:, 1]
    c[0] = 0.0
    c = np.fft.ifftn(c.reshape(n)) * N  # FFTW_BACKWARD, unnormalised
    var_invsq = 1.0 / np.sqrt(_var_first_doubles(c))
    x, y, z = vertices(desc)
    ratio = np.sqrt(_profile(x, y, z, observer, p.r0, p.z0)) * p.rms * var_invsq
    return c.real * ratio


def spectrum_es(k, p):
    """Brnd_es::spectrum (brnd_es.cc:34-49)."""
    p0 = p.rms * p.rms
    unit = 1.0 / (4.0 * PI * k * k)
    band1 = (k < p.k1).astype(np.float64)
    band2 = ((k > p.k1) & (k < p.k0)).astype(np.float64)
    band3 = (k > p.k0).astype(np.float64)
    P = (band1 * (p.k0 / p.k1) ** p.a1 * (k / p.k1) ** 6.0 + band2 / (k / p.k0) ** p.a1
         + band3 / (k / p.k0) ** p.a0)
    return P * p0 * unit


def brnd_es(desc, p, observer, seed, breg_at):
    """Brnd_es::write_grid; breg_at(x, y, z) -> (..., 3) regular field at
    the vertices (Breg::read_field).  Returns (bx, by, bz)."""
    n, _, _ = _box(desc)
    N = n[0] * n[1] * n[2]
    kx, ky, kz = _kgrid(desc)
    ks = np.sqrt(kx * kx + ky * ky + kz * kz).reshape(-1)
    dk3 = KPC ** 3 / np.prod(_box(desc)[2])
    with np.errstate(divide="ignore", invalid="ignore"):
        sigma = np.sqrt(1.0 / 3.0 * spectrum_es(ks, p) * dk3)
    sigma[0] = 0.0
    g = cell_gauss(seed, np.arange(N))
    c0 = sigma * g[:, 0] + 1j * sigma * g[:, 1]
    c1 = sigma * g[:, 2] + 1j * sigma * g[:, 3]
    c0[0] = c1[0] = 0.0
    c0 = np.fft.ifftn(c0.reshape(n)) * N
    c1 = np.fft.ifftn(c1.reshape(n)) * N
    # STEP II: profile and anisotropy (brnd_es.cc:157-204)
    var_invsq = 1.0 / np.sqrt(3.0 * _var_first_doubles(c0))
    x, y, z = vertices(desc)
    ratio = np.sqrt(_profile(x, y, z, observer, p.r0, p.z0)) * p.rms * var_invsq
    b = np.stack([c0.real * ratio, c0.imag * ratio, c1.imag * ratio], axis=-1)
    H = np.asarray(breg_at(x, y, z), dtype=np.float64).reshape(b.shape)
    hl2 = np.sum(H * H, axis=-1, keepdims=True)
    with np.errstate(divide="ignore", invalid="ignore"):
        h = np.where(hl2 != 0, H / np.sqrt(hl2), 0.0)
    rho = p.rho
    rhonorm = 1.0 / np.sqrt(1.0 / 3.0 * rho * rho + 2.0 / 3.0 / (rho * rho))
    par = h * np.sum(h * b, axis=-1, keepdims=True)
    perp = b - par
    bn = (par * rho + perp / rho) * rhonorm
    keep = (np.sum(h * h, axis=-1) < 1e-10)  # no preferred direction: unscaled
    c0 = np.where(keep, c0, bn[..., 0] + 1j * bn[..., 1])
    c1 = np.where(keep, c1, bn[..., 1] + 1j * bn[..., 2])
    c0 = np.fft.fftn(c0)
    c1 = np.fft.fftn(c1)
    # STEP III: Hermitian part, Gram-Schmidt, sqrt(2) (brnd_es.cc:209-259)
    t = np.stack([0.5 * (c0.real + _sym(c0.real)), 0.5 * (c1.real + _sym(c1.real)),
                  0.5 * (c1.imag + _sym(c1.imag))], axis=-1)
    k = np.stack([kx, ky, kz], axis=-1)
    kk = np.sum(k * k, axis=-1, keepdims=True)
    bb = np.sum(t * t, axis=-1, keepdims=True)
    with np.errstate(divide="ignore", invalid="ignore"):
        proj = np.sqrt(3.0) * (t - k * np.sum(k * t, axis=-1, keepdims=True) / kk)
    f = np.where((kk == 0) | (bb == 0), t, proj)
    bx, by, bz = (np.sqrt(2.0) * f[..., a] for a in range(3))
    # re-pack, backward, Hermitian part over N (brnd_es.cc:264-308)
    c0 = np.fft.ifftn(bx + 1j * by) * N
    c1 = np.fft.ifftn(by + 1j * bz) * N
    return (0.5 * (c0.real + _sym(c0.real)) / N, 0.5 * (c1.real + _sym(c1.real)) / N,
            0.5 * (c1.imag + _sym(c1.imag)) / N)
