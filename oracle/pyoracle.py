"""ctypes bindings of the test oracle (test infrastructure only).

- ``Oracle``: the plain-C FP64 restatement, oracle/_build/libhxo.so.
- ``Reference``: the reference hammurabiX integrator compiled from its own
  sources by oracle/Makefile, oracle/_ref/libhxref.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, and only as the checker / the timed CPU baseline.
"""
import ctypes as C
import os

import numpy as np

from hammurabix_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libhxo.so")
REF_SO = os.path.join(HERE, "_ref", "libhxref.so")
REF_HAMX = os.path.join(HERE, "_ref", "hamx")

_dp = C.POINTER(C.c_double)


class Grid(C.Structure):
    _fields_ = [("desc", abi.GridDesc), ("c", _dp * 3)]


class Grids(C.Structure):
    _fields_ = [("slot", Grid * 5)]


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def make_grids(grids):
    """grids: dict field -> (GridDesc, [arrays]) with float64 SoA arrays.

    Returns (Grids struct, keepalive list)."""
    g = Grids()
    keep = []
    for field, (desc, comps) in (grids or {}).items():
        g.slot[field].desc = desc
        for i, a in enumerate(comps):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            g.slot[field].c[i] = _ptr(a)
    return g, keep


def _alloc_outputs(obs):
    ndm, nfd, nsy = abi.obs_output_sizes(obs)
    out = {
        "dm": np.zeros(ndm) if ndm else None,
        "fd": np.zeros(nfd) if nfd else None,
        "is": np.zeros(nsy) if nsy else None,
        "qs": np.zeros(nsy) if nsy else None,
        "us": np.zeros(nsy) if nsy else None,
    }
    return out


class _Lib:
    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run `make -C oracle`)")
        self.lib = C.CDLL(path)


class Oracle(_Lib):
    """The plain-C restatement (oracle/hxo.c)."""

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.hxo_write_grid.restype = C.c_int
        L.hxo_temp_convert.restype = C.c_double
        L.hxo_tereg_field.restype = C.c_double

    def write_grid(self, obs, models, grids=None, mask=None, mask_nside=0):
        g, keep = make_grids(grids)
        out = _alloc_outputs(obs)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        st = self.lib.hxo_write_grid(C.byref(obs), C.byref(models), C.byref(g),
                                     C.c_uint32(mask_nside), _ptr(m),
                                     *(_ptr(out[k]) for k in ("dm", "fd", "is", "qs", "us")))
        if st != 0:
            raise RuntimeError(f"oracle write_grid failed: {abi.STATUS_NAMES.get(st, st)}")
        return out

    def shell_ref(self, obs, shell):
        ds, dd, st = C.c_double(), C.c_double(), C.c_uint64()
        rc = self.lib.hxo_shell_ref(C.byref(obs), C.c_uint32(shell), C.byref(ds),
                                    C.byref(dd), C.byref(st))
        if rc != 0:
            raise ValueError("bad shell")
        return ds.value, dd.value, st.value

    def pix2ang(self, nside):
        n = abi.npix(nside)
        th, ph = np.zeros(n), np.zeros(n)
        self.lib.hxo_pix2ang(C.c_uint32(nside), C.c_uint64(n), _ptr(th), _ptr(ph))
        return th, ph

    def interpolate(self, nside, m, theta, phi):
        m = np.ascontiguousarray(m, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros(len(theta))
        self.lib.hxo_interpolate(C.c_uint32(nside), _ptr(m), C.c_uint64(len(theta)),
                                 _ptr(theta), _ptr(phi), _ptr(out))
        return out

    def accumulate(self, nside_dst, dst, nside_src, src):
        dst = np.array(dst, dtype=np.float64)
        src = np.ascontiguousarray(src, dtype=np.float64)
        self.lib.hxo_accumulate(C.c_uint32(nside_dst), _ptr(dst), C.c_uint32(nside_src),
                                _ptr(src))
        return dst

    def mask_duplicate(self, pivot_nside, mask, nside):
        mask = np.ascontiguousarray(mask, dtype=np.float64)
        out = np.zeros(abi.npix(nside))
        self.lib.hxo_mask_duplicate(C.c_uint32(pivot_nside), _ptr(mask), C.c_uint32(nside),
                                    _ptr(out))
        return out

    def los_geometry(self, theta, phi, b):
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
        n = len(theta)
        ver, par, per, ipa = np.zeros(3 * n), np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.hxo_los_geometry(C.c_uint64(n), _ptr(theta), _ptr(phi), _ptr(b), _ptr(ver),
                                  _ptr(par), _ptr(per), _ptr(ipa))
        return ver.reshape(n, 3), par, per, ipa

    def read_grid(self, desc, comps, pos):
        g = Grid()
        g.desc = desc
        keep = [np.ascontiguousarray(a, dtype=np.float64) for a in comps]
        for i, a in enumerate(keep):
            g.c[i] = _ptr(a)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        n = len(pos) // 3
        nc = len(comps)
        out = np.zeros(n * nc)
        self.lib.hxo_read_grid(C.byref(g), C.c_int(nc), C.c_uint64(n), _ptr(pos), _ptr(out))
        return out.reshape(n, nc) if nc == 3 else out

    def temp_convert(self, t, freq):
        return self.lib.hxo_temp_convert(C.c_double(t), C.c_double(freq))

    def breg_field(self, models, observer, pos):
        """Analytic regular field (hxo_breg_field) at (n, 3) positions."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        out = np.zeros((len(pos), 3))
        obs = (C.c_double * 3)(*observer)
        o = (C.c_double * 3)()
        for i in range(len(pos)):
            self.lib.hxo_breg_field(C.byref(models), obs, (C.c_double * 3)(*pos[i]), o)
            out[i] = o[:]
        return out

    def sync_emissivity(self, models, observer, freq, pos, b_per):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        jt, jp = np.zeros(len(pos)), np.zeros(len(pos))
        obs = (C.c_double * 3)(*observer)
        for i in range(len(pos)):
            p = (C.c_double * 3)(*pos[i])
            a, b = C.c_double(), C.c_double()
            self.lib.hxo_sync_emissivity(C.byref(models), obs, C.c_double(freq), p,
                                         C.c_double(b_per[i]), C.byref(a), C.byref(b))
            jt[i], jp[i] = a.value, b.value
        return jt, jp


class Reference(_Lib):
    """The reference integrator compiled from its own sources (oracle/_ref)."""

    def __init__(self, path=REF_SO):
        super().__init__(path)
        L = self.lib
        L.hxref_write_grid.restype = C.c_int
        L.hxref_temp_convert.restype = C.c_double
        L.hxref_max_threads.restype = C.c_int

    def max_threads(self):
        return self.lib.hxref_max_threads()

    def write_grid(self, obs, models, grids=None, mask=None, mask_nside=0, nthreads=0):
        """Runs Integrator::write_grid; returns (maps, seconds of write_grid)."""
        g, keep = make_grids(grids)
        out = _alloc_outputs(obs)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        secs = C.c_double()
        st = self.lib.hxref_write_grid(C.byref(obs), C.byref(models), C.byref(g),
                                       C.c_uint32(mask_nside), _ptr(m),
                                       *(_ptr(out[k]) for k in ("dm", "fd", "is", "qs", "us")),
                                       C.c_int(nthreads), C.byref(secs))
        if st != 0:
            raise RuntimeError(f"reference write_grid failed: {abi.STATUS_NAMES.get(st, st)}")
        return out, secs.value

    def shell_ref(self, obs, shell):
        ds, dd, st = C.c_double(), C.c_double(), C.c_uint64()
        d0, d1 = obs.radii_shell[shell], obs.radii_shell[shell + 1]
        nmax = int((d1 - d0) / obs.oc_r_res) + 16
        dist = np.zeros(nmax)
        self.lib.hxref_shell_ref(C.byref(obs), C.c_uint32(shell), C.byref(ds), C.byref(dd),
                                 C.byref(st), _ptr(dist))
        return ds.value, dd.value, st.value, dist[:st.value]

    def pix2ang(self, nside):
        n = abi.npix(nside)
        th, ph = np.zeros(n), np.zeros(n)
        self.lib.hxref_pix2ang(C.c_uint32(nside), _ptr(th), _ptr(ph))
        return th, ph

    def interpolate(self, nside, m, theta, phi):
        m = np.ascontiguousarray(m, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros(len(theta))
        self.lib.hxref_interpolate(C.c_uint32(nside), _ptr(m), C.c_uint64(len(theta)),
                                   _ptr(theta), _ptr(phi), _ptr(out))
        return out

    def accumulate(self, nside_dst, dst, nside_src, src):
        dst = np.array(dst, dtype=np.float64)
        src = np.ascontiguousarray(src, dtype=np.float64)
        self.lib.hxref_accumulate(C.c_uint32(nside_dst), _ptr(dst), C.c_uint32(nside_src),
                                  _ptr(src))
        return dst

    def mask_duplicate(self, pivot_nside, mask, nside):
        mask = np.ascontiguousarray(mask, dtype=np.float64)
        out = np.zeros(abi.npix(nside))
        self.lib.hxref_mask_duplicate(C.c_uint32(pivot_nside), _ptr(mask), C.c_uint32(nside),
                                      _ptr(out))
        return out

    def los_geometry(self, theta, phi, b):
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
        n = len(theta)
        ver, par, per, ipa = np.zeros(3 * n), np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.hxref_los_geometry(C.c_uint64(n), _ptr(theta), _ptr(phi), _ptr(b), _ptr(ver),
                                    _ptr(par), _ptr(per), _ptr(ipa))
        return ver.reshape(n, 3), par, per, ipa

    def temp_convert(self, t, freq):
        return self.lib.hxref_temp_convert(C.c_double(t), C.c_double(freq))

    def read_field(self, field, models, grids, observer, pos):
        g, keep = make_grids(grids)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        n = len(pos) // 3
        vec = field in (abi.HXG_FIELD_BREG, abi.HXG_FIELD_BRND)
        out = np.zeros(3 * n if vec else n)
        obs = (C.c_double * 3)(*observer)
        st = self.lib.hxref_read_field(C.c_int(field), C.byref(models), C.byref(g), obs,
                                       C.c_uint64(n), _ptr(pos), _ptr(out))
        if st != 0:
            raise RuntimeError(f"reference read_field failed: {st}")
        return out.reshape(n, 3) if vec else out

    def sync_emissivity(self, models, observer, freq, pos, b_per, grids=None):
        g, keep = make_grids(grids)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        b_per = np.ascontiguousarray(b_per, dtype=np.float64)
        n = len(b_per)
        jt, jp = np.zeros(n), np.zeros(n)
        obs = (C.c_double * 3)(*observer)
        st = self.lib.hxref_sync_emissivity(C.byref(models), C.byref(g), obs, C.c_double(freq),
                                            C.c_uint64(n), _ptr(pos), _ptr(b_per), _ptr(jt),
                                            _ptr(jp))
        if st != 0:
            raise RuntimeError(f"reference sync_emissivity failed: {st}")
        return jt, jp

    def generate_brnd_es(self, models, grids, observer, desc, p, seed):
        """Brnd_es::write_grid on the reference with the cell-indexed
        deviates of the device generator; returns (bx, by, bz) as
        (nx, ny, nz) arrays."""
        g, keep = make_grids(grids)
        n = desc.nx * desc.ny * desc.nz
        out = [np.zeros(n) for _ in range(3)]
        obs = (C.c_double * 3)(*observer)
        st = self.lib.hxref_generate_brnd_es(C.byref(models), C.byref(g), obs, C.byref(desc),
                                             C.byref(p), C.c_uint64(seed), *(_ptr(a) for a in out))
        if st != 0:
            raise RuntimeError(f"reference Brnd_es failed: {st}")
        return [a.reshape(desc.nx, desc.ny, desc.nz) for a in out]

    def generate_ternd_dft(self, observer, desc, p, seed):
        """TErnd_dft::write_grid on the reference (cell-indexed deviates)."""
        n = desc.nx * desc.ny * desc.nz
        out = np.zeros(n)
        obs = (C.c_double * 3)(*observer)
        st = self.lib.hxref_generate_ternd_dft(obs, C.byref(desc), C.byref(p), C.c_uint64(seed),
                                               _ptr(out))
        if st != 0:
            raise RuntimeError(f"reference TErnd_dft failed: {st}")
        return out.reshape(desc.nx, desc.ny, desc.nz)
