"""Python face of the B200 integrator: the reference's
Integrator::write_grid (source/integrator/integrator.cc:23-134) over the C ABI.

    integ = Integrator(precision="fp64")          # or "fp32c"
    integ.set_models(models)                      # abi.Models
    integ.upload_grid(abi.HXG_FIELD_BRND, desc, [bx, by, bz])
    maps = integ.write_grid(obs)                  # dict dm/fd/is/qs/us (numpy)

Device-resident inputs and outputs (torch CUDA tensors) go through
``upload_grid_device`` and ``write_grid_device``.  Those calls are ordered
like torch ops on torch's current stream: the library's stream waits for
the work queued there before the call, and torch's stream waits for the
library's launches after it.
"""
import ctypes as C
import os

import numpy as np

from . import _lib, abi

PRECISIONS = {"fp64": abi.HXG_FP64, "fp32c": abi.HXG_FP32C}


class Integrator:
    def __init__(self, precision="fp64", device=0):
        self._lib = _lib.load()
        self.precision = precision
        h = C.c_void_p()
        _lib.check(self._lib.hxg_create(int(device), PRECISIONS[precision], C.byref(h)))
        self._h = h
        self.device = device
        self._stream = None   # torch stream object of the handle's stream

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hxg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- configuration -------------------------------------------------
    def set_models(self, models):
        _lib.check(self._lib.hxg_set_models(self._h, C.byref(models)), self._h)

    def set_stream(self, stream_ptr):
        """Launch on a CUDA stream (integer cudaStream_t, e.g.
        torch.cuda.current_stream().cuda_stream); 0 = the handle's own."""
        _lib.check(self._lib.hxg_set_stream(self._h, C.c_void_p(stream_ptr or None)), self._h)
        self._stream = None
        if stream_ptr:
            import torch
            self._stream = torch.cuda.ExternalStream(
                stream_ptr, device=torch.device("cuda", self.device))

    def _ordered(self, call):
        """Run call() (a C entry point returning a status) that reads or
        writes torch CUDA tensors, ordered with torch's current stream.  The
        first such call on a handle without a stream of the caller's gives
        the handle a torch stream, so both ends can wait on events."""
        import torch
        if self._stream is None:
            s = torch.cuda.Stream(self.device)
            _lib.check(self._lib.hxg_set_stream(self._h, C.c_void_p(s.cuda_stream)), self._h)
            self._stream = s
        cur = torch.cuda.current_stream(self.device)
        same = cur.cuda_stream == self._stream.cuda_stream
        if not same:
            self._stream.wait_stream(cur)
        try:
            _lib.check(call(), self._h)
        finally:
            if not same:
                cur.wait_stream(self._stream)

    def upload_grid(self, field, desc, comps):
        """Host SoA arrays in the Grid_* layout (x-major, z fastest): FP64
        (hxg_upload_grid), or FP32 when every component is float32
        (hxg_upload_grid_f32: half the bytes, the same slot values)."""
        if all(isinstance(a, np.ndarray) and a.dtype == np.float32 for a in comps):
            arrs = [np.ascontiguousarray(a).reshape(-1) for a in comps]
            ptrs = [C.c_void_p(a.ctypes.data) for a in arrs] + [None] * (3 - len(arrs))
            _lib.check(self._lib.hxg_upload_grid_f32(self._h, int(field), C.byref(desc), *ptrs),
                       self._h)
            return
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in comps]
        ptrs = [_lib.dptr(a) for a in arrs] + [None] * (3 - len(arrs))
        _lib.check(self._lib.hxg_upload_grid(self._h, int(field), C.byref(desc), *ptrs),
                   self._h)

    def upload_grid_device(self, field, desc, comps):
        """Device FP64 SoA arrays (torch CUDA float64 tensors, contiguous)."""
        ptrs = [C.c_void_p(t.data_ptr()) for t in comps] + [None] * (3 - len(comps))
        self._ordered(lambda: self._lib.hxg_upload_grid_device(self._h, int(field),
                                                               C.byref(desc), *ptrs))

    def upload_grid_file(self, field, desc, path):
        """Load a grid from the reference's binary grid file
        (hxg_upload_grid_file: chunked pinned reads, device-side split)."""
        _lib.check(self._lib.hxg_upload_grid_file(self._h, field, C.byref(desc),
                                                  os.fsencode(path)), self._h)

    def download_grid(self, field, desc):
        """A slot's FP64 SoA arrays as numpy arrays (hxg_download_grid),
        shaped (nx, ny, nz) (flat for the CRE slot); desc is the slot's
        geometry."""
        vec = field in (abi.HXG_FIELD_BREG, abi.HXG_FIELD_BRND)
        n = desc.nx * desc.ny * desc.nz * (desc.nE if field == abi.HXG_FIELD_CRE else 1)
        out = [np.zeros(n) for _ in range(3 if vec else 1)]
        ptrs = [_lib.dptr(a) for a in out] + [None] * (3 - len(out))
        _lib.check(self._lib.hxg_download_grid(self._h, int(field), *ptrs), self._h)
        if field != abi.HXG_FIELD_CRE:
            out = [a.reshape(desc.nx, desc.ny, desc.nz) for a in out]
        return out

    def export_grid_file(self, field, path):
        """Write a slot in the reference's binary grid format
        (hxg_export_grid_file, Grid_*::export_grid)."""
        _lib.check(self._lib.hxg_export_grid_file(self._h, int(field), os.fsencode(path)),
                   self._h)

    def generate_brnd_es(self, desc, params, observer, seed):
        """Brnd_es::write_grid on the device into the BRND slot
        (hxg_generate_brnd_es); the anisotropy follows the regular field of
        the models set on this handle."""
        obs = (C.c_double * 3)(*observer)
        _lib.check(self._lib.hxg_generate_brnd_es(self._h, C.byref(desc), C.byref(params), obs,
                                                  C.c_uint64(seed)), self._h)

    def generate_ternd_dft(self, desc, params, observer, seed):
        """TErnd_dft::write_grid on the device into the TERND slot."""
        obs = (C.c_double * 3)(*observer)
        _lib.check(self._lib.hxg_generate_ternd_dft(self._h, C.byref(desc), C.byref(params),
                                                    obs, C.c_uint64(seed)), self._h)

    def set_mask(self, nside, mask):
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        _lib.check(self._lib.hxg_set_mask(self._h, int(nside), _lib.dptr(m)), self._h)

    # ---- integration -----------------------------------------------------
    def write_grid(self, obs, out=None):
        """One frequency pass; returns the Grid_obs maps (before
        Grid_obs::export_grid's unit rescale) as float64 numpy arrays.
        ``out`` may supply the destination arrays (dict dm/fd/is/qs/us of
        C-contiguous float64 arrays of the right sizes, e.g. pinned memory)."""
        ndm, nfd, nsy = abi.obs_output_sizes(obs)
        sizes = {"dm": ndm, "fd": nfd, "is": nsy, "qs": nsy, "us": nsy}
        if out is None:
            out = {k: (np.zeros(n) if n else None) for k, n in sizes.items()}
        else:
            out = {k: (out[k][:n] if n else None) for k, n in sizes.items()}
        _lib.check(self._lib.hxg_write_grid(
            self._h, C.byref(obs), *(_lib.dptr(out[k]) for k in ("dm", "fd", "is", "qs", "us"))),
            self._h)
        return out

    def write_grid_device(self, obs, dm=None, fd=None, is_=None, qs=None, us=None):
        """Asynchronous variant writing into device buffers (torch CUDA
        float64 tensors) on the handle's stream."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        self._ordered(lambda: self._lib.hxg_write_grid_device(
            self._h, C.byref(obs), ptr(dm), ptr(fd), ptr(is_), ptr(qs), ptr(us)))

    def sync(self):
        _lib.check(self._lib.hxg_sync(self._h), self._h)

    def write_grid_multi(self, passes, out=None):
        """hxg_write_grid_multi_host: passes is a list of Obs; returns one
        dict dm/fd/is/qs/us of float64 numpy maps per pass (None where the
        pass writes no such map).  ``out`` may supply them (one dict per
        pass of C-contiguous float64 arrays of the right sizes, e.g. pinned
        memory), as in write_grid."""
        keys = ("dm", "fd", "is", "qs", "us")
        n = len(passes)
        obs = (abi.Obs * n)(*passes)
        given = out
        out, ptrs = [], (C.c_void_p * (5 * n))()
        for k, o in enumerate(passes):
            ndm, nfd, nsy = abi.obs_output_sizes(o)
            sizes = (ndm, nfd, nsy, nsy, nsy)
            if given is None:
                maps = {key: (np.zeros(c) if c else None) for key, c in zip(keys, sizes)}
            else:
                maps = {key: (given[k][key][:c] if c else None) for key, c in zip(keys, sizes)}
            for j, key in enumerate(keys):
                if maps[key] is not None:
                    ptrs[5 * k + j] = maps[key].ctypes.data
            out.append(maps)
        _lib.check(self._lib.hxg_write_grid_multi_host(self._h, n, obs, ptrs), self._h)
        return out

    def write_grid_multi_device(self, passes):
        """Several frequency passes at once (hxg_write_grid_multi): passes is
        a list of (obs, [dm, fd, is, qs, us]) with torch CUDA float64 tensors
        (None where the pass writes no such map).  In the FP32C form up to
        three passes with the same geometry share one traversal per shell."""
        n = len(passes)
        obs = (abi.Obs * n)(*[o for o, _ in passes])
        ptrs = (C.c_void_p * (5 * n))()
        for k, (_, maps) in enumerate(passes):
            for j, t in enumerate(maps):
                ptrs[5 * k + j] = t.data_ptr() if t is not None else None
        self._ordered(lambda: self._lib.hxg_write_grid_multi(self._h, n, obs, ptrs))

    # ---- one shell over a shard of its pixels ---------------------------------
    def shell_integrate_device(self, obs, shell, shard, nshards, fd, tmp):
        """Shell `shell` for the pixels of shard `shard` of `nshards` into the
        shell maps tmp = [dm, fd, is, qs, us] (torch CUDA float64 tensors of
        at least 12 nside_shell^2 elements, or None where obs needs none);
        fd = the accumulated FD output (hxg_shell_integrate_device)."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        self._ordered(lambda: self._lib.hxg_shell_integrate_device(
            self._h, C.byref(obs), int(shell), int(shard), int(nshards), ptr(fd),
            *(ptr(t) for t in tmp)))

    def shell_integrate_multi_device(self, passes, shell, shard, nshards, fd, tmp_dm, tmp_fd,
                                     tmp_iqu):
        """hxg_shell_integrate_multi_device: 2 or 3 fusable passes (list of
        Obs) in one traversal; tmp_iqu = one [I, Q, U] list per pass."""
        n = len(passes)
        obs = (abi.Obs * n)(*passes)
        iqu = (C.c_void_p * (3 * n))(*[t.data_ptr() for maps in tmp_iqu for t in maps])
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        self._ordered(lambda: self._lib.hxg_shell_integrate_multi_device(
            self._h, n, obs, int(shell), int(shard), int(nshards), ptr(fd), ptr(tmp_dm),
            ptr(tmp_fd), iqu))

    def shell_merge_device(self, obs, shell, tmp, outs):
        """Accumulate shell maps tmp into the pass outputs outs = [dm, fd, is,
        qs, us] (hxg_shell_merge_device)."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        self._ordered(lambda: self._lib.hxg_shell_merge_device(
            self._h, C.byref(obs), int(shell), *(ptr(t) for t in tmp),
            *(ptr(t) for t in outs)))

    # ---- adjoint -----------------------------------------------------------
    def set_checkpointing(self, enable=True):
        """Store per-shell checkpoints in write_grid_device for adjoint()."""
        _lib.check(self._lib.hxg_set_checkpointing(self._h, int(bool(enable))), self._h)

    def adjoint_device(self, obs, g_dm=None, g_fd=None, g_is=None, g_qs=None, g_us=None,
                       grad_params=None, grad_b=None, grad_ne=None):
        """dL/d(maps) (torch CUDA float64) -> fills grad_params
        (HXG_NUM_PARAMS), grad_b (3 tensors, one per B component) and
        grad_ne (one tensor) with dL/d(parameters) and dL/d(grid values)."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        gb = list(grad_b) if grad_b is not None else [None, None, None]
        self._ordered(lambda: self._lib.hxg_adjoint_device(
            self._h, C.byref(obs), ptr(g_dm), ptr(g_fd), ptr(g_is), ptr(g_qs), ptr(g_us),
            ptr(grad_params), ptr(gb[0]), ptr(gb[1]), ptr(gb[2]), ptr(grad_ne)))

    # ---- sharded adjoint (one rank's part; sharded.adjoint_sharded) ---------
    def adjoint_shard_begin(self, obs, shard, nshards):
        """hxg_adjoint_shard_begin: after write_grid_sharded's per-shell
        forward of shard `shard` of `nshards` with checkpointing on."""
        self._ordered(lambda: self._lib.hxg_adjoint_shard_begin(
            self._h, C.byref(obs), int(shard), int(nshards)))

    def adjoint_shard_shell(self, obs, shell, g_dm, g_fdmap, g_is, g_qs, g_us, gfd_inc):
        """hxg_adjoint_shard_shell (outermost shell first): gfd_inc receives
        this shard's inner-FD terms of the shell."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        self._ordered(lambda: self._lib.hxg_adjoint_shard_shell(
            self._h, C.byref(obs), int(shell), ptr(g_dm), ptr(g_fdmap), ptr(g_is), ptr(g_qs),
            ptr(g_us), ptr(gfd_inc)))

    def adjoint_shard_finish(self, grad_params=None, grad_b=None, grad_ne=None):
        """hxg_adjoint_shard_finish: this shard's gradients (their sum over
        the shards is the full gradient)."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        gb = list(grad_b) if grad_b is not None else [None, None, None]
        self._ordered(lambda: self._lib.hxg_adjoint_shard_finish(
            self._h, ptr(grad_params), ptr(gb[0]), ptr(gb[1]), ptr(gb[2]), ptr(grad_ne)))

    # ---- batched forward ---------------------------------------------------
    def batch(self, entries, tune=False):
        """Plan a batch of independent passes sharing this handle's grids.
        entries: iterable of (models, obs, outs) with outs a dict of torch
        CUDA float64 tensors keyed "dm", "fd", "is", "qs", "us" (the ones
        obs requests).  Returns a Batch; Batch.run() launches its graph."""
        return Batch(self, list(entries), tune)

    def set_interp_cache(self, nbytes):
        """Bound on the device bytes of the merges' interpolation tables
        (hxg_set_interp_cache; 0: weights found in place)."""
        _lib.check(self._lib.hxg_set_interp_cache(self._h, int(nbytes)), self._h)

    # ---- timing ----------------------------------------------------------
    def set_timing(self, enable=True):
        _lib.check(self._lib.hxg_set_timing(self._h, int(bool(enable))), self._h)

    def get_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        s = C.c_int64()
        _lib.check(self._lib.hxg_get_timing(self._h, C.byref(ms), C.byref(n), C.byref(s)),
                   self._h)
        return ms.value, n.value, s.value

    def launch_count(self):
        n = C.c_int64()
        _lib.check(self._lib.hxg_get_launch_count(self._h, C.byref(n)), self._h)
        return n.value

    def read_grid(self, field, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        n = len(pos) // 3
        vec = field in (abi.HXG_FIELD_BREG, abi.HXG_FIELD_BRND)
        out = np.zeros(3 * n if vec else n)
        _lib.check(self._lib.hxg_read_grid(self._h, int(field), C.c_uint64(n), _lib.dptr(pos),
                                           _lib.dptr(out)), self._h)
        return out.reshape(n, 3) if vec else out


# ---- stateless device helpers (known-answer entry points) -----------------

class Batch:
    """A planned batch (hxg_batch_create): one CUDA graph per run."""

    def __init__(self, integ, entries, tune):
        self._lib = integ._lib
        self._integ = integ
        arr = (abi.BatchEntry * len(entries))()
        self._keep = []
        for k, (models, obs, outs) in enumerate(entries):
            arr[k].models = models
            arr[k].obs = obs
            for key, field in (("dm", "d_dm"), ("fd", "d_fd"), ("is", "d_is"), ("qs", "d_qs"),
                               ("us", "d_us")):
                t = outs.get(key)
                if t is not None:
                    self._keep.append(t)
                    setattr(arr[k], field, t.data_ptr())
        self._b = C.c_void_p()
        integ._ordered(lambda: self._lib.hxg_batch_create(integ._h, len(entries), arr,
                                                          int(bool(tune)), C.byref(self._b)))

    def run(self):
        self._integ._ordered(lambda: self._lib.hxg_batch_run(self._b))

    def info(self):
        lanes, grain, tried = C.c_int(), C.c_int(), C.c_int()
        ms, samples = C.c_double(), C.c_int64()
        _lib.check(self._lib.hxg_batch_info(self._b, C.byref(lanes), C.byref(grain),
                                            C.byref(tried), C.byref(ms), C.byref(samples)))
        return {"lanes_per_pixel": lanes.value, "grain": grain.value, "shapes_tried": tried.value,
                "best_ms": ms.value, "samples": samples.value}

    def close(self):
        if self._b:
            self._lib.hxg_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pix2ang(nside):
    lib = _lib.load()
    n = abi.npix(nside)
    th, ph = np.zeros(n), np.zeros(n)
    _lib.check(lib.hxg_pix2ang(int(nside), n, _lib.dptr(th), _lib.dptr(ph)))
    return th, ph


def interpolate(nside, m, theta, phi):
    lib = _lib.load()
    m = np.ascontiguousarray(m, dtype=np.float64)
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.zeros(len(theta))
    _lib.check(lib.hxg_interpolate(int(nside), _lib.dptr(m), len(theta), _lib.dptr(theta),
                                   _lib.dptr(phi), _lib.dptr(out)))
    return out


def accumulate(nside_dst, dst, nside_src, src):
    lib = _lib.load()
    dst = np.array(dst, dtype=np.float64)
    src = np.ascontiguousarray(src, dtype=np.float64)
    _lib.check(lib.hxg_accumulate(int(nside_dst), _lib.dptr(dst), int(nside_src),
                                  _lib.dptr(src)))
    return dst


def synchrotron(which, x):
    """F(x) (which=1) or G(x) (which=2) from the library's tables
    (hxg_synchrotron)."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    out = np.zeros_like(x)
    _lib.check(lib.hxg_synchrotron(int(which), len(x), _lib.dptr(x), _lib.dptr(out)))
    return out


def los_geometry(theta, phi, b):
    lib = _lib.load()
    theta = np.ascontiguousarray(theta, dtype=np.float64)
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
    n = len(theta)
    ver, par, per = np.zeros(3 * n), np.zeros(n), np.zeros(n)
    c2, s2 = np.zeros(n), np.zeros(n)
    _lib.check(lib.hxg_los_geometry(n, _lib.dptr(theta), _lib.dptr(phi), _lib.dptr(b),
                                    _lib.dptr(ver), _lib.dptr(par), _lib.dptr(per),
                                    _lib.dptr(c2), _lib.dptr(s2)))
    return ver.reshape(n, 3), par, per, c2, s2


def shell_ref(obs, shell):
    lib = _lib.load()
    ds, dd, st = C.c_double(), C.c_double(), C.c_uint64()
    _lib.check(lib.hxg_shell_ref(C.byref(obs), int(shell), C.byref(ds), C.byref(dd),
                                 C.byref(st)))
    return ds.value, dd.value, st.value


def mask_duplicate(pivot_nside, mask, nside):
    lib = _lib.load()
    mask = np.ascontiguousarray(mask, dtype=np.float64)
    out = np.zeros(abi.npix(nside))
    _lib.check(lib.hxg_mask_duplicate(int(pivot_nside), _lib.dptr(mask), int(nside),
                                      _lib.dptr(out)))
    return out
