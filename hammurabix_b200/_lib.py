"""Loader and ctypes signatures of lib/libhxg.so (the C ABI, include/hxg.h).

There is no fallback: if the library is missing or no CUDA device is
visible, every compute call raises HxgError.
"""
import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libhxg.so")

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_h = C.c_void_p

# name -> (restype, argtypes); one entry per function declared in include/hxg.h
SIGNATURES = {
    "hxg_abi_version": (C.c_int, []),
    "hxg_device_count": (C.c_int, []),
    "hxg_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_h)]),
    "hxg_destroy": (C.c_int, [_h]),
    "hxg_last_error": (C.c_char_p, [_h]),
    "hxg_set_stream": (C.c_int, [_h, _vp]),
    "hxg_set_models": (C.c_int, [_h, C.POINTER(abi.Models)]),
    "hxg_upload_grid": (C.c_int, [_h, C.c_int, C.POINTER(abi.GridDesc), _dp, _dp, _dp]),
    "hxg_upload_grid_device": (C.c_int, [_h, C.c_int, C.POINTER(abi.GridDesc), _vp, _vp, _vp]),
    "hxg_upload_grid_f32": (C.c_int, [_h, C.c_int, C.POINTER(abi.GridDesc), _vp, _vp, _vp]),
    "hxg_set_mask": (C.c_int, [_h, C.c_uint32, _dp]),
    "hxg_write_grid": (C.c_int, [_h, C.POINTER(abi.Obs), _dp, _dp, _dp, _dp, _dp]),
    "hxg_write_grid_device": (C.c_int, [_h, C.POINTER(abi.Obs), _vp, _vp, _vp, _vp, _vp]),
    "hxg_sync": (C.c_int, [_h]),
    "hxg_set_timing": (C.c_int, [_h, C.c_int]),
    "hxg_get_timing": (C.c_int, [_h, _dp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "hxg_get_launch_count": (C.c_int, [_h, C.POINTER(C.c_int64)]),
    "hxg_set_interp_cache": (C.c_int, [_h, C.c_uint64]),
    "hxg_write_grid_noalloc": (C.c_int, [C.POINTER(abi.Obs), C.POINTER(abi.Models),
                                         C.POINTER(abi.GridDesc), _vp, _vp, _vp, _vp, _vp,
                                         _vp, _vp]),
    "hxg_set_checkpointing": (C.c_int, [_h, C.c_int]),
    "hxg_adjoint_shard_begin": (C.c_int, [_h, C.POINTER(abi.Obs), C.c_uint32, C.c_uint32]),
    "hxg_adjoint_shard_shell": (C.c_int, [_h, C.POINTER(abi.Obs), C.c_uint32, _vp, _vp, _vp,
                                          _vp, _vp, _vp]),
    "hxg_adjoint_shard_finish": (C.c_int, [_h, _vp, _vp, _vp, _vp, _vp]),
    "hxg_adjoint_device": (C.c_int, [_h, C.POINTER(abi.Obs), _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                     _vp, _vp, _vp]),
    "hxg_shell_ref": (C.c_int, [C.POINTER(abi.Obs), C.c_uint32, _dp, _dp,
                                C.POINTER(C.c_uint64)]),
    "hxg_mask_duplicate": (C.c_int, [C.c_uint32, _dp, C.c_uint32, _dp]),
    "hxg_pix2ang": (C.c_int, [C.c_uint32, C.c_uint64, _dp, _dp]),
    "hxg_interpolate": (C.c_int, [C.c_uint32, _dp, C.c_uint64, _dp, _dp, _dp]),
    "hxg_accumulate": (C.c_int, [C.c_uint32, _dp, C.c_uint32, _dp]),
    "hxg_los_geometry": (C.c_int, [C.c_uint64, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "hxg_read_grid": (C.c_int, [_h, C.c_int, C.c_uint64, _dp, _dp]),
    "hxg_upload_grid_file": (C.c_int, [_h, C.c_int, C.POINTER(abi.GridDesc), C.c_char_p]),
    "hxg_synchrotron": (C.c_int, [C.c_int, C.c_uint64, _dp, _dp]),
    "hxg_download_grid": (C.c_int, [_h, C.c_int, _dp, _dp, _dp]),
    "hxg_write_grid_multi": (C.c_int, [_h, C.c_int, C.POINTER(abi.Obs), C.POINTER(_vp)]),
    "hxg_write_grid_multi_host": (C.c_int, [_h, C.c_int, C.POINTER(abi.Obs), C.POINTER(_vp)]),
    "hxg_shell_integrate_multi_device": (C.c_int, [_h, C.c_int, C.POINTER(abi.Obs), C.c_uint32,
                                                   C.c_uint32, C.c_uint32, _vp, _vp, _vp,
                                                   C.POINTER(_vp)]),
    "hxg_shell_integrate_device": (C.c_int, [_h, C.POINTER(abi.Obs), C.c_uint32, C.c_uint32,
                                             C.c_uint32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hxg_shell_merge_device": (C.c_int, [_h, C.POINTER(abi.Obs), C.c_uint32, _vp, _vp, _vp,
                                         _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hxg_export_grid_file": (C.c_int, [_h, C.c_int, C.c_char_p]),
    "hxg_generate_brnd_es": (C.c_int, [_h, C.POINTER(abi.GridDesc), C.POINTER(abi.BrndEs),
                                       _dp, C.c_uint64]),
    "hxg_generate_ternd_dft": (C.c_int, [_h, C.POINTER(abi.GridDesc), C.POINTER(abi.TerndDft),
                                         _dp, C.c_uint64]),
    "hxg_batch_create": (C.c_int, [_h, C.c_int, C.POINTER(abi.BatchEntry), C.c_int,
                                   C.POINTER(_vp)]),
    "hxg_batch_run": (C.c_int, [_vp]),
    "hxg_batch_info": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int), _dp, C.POINTER(C.c_int64)]),
    "hxg_batch_destroy": (C.c_int, [_vp]),
}


class HxgError(RuntimeError):
    """A non-zero status from the C ABI (the reference throws
    std::runtime_error where this library returns a status)."""

    def __init__(self, status, message=""):
        self.status = status
        name = abi.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{name}: {message}" if message else name)


_LIB = None


def load():
    """Load lib/libhxg.so once; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise HxgError(abi.HXG_ERR_NO_DEVICE,
                       f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.hxg_abi_version() != abi.HXG_ABI_VERSION:
        raise HxgError(abi.HXG_ERR_INVALID, "ABI version mismatch")
    _LIB = lib
    return lib


def check(status, handle=None):
    if status != abi.HXG_OK:
        msg = ""
        if handle is not None:
            m = load().hxg_last_error(handle)
            msg = m.decode() if m else ""
        raise HxgError(status, msg)


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)
