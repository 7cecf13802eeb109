"""hxg_write_grid_noalloc: the integrator for callers that cannot allocate
device memory (host applications that own every device allocation,
real-time loops that must not touch the allocator after start-up).  It must give the same maps as
the ordinary entry point, twice in a row, with its scratch held in a fixed
static device array.  Collected last so that a failure here leaves the rest
of the suite already run."""
import ctypes as C

import numpy as np
import pytest

import cases
from conftest import rel_err
from hammurabix_b200 import _lib, abi
from hammurabix_b200.integrator import Integrator

pytestmark = pytest.mark.gpu

TOL = {"dm": 1e-12, "fd": 1e-12, "is": 1e-12, "qs": 1e-12, "us": 1e-12}
KEYS = ("dm", "fd", "is", "qs", "us")


def _vp(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _outputs(torch, o):
    ndm, nfd, nsy = abi.obs_output_sizes(o)
    mk = lambda n: torch.full((n,), 123.0, dtype=torch.float64, device="cuda") if n else None
    return {"dm": mk(ndm), "fd": mk(nfd), "is": mk(nsy), "qs": mk(nsy), "us": mk(nsy)}


def test_noalloc_matches_write_grid(fields32):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    passes, models, grids, _ = cases.case_grid_small(fields32)
    desc, bcomps = grids[abi.HXG_FIELD_BRND]
    _, tcomps = grids[abi.HXG_FIELD_TEREG]
    # the caller packs its grid: FP64 records {bx, by, bz, ne} per voxel
    rec = torch.tensor(np.stack(list(bcomps) + list(tcomps), axis=1), dtype=torch.float64,
                       device="cuda").contiguous()
    stream = torch.cuda.Stream()
    with Integrator("fp64") as integ:
        integ.set_models(models)
        for field, (d, comps) in grids.items():
            integ.upload_grid(field, d, comps)
        expect = [integ.write_grid(o) for o in passes]
    for call in range(2):
        for o, exp in zip(passes, expect):
            out = _outputs(torch, o)
            # the outputs and records were written on torch's stream; the
            # entry point's stream must not start before those writes land
            stream.wait_stream(torch.cuda.current_stream())
            st = lib.hxg_write_grid_noalloc(
                C.byref(o), C.byref(models), C.byref(desc), _vp(rec),
                *(_vp(out[k]) for k in KEYS), C.c_void_p(stream.cuda_stream))
            assert st == abi.HXG_OK, abi.STATUS_NAMES.get(st, st)
            stream.synchronize()
            for k in KEYS:
                if exp[k] is None:
                    continue
                got = out[k].cpu().numpy()
                assert rel_err(got, exp[k]) <= TOL[k], (call, k, rel_err(got, exp[k]))
                assert np.abs(exp[k]).max() > 0


def test_noalloc_analytic_config1():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    (o,), models, _, _ = cases.case_config1()
    with Integrator("fp64") as integ:
        integ.set_models(models)
        exp = integ.write_grid(o)
    for call in range(2):
        out = _outputs(torch, o)
        st = lib.hxg_write_grid_noalloc(C.byref(o), C.byref(models), None, None,
                                        *(_vp(out[k]) for k in KEYS), None)
        assert st == abi.HXG_OK, abi.STATUS_NAMES.get(st, st)
        torch.cuda.synchronize()
        for k in KEYS:
            assert rel_err(out[k].cpu().numpy(), exp[k]) <= TOL[k], (call, k)


def test_noalloc_rejects_oversized_and_masked():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    (o,), models, _, _ = cases.case_config1()
    big = abi.Obs.from_buffer_copy(o)
    big.nside_shell[0] = 2 * abi.HXG_NOALLOC_MAX_NSIDE
    big.nside_dm = big.nside_fd = big.nside_sync = 2 * abi.HXG_NOALLOC_MAX_NSIDE
    out = _outputs(torch, big)
    st = lib.hxg_write_grid_noalloc(C.byref(big), C.byref(models), None, None,
                                    *(_vp(out[k]) for k in KEYS), None)
    assert st == abi.HXG_ERR_TOO_LARGE
    masked = abi.Obs.from_buffer_copy(o)
    masked.do_mask = 1
    out = _outputs(torch, masked)
    st = lib.hxg_write_grid_noalloc(C.byref(masked), C.byref(models), None, None,
                                    *(_vp(out[k]) for k in KEYS), None)
    assert st == abi.HXG_ERR_UNSUPPORTED
