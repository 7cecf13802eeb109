"""CPU tests of the C ABI: the library loads, exports every entry point
include/hxg.h declares, its struct layouts match the Python mirrors, the
host-only helpers agree with the oracle, and compute calls fail loudly
(HXG_ERR_NO_DEVICE) when no GPU is present."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from hammurabix_b200 import _lib, abi
from hammurabix_b200 import integrator as I

HEADER = os.path.join(ROOT, "include", "hxg.h")


def header_functions():
    src = open(HEADER).read()
    return set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(hxg_\w+)\s*\(", src, re.M))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert declared, "no declarations parsed"
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (hxg_\w+)", out))
    assert declared <= exported, declared - exported


def test_struct_layouts_match_header(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                    'int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                    ' sizeof(hxg_models_t), sizeof(hxg_obs_t), sizeof(hxg_grid_desc_t),'
                    ' offsetof(hxg_models_t, cre_unif), offsetof(hxg_obs_t, sync_freq),'
                    ' offsetof(hxg_models_t, ymw16), offsetof(hxg_grid_desc_t, E_fact),'
                    ' sizeof(hxg_batch_entry_t), offsetof(hxg_batch_entry_t, d_us));'
                    ' printf("%zu %zu\\n", sizeof(hxg_brnd_es_t), sizeof(hxg_ternd_dft_t));}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-o", str(exe), str(prog)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [C.sizeof(abi.Models), C.sizeof(abi.Obs), C.sizeof(abi.GridDesc),
            abi.Models.cre_unif.offset, abi.Obs.sync_freq.offset, abi.Models.ymw16.offset,
            abi.GridDesc.E_fact.offset, C.sizeof(abi.BatchEntry), abi.BatchEntry.d_us.offset,
            C.sizeof(abi.BrndEs), C.sizeof(abi.TerndDft)]
    assert got == want


def test_abi_version():
    assert _lib.load().hxg_abi_version() == abi.HXG_ABI_VERSION


def test_host_shell_ref_matches_oracle(oracle):
    from hammurabix_b200 import workloads as W
    for o in W.config_grid([64, 128, 256], 30.0, 0.01, [23.0]) + [W.config1()[0]]:
        for s in range(o.total_shell):
            assert I.shell_ref(o, s) == oracle.shell_ref(o, s)


def test_host_mask_duplicate_matches_fixtures(fixtures):
    m8 = fixtures["mask_map_nside8"]
    assert np.array_equal(I.mask_duplicate(8, m8, 2), fixtures["mask_map_nside2"])
    assert np.array_equal(I.mask_duplicate(8, m8, 64), fixtures["mask_map_nside64"])


def test_invalid_arguments_rejected():
    lib = _lib.load()
    assert lib.hxg_create(0, 7, C.byref(C.c_void_p())) == abi.HXG_ERR_INVALID
    assert lib.hxg_pix2ang(3, 10, None, None) == abi.HXG_ERR_INVALID
    assert lib.hxg_mask_duplicate(5, None, 4, None) == abi.HXG_ERR_INVALID


@pytest.mark.skipif(_lib.load().hxg_device_count() > 0, reason="a GPU is present")
def test_no_device_fails_loudly():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.hxg_create(0, abi.HXG_FP64, C.byref(h)) == abi.HXG_ERR_NO_DEVICE
    th, ph = np.zeros(48), np.zeros(48)
    assert lib.hxg_pix2ang(2, 48, _lib.dptr(th), _lib.dptr(ph)) == abi.HXG_ERR_NO_DEVICE
    with pytest.raises(_lib.HxgError):
        I.Integrator("fp64")
