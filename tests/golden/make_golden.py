"""Generate the golden fixtures under tests/golden/ (run in the container
that holds the hammurabiX source tree; the outputs are committed).

1. reference_fixtures.npz -- the reference's own unit-test fixtures
   (tests/unit_tests/reference/*.bin of hammurabiX): healpy RING pointings
   (theta, phi) at Nside 2..32 (hamdis_tests.cc:156-232), the random maps of
   the interpolation test (hamdis_tests.cc:320-370) and the mask maps of the
   duplicate test (hamsk_tests.cc:11-56), as raw little-endian FP64.
2. int_tests_01.xml, int_tests_02.xml -- the shell-geometry parameter files
   of integrator_tests.cc:28-139, copied verbatim.
3. ref_maps.npz -- full DM / FD / I / Q / U maps computed by the reference
   integrator itself (compiled from its sources by oracle/Makefile) on the
   small cases of tests/cases.py, plus the FP32 field grids those cases use.
4. ref_models_ext.npz -- the same for the Breg_jaffe (ring and bar),
   Breg_jf12 and TEreg_ymw16 models with the parameter values of the
   reference's templates/params_template.xml (parsed by
   hammurabix_b200.param with Param's unit conversions); the hxg_models_t
   block of each case is stored beside its maps.
5. ref_cre_grid.npz -- the same for the CRE-grid emissivity on the power-law
   CRE grid of tests/cases.py:case_cre_grid (the reference built with the
   oracle's F and G, oracle/shim/shim.cc).
6. ref_rfg.npz -- Brnd_es / TErnd_dft fields generated by the reference's
   own generator code on the cases of tests/cases.py:case_rfg, run on one
   thread with the shim's cell-indexed Philox deviates and its direct-sum
   DFT (oracle/shim), i.e. the deviates the device generators draw; each
   case's hxg_models_t block is stored beside its field.

Usage: python tests/golden/make_golden.py <hammurabiX source dir>
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import cases  # noqa: E402
import pyoracle  # noqa: E402
from hammurabix_b200 import workloads as W  # noqa: E402


def reference_fixtures(src):
    fx = os.path.join(src, "tests", "unit_tests", "reference")
    out = {}
    for ns in (2, 4, 8, 16, 32):
        a = np.fromfile(os.path.join(fx, f"pointing_healpix_nside{ns}.bin"), dtype="<f8")
        out[f"pointing_nside{ns}"] = a.reshape(-1, 2)
    for ns in (2, 4, 8):
        out[f"random_map_nside{ns}"] = np.fromfile(
            os.path.join(fx, f"random_map_nside{ns}.bin"), dtype="<f8")
    for ns in (2, 8, 64):
        out[f"mask_map_nside{ns}"] = np.fromfile(
            os.path.join(fx, f"mask_map_nside{ns}.bin"), dtype="<f8")
    np.savez_compressed(os.path.join(HERE, "reference_fixtures.npz"), **out)
    for name in ("int_tests_01.xml", "int_tests_02.xml"):
        shutil.copyfile(os.path.join(fx, name), os.path.join(HERE, name))


def _run(ref, passes, m, grids, mask, key, out):
    for i, o in enumerate(passes):
        kw = {}
        if mask is not None:
            kw = dict(mask_nside=mask[0], mask=mask[1])
        maps, _ = ref.write_grid(o, m, grids, **kw)
        for k, v in maps.items():
            if v is not None:
                out[f"{key}/pass{i}/{k}"] = v


def reference_maps():
    ref = pyoracle.Reference()
    out = {}
    fields32 = W.random_grids(32, 1, 2)
    for k, a in zip(("bx", "by", "bz", "ne"), fields32):
        out[f"fields32/{k}"] = a
    _run(ref, *cases.case_config1(), "config1", out)
    _run(ref, *cases.case_grid_small(fields32), "grid_small", out)
    _run(ref, *cases.case_grid_lowfreq(fields32), "grid_lowfreq", out)
    _run(ref, *cases.case_mask(), "mask", out)
    for name, passes, m in cases.case_models():
        _run(ref, passes, m, None, None, f"model_{name}", out)
    np.savez_compressed(os.path.join(HERE, "ref_maps.npz"), **out)


def _template_blocks(src):
    """jaffe / jf12 / ymw16 parameter blocks of the reference's template."""
    import tempfile
    import xml.etree.ElementTree as ET
    from hammurabix_b200.param import Param
    tree = ET.parse(os.path.join(src, "templates", "params_template.xml"))
    root = tree.getroot()
    blocks = {}
    for btype, tetype in (("jaffe", "ymw16"), ("jf12", "ymw16")):
        root.find("magneticfield").find("regular").set("type", btype)
        root.find("thermalelectron").find("regular").set("type", tetype)
        with tempfile.NamedTemporaryFile("w", suffix=".xml", delete=False) as f:
            tree.write(f, encoding="unicode")
        try:
            m = Param(f.name).models
        finally:
            os.unlink(f.name)
        blocks[btype] = getattr(m, btype)
        blocks["ymw16"] = m.ymw16
    return blocks


def reference_models_ext(src):
    ref = pyoracle.Reference()
    blocks = _template_blocks(src)
    out = {}
    for name, m in cases.case_models_ext(blocks):
        passes = cases.obs_models_ext()
        _run(ref, passes, m, None, None, name, out)
        out[f"{name}/models"] = np.frombuffer(bytes(m), dtype=np.uint8).copy()
    np.savez_compressed(os.path.join(HERE, "ref_models_ext.npz"), **out)


def reference_cre_grid():
    ref = pyoracle.Reference()
    out = {}
    _run(ref, *cases.case_cre_grid(), None, "cre_grid", out)
    np.savez_compressed(os.path.join(HERE, "ref_cre_grid.npz"), **out)


def reference_rfg(src):
    ref = pyoracle.Reference()
    blocks = _template_blocks(src)
    out = {}
    for name, kind, desc, p, seed, m, grids in cases.case_rfg(blocks["jf12"]):
        if kind == "ternd":
            out[f"{name}/te"] = ref.generate_ternd_dft(cases.RFG_OBSERVER, desc, p, seed)
        else:
            bx, by, bz = ref.generate_brnd_es(m, grids, cases.RFG_OBSERVER, desc, p, seed)
            out[f"{name}/bx"], out[f"{name}/by"], out[f"{name}/bz"] = bx, by, bz
            out[f"{name}/models"] = np.frombuffer(bytes(m), dtype=np.uint8).copy()
    np.savez_compressed(os.path.join(HERE, "ref_rfg.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <hammurabiX source dir>")
    src = sys.argv[1]
    reference_fixtures(src)
    reference_maps()
    reference_models_ext(src)
    reference_cre_grid()
    reference_rfg(src)
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
