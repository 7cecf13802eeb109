"""The link-time drop-in: the reference CLI (source/main/main_std.cc, the
unmodified Pipeline) built with integrator_b200.cc in place of the reference
integrator (hammurabix_b200/dropin/_build/hamx_b200), against the reference
CLI itself (oracle/_ref/hamx), on the same XML parameter file and the same
field-grid files.  Output maps are the files Grid_obs::export_grid writes
(source/grid/grid_obs.cc:53-82): raw FP64, DM in pc/cm^3, FD in rad/m^2,
I/Q/U in K.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err
from hammurabix_b200.param import Param

HAMX_REF = os.path.join(ROOT, "oracle", "_ref", "hamx")
HAMX_B200 = os.path.join(ROOT, "hammurabix_b200", "dropin", "_build", "hamx_b200")

XML = """<?xml version="1.0"?>
<root>
  <observable>
    <dm cue="1" filename="{d}/dm.bin" nside="16"/>
    <faraday cue="1" filename="{d}/fd.bin" nside="16"/>
    <sync cue="1" freq="0.408" filename="{d}/sync_0.408.bin" nside="16"/>
    <sync cue="1" freq="23" filename="{d}/sync_23.bin" nside="8"/>
  </observable>
  <mask cue="{mask}" filename="{d}/mask.bin" nside="8"/>
  <fieldio>
    <breg read="0" write="0" filename="{d}/breg.bin"/>
    <brnd read="1" write="0" filename="{d}/brnd.bin"/>
    <tereg read="1" write="0" filename="{d}/tereg.bin"/>
    <ternd read="0" write="0" filename="{d}/ternd.bin"/>
    <cre read="0" write="0" filename="{d}/cre.bin"/>
  </fieldio>
  <grid>
    <observer><x value="-8.3"/><y value="0"/><z value="0.006"/></observer>
    <box_brnd>
      <nx value="32"/><ny value="32"/><nz value="32"/>
      <x_min value="-20.0"/><x_max value="20.0"/><y_min value="-20.0"/>
      <y_max value="20.0"/><z_min value="-5.0"/><z_max value="5.0"/>
    </box_brnd>
    <box_tereg>
      <nx value="32"/><ny value="32"/><nz value="32"/>
      <x_min value="-20.0"/><x_max value="20.0"/><y_min value="-20.0"/>
      <y_max value="20.0"/><z_min value="-5.0"/><z_max value="5.0"/>
    </box_tereg>
    <shell>
      <layer type="auto">
        <auto><shell_num value="3"/><nside_sim value="4"/></auto>
      </layer>
      <oc_r_min value="0.0"/><oc_r_max value="30.0"/>
      <gc_r_min value="0.0"/><gc_r_max value="20.0"/>
      <gc_z_min value="-10.0"/><gc_z_max value="10.0"/>
      <oc_r_res value="0.05"/>
    </shell>
  </grid>
  <magneticfield>
    <regular cue="1" type="lsa">
      <lsa><b0 value="3.2"/><psi0 value="27.0"/><psi1 value="0.9"/><chi0 value="25.0"/></lsa>
    </regular>
    <random cue="1" type="global" seed="0"/>
  </magneticfield>
  <thermalelectron>
    <regular cue="1" type="unif"><unif><n0 value="0.01"/><r0 value="3.0"/></unif></regular>
    <random cue="0" type="global" seed="0"/>
  </thermalelectron>
  <cre cue="1" type="analytic">
    <analytic>
      <alpha value="3.0"/><beta value="0.0"/><theta value="0.0"/>
      <r0 value="5.0"/><z0 value="1.0"/><E0 value="20.6"/><j0 value="0.0217"/>
    </analytic>
  </cre>
</root>
"""

OUTPUTS = ["dm.bin", "fd.bin", "sync_0.408_I.bin", "sync_0.408_Q.bin", "sync_0.408_U.bin",
           "sync_23_I.bin", "sync_23_Q.bin", "sync_23_U.bin"]


def _write_inputs(d, fields32, mask):
    bx, by, bz, ne = (np.asarray(a, dtype=np.float64).reshape(-1) for a in fields32)
    # Grid_brnd::import_grid reads interleaved (bx, by, bz) per voxel
    # (source/grid/grid_brnd.cc:60-80); Grid_tereg one value per voxel
    np.stack([bx, by, bz], axis=1).tofile(os.path.join(d, "brnd.bin"))
    ne.tofile(os.path.join(d, "tereg.bin"))
    if mask is not None:
        mask.tofile(os.path.join(d, "mask.bin"))
    path = os.path.join(d, "params.xml")
    with open(path, "w") as f:
        f.write(XML.format(d=d, mask=int(mask is not None)))
    return path


def _run(exe, d, xml, env=None):
    r = subprocess.run([exe, xml], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, **(env or {})))
    assert r.returncode == 0, r.stdout + r.stderr
    return {k: np.fromfile(os.path.join(d, k)) for k in OUTPUTS}


def test_dropin_xml_parses_like_reference(tmp_path, fields32):
    """The Python Param mirror reads the same XML into the same shells."""
    xml = _write_inputs(str(tmp_path), fields32, None)
    par = Param(xml)
    assert par.nside_shell == [4, 8, 16]
    assert par.num_passes() == 2
    assert par.obs_pass(0).sync_freq == 23e9 and par.obs_pass(0).do_fd == 1
    assert par.obs_pass(1).do_fd == 0


@pytest.mark.gpu
def test_inprocess_hampyx_matches_reference_cli(tmp_path, fields32):
    """hammurabix_b200.hampyx (in process) vs the reference CLI's exported
    files, keyed the way hampyx keys them (hampyx.py:306-338)."""
    if not os.path.exists(HAMX_REF):
        pytest.skip("reference CLI not built")
    from hammurabix_b200 import hampyx
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    ref = _run(HAMX_REF, str(ref_dir), _write_inputs(str(ref_dir), fields32, None))
    xml = _write_inputs(str(tmp_path), fields32, None)
    obj = hampyx.Hampyx(xml_path=xml)
    sim = obj()
    pairs = {("dm", "nan", "16", "nan"): "dm.bin", ("fd", "nan", "16", "nan"): "fd.bin"}
    for f, ns in (("0.408", "16"), ("23", "8")):
        for s in ("I", "Q", "U"):
            pairs[("sync", f, ns, s)] = f"sync_{f}_{s}.bin"
    for key, fn in pairs.items():
        tol = 1e-10 if key[0] in ("dm", "fd") else 1e-9
        assert rel_err(sim[key], ref[fn]) <= tol, (key, rel_err(sim[key], ref[fn]))
    # XML editing round trip (hampyx.py:364-388): switch the 23 GHz entry off
    obj.mod_par(keychain=["observable", "faraday"], attrib={"cue": "0"})
    obj.sim_map.clear()
    sim2 = obj()
    assert ("fd", "nan", "16", "nan") not in sim2


@pytest.mark.gpu
@pytest.mark.parametrize("with_mask", [False, True])
def test_dropin_matches_reference_cli(tmp_path, fields32, with_mask):
    if not (os.path.exists(HAMX_REF) and os.path.exists(HAMX_B200)):
        pytest.skip("reference CLI or drop-in binary not built")
    mask = None
    if with_mask:
        rng = np.random.Generator(np.random.PCG64(12))
        mask = (rng.random(12 * 8 * 8) > 0.25).astype(np.float64)
    ref_dir = tmp_path / "ref"
    gpu_dir = tmp_path / "gpu"
    ref_dir.mkdir()
    gpu_dir.mkdir()
    ref = _run(HAMX_REF, str(ref_dir), _write_inputs(str(ref_dir), fields32, mask))
    gpu = _run(HAMX_B200, str(gpu_dir), _write_inputs(str(gpu_dir), fields32, mask))
    for k in OUTPUTS:
        assert ref[k].shape == gpu[k].shape, k
        tol = 1e-10 if k in ("dm.bin", "fd.bin") else 1e-9
        assert rel_err(gpu[k], ref[k]) <= tol, (k, rel_err(gpu[k], ref[k]))
        assert np.abs(ref[k]).max() > 0, k
    f32 = tmp_path / "f32"
    f32.mkdir()
    g32 = _run(HAMX_B200, str(f32), _write_inputs(str(f32), fields32, mask),
               env={"HAMMURABIX_PRECISION": "fp32c"})
    for k in OUTPUTS:
        assert rel_err(g32[k], ref[k]) <= 1e-5, (k, rel_err(g32[k], ref[k]))


XML_RND = """<?xml version="1.0"?>
<root>
  <observable>
    <dm cue="1" filename="{d}/dm.bin" nside="16"/>
    <faraday cue="1" filename="{d}/fd.bin" nside="16"/>
    <sync cue="1" freq="1.4" filename="{d}/sync_1.4.bin" nside="16"/>
  </observable>
  <mask cue="0" filename="{d}/mask.bin" nside="8"/>
  <fieldio>
    <breg read="0" write="0" filename="{d}/breg.bin"/>
    <brnd read="0" write="{bcue}" filename="{d}/brnd.bin"/>
    <tereg read="0" write="0" filename="{d}/tereg.bin"/>
    <ternd read="0" write="{tcue}" filename="{d}/ternd.bin"/>
    <cre read="0" write="0" filename="{d}/cre.bin"/>
  </fieldio>
  <grid>
    <observer><x value="-8.3"/><y value="0"/><z value="0.006"/></observer>
    <box_brnd>
      <nx value="16"/><ny value="12"/><nz value="10"/>
      <x_min value="-20.0"/><x_max value="20.0"/><y_min value="-20.0"/>
      <y_max value="20.0"/><z_min value="-5.0"/><z_max value="5.0"/>
    </box_brnd>
    <box_ternd>
      <nx value="12"/><ny value="14"/><nz value="9"/>
      <x_min value="-20.0"/><x_max value="20.0"/><y_min value="-20.0"/>
      <y_max value="20.0"/><z_min value="-5.0"/><z_max value="5.0"/>
    </box_ternd>
    <shell>
      <layer type="auto">
        <auto><shell_num value="2"/><nside_sim value="8"/></auto>
      </layer>
      <oc_r_min value="0.0"/><oc_r_max value="30.0"/>
      <gc_r_min value="0.0"/><gc_r_max value="20.0"/>
      <gc_z_min value="-10.0"/><gc_z_max value="10.0"/>
      <oc_r_res value="0.05"/>
    </shell>
  </grid>
  <magneticfield>
    <regular cue="1" type="lsa">
      <lsa><b0 value="3.2"/><psi0 value="27.0"/><psi1 value="0.9"/><chi0 value="25.0"/></lsa>
    </regular>
    <random cue="{bcue}" type="global" seed="7">
      <global type="es">
        <es>
          <rms value="1.5"/><k0 value="10.0"/><k1 value="0.1"/><a0 value="1.7"/>
          <a1 value="0.0"/><rho value="3.0"/><r0 value="8.0"/><z0 value="1.0"/>
        </es>
      </global>
    </random>
  </magneticfield>
  <thermalelectron>
    <regular cue="1" type="unif"><unif><n0 value="0.01"/><r0 value="3.0"/></unif></regular>
    <random cue="{tcue}" type="global" seed="9">
      <global type="dft">
        <dft><rms value="0.005"/><k0 value="0.05"/><a0 value="-1.7"/><r0 value="8.0"/><z0 value="1.0"/></dft>
      </global>
    </random>
  </thermalelectron>
  <cre cue="1" type="analytic">
    <analytic>
      <alpha value="3.0"/><beta value="0.0"/><theta value="0.0"/>
      <r0 value="5.0"/><z0 value="1.0"/><E0 value="20.6"/><j0 value="0.0217"/>
    </analytic>
  </cre>
</root>
"""
OUTPUTS_RND = ["dm.bin", "fd.bin", "sync_1.4_I.bin", "sync_1.4_Q.bin", "sync_1.4_U.bin"]


@pytest.mark.gpu
@pytest.mark.parametrize("fields,cells", [(("brnd",), "4"), (("ternd", "brnd"), "2,4")])
def test_dropin_generators_match_reference_cli(tmp_path, fields, cells):
    """Random fields made inside the pipeline: the drop-in's device
    generators against the reference CLI's own Brnd_es / TErnd_dft, which
    run on one thread with the shim's cell-indexed Philox deviates
    (HXO_SHIM_CELL_STREAM = deviates per k-space cell for each generator in
    the Pipeline's order, TErnd_dft before Brnd_es), so both draw the same
    deviates.  Compared: the exported field grids and the maps.  TErnd_dft
    runs only together with Brnd_es: it seeds from brnd_seed
    (ternd_dft.cc:42-49), which Param reads only when the random B field is
    on, so alone its seed is undefined.  Only generated fields are
    exported: the Pipeline exports a grid with write permission even when it
    was never built (pipeline.cc:104-107) and dereferences an unallocated
    array."""
    if not (os.path.exists(HAMX_REF) and os.path.exists(HAMX_B200)):
        pytest.skip("reference CLI or drop-in binary not built")
    out = {}
    files = [f"{f}.bin" for f in fields]
    for name, exe, env in (("ref", HAMX_REF, {"OMP_NUM_THREADS": "1",
                                               "HXO_SHIM_CELL_STREAM": cells}),
                           ("gpu", HAMX_B200, {})):
        d = tmp_path / name
        d.mkdir()
        xml = d / "params.xml"
        xml.write_text(XML_RND.format(d=str(d), bcue=int("brnd" in fields),
                                      tcue=int("ternd" in fields)))
        r = subprocess.run([exe, str(xml)], capture_output=True, text=True, timeout=600,
                           env=dict(os.environ, **env))
        assert r.returncode == 0, r.stdout + r.stderr
        out[name] = {k: np.fromfile(str(d / k)) for k in OUTPUTS_RND + files}
    for g in files:
        e = rel_err(out["gpu"][g], out["ref"][g])
        assert e <= 1e-12, (g, e)
    for k in OUTPUTS_RND:
        tol = 1e-10 if k in ("dm.bin", "fd.bin") else 1e-9
        assert rel_err(out["gpu"][k], out["ref"][k]) <= tol, (k, rel_err(out["gpu"][k],
                                                                        out["ref"][k]))


# Random B generators the B200 build does not replace (Brnd_jf12,
# source/field/b/brnd_jf12.cc:137-211; Brnd_mhd, brnd_mhd.cc:15-135): the
# drop-in CLI has no GSL or FFTW behind them, so it must stop with an error
# instead of running them on stand-ins.
_BRND_ES = XML_RND[XML_RND.index('    <random cue="{bcue}"'):XML_RND.index("  </magneticfield>")]
_BRND_OTHER = {
    "jf12": """    <random cue="1" type="global" seed="7">
      <global type="jf12">
        <jf12>
          <rms value="1.0"/><k0 value="10.0"/><k1 value="0.1"/><a0 value="1.7"/>
          <a1 value="0.0"/><rho value="1.0"/>
          <b0_1 value="10.81"/><b0_2 value="6.96"/><b0_3 value="9.59"/><b0_4 value="6.96"/>
          <b0_5 value="1.96"/><b0_6 value="16.34"/><b0_7 value="37.29"/><b0_8 value="10.35"/>
          <b0_int value="7.63"/><z0_spiral value="0.61"/>
          <b0_halo value="4.68"/><r0_halo value="10.97"/><z0_halo value="2.84"/>
        </jf12>
      </global>
    </random>
""",
    "mhd": """    <random cue="1" type="local" seed="7">
      <local type="mhd">
        <mhd>
          <pa0 value="1"/><pf0 value="1"/><ps0 value="1"/><k0 value="10.0"/>
          <aa0 value="1.7"/><af0 value="1.5"/><as0 value="1.7"/><k1 value="0.1"/>
          <a1 value="0.0"/><beta value="0.1"/><ma value="0.5"/>
        </mhd>
      </local>
    </random>
""",
}


@pytest.mark.parametrize("kind", sorted(_BRND_OTHER))
def test_dropin_refuses_unreplaced_generators(tmp_path, kind):
    """The generator throws before any device work, so this runs without a
    GPU: the process exits non-zero and names the missing replacement."""
    if not os.path.exists(HAMX_B200):
        pytest.skip("drop-in binary not built")
    xml = XML_RND.replace(_BRND_ES, _BRND_OTHER[kind]).format(d=str(tmp_path), bcue=1, tcue=0)
    path = tmp_path / "params.xml"
    path.write_text(xml)
    r = subprocess.run([HAMX_B200, str(path)], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "not replaced on the B200 build" in r.stderr, r.stdout + r.stderr
    assert not (tmp_path / "dm.bin").exists()


def test_dropin_links_no_oracle_code():
    """The drop-in CLI is product code: none of the oracle's stand-ins (its
    GSL/FFTW shim, cell-stream RNG, direct-sum DFT) are linked into it."""
    if not os.path.exists(HAMX_B200):
        pytest.skip("drop-in binary not built")
    r = subprocess.run(["nm", "-C", HAMX_B200], capture_output=True, text=True, check=True)
    syms = r.stdout
    for marker in ("hxo_", "philox", "splitmix", "cells_for_next_seed"):
        assert marker not in syms, marker
    assert "fftw_execute_dft" in syms and "gsl_rng_alloc" in syms


HAMX_B200_MULTI = os.path.join(ROOT, "hammurabix_b200", "dropin", "_build", "hamx_b200_multi")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_dropin_second_pipeline_sees_new_grids(tmp_path, fields32, precision):
    """Two Pipelines in one process (hamx_b200_multi), each reading its own
    grid files of the same size: the second run's Grid_* arrays are new
    allocations of the same size, which the allocator can hand out at the
    first run's addresses, and its grids differ from the first run's.  Each
    run must match the reference CLI on its own inputs; a device slot or a
    kept FP32C pass keyed on host addresses alone would give the second run
    the first run's maps."""
    if not (os.path.exists(HAMX_REF) and os.path.exists(HAMX_B200_MULTI)):
        pytest.skip("reference CLI or multi-run drop-in not built")
    bx, by, bz, ne = fields32
    second = (-0.7 * np.asarray(by), 1.3 * np.asarray(bx), np.asarray(bz)[::-1].copy(),
              0.5 * np.asarray(ne)[::-1].copy())
    runs = [("a", fields32), ("b", second)]
    xmls, ref = [], {}
    for name, f in runs:
        rd = tmp_path / f"ref_{name}"
        gd = tmp_path / f"gpu_{name}"
        rd.mkdir()
        gd.mkdir()
        ref[name] = _run(HAMX_REF, str(rd), _write_inputs(str(rd), f, None))
        xmls.append(_write_inputs(str(gd), f, None))
    env = dict(os.environ, HAMMURABIX_PRECISION=precision)
    r = subprocess.run([HAMX_B200_MULTI] + xmls, capture_output=True, text=True, timeout=600,
                       env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    for name, _ in runs:
        got = {k: np.fromfile(str(tmp_path / f"gpu_{name}" / k)) for k in OUTPUTS}
        for k in OUTPUTS:
            if precision == "fp64":
                tol = 1e-10 if k in ("dm.bin", "fd.bin") else 1e-9
            else:
                tol = 1e-5
            assert rel_err(got[k], ref[name][k]) <= tol, (name, k, rel_err(got[k], ref[name][k]))
    # the two runs' maps really differ, so a stale slot could not pass
    assert rel_err(ref["a"]["dm.bin"], ref["b"]["dm.bin"]) > 1e-3
