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
