"""In-process mirror of the reference's Pipeline for the LOS path
(source/pipeline/pipeline.cc) on the B200 integrator.

    pipe = Pipeline("params.xml", precision="fp64")
    maps = pipe.run()            # {(kind, freq, nside, stokes): numpy map}
    pipe.export()                # the files Grid_obs::export_grid writes

Grid files are read in the reference's format (Grid_*::import_grid:
interleaved FP64 per voxel for B, one FP64 per voxel for n_e;
source/grid/grid_breg.cc:60-80, grid_tereg.cc).  The frequency loop follows
Pipeline::assemble_obs (pipeline.cc:165-190): the last <sync> entry first,
DM and FD only on the first pass.  Map units are those of
Grid_obs::export_grid (source/grid/grid_obs.cc:53-82): DM in pc/cm^3, FD in
rad/m^2, I/Q/U in K.
"""
import os

import numpy as np

from . import abi
from . import units as U
from .integrator import Integrator
from .param import Param, ParamError


def _sync_freq_string(par, idx):
    """The frequency string of a <sync> entry as written in the XML (the key
    hampyx uses, hampyx.py:284-290)."""
    syncs = par.root.findall("observable/sync")
    return str(syncs[idx].get("freq"))


class Pipeline:
    def __init__(self, xml_path, precision="fp64", device=0, integrator=None):
        self.par = Param(xml_path)
        self.xml_path = xml_path
        self.integ = integrator or Integrator(precision, device=device)
        self.maps = {}
        self._grids_loaded = False

    # Pipeline::assemble_grid + assemble_* (pipeline.cc:23-162): the grid
    # imports and the model selection (already resolved by Param).
    def assemble_fields(self):
        par = self.par
        m = par.models
        self.integ.set_models(m)
        readers = {
            abi.HXG_FIELD_BREG: m.breg == abi.HXG_BREG_GRID,
            abi.HXG_FIELD_BRND: m.brnd == abi.HXG_BRND_GRID,
            abi.HXG_FIELD_TEREG: m.tereg == abi.HXG_TEREG_GRID,
            abi.HXG_FIELD_TERND: m.ternd == abi.HXG_TERND_GRID,
        }
        for slot, active in readers.items():
            if not active:
                continue
            desc, fname = par.grids[slot]
            self.integ.upload_grid_file(slot, desc, fname)
        if par.do_mask:
            mask = np.fromfile(par.mask_name, dtype="<f8")
            if mask.size != abi.npix(par.nside_mask):
                raise ParamError("mask file size does not match its nside")
            self.integ.set_mask(par.nside_mask, mask)
        else:
            self.integ.set_mask(0, None)
        self._grids_loaded = True

    # Pipeline::assemble_obs (pipeline.cc:165-190)
    def assemble_obs(self):
        par = self.par
        if not self._grids_loaded:
            self.assemble_fields()
        self.maps = {}
        self.raw = []
        # all passes in one call: the FP32C form runs passes of the same
        # geometry in one traversal per shell (hxg_write_grid_multi)
        obs = [par.obs_pass(k) for k in range(par.num_passes())]
        outs = self.integ.write_grid_multi(obs)
        for k, (o, out) in enumerate(zip(obs, outs)):
            self.raw.append((o, out))
            idx = len(par.do_sync) - 1 - k
            if o.do_dm:
                self.maps[("dm", "nan", str(o.nside_dm), "nan")] = out["dm"] * (U.ccm / U.pc)
            if o.do_fd:
                self.maps[("fd", "nan", str(o.nside_fd), "nan")] = out["fd"] * (U.m * U.m)
            if o.do_sync:
                f = _sync_freq_string(par, idx)
                for s, key in (("I", "is"), ("Q", "qs"), ("U", "us")):
                    self.maps[("sync", f, str(o.nside_sync), s)] = out[key]
        return self.maps

    def run(self):
        self.assemble_fields()
        return self.assemble_obs()

    # Grid_obs::export_grid (grid_obs.cc:53-82): raw FP64 dumps with
    # _I/_Q/_U inserted before the extension of the sync file names.
    def export(self):
        par = self.par
        for k, (o, out) in enumerate(self.raw):
            idx = len(par.do_sync) - 1 - k
            if o.do_dm:
                (out["dm"] * (U.ccm / U.pc)).astype("<f8").tofile(par.sim_dm_name)
            if o.do_sync:
                name = par.sim_sync_names[idx]
                for s, key in (("_I", "is"), ("_Q", "qs"), ("_U", "us")):
                    fn = name[:-4] + s + name[-4:]
                    out[key].astype("<f8").tofile(fn)
            if o.do_fd:
                (out["fd"] * (U.m * U.m)).astype("<f8").tofile(par.sim_fd_name)
