"""hammurabiX XML parameters (the reference's Param, source/param/param.cc).

Parses the same XML files as the reference, with the same unit conversions
(every value is multiplied by the same CGS constant, include/hamunits.h),
into the hxg ABI structs:

    par = Param("params.xml")
    par.obs           # abi.Obs for the first frequency pass
    par.models        # abi.Models (regular/random B, n_e, CRE selection)
    par.grids         # field slot -> (abi.GridDesc, filename) for grid reads

The frequency list keeps the reference's order (par.sync_freqs etc.);
Pipeline applies the reference's back-to-front loop over it.

Two model types that the reference does not have are accepted as
extensions: <regular type="spiral"> for magnetic fields and
<regular type="expdisk"> for thermal electrons (see include/hxg.h).
"""
import math
import xml.etree.ElementTree as ET

from . import abi
from . import units as U


class ParamError(RuntimeError):
    """Raised where the reference throws std::runtime_error."""


def _find(el, path):
    e = el.find(path)
    if e is None:
        raise ParamError(f"missing XML element <{path}>")
    return e


def _f(el, key, attr="value"):
    return float(_find(el, key).get(attr))


def _u(el, key, attr="value"):
    return int(_find(el, key).get(attr))


def _b(el, key=None, attr="cue"):
    e = _find(el, key) if key else el
    v = e.get(attr)
    if v is None:
        raise ParamError(f"missing attribute {attr}")
    return v.strip().lower() in ("1", "true")


class Param:
    def __init__(self, filename):
        self.filename = filename
        tree = ET.parse(filename)
        self.root = tree.getroot()
        r = self.root
        obsv = _find(r, "grid/observer")
        # Param::Param (param.cc:12-20)
        self.observer = (U.kpc * _f(obsv, "x"), U.kpc * _f(obsv, "y"), U.kpc * _f(obsv, "z"))
        self.models = abi.Models()
        self.grids = {}
        self._obs_param()
        self._breg_param()
        self._brnd_param()
        self._tereg_param()
        self._ternd_param()
        self._cre_param()

    # ---- Param::obs_param (param.cc:30-144) -------------------------------
    def _obs_param(self):
        r = self.root
        ob = _find(r, "observable")
        self.write_permission = False
        dm = ob.find("dm")
        self.do_dm = False
        self.nside_dm = 0
        self.sim_dm_name = None
        if dm is not None:
            self.write_permission = True
            self.do_dm = _b(dm)
            self.sim_dm_name = dm.get("filename")
            self.nside_dm = int(dm.get("nside"))
        fd = ob.find("faraday")
        self.do_fd = False
        self.nside_fd = 0
        self.sim_fd_name = None
        if fd is not None:
            self.write_permission = True
            self.do_fd = _b(fd)
            self.sim_fd_name = fd.get("filename")
            self.nside_fd = int(fd.get("nside"))
        self.do_sync, self.sync_freqs, self.sim_sync_names, self.nside_sync = [], [], [], []
        syncs = ob.findall("sync")
        if syncs:
            self.write_permission = True
            for s in syncs:
                self.do_sync.append(_b(s))
                self.sync_freqs.append(float(s.get("freq")) * U.GHz)
                self.sim_sync_names.append(s.get("filename"))
                self.nside_sync.append(int(s.get("nside")))
        else:
            self.do_sync.append(False)
        self.nside_shell, self.radii_shell = [], []
        self.total_shell = 0
        self.do_mask = False
        if not self.write_permission:
            return
        sh = _find(r, "grid/shell")
        self.oc_r_min = _f(sh, "oc_r_min") * U.kpc
        self.oc_r_max = _f(sh, "oc_r_max") * U.kpc
        self.gc_r_min = _f(sh, "gc_r_min") * U.kpc
        self.gc_r_max = _f(sh, "gc_r_max") * U.kpc
        self.gc_z_min = _f(sh, "gc_z_min") * U.kpc
        self.gc_z_max = _f(sh, "gc_z_max") * U.kpc
        self.oc_r_res = _f(sh, "oc_r_res") * U.kpc
        layer = _find(sh, "layer").get("type")
        if layer == "auto":
            a = _find(sh, "layer/auto")
            self.total_shell = _u(a, "shell_num")
            nside_sim = _u(a, "nside_sim")
            self.nside_shell = [int(math.pow(2, i) * nside_sim) for i in range(self.total_shell)]
            self.radii_shell = [self.oc_r_min]
            for i in range(self.total_shell):
                self.radii_shell.append((self.oc_r_max - self.oc_r_min)
                                        * math.pow(0.5, self.total_shell - i - 1)
                                        + self.oc_r_min)
        elif layer == "manual":
            mnl = _find(sh, "layer/manual")
            self.nside_shell = [int(e.get("value")) for e in mnl.findall("nside_sim")]
            self.total_shell = len(self.nside_shell)
            cuts = [float(e.get("value")) for e in mnl.findall("cut")] + [1.]
            if len(cuts) != self.total_shell:
                raise ParamError("manual shell cuts and nside_sim counts differ")
            self.radii_shell = [self.oc_r_min]
            for c in cuts:
                self.radii_shell.append((self.oc_r_max - self.oc_r_min) * c + self.oc_r_min)
        else:
            raise ParamError("unsupported layer option")
        if self.total_shell > abi.HXG_MAX_SHELLS:
            raise ParamError(f"more than {abi.HXG_MAX_SHELLS} shells")
        mk = _find(r, "mask")
        if _b(mk):
            self.do_mask = True
            self.mask_name = mk.get("filename")
            self.nside_mask = int(mk.get("nside"))

    def obs_pass(self, k):
        """abi.Obs for the k-th pass of Pipeline::assemble_obs
        (pipeline.cc:165-190): sync entry len-1-k, DM/FD only on pass 0."""
        o = abi.Obs()
        for i in range(3):
            o.observer[i] = self.observer[i]
        o.gc_r_min, o.gc_r_max = self.gc_r_min, self.gc_r_max
        o.gc_z_min, o.gc_z_max = self.gc_z_min, self.gc_z_max
        o.oc_r_res = self.oc_r_res
        o.total_shell = self.total_shell
        for i, n in enumerate(self.nside_shell):
            o.nside_shell[i] = n
        for i, rr in enumerate(self.radii_shell):
            o.radii_shell[i] = rr
        o.do_dm = int(self.do_dm and k == 0)
        o.do_fd = int(self.do_fd and k == 0)
        o.nside_dm = self.nside_dm if o.do_dm else 0
        o.nside_fd = self.nside_fd if o.do_fd else 0
        idx = len(self.do_sync) - 1 - k
        if self.do_sync[idx] and self.sync_freqs:
            o.do_sync = 1
            o.sync_freq = self.sync_freqs[idx]
            o.nside_sync = self.nside_sync[idx]
        o.do_mask = int(self.do_mask)
        return o

    def num_passes(self):
        return len(self.do_sync) if self.write_permission else 0

    @property
    def obs(self):
        return self.obs_pass(0)

    # ---- field boxes --------------------------------------------------
    def _box(self, name):
        b = _find(self.root, f"grid/{name}")
        d = abi.GridDesc()
        d.nx, d.ny, d.nz = _u(b, "nx"), _u(b, "ny"), _u(b, "nz")
        d.x_max = U.kpc * _f(b, "x_max")
        d.x_min = U.kpc * _f(b, "x_min")
        d.y_max = U.kpc * _f(b, "y_max")
        d.y_min = U.kpc * _f(b, "y_min")
        d.z_max = U.kpc * _f(b, "z_max")
        d.z_min = U.kpc * _f(b, "z_min")
        return d

    def _fieldio(self, key):
        fio = self.root.find("fieldio")
        e = fio.find(key) if fio is not None else None
        if e is None:
            return False, False, None
        return _b(e, attr="read"), _b(e, attr="write"), e.get("filename")

    # ---- Param::breg_param (param.cc:146-340) -------------------------
    def _breg_param(self):
        m = self.models
        read, write, fname = self._fieldio("breg")
        mf = _find(self.root, "magneticfield")
        build = _b(mf, "regular")
        self.breg_type = None
        if build and not read:
            reg = _find(mf, "regular")
            t = reg.get("type")
            self.breg_type = t
            if t == "lsa":
                s = _find(reg, "lsa")
                m.breg = abi.HXG_BREG_LSA
                m.lsa.b0 = _f(s, "b0") * U.muGauss
                m.lsa.psi0 = _f(s, "psi0") * U.rad
                m.lsa.psi1 = _f(s, "psi1") * U.rad
                m.lsa.chi0 = _f(s, "chi0") * U.rad
            elif t == "unif":
                s = _find(reg, "unif")
                m.breg = abi.HXG_BREG_UNIF
                m.unif.bp = _f(s, "bp") * U.muGauss
                m.unif.bv = _f(s, "bv") * U.muGauss
                m.unif.l0 = _f(s, "l0") * U.rad
            elif t == "cart":
                s = _find(reg, "cart")
                m.breg = abi.HXG_BREG_CART
                m.cart.bx = _f(s, "bx") * U.muGauss
                m.cart.by = _f(s, "by") * U.muGauss
                m.cart.bz = _f(s, "bz") * U.muGauss
            elif t == "helix":
                s = _find(reg, "helix")
                m.breg = abi.HXG_BREG_HELIX
                m.helix.bx = _f(s, "bx") * U.muGauss
                m.helix.by = _f(s, "by") * U.muGauss
                m.helix.bz = _f(s, "bz") * U.muGauss
                m.helix.r_min = _f(s, "r_min") * U.kpc
                m.helix.r_max = _f(s, "r_max") * U.kpc
            elif t == "jaffe":
                self._jaffe(_find(reg, "jaffe"))
            elif t == "jf12":
                self._jf12(_find(reg, "jf12"))
            elif t == "spiral":
                s = _find(reg, "spiral")
                m.breg = abi.HXG_BREG_SPIRAL
                m.spiral.b0 = _f(s, "b0") * U.muGauss
                m.spiral.pitch = _f(s, "pitch") * U.rad
                m.spiral.r_scale = _f(s, "r0") * U.kpc
                m.spiral.h_scale = _f(s, "z0") * U.kpc
            else:
                raise ParamError("unsupported breg model")
        elif build and read:
            m.breg = abi.HXG_BREG_GRID
        else:
            m.breg = abi.HXG_BREG_NONE
        if read or write:
            self.grids[abi.HXG_FIELD_BREG] = (self._box("box_breg"), fname)

    def _jaffe(self, s):
        m = self.models
        j = m.jaffe
        m.breg = abi.HXG_BREG_JAFFE
        j.quadruple = int(_b(s, "quadruple"))
        j.bss = int(_b(s, "bss"))
        j.disk_amp = _f(s, "disk_amp") * U.muGauss
        j.disk_z0 = _f(s, "disk_z0") * U.kpc
        j.halo_amp = _f(s, "halo_amp") * U.muGauss
        j.halo_z0 = _f(s, "halo_z0") * U.kpc
        j.r_inner = _f(s, "r_inner") * U.kpc
        j.r_scale = _f(s, "r_scale") * U.kpc
        j.r_peak = _f(s, "r_peak") * U.kpc
        j.ring = int(_b(s, "ring"))
        j.ring_amp = _f(s, "ring_amp") * U.muGauss
        j.ring_r = _f(s, "ring_r") * U.kpc
        j.bar = int(_b(s, "bar"))
        j.bar_amp = _f(s, "bar_amp") * U.muGauss
        j.bar_a = _f(s, "bar_a") * U.kpc
        j.bar_b = _f(s, "bar_b") * U.kpc
        j.bar_phi0 = _f(s, "bar_phi0") * U.rad
        j.arm_num = _u(s, "arm_num")
        # Param reads four arms (param.cc:207-227); more would be read past
        # its vectors
        if j.arm_num > 4:
            raise ParamError(f"Breg_jaffe arm_num {j.arm_num} exceeds the 4 arms given")
        j.arm_r0 = _f(s, "arm_r0") * U.kpc
        j.arm_z0 = _f(s, "arm_z0") * U.kpc
        for i in range(4):
            j.arm_phi0[i] = _f(s, f"arm_phi{i + 1}") * U.rad
            j.arm_amp[i] = _f(s, f"arm_amp{i + 1}") * U.muGauss
        j.arm_pitch = _f(s, "arm_pitch") * U.rad
        j.comp_c = _f(s, "comp_c")
        j.comp_d = _f(s, "comp_d") * U.kpc
        j.comp_r = _f(s, "comp_r") * U.kpc
        j.comp_p = _f(s, "comp_p")

    def _jf12(self, s):
        m = self.models
        j = m.jf12
        m.breg = abi.HXG_BREG_JF12
        for k in ("b_arm1", "b_arm2", "b_arm3", "b_arm4", "b_arm5", "b_arm6", "b_arm7",
                  "b_ring", "Bn", "Bs", "B0_X"):
            setattr(j, k, _f(s, k) * U.muGauss)
        for k in ("h_disk", "w_disk", "rn", "rs", "wh", "z0", "rpc_X", "r0_X"):
            setattr(j, k, _f(s, k) * U.kpc)
        j.Xtheta = _f(s, "Xtheta") * U.rad

    # ---- Param::brnd_param (param.cc:342-464) -------------------------
    def _brnd_param(self):
        read, write, fname = self._fieldio("brnd")
        mf = _find(self.root, "magneticfield")
        build = _b(mf, "random")
        if read:
            self.models.brnd = abi.HXG_BRND_GRID
        elif build:
            raise ParamError("random-field generators are outside the integrator; "
                             "write the grid to a file and read it (<fieldio><brnd read=\"1\">)")
        else:
            self.models.brnd = abi.HXG_BRND_NONE
        if read or write or build:
            self.grids[abi.HXG_FIELD_BRND] = (self._box("box_brnd"), fname)

    # ---- Param::tereg_param (param.cc:466-668) ------------------------
    def _tereg_param(self):
        m = self.models
        read, write, fname = self._fieldio("tereg")
        te = _find(self.root, "thermalelectron")
        build = _b(te, "regular")
        if build:
            reg = _find(te, "regular")
            t = reg.get("type")
            self.tereg_type = t
            if t == "ymw16":
                self._ymw16(_find(reg, "ymw16"))
            elif t == "unif":
                s = _find(reg, "unif")
                m.te_unif.n0 = _f(s, "n0")
                m.te_unif.r0 = _f(s, "r0") * U.kpc
                m.tereg = abi.HXG_TEREG_UNIF
            elif t == "expdisk":
                s = _find(reg, "expdisk")
                m.te_exp.n0 = _f(s, "n0")
                m.te_exp.r_scale = _f(s, "r0") * U.kpc
                m.te_exp.h_scale = _f(s, "z0") * U.kpc
                m.tereg = abi.HXG_TEREG_EXPDISK
            else:
                raise ParamError("unsupported tereg model")
            # Pipeline::assemble_tereg (pipeline.cc:33-54): a read grid
            # replaces the model
            if read:
                m.tereg = abi.HXG_TEREG_GRID
        else:
            m.tereg = abi.HXG_TEREG_NONE
        if read or write:
            self.grids[abi.HXG_FIELD_TEREG] = (self._box("box_tereg"), fname)

    def _ymw16(self, s):
        y = self.models.ymw16
        self.models.tereg = abi.HXG_TEREG_YMW16
        w = _find(s, "warp")
        y.r_warp = _f(w, "r_warp") * U.kpc
        y.r0 = _f(w, "r0") * U.kpc
        y.t0_gamma_w = _f(w, "gamma_w")
        t = _find(s, "thickdisk")
        y.t1_ad = _f(t, "ad") * U.pc
        y.t1_bd = _f(t, "bd") * U.pc
        y.t1_n1 = _f(t, "n1")
        y.t1_h1 = _f(t, "h1") * U.pc
        t = _find(s, "thindisk")
        y.t2_a2 = _f(t, "a2") * U.pc
        y.t2_b2 = _f(t, "b2") * U.pc
        y.t2_n2 = _f(t, "n2")
        y.t2_k2 = _f(t, "k2")
        t = _find(s, "spiralarm")
        y.t3_b2s = _f(t, "b2s") * U.pc
        for i in range(5):
            y.t3_narm[i] = _f(t, f"ele_arm_{i}")
            y.t3_warm[i] = _f(t, f"wid_arm_{i}") * U.pc
            y.t3_rmin[i] = _f(t, f"rref_arm_{i}") * U.kpc
            y.t3_phimin[i] = _f(t, f"phiref_arm_{i}") * U.rad
            y.t3_tpitch[i] = math.tan(_f(t, f"pitch_arm_{i}") * U.rad)
            y.t3_cpitch[i] = math.cos(_f(t, f"pitch_arm_{i}") * U.rad)
        y.t3_aa = _f(t, "aa") * U.pc
        y.t3_ka = _f(t, "ka")
        y.t3_ncn = _f(t, "ncn")
        y.t3_thetacn = _f(t, "thetacn")
        y.t3_wcn = _f(t, "wcn")
        y.t3_nsg = _f(t, "nsg")
        y.t3_thetasg = _f(t, "thetasg")
        y.t3_wsg = _f(t, "wsg")
        t = _find(s, "galcenter")
        y.t4_ngc = _f(t, "ngc")
        y.t4_agc = _f(t, "agc") * U.pc
        y.t4_hgc = _f(t, "hgc") * U.pc
        t = _find(s, "gumnebula")
        y.t5_ngn = _f(t, "ngn")
        y.t5_wgn = _f(t, "wgn") * U.pc
        y.t5_agn = _f(t, "agn") * U.pc
        y.t5_kgn = _f(t, "kgn")
        t = _find(s, "localbubble")
        y.t6_j_lb = _f(t, "j_lb")
        y.t6_nlb1 = _f(t, "nlb1")
        y.t6_thetalb1 = _f(t, "thetalb1")
        y.t6_detlb1 = _f(t, "detlb1")
        y.t6_wlb1 = _f(t, "wlb1") * U.pc
        y.t6_hlb1 = _f(t, "hlb1") * U.pc
        y.t6_nlb2 = _f(t, "nlb2")
        y.t6_thetalb2 = _f(t, "thetalb2")
        y.t6_detlb2 = _f(t, "detlb2")
        y.t6_wlb2 = _f(t, "wlb2") * U.pc
        y.t6_hlb2 = _f(t, "hlb2") * U.pc
        t = _find(s, "loopi")
        y.t7_nli = _f(t, "nli")
        y.t7_rli = _f(t, "rli") * U.pc
        y.t7_wli = _f(t, "wli") * U.pc
        y.t7_detthetali = _f(t, "detthetali")
        y.t7_thetali = _f(t, "thetali")

    # ---- Param::ternd_param (param.cc:670-718) ------------------------
    def _ternd_param(self):
        read, write, fname = self._fieldio("ternd")
        te = _find(self.root, "thermalelectron")
        build = _b(te, "random")
        if read:
            self.models.ternd = abi.HXG_TERND_GRID
        elif build:
            raise ParamError("random-field generators are outside the integrator; "
                             "write the grid to a file and read it (<fieldio><ternd read=\"1\">)")
        else:
            self.models.ternd = abi.HXG_TERND_NONE
        if read or write or build:
            self.grids[abi.HXG_FIELD_TERND] = (self._box("box_ternd"), fname)

    # ---- Param::cre_param (param.cc:720-778) ---------------------------
    def _cre_param(self):
        m = self.models
        read, write, fname = self._fieldio("cre")
        c = _find(self.root, "cre")
        build = _b(c)
        if build:
            t = c.get("type")
            if t == "analytic":
                s = _find(c, "analytic")
                m.cre = abi.HXG_CRE_ANA
                a = m.cre_ana
                a.alpha = _f(s, "alpha")
                a.beta = _f(s, "beta")
                a.theta = _f(s, "theta")
                a.r0 = _f(s, "r0") * U.kpc
                a.z0 = _f(s, "z0") * U.kpc
                a.E0 = _f(s, "E0") * U.GeV
                a.j0 = _f(s, "j0")
            elif t == "unif":
                s = _find(c, "unif")
                m.cre = abi.HXG_CRE_UNIF
                u = m.cre_unif
                u.alpha = _f(s, "alpha")
                u.r0 = _f(s, "r0") * U.kpc
                u.E0 = _f(s, "E0") * U.GeV
                u.j0 = _f(s, "j0")
            else:
                raise ParamError("unsupported cre model")
        if read:
            m.cre = abi.HXG_CRE_GRID
        if read or write:
            b = _find(self.root, "grid/box_cre")
            d = abi.GridDesc()
            d.E_min = U.GeV * _f(b, "E_min")
            d.E_max = U.GeV * _f(b, "E_max")
            d.nE = _u(b, "nE")
            d.E_fact = math.log(d.E_max / d.E_min) / (d.nE - 1)
            d.nz, d.nx, d.ny = _u(b, "nz"), _u(b, "nx"), _u(b, "ny")
            d.x_max = U.kpc * _f(b, "x_max")
            d.x_min = U.kpc * _f(b, "x_min")
            d.y_max = U.kpc * _f(b, "y_max")
            d.y_min = U.kpc * _f(b, "y_min")
            d.z_max = U.kpc * _f(b, "z_max")
            d.z_min = U.kpc * _f(b, "z_min")
            self.grids[abi.HXG_FIELD_CRE] = (d, fname)
