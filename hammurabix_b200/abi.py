"""ctypes mirrors of the C ABI structs in include/hxg.h.

The field order and types match include/hxg.h exactly; tests check the
sizes against the compiled library.
"""
import ctypes as C

HXG_ABI_VERSION = 1
HXG_MAX_SHELLS = 16

# status codes
HXG_OK = 0
HXG_ERR_INVALID = 1
HXG_ERR_UNSUPPORTED = 2
HXG_ERR_CUDA = 3
HXG_ERR_OOM = 4
HXG_ERR_TIMEOUT = 5
HXG_ERR_STATE = 6
HXG_ERR_NO_DEVICE = 7
HXG_ERR_TOO_LARGE = 8
HXG_NOALLOC_MAX_NSIDE = 128

STATUS_NAMES = {
    0: "HXG_OK", 1: "HXG_ERR_INVALID", 2: "HXG_ERR_UNSUPPORTED",
    3: "HXG_ERR_CUDA", 4: "HXG_ERR_OOM", 5: "HXG_ERR_TIMEOUT",
    6: "HXG_ERR_STATE", 7: "HXG_ERR_NO_DEVICE", 8: "HXG_ERR_TOO_LARGE",
}

# precision forms
HXG_FP64 = 0
HXG_FP32C = 1

# field slots
HXG_FIELD_BREG, HXG_FIELD_BRND, HXG_FIELD_TEREG, HXG_FIELD_TERND, HXG_FIELD_CRE = range(5)

# model enums
HXG_BREG_NONE, HXG_BREG_GRID, HXG_BREG_LSA, HXG_BREG_UNIF, HXG_BREG_CART, \
    HXG_BREG_HELIX, HXG_BREG_JAFFE, HXG_BREG_JF12, HXG_BREG_SPIRAL = range(9)
HXG_BRND_NONE, HXG_BRND_GRID = range(2)
HXG_TEREG_NONE, HXG_TEREG_GRID, HXG_TEREG_UNIF, HXG_TEREG_YMW16, HXG_TEREG_EXPDISK = range(5)
HXG_TERND_NONE, HXG_TERND_GRID = range(2)
HXG_CRE_NONE, HXG_CRE_ANA, HXG_CRE_UNIF, HXG_CRE_GRID = range(4)

_d = C.c_double
_i32 = C.c_int32
_u32 = C.c_uint32


def _fields(names, typ=_d):
    return [(n, typ) for n in names]


class BregLsa(C.Structure):
    _fields_ = _fields(["b0", "psi0", "psi1", "chi0"])


class BregUnif(C.Structure):
    _fields_ = _fields(["bp", "bv", "l0"])


class BregCart(C.Structure):
    _fields_ = _fields(["bx", "by", "bz"])


class BregHelix(C.Structure):
    _fields_ = _fields(["bx", "by", "bz", "r_min", "r_max"])


class BregJaffe(C.Structure):
    _fields_ = (_fields(["quadruple", "bss", "ring", "bar"], _i32)
                + _fields(["arm_num", "_pad"], _u32)
                + _fields(["disk_amp", "disk_z0", "halo_amp", "halo_z0",
                           "r_inner", "r_scale", "r_peak",
                           "ring_amp", "bar_amp", "ring_r", "bar_a", "bar_b", "bar_phi0"])
                + [("arm_amp", _d * 8), ("arm_phi0", _d * 8)]
                + _fields(["arm_pitch", "arm_r0", "arm_z0",
                           "comp_r", "comp_c", "comp_d", "comp_p"]))


class BregJf12(C.Structure):
    _fields_ = _fields(["b_arm1", "b_arm2", "b_arm3", "b_arm4", "b_arm5", "b_arm6",
                        "b_arm7", "b_ring", "h_disk", "w_disk", "Bn", "Bs", "rn", "rs",
                        "wh", "z0", "B0_X", "Xtheta", "rpc_X", "r0_X"])


class BregSpiral(C.Structure):
    _fields_ = _fields(["b0", "pitch", "r_scale", "h_scale"])


class TeregUnif(C.Structure):
    _fields_ = _fields(["n0", "r0"])


class TeregExpdisk(C.Structure):
    _fields_ = _fields(["n0", "r_scale", "h_scale"])


class TeregYmw16(C.Structure):
    _fields_ = (_fields(["r_warp", "r0", "t0_gamma_w", "t1_ad", "t1_bd", "t1_n1", "t1_h1",
                         "t2_a2", "t2_b2", "t2_n2", "t2_k2", "t3_b2s", "t3_ka"])
                + [("t3_narm", _d * 5), ("t3_warm", _d * 5)]
                + _fields(["t3_aa", "t3_ncn", "t3_wcn", "t3_thetacn", "t3_nsg", "t3_wsg",
                           "t3_thetasg"])
                + [("t3_rmin", _d * 5), ("t3_phimin", _d * 5), ("t3_tpitch", _d * 5),
                   ("t3_cpitch", _d * 5)]
                + _fields(["t4_ngc", "t4_agc", "t4_hgc", "t5_kgn", "t5_ngn", "t5_wgn",
                           "t5_agn", "t6_j_lb", "t6_nlb1", "t6_detlb1", "t6_wlb1",
                           "t6_hlb1", "t6_thetalb1", "t6_nlb2", "t6_detlb2", "t6_wlb2",
                           "t6_hlb2", "t6_thetalb2", "t7_nli", "t7_rli", "t7_wli",
                           "t7_detthetali", "t7_thetali"]))


class BrndEs(C.Structure):
    """hxg_brnd_es_t (Param::brnd_es)."""
    _fields_ = _fields(["rms", "k0", "k1", "a0", "a1", "rho", "r0", "z0"])


class TerndDft(C.Structure):
    """hxg_ternd_dft_t (Param::ternd_dft)."""
    _fields_ = _fields(["rms", "k0", "a0", "r0", "z0"])


class CreAna(C.Structure):
    _fields_ = _fields(["alpha", "beta", "theta", "r0", "z0", "E0", "j0"])


class CreUnif(C.Structure):
    _fields_ = _fields(["alpha", "r0", "E0", "j0"])


class Models(C.Structure):
    _fields_ = (_fields(["breg", "brnd", "tereg", "ternd", "cre", "_pad"], _i32)
                + [("lsa", BregLsa), ("unif", BregUnif), ("cart", BregCart),
                   ("helix", BregHelix), ("jaffe", BregJaffe), ("jf12", BregJf12),
                   ("spiral", BregSpiral), ("te_unif", TeregUnif), ("ymw16", TeregYmw16),
                   ("te_exp", TeregExpdisk), ("cre_ana", CreAna), ("cre_unif", CreUnif)])


class GridDesc(C.Structure):
    _fields_ = (_fields(["nx", "ny", "nz", "nE"], _u32)
                + _fields(["x_min", "x_max", "y_min", "y_max", "z_min", "z_max",
                           "E_min", "E_max", "E_fact"]))


class Obs(C.Structure):
    _fields_ = [("observer", _d * 3),
                ("gc_r_min", _d), ("gc_r_max", _d), ("gc_z_min", _d), ("gc_z_max", _d),
                ("oc_r_res", _d),
                ("total_shell", _u32),
                ("nside_shell", _u32 * HXG_MAX_SHELLS),
                ("radii_shell", _d * (HXG_MAX_SHELLS + 1)),
                ("do_dm", _i32), ("do_fd", _i32), ("do_sync", _i32), ("do_mask", _i32),
                ("nside_dm", _u32), ("nside_fd", _u32), ("nside_sync", _u32), ("_pad", _u32),
                ("sync_freq", _d)]


class BatchEntry(C.Structure):
    """hxg_batch_entry_t: one pass of a batch (models, obs, device outputs)."""
    _fields_ = [("models", Models), ("obs", Obs),
                ("d_dm", C.c_void_p), ("d_fd", C.c_void_p), ("d_is", C.c_void_p),
                ("d_qs", C.c_void_p), ("d_us", C.c_void_p)]


def npix(nside):
    return 12 * int(nside) * int(nside)


def obs_output_sizes(obs):
    """Number of pixels of each output map (dm, fd, is/qs/us) of an Obs."""
    return (npix(obs.nside_dm) if obs.do_dm else 0,
            npix(obs.nside_fd) if obs.do_fd else 0,
            npix(obs.nside_sync) if obs.do_sync else 0)

# adjoint parameter slots (include/hxg.h HXG_PARAM_*)
HXG_PARAM_SPIRAL_B0, HXG_PARAM_SPIRAL_PITCH, HXG_PARAM_SPIRAL_R, HXG_PARAM_SPIRAL_H, \
    HXG_PARAM_EXPDISK_N0, HXG_PARAM_EXPDISK_R, HXG_PARAM_EXPDISK_H, HXG_PARAM_CRE_J0 = range(8)
HXG_NUM_PARAMS = 8
