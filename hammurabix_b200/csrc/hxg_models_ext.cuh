// hxg_models_ext.cuh -- the reference's large analytic models on the
// device, in FP64 and in the reference's operation order:
//   Breg_jaffe  (source/field/b/breg_jaffe.cc:11-243, include/bfield.h:202-224)
//   Breg_jf12   (source/field/b/breg_jf12.cc:8-189)
//   TEreg_ymw16 (source/field/te/tereg_ymw16.cc:10-333)
// Constants the reference computes from parameters alone (cos/sin of the
// pitch, the flux-conserving eighth JF12 arm, the Gum-nebula centre, ...)
// are computed once on the host with the same expressions.  Lengths and
// fields arrive in the working units of the form (DevModels::kpc, ::pc).
// Both forms evaluate these models in FP64; the FP32-compensated form calls
// them through its FP64 model path.
#pragma once

#include "../../include/hxg.h"
#include "hxg_common.cuh"

namespace hxg {

// pow(1 / cosh(x), 2) as TEreg_ymw16 writes it
__device__ __forceinline__ double sech2(double x) {
  const double c = 1. / cosh(x);
  return c * c;
}

// 1 / (cosh(x) * cosh(x)) as Breg_jaffe writes it (bfield.h:202-224)
__device__ __forceinline__ double inv_cosh2(double x) {
  const double c = cosh(x);
  return 1. / (c * c);
}

// ---- Breg_jaffe -------------------------------------------------------
struct JaffeDev {
  hxg_breg_jaffe_t p;  // the Param block (working units)
  double cos_p, sin_p, beta_inv;   // arm pitch: cos, sin, -tan^-1
  double cos_b, sin_b;             // bar_phi0
  double bar_lim, c0;              // bar_a + comp_d/2, 1/comp_c - 1
  double r_forbid;                 // 0.5 kpc
};

// radial_scaling (breg_jaffe.cc:87-101)
__device__ __forceinline__ double jaffe_radial(const JaffeDev &J, double x, double y) {
  const double r2 = x * x + y * y;
  const double s1 = 1. - exp(-r2 / (J.p.r_inner * J.p.r_inner));
  const double s2 = exp(-r2 / (J.p.r_scale * J.p.r_scale));
  const double s3 = exp(-r2 * r2 / (J.p.r_peak * J.p.r_peak * J.p.r_peak * J.p.r_peak));
  return s1 * (s2 + s3);
}

// dist2arm (breg_jaffe.cc:175-243): distances to the ring/bar (one entry)
// or to each spiral arm (arm_num entries); no entry without ring and bar.
__device__ __forceinline__ int jaffe_dist2arm(const JaffeDev &J, double x, double y,
                                              double d[8]) {
  const double r = sqrt(x * x + y * y);
  double theta = atan2(y, x);
  if (theta < 0) theta += 2 * cgs::pi;
  const int na = (int)min(J.p.arm_num, 8u);
  const auto arms = [&]() {
    for (int i = 0; i < na; ++i) {
      const double d_ang = J.p.arm_phi0[i] - theta;
      const double d_rad = fabs(J.p.arm_r0 * exp(d_ang * J.beta_inv) - r);
      const double d_rad_p = fabs(J.p.arm_r0 * exp((d_ang + 2 * cgs::pi) * J.beta_inv) - r);
      const double d_rad_m = fabs(J.p.arm_r0 * exp((d_ang - 2 * cgs::pi) * J.beta_inv) - r);
      d[i] = fmin(fmin(d_rad, d_rad_p), d_rad_m) * J.cos_p;
    }
    return na;
  };
  if (J.p.ring) {
    if (r < J.p.ring_r) {
      d[0] = fabs(J.p.ring_r - r);
      return 1;
    }
    return arms();
  }
  if (J.p.bar) {
    const double cos_tmp = J.cos_b * x / r - J.sin_b * y / r;
    const double sin_tmp = J.cos_b * y / r + J.sin_b * x / r;
    if (r < J.bar_lim) {
      d[0] = fabs(J.p.bar_a * J.p.bar_b /
                      sqrt(J.p.bar_a * J.p.bar_a * sin_tmp * sin_tmp +
                           J.p.bar_b * J.p.bar_b * cos_tmp * cos_tmp) -
                  r);
      return 1;
    }
    return arms();
  }
  return 0;
}

static __device__ __noinline__ void breg_jaffe(const JaffeDev &J, double x, double y, double z,
                                        double b[3]) {
  b[0] = b[1] = b[2] = 0.;
  const double r = sqrt(x * x + y * y);
  // orientation (breg_jaffe.cc:38-85): zero in the forbidden centre
  if (r < J.r_forbid) return;
  double t0 = 0., t1 = 0., t2 = 0.;
  double quadruple = 1;
  if (z > J.p.disk_z0) quadruple = (1 - 2 * J.p.quadruple);
  const double sgn_bss = (1 - 2 * J.p.bss);
  if (J.p.ring) {
    if (r > J.p.ring_r) {
      t0 = (J.cos_p * (y / r) - J.sin_p * (x / r)) * quadruple;
      t1 = (-J.cos_p * (x / r) - J.sin_p * (y / r)) * quadruple;
    } else {
      t0 = sgn_bss * y / r;
      t1 = (2 * J.p.bss - 1) * x / r;
    }
  } else if (J.p.bar) {
    const double xx = J.cos_b * x - J.sin_b * y;
    const double yy = J.sin_b * x + J.cos_b * y;
    if (r > J.bar_lim) {
      t0 = (J.cos_p * (y / r) - J.sin_p * (x / r)) * quadruple;
      t1 = (-J.cos_p * (x / r) - J.sin_p * (y / r)) * quadruple;
    } else if (yy != 0) {
      const double new_x = copysign(1., yy);
      const double new_y = -copysign(1., yy) * (xx / yy) * J.p.bar_b * J.p.bar_b /
                           (J.p.bar_a * J.p.bar_a);
      t0 = (J.cos_b * new_x + J.sin_b * new_y) * sgn_bss;
      t1 = (-J.sin_b * new_x + J.cos_b * new_y) * sgn_bss;
      const double len = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
      t0 = t0 / len;
      t1 = t1 / len;
      t2 = t2 / len;
    } else {
      t0 = (2 * J.p.bss - 1) * copysign(1., xx) * J.sin_b;
      t1 = (2 * J.p.bss - 1) * copysign(1., xx) * J.cos_b;
    }
  }
  // btot = bhat * radial * (disk_amp * disk + halo_amp * halo)  (:11-36)
  const double rs = jaffe_radial(J, x, y);
  const double hs = J.p.disk_amp * inv_cosh2(z / J.p.disk_z0) + J.p.halo_amp * inv_cosh2(z / J.p.halo_z0);
  b[0] = t0 * rs * hs;
  b[1] = t1 * rs * hs;
  b[2] = t2 * rs * hs;
  // arm compression (arm_compress, :103-129)
  double a0[8];
  const int na = jaffe_dist2arm(J, x, y, a0);
  const double rc = r / J.p.comp_r;
  const double zs = inv_cosh2(z / J.p.arm_z0);
  const double d0_inv = (rs * zs) / J.p.comp_d;
  const double factor = J.c0 * rs * zs;
  if (rc > 1) {
    const double cdrop = pow(rc, -J.p.comp_p);
    for (int i = 0; i < na; ++i)
      a0[i] = factor * cdrop * exp(-a0[i] * a0[i] * cdrop * cdrop * d0_inv * d0_inv);
  } else {
    for (int i = 0; i < na; ++i) a0[i] = factor * exp(-a0[i] * a0[i] * d0_inv * d0_inv);
  }
  if (na == 1) {
    const double inner_b = J.p.ring ? J.p.ring_amp : (J.p.bar ? J.p.bar_amp : 0.);
    b[0] += t0 * a0[0] * inner_b;
    b[1] += t1 * a0[0] * inner_b;
    b[2] += t2 * a0[0] * inner_b;
  } else {
    for (int i = 0; i < na; ++i) {
      b[0] += t0 * a0[i] * J.p.arm_amp[i];
      b[1] += t1 * a0[i] * J.p.arm_amp[i];
      b[2] += t2 * a0[i] * J.p.arm_amp[i];
    }
  }
}

// ---- Breg_jf12 ------------------------------------------------------
struct Jf12Dev {
  hxg_breg_jf12_t p;     // the Param block (working units)
  double bv[8];          // the 8 arm fields, the 8th from flux conservation
  double rc_b[8];        // arm boundaries on the negative x axis
  double cot_inc, sin_inc, cos_inc;  // 1/tan(90 - 11.5 deg), sin/cos 11.5 deg
  double tan_x;          // tan(Xtheta)
  double r_max, rho_gc, r_min, r_cent;  // 20, 1, 5, 3 kpc
  double tiny;           // 1e-12 G: the value the reference returns outside
};

static __device__ __noinline__ void breg_jf12(const Jf12Dev &J, double x, double y, double z,
                                       double b[3]) {
  const double r = sqrt(x * x + y * y);
  const double rho = sqrt(x * x + y * y + z * z);
  const double phi = atan2(y, x);
  if (r > J.r_max || rho < J.rho_gc) {
    b[0] = b[1] = b[2] = J.tiny;
    return;
  }
  // disk (breg_jf12.cc:72-120)
  const double B0 = (J.r_min / r);
  const double zprofile = 1. / (1 + exp(-2. / J.p.w_disk * (fabs(z) - J.p.h_disk)));
  double cyl0 = 0., cyl1 = 0., cyl2 = 0.;
  if (r > J.r_cent) {
    if (r < J.r_min) {
      cyl1 = B0 * J.p.b_ring * (1 - zprofile);
    } else {
      double b_disk = 0.;
      double r_negx = r * exp(-J.cot_inc * (phi - cgs::pi));
      if (r_negx > J.rc_b[7]) r_negx = r * exp(-J.cot_inc * (phi + cgs::pi));
      if (r_negx > J.rc_b[7]) r_negx = r * exp(-J.cot_inc * (phi + 3 * cgs::pi));
      for (int i = 7; i >= 0; i--)
        if (r_negx < J.rc_b[i]) b_disk = J.bv[i];
      cyl0 = b_disk * B0 * J.sin_inc * (1 - zprofile);
      cyl1 = b_disk * B0 * J.cos_inc * (1 - zprofile);
    }
  }
  // toroidal halo (:122-139)
  double b1, rh;
  if (z >= 0) {
    b1 = J.p.Bn;
    rh = J.p.rn;
  } else {
    b1 = J.p.Bs;
    rh = J.p.rs;
  }
  const double B_h = b1 * (1. - 1. / (1. + exp(-2. / J.p.wh * (r - rh)))) * exp(-(fabs(z)) / (J.p.z0));
  cyl1 += B_h * zprofile;
  // X field (:141-170)
  double Xtheta, rp_X, B_X;
  const double r_sign = z < 0 ? -1. : 1.;
  const double rc_X = J.p.rpc_X + fabs(z) / J.tan_x;
  if (r < rc_X) {
    rp_X = r * J.p.rpc_X / rc_X;
    const double q = J.p.rpc_X / rc_X;
    B_X = J.p.B0_X * (q * q) * exp(-rp_X / J.p.r0_X);
    Xtheta = atan(fabs(z) / (r - rp_X));
    if (z == 0.) Xtheta = cgs::pi / 2.;
  } else {
    Xtheta = J.p.Xtheta;
    rp_X = r - fabs(z) / J.tan_x;
    B_X = J.p.B0_X * rp_X / r * exp(-rp_X / J.p.r0_X);
  }
  cyl0 += B_X * cos(Xtheta) * r_sign;
  cyl2 += B_X * sin(Xtheta);
  // cylindrical -> Cartesian (:178-186)
  const double cp = cos(phi), sp = sin(phi);
  b[0] = cyl0 * cp - cyl1 * sp;
  b[1] = cyl0 * sp + cyl1 * cp;
  b[2] = cyl2;
}

// ---- TEreg_ymw16 ----------------------------------------------------
struct Ymw16Dev {
  hxg_tereg_ymw16_t p;   // the Param block (working units)
  double pc, kpc;        // one pc / kpc in working units
  double gum_xc, gum_yc, gum_zc;   // Gum nebula centre (tereg_ymw16.cc:234-240)
  double cos_li, sin_li;           // Loop I orientation (:307)
};

__device__ __forceinline__ double ymw_thick(const Ymw16Dev &Y, double zz, double rr) {
  if (zz > 10. * Y.p.t1_h1) return 0.;
  double gd = 1.;
  if (rr > Y.p.t1_bd) gd = sech2((rr - Y.p.t1_bd) / Y.p.t1_ad);
  return Y.p.t1_n1 * gd * sech2(zz / Y.p.t1_h1);
}

__device__ __forceinline__ double ymw_thin(const Ymw16Dev &Y, double zz, double rr) {
  const double h0 = Y.p.t2_k2 * (32 * Y.pc + 1.6e-3 * rr + (4.e-7 / Y.pc) * rr * rr);
  if (zz > 10. * h0) return 0.;
  double gd = 1.;
  if (rr > Y.p.t1_bd) gd = sech2((rr - Y.p.t1_bd) / Y.p.t1_ad);
  return Y.p.t2_n2 * gd * sech2((rr - Y.p.t2_b2) / Y.p.t2_a2) * sech2(zz / h0);
}

__device__ __forceinline__ double ymw_spiral(const Ymw16Dev &Y, double xx, double yy,
                                             double zz, double rr) {
  double scaling = 1.;
  if (rr > Y.p.t1_bd) {
    if ((rr - Y.p.t1_bd) > 10. * Y.p.t1_ad) return 0.;
    scaling = sech2((rr - Y.p.t1_bd) / Y.p.t1_ad);
  }
  const double h0 = Y.p.t3_ka * (32 * Y.pc + 1.6e-3 * rr + (4.e-7 / Y.pc) * (rr * rr));
  if (zz > 10. * h0) return 0.;
  scaling *= sech2(zz / h0);
  if ((rr - Y.p.t3_b2s) > 10. * Y.p.t3_aa) return 0.;
  scaling *= sech2((rr - Y.p.t3_b2s) / Y.p.t3_aa);
  double theta = atan2(yy, xx);
  if (theta < 0) theta += 2 * cgs::pi;
  double ne3s = 0.;
  // the reference loops over arms 0..3 (its local-arm branch for i == 4
  // is never reached)
  for (int i = 0; i < 4; ++i) {
    double d_phi = theta - Y.p.t3_phimin[i];
    if (d_phi < 0) d_phi += 2. * cgs::pi;
    const double d = fabs(Y.p.t3_rmin[i] * exp(d_phi * Y.p.t3_tpitch[i]) - rr);
    const double d_p = fabs(Y.p.t3_rmin[i] * exp((d_phi + 2. * cgs::pi) * Y.p.t3_tpitch[i]) - rr);
    const double smin = fmin(d, d_p) * Y.p.t3_cpitch[i];
    if (smin > 10. * Y.p.t3_warm[i]) continue;
    if (i != 2) {
      ne3s += Y.p.t3_narm[i] * scaling * sech2(smin / Y.p.t3_warm[i]);
    } else {
      const double tr = theta * cgs::rad;  // as the reference writes it
      const double qs = (tr - Y.p.t3_thetasg) / Y.p.t3_wsg;
      double ga;
      if (rr > 6 * Y.kpc && tr > Y.p.t3_thetacn) {
        ga = (1. - (Y.p.t3_nsg) * (exp(-(qs * qs)))) * (1. + Y.p.t3_ncn) *
             sech2(smin / Y.p.t3_warm[i]);
      } else {
        const double qc = (tr - Y.p.t3_thetacn) / Y.p.t3_wcn;
        ga = (1. - (Y.p.t3_nsg) * (exp(-(qs * qs)))) * (1. + Y.p.t3_ncn * exp(-(qc * qc))) *
             sech2(smin / Y.p.t3_warm[i]);
      }
      ne3s += Y.p.t3_narm[i] * scaling * ga;
    }
  }
  return ne3s;
}

__device__ __forceinline__ double ymw_galcen(const Ymw16Dev &Y, double xx, double yy,
                                             double zz) {
  const double Xgc = 50. * Y.pc, Ygc = 0., Zgc = -7. * Y.pc;
  const double R2gc = (xx - Xgc) * (xx - Xgc) + (yy - Ygc) * (yy - Ygc);
  if (R2gc > 10. * Y.p.t4_agc * Y.p.t4_agc) return 0.;
  const double Ar = exp(-R2gc / (Y.p.t4_agc * Y.p.t4_agc));
  if (fabs(zz - Zgc) > 10. * Y.p.t4_hgc) return 0.;
  const double Az = sech2((zz - Zgc) / Y.p.t4_hgc);
  return Y.p.t4_ngc * Ar * Az;
}

__device__ __forceinline__ double ymw_gum(const Ymw16Dev &Y, double xx, double yy,
                                          double zz) {
  if (yy < 0 || xx > 0) return 0.;
  const double xc = Y.gum_xc, yc = Y.gum_yc, zc = Y.gum_zc;
  const double theta =
      atan2(fabs(zz - zc), sqrt((xx - xc) * (xx - xc) + (yy - yc) * (yy - yc)));
  const double tantheta = tan(theta);
  const double zp = (Y.p.t5_agn * Y.p.t5_kgn) /
                    sqrt(1. + Y.p.t5_kgn * Y.p.t5_kgn / (tantheta * tantheta));
  const double xyp = zp / tantheta;
  const double xy_dist = sqrt(Y.p.t5_agn * Y.p.t5_agn - xyp * xyp) * double(Y.p.t5_agn > xyp);
  const double alpha = atan2(Y.p.t5_kgn * xyp, xy_dist) + theta;
  const double R2 = (xx - xc) * (xx - xc) + (yy - yc) * (yy - yc) + (zz - zc) * (zz - zc);
  const double r2 = zp * zp + xyp * xyp;
  const double sa = sin(alpha);
  const double D2min = (R2 + r2 - 2. * sqrt(R2 * r2)) * sa * sa;
  if (D2min > 10. * Y.p.t5_wgn * Y.p.t5_wgn) return 0.;
  return Y.p.t5_ngn * exp(-D2min / (Y.p.t5_wgn * Y.p.t5_wgn));
}

__device__ __forceinline__ double ymw_localbubble(const Ymw16Dev &Y, double xx, double yy,
                                                  double zz, double ll, double Rlb) {
  if (yy < 0) return 0.;
  double nel = 0.;
  const double u = (yy - 8.34 * Y.kpc) * 0.94 - 0.34 * zz;
  const double rLB = sqrt(u * u + xx * xx);
  const double dl1 = fmin(fabs(ll + 360. - Y.p.t6_thetalb1), fabs(Y.p.t6_thetalb1 - (ll)));
  if (dl1 < 10. * Y.p.t6_detlb1 || (rLB - Rlb) < 10. * Y.p.t6_wlb1 || zz < 10. * Y.p.t6_hlb1)
    nel += Y.p.t6_nlb1 * sech2(dl1 / Y.p.t6_detlb1) * sech2((rLB - Rlb) / Y.p.t6_wlb1) *
           sech2(zz / Y.p.t6_hlb1);
  const double dl2 = fmin(fabs(ll + 360 - Y.p.t6_thetalb2), fabs(Y.p.t6_thetalb2 - (ll)));
  if (dl2 < 10. * Y.p.t6_detlb2 || (rLB - Rlb) < 10. * Y.p.t6_wlb2 || zz < 10. * Y.p.t6_hlb2)
    nel += Y.p.t6_nlb2 * sech2(dl2 / Y.p.t6_detlb2) * sech2((rLB - Rlb) / Y.p.t6_wlb2) *
           sech2(zz / Y.p.t6_hlb2);
  return nel;
}

__device__ __forceinline__ double ymw_nps(const Ymw16Dev &Y, double xx, double yy,
                                          double zz) {
  if (yy < 0) return 0.;
  const double x_c = -10.156 * Y.pc, y_c = 8106.207 * Y.pc, z_c = 10.467 * Y.pc;
  const double rLI = sqrt((xx - x_c) * (xx - x_c) + (yy - y_c) * (yy - y_c) + (zz - z_c) * (zz - z_c));
  const double theta = acos(((xx - x_c) * (Y.cos_li) + (zz - z_c) * (Y.sin_li)) / rLI) / cgs::rad;
  if (theta > 10. * Y.p.t7_detthetali || (rLI - Y.p.t7_rli) > 10. * Y.p.t7_wli) return 0.;
  const double a = (rLI - Y.p.t7_rli) / Y.p.t7_wli, t = theta / Y.p.t7_detthetali;
  return (Y.p.t7_nli) * exp(-(a * a)) * exp(-(t * t));
}

// write_field (tereg_ymw16.cc:10-75): YMW16 frame (y, -x, z), warp,
// 25-kpc cut, components and their combination rules
static __device__ __noinline__ double tereg_ymw16(const Ymw16Dev &Y, double x, double y, double z) {
  double gx = y, gy = -x, gz = z;
  const double r_cyl = sqrt(gx * gx + gy * gy);
  if (r_cyl >= Y.p.r_warp) {
    const double theta_warp = atan2(gy, gx);
    gz -= Y.p.t0_gamma_w * (r_cyl - Y.p.r_warp) * cos(theta_warp);
  }
  if (sqrt(gx * gx + gy * gy + gz * gz) > 25 * Y.kpc) return 0.;
  double ne_comp[8] = {0., 0., 0., 0., 0., 0., 0., 0.};
  double w_lb = 0., w_gum = 0., w_loop = 0.;
  const double ec_l = atan2(gx, Y.p.r0 - gy) / cgs::rad;
  ne_comp[1] = ymw_thick(Y, gz, r_cyl);
  ne_comp[2] = ymw_thin(Y, gz, r_cyl);
  ne_comp[3] = ymw_spiral(Y, gx, gy, gz, r_cyl);
  ne_comp[4] = ymw_galcen(Y, gx, gy, gz);
  ne_comp[5] = ymw_gum(Y, gx, gy, gz);
  const double lb_boundary = 110. * Y.pc;
  ne_comp[6] = ymw_localbubble(Y, gx, gy, gz, ec_l, lb_boundary);
  ne_comp[7] = ymw_nps(Y, gx, gy, gz);
  ne_comp[0] = ne_comp[1] + fmax(ne_comp[2], ne_comp[3]);
  const double u = (gy - 8.34 * Y.kpc) * 0.94 - 0.34 * gz;
  const double rlb = sqrt(u * u + gx * gx);
  if (rlb < lb_boundary) {
    ne_comp[0] = Y.p.t6_j_lb * ne_comp[1] + fmax(ne_comp[2], ne_comp[3]);
    if (ne_comp[6] > ne_comp[0]) w_lb = 1;
  } else {
    if (ne_comp[6] > ne_comp[0] && ne_comp[6] > ne_comp[5]) w_lb = 1;
  }
  if (ne_comp[7] > ne_comp[0]) w_loop = 1;
  if (ne_comp[5] > ne_comp[0]) w_gum = 1;
  return (1 - w_lb) * ((1 - w_gum) * ((1 - w_loop) * (ne_comp[0] + ne_comp[4]) +
                                      w_loop * ne_comp[7]) +
                       w_gum * ne_comp[5]) +
         (w_lb) * (ne_comp[6]);
}

// ---- CRE-grid synchrotron emissivity ---------------------------------
// (integrator.cc:282-330 total, 351-400 polarised; CREfield::read_grid_num,
// cre.cc:144-199).  The energy integral uses the midpoint rule over the
// grid's energy bins with F(x) (total) and G(x) (polarised); both come from
// tables of ln(F(x)/x^(1/3)), ln(G(x)/x^(1/3)) on u = ln x (smooth in u, so
// the relative error stays uniform where F decays like e^-x), built on the
// host from the integral definitions and read with 4-point Lagrange
// interpolation.
struct CreGridDev {
  const double *flux;         // [((i*ny + j)*nz + k)*nE + e], (GeV m^2 s sr)^-1
  int nx, ny, nz, nE;
  double lo[3], hi[3];        // box (working length units)
  const double *inv_ke2;      // [nE] 1 / KE_e^2, KE_e = E_min exp(e E_fact) (erg)
  const double *beta;         // [nE] sqrt(1 - mec2 / KE_e)
  const double *dke;          // [nE - 1] |KE_{e+1} - KE_e|
  const double *tab_f, *tab_g;
  double u0, inv_du;          // table abscissae u_k = u0 + k / inv_du
  int ntab, _pad;
  double xnum_t, xnum_p;      // numerators of x_fact (t, p) in the reference's order
  double fore_num, fore_den;  // 1.73205081 qe^3 ; mec2 c GeV m^2 s
  double bunit;               // G per working field unit
};

// F(x) or G(x) from its table: tab[k] = ln(fn(x_k) / x_k^(1/3)), x_k = e^(u0+k du)
__host__ __device__ __forceinline__ double synchro_fn(const double *tab, double u0,
                                                      double inv_du, int n, double x) {
  const double t = (log(x) - u0) * inv_du;
  if (!(t >= 1.)) return exp(tab[0]) * cbrt(x);  // below the table: x^(1/3) law
  const int k = (int)t < n - 3 ? (int)t : n - 3;
  const double f = t - k;
  const double wm = -f * (f - 1.) * (f - 2.) * (1. / 6.);
  const double w0 = (f + 1.) * (f - 1.) * (f - 2.) * 0.5;
  const double w1 = -(f + 1.) * f * (f - 2.) * 0.5;
  const double w2 = (f + 1.) * f * (f - 1.) * (1. / 6.);
  return exp(wm * tab[k - 1] + w0 * tab[k] + w1 * tab[k + 1] + w2 * tab[k + 2]) * cbrt(x);
}

// J_tot and J_pol (erg s^-1 cm^-3 Hz^-1 sr^-1, before the step and the
// brightness conversion) at position p for |B_perp| = bper (working units)
static __device__ __noinline__ void cre_grid_j(const CreGridDev &C, double px, double py,
                                        double pz, double bper, double &jt, double &jp) {
  jt = jp = 0.;
  const double p[3] = {px, py, pz};
  const int n[3] = {C.nx, C.ny, C.nz};
  int il[3];
  double fr[3];
  for (int a = 0; a < 3; ++a) {
    const double tmp = (n[a] - 1) * (p[a] - C.lo[a]) / (C.hi[a] - C.lo[a]);
    if (tmp <= 0 || tmp >= n[a] - 1) return;  // read_grid_num returns 0
    il[a] = (int)floor(tmp);
    fr[a] = tmp - il[a];
  }
  const double b = fabs(bper) * C.bunit;
  const double xf_t = C.xnum_t / (3. * cgs::qe * b);
  const double xf_p = C.xnum_p / (3. * cgs::qe * b);
  const long long sz = (long long)C.nz * C.nE, sy = (long long)C.ny * sz;
  const double *c000 = C.flux + il[0] * sy + il[1] * sz + (long long)il[2] * C.nE;
  const double xd = fr[0], yd = fr[1], zd = fr[2];
  // trilinear flux at energy e in read_grid_num's order: z, then y, then x
  const auto flux_at = [&](int e) {
    const double *q = c000 + e;
    const double i1 = q[0] * (1. - zd) + q[C.nE] * zd;
    const double i2 = q[sz] * (1 - zd) + q[sz + C.nE] * zd;
    const double j1 = q[sy] * (1 - zd) + q[sy + C.nE] * zd;
    const double j2 = q[sy + sz] * (1 - zd) + q[sy + sz + C.nE] * zd;
    const double w1 = i1 * (1 - yd) + i2 * yd;
    const double w2 = j1 * (1 - yd) + j2 * yd;
    return w1 * (1 - xd) + w2 * xd;
  };
  double v_lo = flux_at(0) / C.beta[0];
  double st = 0., sp = 0.;
  for (int e = 0; e < C.nE - 1; ++e) {
    const double v_hi = flux_at(e + 1) / C.beta[e + 1];
    const double flux = 0.5 * (v_hi + v_lo);
    v_lo = v_hi;
    const double xt = 0.5 * (xf_t * C.inv_ke2[e + 1] + xf_t * C.inv_ke2[e]);
    const double xp = 0.5 * (xf_p * C.inv_ke2[e + 1] + xf_p * C.inv_ke2[e]);
    if (!(xt > 100)) st += synchro_fn(C.tab_f, C.u0, C.inv_du, C.ntab, xt) * flux * C.dke[e];
    if (!(xp > 100)) sp += synchro_fn(C.tab_g, C.u0, C.inv_du, C.ntab, xp) * flux * C.dke[e];
  }
  const double fore = C.fore_num * b / C.fore_den;
  jt = st * fore;
  jp = sp * fore;
}

// The three models' parameter blocks and the CRE grid of one launch, in
// device memory (the kernels that read them are separate instantiations, so
// the common path carries neither their code nor their parameters).
struct ExtModels {
  JaffeDev jaffe;
  Jf12Dev jf12;
  Ymw16Dev ymw16;
  CreGridDev cre;
};

}  // namespace hxg
