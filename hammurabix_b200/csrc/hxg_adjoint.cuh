// hxg_adjoint.cuh -- adjoint (reverse-mode) shell kernel of the FP64 form.
//
// Given dL/d(shell maps) of one shell, it accumulates dL/d(packed grid
// records), dL/d(model parameters) and dL/d(inner-shell Faraday-depth map).
// Per-shell checkpointing: the forward kernel stored, for every (pixel,
// chunk), the chunk's Faraday depth and its local-frame Q, U sums, plus the
// pixel's inner-shell Faraday depth.  From those the backward kernel gets,
// with warp shuffles, the pixel totals Q, U and each chunk's prefix, so a
// single forward-ordered sweep suffices: the reverse-accumulated phase
// sensitivity S_i = sum_{k >= i} dL/dchi_k equals
// 2 (gU (Q - Q_{<i}) - gQ (U - U_{<i})).
//
// Per sample i (symbols of integrator.cc:173-226):
//   t_i   = n_e B_par K dl           (Faraday-depth term, K = fd_forefactor)
//   chi_i = (FD_inner + sum_{k<=i} t_k) lambda^2 + ipa_i
//   dL/dt_i   = gFD + lambda^2 S_i
//   dL/dJt_i  = gI,  dL/dJp_i = gQ cos 2chi_i + gU sin 2chi_i
//   J ~ |B_perp|^(1-e), e = (index+1)/2  ->  dJ/d|B_perp| = (1-e) J / |B_perp|
//   dipa/dB = (-x e_theta + y e_phi) / (x^2 + y^2),  y = -e_theta.B,
//   x = -e_phi.B
#pragma once

#include "hxg_integrate.cuh"

namespace hxg {

// Parameter-gradient slots: spiral B (b0, pitch, r_scale, h_scale),
// exponential n_e disk (n0, r_scale, h_scale), CRE normalisation j0.
constexpr int kNumParams = 8;

struct AdjointLaunch {
  ShellLaunch F;            // the forward launch of this shell
  const double *ck;         // [(nest * C + c) * 3]: chunk FD, Q, U (local frame)
  const double *ck_inner;   // [ring]: inner-shell FD of each pixel
  const double *g[5];       // dL/d(shell maps) (ring): dm, fd, I, Q, U (I,Q,U
                            // already times the temp_convert factor)
  double *grad_rec;         // [N * 4] dL/d(group-0 records), or null
  double *grad_par;         // [kNumParams], or null
  double *g_fdmap;          // [npix(nside_fdmap)] dL/d(accumulated FD map), or null
  int want_j0;              // 1 when the CRE normalisation gradient is wanted
};

__device__ __forceinline__ void flush_cell(double *grad_rec, long long key,
                                           int ny, int nz, double acc[8][4]) {
  if (key < 0 || grad_rec == nullptr) return;
  const long long nyz = (long long)ny * nz;
  const long long xl = key / nyz;
  const long long yl = (key - xl * nyz) / nz;
  const long long zl = key - xl * nyz - yl * nz;
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz) {
        const int k = dx * 4 + dy * 2 + dz;
        const long long idx = (xl + dx) * nyz + (yl + dy) * nz + (zl + dz);
        double *p = grad_rec + 4 * idx;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (acc[k][c] != 0.) atomicAdd(p + c, acc[k][c]);
          acc[k][c] = 0.;
        }
      }
}

// Launch shape of the adjoint shell kernel (threads per block, resident
// blocks per SM its register allocation must allow).  128 x 3 (168
// registers, 12 warps per SM; the per-cell gradient accumulators take 64)
// ran the config-4 adjoint in 49.9 ms against 52.4 ms at 128 x 4 (128
// registers, more spills) and 62.2 ms at 256 x 1 (254 registers, 8 warps).
#ifndef HXG_ADJ_THREADS
#define HXG_ADJ_THREADS 128
#endif
#ifndef HXG_ADJ_MIN_BLOCKS
#define HXG_ADJ_MIN_BLOCKS 3
#endif

// kFast: the forward launch's models satisfy fast_models (the other models
// compiled out).
template <int NG, bool kExt, bool kFast>
__global__ void __launch_bounds__(HXG_ADJ_THREADS, HXG_ADJ_MIN_BLOCKS)
shell_fp64_adjoint_kernel(const AdjointLaunch A) {
  const ShellLaunch &P = A.F;
  const int lane = threadIdx.x & 31;
  const long long gw =
      ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int C = P.chunks;
  const int seg = lane >> P.log2_chunks;
  const int c = lane & (C - 1);
  const Hpx h = hpx_make((uint64_t)P.nside);
  // shard `shard` of `nshards` of the shell (the forward's pixels)
  const unsigned long long nest =
      shard_nest(P, (unsigned long long)gw * (32 >> P.log2_chunks) + seg);
  const bool valid = nest < h.npix;
  uint64_t ring = 0;
  bool live = false;
  if (valid) {
    ring = hpx_nest2ring(h, nest);
    live = (P.mask == nullptr) || (P.mask[ring] != 0);
  }
  // checkpointed chunk sums; dead lanes contribute zeros to the shuffles
  double fdc = 0., qc = 0., uc = 0.;
  if (live) {
    const unsigned long long ci = nest * (unsigned long long)C + c;
    fdc = A.ck[3 * ci];
    qc = A.ck[3 * ci + 1];
    uc = A.ck[3 * ci + 2];
  }
  const double l2 = P.lambda2;
  // exclusive Faraday-depth prefix F_c of the chunks before this one
  double incl = fdc;
  for (int o = 1; o < C; o <<= 1) {
    const double v = __shfl_up_sync(0xffffffffu, incl, o);
    if (c >= o) incl += v;
  }
  double Fc = __shfl_up_sync(0xffffffffu, incl, 1);
  if (c == 0) Fc = 0.;
  // chunk Q, U in the pixel's (global) phase frame
  double qg = qc, ug = uc;
  if (P.do_sync && c > 0) {
    double sr, cr;
    sincos(2. * l2 * Fc, &sr, &cr);
    qg = qc * cr - uc * sr;
    ug = qc * sr + uc * cr;
  }
  double qi = qg, ui = ug;
  for (int o = 1; o < C; o <<= 1) {
    const double vq = __shfl_up_sync(0xffffffffu, qi, o);
    const double vu = __shfl_up_sync(0xffffffffu, ui, o);
    if (c >= o) {
      qi += vq;
      ui += vu;
    }
  }
  const int last = (seg << P.log2_chunks) + C - 1;
  const double Qp = __shfl_sync(0xffffffffu, qi, last);
  const double Up = __shfl_sync(0xffffffffu, ui, last);
  double Qrun = qi - qg, Urun = ui - ug;  // Q, U of the chunks before this one
  if (c == 0) {
    Qrun = 0.;
    Urun = 0.;
  }
  double gp[kNumParams];
#pragma unroll
  for (int k = 0; k < kNumParams; ++k) gp[k] = 0.;
  if (live) {
    const double gdm = P.do_dm ? A.g[0][ring] : 0.;
    const double gfd = (P.do_fd || P.do_sync) ? A.g[1][ring] : 0.;
    const double gI = P.do_sync ? A.g[2][ring] : 0.;
    const double gQ = P.do_sync ? A.g[3][ring] : 0.;
    const double gU = P.do_sync ? A.g[4][ring] : 0.;
    double th, ph;
    hpx_pix2ang(h, ring, th, ph);
    const double inner = A.ck_inner[ring];
    // dL/d(inner FD) = lambda^2 sum_i dL/dchi_i, scattered through the
    // transpose of the HEALPix interpolation that produced it
    if (c == 0 && A.g_fdmap != nullptr && P.fdmap != nullptr && P.do_sync) {
      const double g_inner = l2 * 2. * (gU * Qp - gQ * Up);
      const Hpx hf = hpx_make((uint64_t)P.nside_fdmap);
      uint64_t pix[4];
      double w[4];
      hpx_interp_weights(hf, th, ph, pix, w);
      const double wtot = w[0] + w[1] + w[2] + w[3];
      if (wtot != 0.)
        for (int k = 0; k < 4; ++k) atomicAdd(A.g_fdmap + pix[k], g_inner * w[k] / wtot);
    }
    const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
    const double ux = cp * st, uy = sp * st, uz = ct;
    const double etx = ct * cp, ety = ct * sp, etz = -st;
    const double epx = -sp, epy = cp;
    const DevModels &M = P.models;
    double acc[8][4];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[k][q] = 0.;
    long long acc_key = -1;
    double gt = P.em_gt, gpp = P.em_gp, last_index = nan("");
    double fdl = 0.;  // running FD of this chunk
    long long wlo, whi, slo_unused, shi_unused;
    ray_window(P, ux, uy, uz, wlo, whi, slo_unused, shi_unused);
    const long long i0 = max((P.step * c) >> P.log2_chunks, wlo);
    const long long i1 = min((P.step * (c + 1)) >> P.log2_chunks, whi);
    for (long long i = i0; i < i1; ++i) {
      const double d = P.d_start + ((double)i + 0.5) * P.delta;
      const double px = ux * d + P.obs[0];
      const double py = uy * d + P.obs[1];
      const double pz = uz * d + P.obs[2];
      // every sample is tested (the certain window measured slower here)
      const double len = sqrt(px * px + py * py + pz * pz);
      if (len < P.gc_r_min || len > P.gc_r_max || pz < P.gc_z_min ||
          pz > P.gc_z_max)
        continue;
      const double p3[3] = {px, py, pz};
      V3<double> Breg{0., 0., 0.};
      double tereg = 0.;
      if (kFast) {
        if (M.breg == kBregSpiral) Breg = breg_spiral<double>(M, px, py, pz, p3);
        if (M.tereg == kTeregExpdisk) tereg = tereg_expdisk<double>(M, px, py, pz);
      } else {
        Breg = breg_model_x<kExt>(M, P.ext, px, py, pz, p3);
        tereg = tereg_model_x<kExt>(M, P.ext, px, py, pz, p3);
      }
      double b3[3] = {Breg.x, Breg.y, Breg.z};
      double te = tereg;
      bool in_grid = false;
      int xl = 0, yl = 0, zl = 0;
      double xd = 0., yd = 0., zd = 0.;
      if (NG > 0) {
        const DevGridGroup &G = P.groups[0];
        if (grid_coords(G, px, py, pz, xl, yl, zl, xd, yd, zd)) {
          in_grid = true;
          CellCache<double> cc;
          fill_cell<double>(G, xl, yl, zl, cc);
          double out[4];
          trilinear<double>(cc, xd, yd, zd, out);
          b3[0] += out[0];
          b3[1] += out[1];
          b3[2] += out[2];
          te += out[3];
        }
      }
      const double te_raw = te;
      te *= (double)(te > 0.);
      const double bx = b3[0], by = b3[1], bz = b3[2];
      const double bpar = bx * ux + by * uy + bz * uz;
      const double cx = by * uz - bz * uy, cy = bz * ux - bx * uz,
                   cz = bx * uy - by * ux;
      const double bper = sqrt(cx * cx + cy * cy + cz * cz);
      const double t = te * bpar * P.fd_fore * P.delta;
      fdl += t;
      double g_te = gdm * P.delta;
      double g_bpar = 0., g_bper = 0., g_ipa = 0.;
      double xv = 0., yv = 0.;
      double jt = 0., jp = 0., e = 0.;
      if (P.do_fd || P.do_sync) {
        double gtt = gfd;
        if (P.do_sync) {
          double index = P.em_index;
          if (!kFast && !P.em_const) {
            index = cre_index<double>(M, px, py, pz);
            if (index != last_index) {
              gt = tgamma(-0.25 * index + 19. / 12.) * tgamma(-0.25 * index - 1. / 12.);
              gpp = tgamma(-0.25 * index + 7. / 12.) * tgamma(-0.25 * index - 1. / 12.);
              last_index = index;
            }
          }
          e = 0.5 * (index + 1);
          const double fn = P.em_n0u * (kFast ? cre_profile_ana<double>(M, px, py, pz)
                                              : cre_profile<double>(M, px, py, pz, p3));
          const double absb = fabs(bper);
          const double Aa = P.em_anum / (P.em_3qe * absb);
          double Ae;
          if (P.em_const && P.em_pow_kind == 1)
            Ae = 1. / Aa;
          else if (P.em_const && P.em_pow_kind == 2)
            Ae = 1.;
          else
            Ae = pow(Aa, e);
          const double den_t = P.em_const ? P.em_den_t
                                          : 4. * cgs::pi * cgs::mec2 * (1. - index);
          jt = fn * 1.73205081 * P.em_qe3 * absb / den_t * (Ae * gt) * P.delta * P.i2bt;
          jp = fn * 1.73205081 * P.em_qe3 * absb / P.em_den_p * (Ae * gpp) * P.delta *
               P.i2bt;
          xv = -(epx * bx + epy * by);
          yv = -(etx * bx + ety * by + etz * bz);
          double c2, s2;
          ipa2<double>(xv, yv, c2, s2);
          double sf, cf;
          sincos(2. * ((inner + Fc + fdl) * l2), &sf, &cf);
          const double cos2 = cf * c2 - sf * s2;
          const double sin2 = sf * c2 + cf * s2;
          // S_i: sensitivity of the loss to the phase of samples k >= i
          const double Si = 2. * (gU * (Qp - Qrun) - gQ * (Up - Urun));
          Qrun += jp * cos2;
          Urun += jp * sin2;
          gtt += l2 * Si;
          const double gjt = gI, gjp = gQ * cos2 + gU * sin2;
          g_ipa = 2. * jp * (gU * cos2 - gQ * sin2);
          if (bper > 0.) g_bper = (gjt * jt + gjp * jp) * (1. - e) / bper;
          if (A.want_j0) gp[7] += gjt * jt + gjp * jp;
        }
        g_te += gtt * bpar * P.fd_fore * P.delta;
        g_bpar = gtt * te * P.fd_fore * P.delta;
      }
      if (!(te_raw > 0.)) g_te = 0.;
      // dL/dB
      double gbx = g_bpar * ux, gby = g_bpar * uy, gbz = g_bpar * uz;
      if (bper > 0.) {
        const double k = g_bper / bper;
        gbx += k * (bx - bpar * ux);
        gby += k * (by - bpar * uy);
        gbz += k * (bz - bpar * uz);
      }
      const double r2 = xv * xv + yv * yv;
      if (g_ipa != 0. && r2 > 0.) {
        const double k = g_ipa / r2;
        gbx += k * (-xv * etx + yv * epx);
        gby += k * (-xv * ety + yv * epy);
        gbz += k * (-xv * etz);
      }
      // analytic-model parameter gradients
      if (M.breg == kBregSpiral && (Breg.x != 0. || Breg.y != 0.)) {
        const double r = sqrt(px * px + py * py);
        const double gdotb = gbx * Breg.x + gby * Breg.y;
        gp[0] += gdotb / M.sp_b0;
        // B = amp (sin(pitch - phi), cos(pitch - phi)), so dB/dpitch is B
        // turned by -90 degrees: (B_y, -B_x)
        gp[1] += gbx * Breg.y - gby * Breg.x;
        gp[2] += gdotb * (r - M.sp_rsun) / (M.sp_rs * M.sp_rs);
        gp[3] += gdotb * fabs(pz) / (M.sp_hs * M.sp_hs);
      }
      if (M.tereg == kTeregExpdisk && tereg != 0.) {
        const double r = sqrt(px * px + py * py);
        gp[4] += g_te * tereg / M.tex_n0;
        gp[5] += g_te * tereg * r / (M.tex_rs * M.tex_rs);
        gp[6] += g_te * tereg * fabs(pz) / (M.tex_hs * M.tex_hs);
      }
      // grid-record gradients, accumulated per cell
      if (NG > 0 && in_grid && A.grad_rec != nullptr) {
        const DevGridGroup &G = P.groups[0];
        const long long key = (long long)xl * ((long long)G.ny * G.nz) +
                              (long long)yl * G.nz + zl;
        if (key != acc_key) {
          flush_cell(A.grad_rec, acc_key, G.ny, G.nz, acc);
          acc_key = key;
        }
        const double wx[2] = {1. - xd, xd}, wy[2] = {1. - yd, yd},
                     wz[2] = {1. - zd, zd};
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
          for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
              const double w = wx[dx] * wy[dy] * wz[dz];
              const int k = dx * 4 + dy * 2 + dz;
              acc[k][0] += w * gbx;
              acc[k][1] += w * gby;
              acc[k][2] += w * gbz;
              acc[k][3] += w * g_te;
            }
      }
    }
    if (NG > 0)
      flush_cell(A.grad_rec, acc_key, P.groups[0].ny, P.groups[0].nz, acc);
  }
  // parameter gradients: warp reduction, one atomic per warp and slot
  if (A.grad_par != nullptr) {
#pragma unroll
    for (int k = 0; k < kNumParams; ++k) {
      double v = gp[k];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0 && v != 0.) atomicAdd(A.grad_par + k, v);
    }
  }
}

}  // namespace hxg
