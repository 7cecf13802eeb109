// hxg_adjoint32.cuh -- adjoint (reverse-mode) shell kernel of the
// FP32-compensated form.
//
// The reverse of fp32c_tile (one frequency pass, the grid workloads'
// models: spiral or no regular B, exponential-disk or no regular n_e, one
// grid geometry, CRE_ana with a constant index) in the same precision split
// as that forward: the ray, the Faraday-depth path (n_e B_par, its running
// sum, the phase) and the reverse phase sensitivity in FP64; the grid
// interpolation, the synchrotron emissivity, the polarisation angle and the
// field gradients in FP32.  The structure follows shell_fp64_adjoint_kernel
// (hxg_adjoint.cuh): the forward stored, per (pixel, chunk), the chunk's FD
// and local-frame Q, U, and per pixel the inner-shell FD; one forward-ordered
// sweep per chunk then forms S_i = 2 (gU (Q - Q_{<i}) - gQ (U - U_{<i})), the
// sensitivity of the loss to the phase of the samples k >= i.
//
// Per sample, with J_t, Q_i, U_i the sample's emissivity terms in output
// units and B in 2^-20 G:
//   dL/dt_i  = gFD + lambda^2 S_i                (t_i: the sample's FD term)
//   e_i      = gI J_t + gQ Q_i + gU U_i          (= sum dL/dJ J)
//   dL/dB    = dL/dt_i dt_i/dB_par u + e_i pe/|B_perp|^2 B_perp
//              + 2 (gU Q_i - gQ U_i) dipa/dB     (J ~ |B_perp|^pe)
// The per-cell gradient of the grid records is summed in 32 FP32 registers
// while the ray stays in a cell (half the FP64 kernel's 64) and flushed
// into the FP64 record gradient with FP64 atomics.  Gradients come out in
// the form's units (kpc, 2^-20 G); the host converts them to CGS.
#pragma once

#include "hxg_adjoint.cuh"
#include "hxg_fp32c.cuh"

// Launch shape of the FP32C adjoint kernel (threads per block, resident
// blocks per SM its register allocation must allow).  128 x 4 (128
// registers) ran the config-4 adjoint in 18.1 ms against 19.3 ms at 128 x 3,
// 24.4 ms at 128 x 2, 20.3 ms at 128 x 5 and 22.6 ms at 128 x 6.
#ifndef HXG_ADJ32_THREADS
#define HXG_ADJ32_THREADS 128
#endif
#ifndef HXG_ADJ32_MIN_BLOCKS
#define HXG_ADJ32_MIN_BLOCKS 4
#endif

namespace hxg {

constexpr unsigned kNoCell = 0xFFFFFFFFu;

// Adds the accumulators of the cell whose corner 000 is record `key` into
// the FP64 record gradient and clears them.
__device__ __forceinline__ void flush_cell32(double *grad_rec, unsigned key, unsigned ny,
                                             unsigned nz, float acc[8][4]) {
  if (key == kNoCell) return;
  const unsigned nyz = ny * nz;
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz) {
        const int k = dx * 4 + dy * 2 + dz;
        double *p = grad_rec + 4 * (size_t)(key + dx * nyz + dy * nz + dz);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (acc[k][q] != 0.f) atomicAdd(p + q, (double)acc[k][q]);
          acc[k][q] = 0.f;
        }
      }
}

// Parameter-gradient accumulators of the FP32C adjoint, in the form's units
// (the host converts): 0 sum B.gB over the spiral samples (dL/dln b0),
// 1 dL/dpitch, 2 dL/dr_s and 3 dL/dh_s of the spiral (per kpc), 4 sum
// n_e,disk dL/dn_e (dL/dln n0), 5 dL/dr_s and 6 dL/dh_s of the disk (per
// kpc), 7 sum dL/dJ J (dL/dln j0).
template <int NG>
__global__ void __launch_bounds__(HXG_ADJ32_THREADS, HXG_ADJ32_MIN_BLOCKS)
shell_fp32c_adjoint_kernel(const AdjointLaunch A) {
  const ShellLaunch &P = A.F;
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
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
  // exclusive Faraday-depth prefix Fc of the chunks before this one
  double incl = fdc;
  for (int o = 1; o < C; o <<= 1) {
    const double v = __shfl_up_sync(0xffffffffu, incl, o);
    if (c >= o) incl += v;
  }
  double Fc = __shfl_up_sync(0xffffffffu, incl, 1);
  if (c == 0) Fc = 0.;
  // chunk Q, U in the pixel's (global) phase frame, their prefix and totals
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
    const float etx = float(ct * cp), ety = float(ct * sp), etz = float(-st);
    const float epx = float(-sp), epy = float(cp);
    const double ox = P.obs[0], oy = P.obs[1], oz = P.obs[2];
    const double ou2 = 2. * (ox * ux + oy * uy + oz * uz);
    const double oo = ox * ox + oy * oy + oz * oz;
    const DevModels &M = P.models;
    const FastModels &F = P.fast;
    const bool fast_b = M.breg == kBregSpiral;
    const bool fast_t = M.tereg == kTeregExpdisk;
    const double rc2_hi = F.rc2_hi, rc2_lo = F.rc2_lo;
    const double K0 = F.sp_sin_s * (ox * ux + oy * uy) + F.sp_cos_s * (ox * uy - oy * ux);
    const double K1 = F.sp_sin_s * (ux * ux + uy * uy);
    const float spf = F.sp_sinf_s, cpf = F.sp_cosf_s;
    const float pe = F.pe;
    const bool pe2 = P.em_const && P.em_pe == 2.;
    // Faraday phase in turns of the pixel frame: inner + Fc + the running
    // chunk FD (the sample's own term included), rounded as in fp32c_tile
    const double rev0 = l2 * (inner + Fc) * (1. / cgs::pi) + (1572864.0 + 0x1p-24);
    const double rev_k = P.phase_k * (0.5 / cgs::pi);
    double g0x = 0., g0y = 0., g0z = 0., gvx = 0., gvy = 0., gvz = 0.;
    if (NG == 1) {
      const DevGridGroup &G = P.groups[0];
      g0x = (ox - G.lo[0]) * G.scale[0];
      g0y = (oy - G.lo[1]) * G.scale[1];
      g0z = (oz - G.lo[2]) * G.scale[2];
      gvx = ux * G.scale[0];
      gvy = uy * G.scale[1];
      gvz = uz * G.scale[2];
    }
    long long wlo, whi, slo_unused, shi_unused;
    ray_window(P, ux, uy, uz, wlo, whi, slo_unused, shi_unused);
    exact_cut_window(P, uz, ou2, oo, wlo, whi);
    const int i0 = (int)max((P.step * c) >> P.log2_chunks, wlo);
    const int i1 = (int)min((P.step * (c + 1)) >> P.log2_chunks, whi);
    double d = P.d_start + ((double)i0 + 0.5) * P.delta;
    FixAxis fx, fy, fz;
    int ga = i1, gb = i1;
    if (NG == 1) {
      const double g0[3] = {g0x, g0y, g0z}, gv[3] = {gvx, gvy, gvz};
      grid_window(P, P.groups[0], g0, gv, i0, i1, ga, gb);
      const double dg = P.d_start + ((double)ga + 0.5) * P.delta;
      fx.start(fma(gvx, dg, g0x), gvx * P.delta);
      fy.start(fma(gvy, dg, g0y), gvy * P.delta);
      fz.start(fma(gvz, dg, g0z), gvz * P.delta);
    }
    float acc[8][4];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[k][q] = 0.f;
    unsigned acc_key = kNoCell;
    double sfd = 0.;  // running FD of this chunk (FD-sum units)
    for (int i = i0; i < i1; ++i, d += P.delta) {
      const double pz = fma(uz, d, oz);
      const double px = fma(ux, d, ox);
      const double py = fma(uy, d, oy);
      const float xf = float(px), yf = float(py), zf = float(pz);
      double bp_d = 0., te_d = 0., r = 0.;
      float bxr = 0.f, byr = 0.f, rcf = 0.f;
      bool in_b = false;
      if (fast_b || fast_t) {
        const double rc2 = fma(px, px, py * py);
        const double rc2m = fmax(rc2, 1e-300);
        const double y = rsqrt_fd(rc2m);
        r = rc2m * y;
        rcf = float(r);
        in_b = fast_b && !(rc2 > rc2_hi || rc2 < rc2_lo);
        if (in_b) {
          const double ay =
              exp_tab(fma(-r, F.sp_irs, fma(-fabs(pz), F.sp_ihs, F.sp_crs_l))) * y;
          bp_d = ay * fma(K1, d, K0);
          const float ayf = float(ay);
          bxr = ayf * (spf * xf - cpf * yf);
          byr = ayf * (spf * yf + cpf * xf);
        }
        if (fast_t) te_d = exp_tab(fma(-r, F.ex_irn, fma(-fabs(pz), F.ex_ihn, F.ex_ln0)));
      }
      float bg[4] = {0.f, 0.f, 0.f, 0.f};
      unsigned key = kNoCell;
      float tx = 0.f, ty = 0.f, tz = 0.f;
      if (NG == 1) {
        const DevGridGroup &G = P.groups[0];
        if ((unsigned)(i - ga) < (unsigned)(gb - ga)) {
          if (fx.inside(G.nx) && fy.inside(G.ny) && fz.inside(G.nz)) {
            int cx, cy, cz;
            fx.split(cx, tx);
            fy.split(cy, ty);
            fz.split(cz, tz);
            trilinear_f32(reinterpret_cast<const float4 *>(G.rec), G.ny, G.nz, cx, cy, cz,
                          tx, ty, tz, bg);
            key = ((unsigned)cx * (unsigned)G.ny + (unsigned)cy) * (unsigned)G.nz +
                  (unsigned)cz;
          }
          fx.next();
          fy.next();
          fz.next();
        }
      }
      const double te_raw = te_d + double(bg[3]);
      const double te = fmax(te_raw, 0.);
      const double bpar =
          bp_d + fma(double(bg[0]), ux, fma(double(bg[1]), uy, double(bg[2]) * uz));
      sfd = fma(te, bpar, sfd);
      double g_te = gdm * P.k_dm;
      double g_bpar = 0.;
      float gbx = 0.f, gby = 0.f, gbz = 0.f;
      if (P.do_fd || P.do_sync) {
        double gtt = gfd;  // dL/d(sample FD term)
        if (P.do_sync) {
          const float bx = bxr + bg[0], by = byr + bg[1], bz = bg[2];
          const float xv = -(epx * bx + epy * by);
          const float yv = -(etx * bx + ety * by + etz * bz);
          const float rr = fmaf(xv, xv, yv * yv);
          const float cc2 = fmaf(xv, xv, -yv * yv), ss2 = 2.f * xv * yv;
          const float prof = cre_ana_prof32(F, rcf, zf);
          float wt, wpc, wps;
          if (pe2) {
            wt = prof * rr;
            wpc = prof * cc2;
            wps = prof * ss2;
          } else {
            const float wp = prof * ((pe == 1.f) ? sqrtf(rr) : powf(rr, 0.5f * pe));
            const float inv = rr > 0.f ? __frcp_rn(rr) : 0.f;
            wt = wp;
            wpc = rr > 0.f ? wp * cc2 * inv : wp;
            wps = wp * ss2 * inv;
          }
          const double rev = fma(rev_k, sfd, rev0);
          const int q = __double2loint(rev) >> 9;
          const float ang = (__int_as_float(0x4B400000 + q) - 12582912.0f) * 7.490140565847857e-07f;
          float sf, cf;
          __sincosf(ang, &sf, &cf);
          const double Qi = P.k_p * (double)fmaf(wpc, cf, -wps * sf);
          const double Ui = P.k_p * (double)fmaf(wpc, sf, wps * cf);
          const double Ji = P.k_t * (double)wt;
          // S_i counts the sample's own phase (k >= i): Q_{<i} before it
          const double Si = 2. * (gU * (Qp - Qrun) - gQ * (Up - Urun));
          Qrun += Qi;
          Urun += Ui;
          gtt = fma(l2, Si, gtt);
          const double ej = fma(gI, Ji, fma(gQ, Qi, gU * Ui));
          if (A.want_j0) gp[7] += ej;
          // |B_perp|^pe: e_i pe / |B_perp|^2 B_perp with B_perp =
          // -(xv e_phi + yv e_theta); the angle ipa = atan2(yv, xv)
          const float kb = rr > 0.f ? float(ej) * pe / rr : 0.f;
          const float ki = rr > 0.f ? float(2. * (gU * Qi - gQ * Ui)) / rr : 0.f;
          gbx = -kb * fmaf(xv, epx, yv * etx) + ki * fmaf(-xv, etx, yv * epx);
          gby = -kb * fmaf(xv, epy, yv * ety) + ki * fmaf(-xv, ety, yv * epy);
          gbz = -kb * (yv * etz) - ki * (xv * etz);
        }
        g_te = fma(gtt * bpar, P.fd_fore, g_te);
        g_bpar = gtt * te * P.fd_fore;
      }
      if (!(te_raw > 0.)) g_te = 0.;
      gbx += float(g_bpar * ux);
      gby += float(g_bpar * uy);
      gbz += float(g_bpar * uz);
      // analytic-model parameter gradients (form units; the host converts)
      if (in_b) {
        const double gdotb = (double)fmaf(gbx, bxr, gby * byr);
        gp[0] += gdotb;
        // B = amp (sin(pitch - phi), cos(pitch - phi)): dB/dpitch = (B_y, -B_x)
        gp[1] += (double)fmaf(gbx, byr, -gby * bxr);
        gp[2] += gdotb * fma(r, F.sp_irs, -F.sp_crs) * F.sp_irs;
        gp[3] += gdotb * fabs(pz) * F.sp_ihs * F.sp_ihs;
      }
      if (fast_t) {
        const double gt = g_te * te_d;
        gp[4] += gt;
        gp[5] += gt * r * F.ex_irn * F.ex_irn;
        gp[6] += gt * fabs(pz) * F.ex_ihn * F.ex_ihn;
      }
      // grid-record gradients, summed per cell
      if (NG == 1 && key != kNoCell && A.grad_rec != nullptr) {
        const DevGridGroup &G = P.groups[0];
        if (key != acc_key) {
          flush_cell32(A.grad_rec, acc_key, (unsigned)G.ny, (unsigned)G.nz, acc);
          acc_key = key;
        }
        const float wx[2] = {1.f - tx, tx}, wy[2] = {1.f - ty, ty}, wz[2] = {1.f - tz, tz};
        const float gt = float(g_te);
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
          for (int dy = 0; dy < 2; ++dy) {
            const float wxy = wx[dx] * wy[dy];
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
              const float w = wxy * wz[dz];
              const int k = dx * 4 + dy * 2 + dz;
              acc[k][0] = fmaf(w, gbx, acc[k][0]);
              acc[k][1] = fmaf(w, gby, acc[k][1]);
              acc[k][2] = fmaf(w, gbz, acc[k][2]);
              acc[k][3] = fmaf(w, gt, acc[k][3]);
            }
          }
      }
    }
    if (NG == 1 && A.grad_rec != nullptr)
      flush_cell32(A.grad_rec, acc_key, (unsigned)P.groups[0].ny, (unsigned)P.groups[0].nz,
                   acc);
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
