// hxg_integrate.cuh -- shell integration kernels (the per-pixel radial loop
// of Integrator::radial_integration, source/integrator/integrator.cc:136-228,
// run for every pixel of one shell, integrator.cc:60-116).
//
// Mapping: each warp owns 32/C pixels of a compact NESTED sky patch (so
// neighbouring rays share grid cache lines) and C lanes split each pixel's
// radial range into contiguous chunks.  Chunk c integrates with the phase of
// its own partial Faraday depth; once the chunk sums are known, its Stokes
// Q/U are rotated by 2*lambda^2*(Faraday depth of the chunks before it) --
// algebraically identical to the reference's running phase
// (integrator.cc:221-225) -- and the chunks are reduced with warp shuffles.
// With C = 1 (large shells) each lane is one pixel in the reference's order.
#pragma once

#include "hxg_common.cuh"
#include "hxg_fields.cuh"

namespace hxg {

constexpr int kMaxGroups = 4;

// FP32C evaluation of the spiral B and exponential n_e models (FP64, kpc
// and 2^-20 G, reciprocals precomputed).
struct FastModels {
  double sp_b0, sp_irs, sp_crs, sp_ihs;  // amplitude, 1/r_s, r_sun/r_s, 1/h_s
  double sp_sin, sp_cos;                 // sin, cos of the pitch angle
  double ex_n0, ex_irn, ex_ihn;          // exp-disk n0, 1/r_s, 1/h_s
  // the kFast sample loop folds the amplitudes into the exponents:
  // r_sun/r_s + ln|b0| and ln n0, the sign of b0 into sp_*_s
  double sp_crs_l, ex_ln0;
  double sp_sin_s, sp_cos_s;             // sign(b0) sin, sign(b0) cos
  float sp_sinf_s, sp_cosf_s;            // the same in FP32
  // launch constants in the types the sample loop uses, so that the loop
  // reads them as operands instead of converting them
  double r2min, r2max;                   // gc_r_min^2, gc_r_max^2
  double rc2_hi, rc2_lo;                 // spiral cylinder: (20 kpc)^2, (3 kpc)^2
  float sp_sinf, sp_cosf;                // sp_sin, sp_cos
  float cre_ir0, cre_2iz0, cre_R0;       // CRE_ana: 1/r0, 2/z0, R0
  // the same for base-2 exponentials: log2(e)/r0, 2 log2(e)/z0 and
  // 2 + R0 log2(e)/r0 (the factor 4 of 4 e^x / (1 + t)^2 folded in)
  float cre_ir0_l2, cre_2iz0_l2, cre_R0_l2;
  float pe;                              // em_pe
};

// Everything one shell launch needs, in the working units of its form.
struct ShellLaunch {
  double obs[3];             // observer
  double d_start, delta;     // first-sample distance and radial step
  long long step;            // samples per ray (integrator.cc:237-240)
  double gc_r_min, gc_r_max, gc_z_min, gc_z_max;
  int nside, chunks, log2_chunks;
  // shard `shard` of `nshards` of the shell: the NESTED blocks of
  // 2^shard_log2 pixels b with b % nshards == shard (interleaved over the
  // sky, so that the shards see the same mix of ray lengths; a block is a
  // compact sky patch); 0 of 1 for the whole shell
  unsigned shard, nshards, shard_log2;
  int do_dm, do_fd, do_sync;
  const double *fdmap;       // accumulated FD map of inner shells (or null)
  int nside_fdmap;
  const unsigned char *mask; // 1 = integrate (integrator.cc:69-70), or null
  double *out[5];            // shell maps (RING): dm, fd, is, qs, us
  // FD and synchrotron constants
  double fd_fore;            // FP64: -qe^3/(2 pi mec2^2); FP32C: that * delta * 2^-20 G
  double lambda2;            // (c/nu)^2
  double i2bt;               // c^2 / (2 kB nu^2)
  double tc_a, tc_b;         // temp_convert(t) = t*a*a/b (integrator.cc:275-279)
  // analytic synchrotron emissivity (integrator.cc:332-346, 401-415)
  int em_const;              // spectral index constant over space
  int em_pow_kind;           // 0: pow(); 1: exponent == -1; 2: exponent == 0
  double em_index;           // constant index
  double em_n0u;             // j0 * gamma0^-index(observer) * unit
  double em_qe3, em_den_t, em_den_p, em_anum, em_3qe;
  double em_gt, em_gp;       // Gamma products at the constant index
  // FP32C scales (applied in FP64 after the sums)
  double k_t, k_p, k_dm;     // I, Q/U and DM scale factors
  double phase_k;            // 2 lambda^2 * fd_fore (per FP64 FD-sum unit)
  double a_s;                // A * |B_perp| in 2^-20 G (variable-index path)
  double em_pe;              // exponent of |B_perp| (constant index, FP32C)
  DevModels models;
  DevGridGroup groups[kMaxGroups];
  int ngroups;
  // adjoint checkpoint (FP64 form): per (pixel, chunk) the chunk's FD, Q, U
  // before the chunk combination, per pixel the inner-shell FD; null = off
  double *ck;
  double *ck_inner;
  FastModels fast;  // FP32C only
  const ExtModels *ext;  // Jaffe / JF12 / YMW16 blocks (device), or null
};

// The models of the grid workloads: B none, grid or spiral; n_e none, grid
// or exponential disk; CRE_ana with a constant index; no inner radius cut
// (gc_r_min = 0, so that the samples of a ray that pass the cuts are one
// contiguous run).  The shell kernels have an instantiation (kFast) for
// launches whose models are among these, with the other models' paths
// compiled out, so that its registers are allocated for this path alone.
__host__ __device__ inline bool fast_models(const ShellLaunch &P) {
  const DevModels &M = P.models;
  return P.ext == nullptr && !(P.gc_r_min > 0.) &&
         // amplitudes folded into the exponents as logarithms (FastModels)
         (M.breg != kBregSpiral || M.sp_b0 != 0.) &&
         (M.tereg != kTeregExpdisk || M.tex_n0 > 0.) &&
         (M.breg == kBregNone || M.breg == kBregGrid || M.breg == kBregSpiral) &&
         (M.tereg == kTeregNone || M.tereg == kTeregGrid || M.tereg == kTeregExpdisk) &&
         (!P.do_sync || (M.cre == kCreAna && P.em_const));
}

// The frequency-dependent constants of NF frequency passes that share one
// shell traversal (same observer, shells, limits and models): each pass's
// phase scale, emissivity scales, temp_convert and I/Q/U shell maps.  The
// positions, field samples, emissivity weights, DM and FD of a sample do not
// depend on the frequency and are computed once for all NF passes.
// Launch shape of the fused-frequency shell kernel: threads per block and
// the resident blocks per SM its register budget is cut for.  128 x 5
// (96 registers) keeps 20 warps per SM; for the general instantiation it ran
// config 3 in 91.3 ms against 92.8 ms at 256 x 2 (128 registers) and
// 97.2 ms at 128 x 6 (80 registers, more spills).  The kFast instantiation
// runs 128 x 7 (72 registers, 28 warps): config 3's fused step 59.1 ms
// against 59.5 ms at 128 x 5, 59.7 ms at 128 x 6, 61.3 ms at 128 x 8 and
// 68.5 ms at 128 x 9 (the spills grow with each step).
#ifndef HXG_FP32C_MULTI_THREADS
#define HXG_FP32C_MULTI_THREADS 128
#endif
#ifndef HXG_FP32C_MULTI_MIN_BLOCKS_FAST
#define HXG_FP32C_MULTI_MIN_BLOCKS_FAST 7
#endif
#ifndef HXG_FP32C_MULTI_MIN_BLOCKS
#define HXG_FP32C_MULTI_MIN_BLOCKS 5
#endif

template <int NF>
struct FreqSet {
  double lambda2[NF];   // (c/nu)^2
  double phase_k[NF];   // 2 lambda^2 * fd_fore (per FP64 FD-sum unit)
  double k_t[NF], k_p[NF];
  double tc_a[NF], tc_b[NF];
  double a_s[NF];       // A * |B_perp| scale of the variable-index emissivity
  int inner[NF];        // 1: the pass reads the inner-shell FD (its do_fd)
  double *out[NF][3];   // I, Q, U shell maps
};

// NESTED index of the shard's local pixel `local`: local pixels run through
// the shard's blocks in order.
__device__ __forceinline__ unsigned long long shard_nest(const ShellLaunch &P,
                                                         unsigned long long local) {
  if (P.nshards == 1) return local;
  const unsigned L = P.shard_log2;
  return (((local >> L) * P.nshards + P.shard) << L) + (local & ((1ull << L) - 1));
}

// Sample window [lo, hi) of one ray: the samples that can pass the
// spherical |pos| <= r_max and vertical z_min <= z <= z_max cuts
// (integrator.cc:179-182), from the roots of |o + u d|^2 = r_max^2 and
// o_z + u_z d = z_min / z_max, widened by two samples on each side.  Samples
// outside the window fail the cuts; the samples of [slo, shi) lie two or
// more steps inside it and pass them for certain, the others inside the
// window are tested exactly, so the result is the per-sample test's.
__device__ __forceinline__ void ray_window(const ShellLaunch &P, double ux,
                                           double uy, double uz,
                                           long long &lo, long long &hi,
                                           long long &slo, long long &shi) {
  const double ox = P.obs[0], oy = P.obs[1], oz = P.obs[2];
  const double b = ox * ux + oy * uy + oz * uz;  // o.u
  const double c = (ox * ox + oy * oy + oz * oz) - P.gc_r_max * P.gc_r_max;
  const double disc = b * b - c;
  lo = 0;
  hi = 0;
  slo = 0;
  shi = 0;
  if (!(disc >= 0.)) return;  // the ray misses the r_max sphere
  const double sq = sqrt(disc);
  double da = -b - sq, db = -b + sq;
  if (uz > 0.) {
    da = fmax(da, (P.gc_z_min - oz) / uz);
    db = fmin(db, (P.gc_z_max - oz) / uz);
  } else if (uz < 0.) {
    da = fmax(da, (P.gc_z_max - oz) / uz);
    db = fmin(db, (P.gc_z_min - oz) / uz);
  } else if (oz < P.gc_z_min || oz > P.gc_z_max) {
    return;
  }
  if (!(da <= db)) return;
  // d_i = d_start + (i + 1/2) delta
  const double n = (double)P.step;
  const double xa = (da - P.d_start) / P.delta - 0.5, xb = (db - P.d_start) / P.delta - 0.5;
  const double fa = fmin(fmax(floor(xa) - 2., 0.), n);
  const double fb = fmin(fmax(ceil(xb) + 3., 0.), n);
  lo = (long long)fa;
  hi = (long long)fb;
  // samples two or more steps inside both ends pass the cuts for certain
  // (the rounding of da, db and of the sample positions is ~1e-12 of a
  // step); with an inner radius the ray may cross the r_min ball, so every
  // sample is tested
  if (!(P.gc_r_min > 0.)) {
    slo = (long long)fmin(fmax(ceil(xa) + 2., 0.), n);
    shi = (long long)fmin(fmax(floor(xb) - 1., 0.), n);
  }
}

// Kahan-compensated FP32 accumulator.
struct KahanF {
  float s, c;
  __device__ __forceinline__ void add(float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const {
    return double(s) - double(c);
  }
};

// Two-level FP32 sum: a plain running sum over a block of samples, folded
// into a Kahan-compensated total by flush() (the caller flushes every 16
// sample indices).  The block sums' rounding (a few ulp of at most 16
// terms) is random from block to block, and the total is compensated.
struct BlockKahanF {
  float acc;
  KahanF tot;
  __device__ __forceinline__ void add(float v) { acc += v; }
  __device__ __forceinline__ void flush() {
    tot.add(acc);
    acc = 0.f;
  }
  __device__ __forceinline__ double value() const {
    KahanF t = tot;
    t.add(acc);
    return t.value();
  }
};

__device__ __forceinline__ double shfl_xor_d(double v, int o) {
  return __shfl_xor_sync(0xffffffffu, v, o);
}

// Combine the C chunk partial sums of each pixel: exclusive FD prefix over
// the chunks, rotation of each chunk's Q/U by 2*lambda^2*prefix, butterfly
// reduction inside the C-lane segment.  All 32 lanes participate.
__device__ __forceinline__ void combine_chunks(const ShellLaunch &P, int c,
                                               double rot_k, double &dm,
                                               double &fd, double &si,
                                               double &sq, double &su) {
  const int C = P.chunks;
  if (C == 1) return;
  // inclusive scan of fd within the segment
  double incl = fd;
  for (int o = 1; o < C; o <<= 1) {
    const double v = __shfl_up_sync(0xffffffffu, incl, o);
    if (c >= o) incl += v;
  }
  double excl = __shfl_up_sync(0xffffffffu, incl, 1);
  if (c == 0) excl = 0.;
  if (P.do_sync && c > 0) {
    double sr, cr;
    sincos(rot_k * excl, &sr, &cr);
    const double q = sq * cr - su * sr;
    const double u = sq * sr + su * cr;
    sq = q;
    su = u;
  }
  for (int o = C >> 1; o > 0; o >>= 1) {
    dm += shfl_xor_d(dm, o);
    fd += shfl_xor_d(fd, o);
    si += shfl_xor_d(si, o);
    sq += shfl_xor_d(sq, o);
    su += shfl_xor_d(su, o);
  }
}

// cos(2*ipa), sin(2*ipa) of the IAU polarisation angle
// ipa = atan2(-e_theta.B, -e_phi.B) (integrator.cc:257-265), from the
// double-angle identities (no atan2).
template <typename T>
__device__ __forceinline__ void ipa2(T xv, T yv, T &c2, T &s2) {
  const T r2 = xv * xv + yv * yv;
  if (r2 > T(0)) {
    const T inv = T(1) / r2;
    c2 = (xv * xv - yv * yv) * inv;
    s2 = T(2) * xv * yv * inv;
  } else {
    c2 = T(1);
    s2 = T(0);
  }
}

// ===================================================================
// FP64 parity form
// ===================================================================
// Warp gw of shell launch P (32/C pixels, C lanes each).  All 32 lanes of
// the warp call it with the same gw.  kFast: the launch's models satisfy
// fast_models (the same arithmetic, the other models compiled out).
template <int NG, bool kCache, bool kExt, bool kFast = false>
__device__ __forceinline__ void fp64_tile(const ShellLaunch &P, long long gw,
                                          int lane) {
  const int C = P.chunks;
  const int seg = lane >> P.log2_chunks;
  const int c = lane & (C - 1);
  const Hpx h = hpx_make((uint64_t)P.nside);
  const unsigned long long nest =
      shard_nest(P, (unsigned long long)gw * (32 >> P.log2_chunks) + seg);
  const bool valid = nest < h.npix;
  uint64_t ring = 0;
  bool live = false;
  if (valid) {
    ring = hpx_nest2ring(h, nest);
    live = (P.mask == nullptr) || (P.mask[ring] != 0);
  }
  double dm = 0., fd = 0., si = 0., sq = 0., su = 0.;
  const double rot_k = 2. * P.lambda2;
  if (live) {
    double th, ph;
    hpx_pix2ang(h, ring, th, ph);
    double inner = 0.;
    if (P.fdmap != nullptr) {
      const Hpx hf = hpx_make((uint64_t)P.nside_fdmap);
      inner = hpx_interpolate(hf, P.fdmap, th, ph);
    }
    if (P.ck_inner != nullptr && c == 0) P.ck_inner[ring] = inner;
    const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
    // los_versor (integrator.cc:268-272)
    const double ux = cp * st, uy = sp * st, uz = ct;
    // spherical unit vectors of sync_ipa (integrator.cc:260-262)
    const double etx = ct * cp, ety = ct * sp, etz = -st;
    const double epx = -sp, epy = cp;
    const DevModels &M = P.models;
    CellCache<double> cache;
    cache.key = -1;
    double last_index = nan(""), gt = P.em_gt, gp = P.em_gp;
    long long wlo, whi, slo, shi;
    ray_window(P, ux, uy, uz, wlo, whi, slo, shi);
    const long long i0 = max((P.step * c) >> P.log2_chunks, wlo);
    const long long i1 = min((P.step * (c + 1)) >> P.log2_chunks, whi);
    for (long long i = i0; i < i1; ++i) {
      const double d = P.d_start + ((double)i + 0.5) * P.delta;
      const double px = ux * d + P.obs[0];
      const double py = uy * d + P.obs[1];
      const double pz = uz * d + P.obs[2];
      if (i < slo || i >= shi) {
        const double len = sqrt(px * px + py * py + pz * pz);
        if (len < P.gc_r_min || len > P.gc_r_max || pz < P.gc_z_min ||
            pz > P.gc_z_max)
          continue;
      }
      const double p3[3] = {px, py, pz};
      V3<double> B{0., 0., 0.};
      double te = 0.;
      if (kFast) {
        if (M.breg == kBregSpiral) B = breg_spiral<double>(M, px, py, pz, p3);
        if (M.tereg == kTeregExpdisk) te = tereg_expdisk<double>(M, px, py, pz);
      } else {
        B = breg_model_x<kExt>(M, P.ext, px, py, pz, p3);
        te = tereg_model_x<kExt>(M, P.ext, px, py, pz, p3);
      }
      if (NG > 0) {
        double b3[3] = {B.x, B.y, B.z};
#pragma unroll 1
        for (int g = 0; g < (NG == 1 ? 1 : P.ngroups); ++g)
          sample_group<double, kCache>(P.groups[g], px, py, pz, cache, b3, te);
        B.x = b3[0];
        B.y = b3[1];
        B.z = b3[2];
      }
      te *= (double)(te > 0.);
      const double bpar = B.x * ux + B.y * uy + B.z * uz;
      const double cx = B.y * uz - B.z * uy;
      const double cy = B.z * ux - B.x * uz;
      const double cz = B.x * uy - B.y * ux;
      const double bper = sqrt(cx * cx + cy * cy + cz * cz);
      if (P.do_dm) dm += te * P.delta;
      if (P.do_fd || P.do_sync) fd += te * bpar * P.fd_fore * P.delta;
      if (P.do_sync) {
        double jtot, jpol;
        if (kExt && M.cre == kCreGrid) {
          // spectral integral over the CRE grid (integrator.cc:288-330, 357-400)
          double jt, jp;
          cre_grid_j(P.ext->cre, px, py, pz, bper, jt, jp);
          jtot = jt * P.delta * P.i2bt;
          jpol = jp * P.delta * P.i2bt;
        } else {
          double index = P.em_index;
          if (!kFast && !P.em_const) {
            index = cre_index<double>(M, px, py, pz);
            if (index != last_index) {
              gt = tgamma(-0.25 * index + 19. / 12.) * tgamma(-0.25 * index - 1. / 12.);
              gp = tgamma(-0.25 * index + 7. / 12.) * tgamma(-0.25 * index - 1. / 12.);
              last_index = index;
            }
          }
          const double fn = P.em_n0u * (kFast ? cre_profile_ana<double>(M, px, py, pz)
                                              : cre_profile<double>(M, px, py, pz, p3));
          const double absb = fabs(bper);
          const double A = P.em_anum / (P.em_3qe * absb);
          double Ae;
          if (P.em_const && P.em_pow_kind == 1)
            Ae = 1. / A;
          else if (P.em_const && P.em_pow_kind == 2)
            Ae = 1.;
          else
            Ae = pow(A, 0.5 * (index + 1));
          const double den_t = P.em_const ? P.em_den_t
                                          : 4. * cgs::pi * cgs::mec2 * (1. - index);
          const double norm_t = fn * 1.73205081 * P.em_qe3 * absb / den_t;
          const double norm_p = fn * 1.73205081 * P.em_qe3 * absb / P.em_den_p;
          jtot = norm_t * (Ae * gt) * P.delta * P.i2bt;
          jpol = norm_p * (Ae * gp) * P.delta * P.i2bt;
        }
        si += jtot;
        double c2, s2;
        ipa2<double>(-(epx * B.x + epy * B.y), -(etx * B.x + ety * B.y + etz * B.z),
                     c2, s2);
        double sf, cf;
        sincos(2. * ((inner + fd) * P.lambda2), &sf, &cf);
        sq += (cf * c2 - sf * s2) * jpol;
        su += (sf * c2 + cf * s2) * jpol;
      }
    }
  }
  if (P.ck != nullptr && live) {
    const unsigned long long ci = nest * (unsigned long long)C + c;
    P.ck[3 * ci] = fd;
    P.ck[3 * ci + 1] = sq;
    P.ck[3 * ci + 2] = su;
  }
  combine_chunks(P, c, rot_k, dm, fd, si, sq, su);
  if (live && c == 0) {
    if (P.do_dm) P.out[0][ring] = dm;
    if (P.do_fd || P.do_sync) P.out[1][ring] = fd;
    if (P.do_sync) {
      P.out[2][ring] = si * P.tc_a * P.tc_a / P.tc_b;
      P.out[3][ring] = sq * P.tc_a * P.tc_a / P.tc_b;
      P.out[4][ring] = su * P.tc_a * P.tc_a / P.tc_b;
    }
  } else if (valid && !live && c == 0) {
    // masked pixel: every observable is zero (integrator.cc:63-67, 98-115)
    if (P.do_dm) P.out[0][ring] = 0.;
    if (P.do_fd || P.do_sync) P.out[1][ring] = 0.;
    if (P.do_sync) P.out[2][ring] = P.out[3][ring] = P.out[4][ring] = 0.;
  }
}

// Launch shape of the FP64 shell kernel: threads per block and the resident
// blocks per SM its register allocation must allow.  128 x 7 (72
// registers, 28 warps per SM) ran the config-3 FP64 passes in 490.6 ms
// against 492.7 ms at 128 x 6, 494.0 ms at 256 x 3, 499.5 ms at 256 x 4,
// 513 ms at 128 x 5, 566 ms at 128 x 4 and 574 ms with the compiler's own
// choice at 256 threads (104 registers, 16 warps).
#ifndef HXG_FP64_THREADS
#define HXG_FP64_THREADS 128
#endif
#ifndef HXG_FP64_MIN_BLOCKS
#define HXG_FP64_MIN_BLOCKS 7
#endif

template <int NG, bool kCache, bool kExt, bool kFast = false>
__global__ void __launch_bounds__(HXG_FP64_THREADS, HXG_FP64_MIN_BLOCKS)
shell_fp64_kernel(const ShellLaunch P) {
  fp64_tile<NG, kCache, kExt, kFast>(P, ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                              threadIdx.x & 31);
}

}  // namespace hxg
