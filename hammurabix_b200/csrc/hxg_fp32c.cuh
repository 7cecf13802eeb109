// hxg_fp32c.cuh -- the FP32-compensated shell kernel.
//
// Precision split.  The Faraday depth n_e B_par is summed along the ray and
// its running value sets every later sample's rotation 2 lambda^2 FD, which
// reaches thousands of radians at 0.4 GHz.  A relative error rho in each
// sample's n_e B_par therefore random-walks into a phase error of about
// rho * phase / sqrt(samples); FP32 rounding of the analytic models (a few
// ulp per sample) alone costs ~1e-5 in Q/U there.  So everything that feeds
// n_e B_par is FP64 or exact:
//   - the ray (observer, LOS versor, sample distance), the grid coordinates
//     (64-bit fixed point stepped by integer adds, FixAxis), the cuts;
//   - the analytic regular field and n_e (FP64; the spiral and exponential
//     disk use a table-driven exp and a Newton-refined rsqrt, and the
//     spiral's B_par along the ray is amp/r * (K0 + K1 d) with per-ray K0,
//     K1);
//   - the grid field's B_par (its three FP32 values projected in FP64), the
//     product n_e B_par, the Faraday-depth and DM sums (FP64);
//   - the phase, reduced to a fraction of a turn with integer operations.
// FP32 carries the trilinear grid interpolation (FP32 voxel records, whose
// rounding is random from sample to sample), the synchrotron emissivity and
// polarisation angle, and the I, Q, U sums (FP32 over blocks of 16 samples,
// Kahan-compensated across blocks).
//
// Speed.  The kernel is bound by instruction issue (the grids stay in
// L1/L2), so the sample loop is cut to few instructions: in the
// instantiation for the grid workloads' models (kFast) a ray's window is
// trimmed to the samples that pass the cuts (no per-sample cut test), grid
// coordinates advance by 64-bit integer adds and split into cell and FP32
// fraction with shifts, model amplitudes sit in the exponents, the phase
// fraction comes from integer operations, the |B_perp|^2 emissivity (CRE
// index 3) needs no reciprocal and the CRE profile two base-2 exponentials.
#pragma once

#include "hxg_integrate.cuh"

// Launch shape of the one-pass shell kernel: threads per block and the
// resident blocks per SM its register allocation must allow.  128 x 7 (72
// registers, 28 warps per SM) ran the config-3 passes one by one in
// 172.7 ms against 176.2 ms at 128 x 6 (80 registers) and 181.7 ms at
// 128 x 8 (64; measured before the last two loop changes): more resident
// warps hide the FP64 and MUFU latencies better than the spills they cost.
#ifndef HXG_FP32C_THREADS
#define HXG_FP32C_THREADS 128
#endif
#ifndef HXG_FP32C_MIN_BLOCKS
#define HXG_FP32C_MIN_BLOCKS 7
#endif

namespace hxg {

// Cell index and fractional position along one axis from an FP64 grid
// coordinate g with 0 < g < n-1 < 2^19.  Adding 1.5 * 2^20 leaves floor(g)
// in the low 20 mantissa bits of the high word and frac(g) * 2^32, rounded,
// in the low word; the fraction is rounded to 23 bits into [0, 1].
__device__ __forceinline__ void cell_split(double g, int nmax2, int &cell,
                                           float &frac) {
  const double t = g + 1572864.0;
  const unsigned lo = (unsigned)__double2loint(t);
  const int hi = __double2hiint(t);
  cell = (hi & 0xFFFFF) - 0x80000;
  const unsigned long long r = ((unsigned long long)lo + 256ull) >> 9;
  frac = __uint_as_float(0x3F800000u + (unsigned)r) - 1.0f;
  if (cell > nmax2) {  // g within 2^-33 of n-1: stay in the last cell
    cell = nmax2;
    frac = 1.0f;
  }
}

// Trilinear sample of one FP32 record group at the cell (x, y, z) with
// fractions (fx, fy, fz): out[0..2] = B (2^-20 G), out[3] = n_e.  Each
// record is two (x, y) / (z, w) pairs, interpolated with paired-FP32 lerps
// a + t (b - a) along z, then y, then x (the reference's order, breg.cc:58-96):
// half the instructions of eight weighted sums and a smaller rounding error.
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t) {
  return __ffma2_rn(t, __ffma2_rn(a, make_float2(-1.f, -1.f), b), a);
}
__device__ __forceinline__ void trilinear_f32(const float4 *rec, int ny,
                                              int nz, int x, int y, int z,
                                              float fx, float fy, float fz,
                                              float out[4]) {
  // record indices fit 32 bits (the host refuses larger record arrays)
  const unsigned i00 = ((unsigned)x * (unsigned)ny + (unsigned)y) * (unsigned)nz + (unsigned)z;
  const float4 *p00 = rec + i00;
  const float4 *p01 = p00 + nz;
  const float4 *p10 = p00 + (unsigned)ny * (unsigned)nz;
  const float4 *p11 = p10 + nz;
  const float4 c000 = __ldg(p00), c001 = __ldg(p00 + 1);
  const float4 c010 = __ldg(p01), c011 = __ldg(p01 + 1);
  const float4 c100 = __ldg(p10), c101 = __ldg(p10 + 1);
  const float4 c110 = __ldg(p11), c111 = __ldg(p11 + 1);
  const float2 tz = make_float2(fz, fz), ty = make_float2(fy, fy), tx = make_float2(fx, fx);
  // along z: (x, y) and (z, w) halves of the four corner pairs
  float2 za[4], zb[4];
  const float4 *lo[4] = {&c000, &c010, &c100, &c110}, *hi[4] = {&c001, &c011, &c101, &c111};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    za[k] = lerp2(make_float2(lo[k]->x, lo[k]->y), make_float2(hi[k]->x, hi[k]->y), tz);
    zb[k] = lerp2(make_float2(lo[k]->z, lo[k]->w), make_float2(hi[k]->z, hi[k]->w), tz);
  }
  // along y, then x
  const float2 w1a = lerp2(za[0], za[1], ty), w1b = lerp2(zb[0], zb[1], ty);
  const float2 w2a = lerp2(za[2], za[3], ty), w2b = lerp2(zb[2], zb[3], ty);
  const float2 ra = lerp2(w1a, w2a, tx), rb = lerp2(w1b, w2b, tx);
  out[0] = ra.x;
  out[1] = ra.y;
  out[2] = rb.x;
  out[3] = rb.y;
}

// 2^(j/64) for j = 0..63, correctly rounded to FP64.
__device__ const double kExp2Tab64[64] = {
    1.0, 1.0108892860517005, 1.0218971486541166, 1.0330248790212284,
    1.0442737824274138, 1.0556451783605572, 1.0671404006768237, 1.0787607977571199,
    1.0905077326652577, 1.102382583307841, 1.1143867425958924, 1.1265216186082418,
    1.1387886347566916, 1.1511892299529827, 1.1637248587775775, 1.1763969916502812,
    1.189207115002721, 1.202156731452703, 1.215247359980469, 1.22848053610687,
    1.241857812073484, 1.255380757024691, 1.2690509571917332, 1.2828700160787783,
    1.2968395546510096, 1.3109612115247644, 1.3252366431597413, 1.339667524053303,
    1.3542555469368927, 1.3690024229745905, 1.383909881963832, 1.3989796725383112,
    1.4142135623730951, 1.42961333839197, 1.4451808069770467, 1.460917794180647,
    1.4768261459394993, 1.4929077282912648, 1.5091644275934228, 1.5255981507445384,
    1.5422108254079407, 1.559004400237837, 1.5759808451078865, 1.593142151342267,
    1.6104903319492543, 1.6280274218573478, 1.645755478153965, 1.6636765803267364,
    1.681792830507429, 1.7001063537185235, 1.718619298122478, 1.7373338352737062,
    1.7562521603732995, 1.7753764925265212, 1.7947090750031072, 1.8142521755003989,
    1.8340080864093424, 1.8539791250833855, 1.8741676341103, 1.8945759815869656,
    1.9152065613971474, 1.9360617934922943, 1.9571441241754002, 1.978456026387951,
};

// e^a for a < 700 (a below -700 is taken as -700) by table-driven range
// reduction (Tang, ACM TOMS 15, 1989): k = nearest integer of 64 a / ln2,
// r = a - k ln2/64 with |r| <= ln2/128, e^a = 2^(k >> 6) 2^((k & 63)/64) e^r,
// e^r from its Taylor series to degree 4 (truncation below 4e-14
// relative; the rounding of ln2/64 times k adds below 6e-14): a systematic
// error that moves the Faraday phase at 0.408 GHz, thousands of radians,
// by under 1e-9 rad.
__device__ __forceinline__ double exp_tab(double a) {
  const double kMagic = 6755399441055744.0;  // 1.5 * 2^52
  a = fmax(a, -700.);
  const double t = fma(a, 92.33248261689366, kMagic);   // 64 / ln2
  const int k = __double2loint(t);
  const double kd = t - kMagic;
  const double r = fma(-kd, 0.010830424696249145, a);   // ln2 / 64
  double p = 4.1666666666666664e-02;                    // 1/4!
  p = fma(p, r, 1.6666666666666666e-01);                // 1/3!
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  const double e = p * __ldg(&kExp2Tab64[k & 63]);
  return __hiloint2double(__double2hiint(e) + ((k >> 6) << 20), __double2loint(e));
}

// 1/sqrt(t) for t > 0: the FP64 hardware estimate (relative error below
// 2^-20, measured over 2^-30..2^30) refined by one Newton step, which
// squares that error: 1.3e-12 relative (measured), systematic, and under
// 1e-8 rad of Faraday phase at 0.408 GHz.
__device__ __forceinline__ double rsqrt_fd(double t) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(t));
  const double e = fma(-t * y, y, 1.0);
  return fma(0.5 * y, e, y);
}

// The samples [lo, hi) of the ray window (ray_window) that pass the cuts
// gc_r <= r_max, z_min <= z <= z_max (integrator.cc:179-182) with the
// per-sample test itself, evaluated at the ends: without an inner radius
// the passing samples of a ray are one contiguous run (a ball and a slab
// are convex), so the window shrinks from both ends to the first and the
// last passing sample and the samples between need no test.
__device__ __forceinline__ void exact_cut_window(const ShellLaunch &P, double uz, double ou2,
                                                 double oo, long long &lo, long long &hi) {
  const double oz = P.obs[2], r2max = P.fast.r2max;
  const auto pass = [&](long long i) {
    const double d = P.d_start + ((double)i + 0.5) * P.delta;
    const double pz = fma(uz, d, oz);
    const double r2 = fma(d, d + ou2, oo);
    return !(r2 > r2max || pz < P.gc_z_min || pz > P.gc_z_max);
  };
  while (lo < hi && !pass(lo)) ++lo;
  while (hi > lo && !pass(hi - 1)) --hi;
}

// Fixed-point grid coordinate of one axis along a ray.  The coordinate
// g(d) = (p(d) - min) (n - 1) / (max - min) (breg.cc:34-54) is linear in
// the sample index, so it is stepped by an integer add: a holds
// round(g * 2^44) - 1 of the current sample, s the step.  44 fraction bits
// keep the FP64 resolution of g for n - 1 < 2^19 (the drift over 2^12
// steps is below 1e-10 of a cell).  The cell is the integer part of a and
// the FP32 fraction the nearest FP32 to its leading 32 fraction bits, i.e.
// within half an FP32 ulp of the exact fraction; it may round up to 1, the
// next vertex, which is in the grid since the cell is below n - 1.  A ray
// along which a coordinate is constant (the equator, z = const) repeats
// the same rounding at every sample, so it adds up along the ray: the
// nearest FP32 keeps that error the smallest FP32 allows.
constexpr double kFix = 17592186044416.0;  // 2^44
struct FixAxis {
  long long a, s;
  __device__ __forceinline__ void start(double g, double step) {
    a = __double2ll_rn(g * kFix) - 1;
    s = __double2ll_rn(step * kFix);
  }
  // n: grid points on this axis (a launch constant).  The high word of a
  // alone decides: a >= 0 (0 < g) and a < (n - 1) 2^44, i.e. g <= n - 1;
  // g == n - 1 exactly -- a sample on the upper box face, where the
  // reference returns 0 -- then reads the face value (cell n - 2, fraction
  // 1), a case of measure zero that stays in bounds.
  __device__ __forceinline__ bool inside(int n) const {
    return (unsigned)(a >> 32) < ((unsigned)(n - 1) << 12);
  }
  __device__ __forceinline__ void split(int &cell, float &frac) const {
    const unsigned lo = (unsigned)a, hi = (unsigned)(a >> 32);
    cell = (int)hi >> 12;
    // the leading 32 fraction bits, rounded to the nearest FP32
    frac = __uint2float_rn(__funnelshift_r(lo, hi, 12)) * 0x1p-32f;
  }
  __device__ __forceinline__ void next() { a += s; }
};

// Sample range [ga, gb) of [i0, i1) in which the ray can be inside the grid
// box 0 < g < n - 1 on every axis (from the slab intersections in FP64,
// widened by two samples; the fixed-point test decides each sample).
__device__ __forceinline__ void grid_window(const ShellLaunch &P, const DevGridGroup &G,
                                            const double g0[3], const double gv[3],
                                            int i0, int i1, int &ga, int &gb) {
  double da = -1e300, db = 1e300;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (gv[k] != 0.) {
      const double t0 = -g0[k] / gv[k], t1 = (G.gmax[k] - g0[k]) / gv[k];
      da = fmax(da, fmin(t0, t1));
      db = fmin(db, fmax(t0, t1));
    } else if (!(g0[k] > 0. && g0[k] < G.gmax[k])) {
      db = -1e300;
    }
  }
  ga = i1;
  gb = i1;
  if (!(da <= db)) return;
  const double xa = (da - P.d_start) / P.delta - 0.5, xb = (db - P.d_start) / P.delta - 0.5;
  ga = (int)fmin(fmax(floor(xa) - 2., (double)i0), (double)i1);
  gb = (int)fmin(fmax(ceil(xb) + 3., (double)ga), (double)i1);
}

// 2^x in FP32 (the approximate hardware exponential, as __expf uses it).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// CRE_ana spatial profile exp((R0 - r)/r0) sech^2(z/z0) (cre_ana.cc:11-63)
// in FP32 at cylindrical radius rf and height zf (kpc):
//   = 2^(2 + (R0 - r) log2(e)/r0) t / (1 + t)^2, t = 2^(-2|z| log2(e)/z0).
__device__ __forceinline__ float cre_ana_prof32(const FastModels &F, float rf, float zf) {
  const float t = ex2_approx(-fabsf(zf) * F.cre_2iz0_l2);
  const float den = 1.f + t;
  return __fdividef(ex2_approx(fmaf(-rf, F.cre_ir0_l2, F.cre_R0_l2)) * t, den * den);
}

template <int NF>
__device__ __forceinline__ void combine_chunks_nf(const ShellLaunch &P, const FreqSet<NF> &Fq,
                                                  int c, double &dm, double &fd, double si[NF],
                                                  double sq[NF], double su[NF]) {
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
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    if (P.do_sync && c > 0) {
      double sr, cr;
      sincos(2. * Fq.lambda2[f] * excl, &sr, &cr);
      const double q = sq[f] * cr - su[f] * sr;
      const double u = sq[f] * sr + su[f] * cr;
      sq[f] = q;
      su[f] = u;
    }
  }
  for (int o = C >> 1; o > 0; o >>= 1) {
    dm += shfl_xor_d(dm, o);
    fd += shfl_xor_d(fd, o);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      si[f] += shfl_xor_d(si[f], o);
      sq[f] += shfl_xor_d(sq[f], o);
      su[f] += shfl_xor_d(su[f], o);
    }
  }
}

// Warp gw of shell launch P (32/C pixels, C lanes each) for the NF
// frequency passes of Fq.  All 32 lanes of the warp call it with the same gw.
// kFast: the launch's models are among B none/grid/spiral, n_e
// none/grid/exponential disk and CRE_ana with a constant index (the host
// checks, fast_models); the other models' paths are compiled out, so
// the registers are allocated for this path alone.
template <int NG, bool kExt, int NF, bool kFast = false>
__device__ __forceinline__ void fp32c_tile(const ShellLaunch &P, const FreqSet<NF> &Fq,
                                           long long gw, int lane) {
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
  double dm = 0., fd = 0., si[NF], sq[NF], su[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) si[f] = sq[f] = su[f] = 0.;
  if (live) {
    double th, ph;
    hpx_pix2ang(h, ring, th, ph);
    double inner = 0.;
    if (P.fdmap != nullptr) {
      const Hpx hf = hpx_make((uint64_t)P.nside_fdmap);
      inner = hpx_interpolate(hf, P.fdmap, th, ph);
    }
    if (NF == 1 && P.ck_inner != nullptr && c == 0) P.ck_inner[ring] = inner;
    const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
    const double ux = cp * st, uy = sp * st, uz = ct;
    const float etx = float(ct * cp), ety = float(ct * sp), etz = float(-st);
    const float epx = float(-sp), epy = float(cp);
    const double ox = P.obs[0], oy = P.obs[1], oz = P.obs[2];
    // |pos|^2 along the ray: |o|^2 + 2 (o.u) d + d^2
    const double ou2 = 2. * (ox * ux + oy * uy + oz * uz);
    const double oo = ox * ox + oy * oy + oz * oz;
    const double r2min = P.fast.r2min, r2max = P.fast.r2max;
    // Faraday phase in turns: rev0 + rev_k * (FD sum), per pass
    double rev0[NF], rev_k[NF];
    float a_s[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      // + 1.5 * 2^20: the low word of the sum then holds the fraction of a
      // turn in units of 2^-32; + 2^-24 rounds it to 2^-23 below
      rev0[f] = Fq.lambda2[f] * (Fq.inner[f] ? inner : 0.) * (1. / cgs::pi) +
                (1572864.0 + 0x1p-24);
      rev_k[f] = Fq.phase_k[f] * (0.5 / cgs::pi);
      a_s[f] = float(Fq.a_s[f]);
    }
    const DevModels &M = P.models;
    const FastModels &F = P.fast;
    const float pe = P.fast.pe;
    const bool pe2 = P.em_const && P.em_pe == 2.;

    // grid-space ray of group 0: g(d) = g0 + gv d
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
    // spiral B_par along the ray: amp/r * (K0 + K1 d)
    // kFast folds b0 into the exponent and its sign into the pitch terms
    const double ss = kFast ? F.sp_sin_s : F.sp_sin, cs = kFast ? F.sp_cos_s : F.sp_cos;
    const double K0 = ss * (ox * ux + oy * uy) + cs * (ox * uy - oy * ux);
    const double K1 = ss * (ux * ux + uy * uy);
    const float spf = kFast ? F.sp_sinf_s : F.sp_sinf, cpf = kFast ? F.sp_cosf_s : F.sp_cosf;
    // I is one sum for all passes when the emissivity weight is frequency
    // independent (constant index); Q, U always one sum per pass
    constexpr int NI = NF;
    BlockKahanF ki[NI], kq[NF], ku[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) ki[f] = kq[f] = ku[f] = BlockKahanF{0.f, KahanF{0.f, 0.f}};
    bool i_shared = true;
    double sfd = 0., sdm = 0.;
    const bool fast_b = M.breg == kBregSpiral;
    const bool slow_b = !kFast && M.breg != kBregNone && M.breg != kBregGrid && !fast_b;
    const bool fast_t = M.tereg == kTeregExpdisk;
    const bool slow_t = !kFast && M.tereg != kTeregNone && M.tereg != kTeregGrid && !fast_t;
    const double rc2_hi = F.rc2_hi, rc2_lo = F.rc2_lo;
    float last_index = __int_as_float(0x7fc00000), gt = float(P.em_gt),
          gp = float(P.em_gp), inv1mi = 1.f;
    long long wlo, whi, slo_unused, shi_unused;
    ray_window(P, ux, uy, uz, wlo, whi, slo_unused, shi_unused);
    // kFast: no inner radius, so the window is cut to the passing samples
    if (kFast) exact_cut_window(P, uz, ou2, oo, wlo, whi);
    // sample indices fit 32 bits (step < 2^31, checked on the host)
    const int i0 = (int)max((P.step * c) >> P.log2_chunks, wlo);
    const int i1 = (int)min((P.step * (c + 1)) >> P.log2_chunks, whi);
    double d = P.d_start + ((double)i0 + 0.5) * P.delta;
    // kFast, one grid group: fixed-point grid coordinates from sample ga on
    FixAxis fx, fy, fz;
    int ga = i1, gb = i1;
    if (kFast && NG == 1) {
      const DevGridGroup &G = P.groups[0];
      const double g0[3] = {g0x, g0y, g0z}, gv[3] = {gvx, gvy, gvz};
      grid_window(P, G, g0, gv, i0, i1, ga, gb);
      const double dg = P.d_start + ((double)ga + 0.5) * P.delta;
      fx.start(fma(gvx, dg, g0x), gvx * P.delta);
      fy.start(fma(gvy, dg, g0y), gvy * P.delta);
      fz.start(fma(gvz, dg, g0z), gvz * P.delta);
    }
    // blocks of 16 sample indices (aligned): the block sums fold into the
    // Kahan totals after each block
    for (int i = i0; i < i1;) {
     const int iend = min(i1, (i | 15) + 1);
     for (; i < iend; ++i, d += P.delta) {
      // the general instantiation tests every sample (an inner radius can
      // split a ray's passing samples in two runs)
      const double pz = fma(uz, d, oz);
      if (!kFast) {
        const double r2 = fma(d, d + ou2, oo);
        if (r2 < r2min || r2 > r2max || pz < P.gc_z_min || pz > P.gc_z_max) continue;
      }
      const double px = fma(ux, d, ox);
      const double py = fma(uy, d, oy);
      const double p3[3] = {px, py, pz};
      const float xf = float(px), yf = float(py), zf = float(pz);
      // FP64 analytic part of B_par and n_e; FP32 field for the synchrotron
      double bp_d = 0., te_d = 0.;
      float bxr = 0.f, byr = 0.f, bzr = 0.f;
      float rcf = 0.f;
      if (fast_b || fast_t) {
        const double rc2 = fma(px, px, py * py);
        // on the z axis r is 1e-150 instead of 0 (y finite; the spiral is
        // cut there)
        const double rc2m = fmax(rc2, 1e-300);
        const double y = rsqrt_fd(rc2m);
        const double r = rc2m * y;
        rcf = float(r);
        if (fast_b && !(rc2 > rc2_hi || rc2 < rc2_lo)) {
          // kFast: b0 exp(a) = sign(b0) exp(a + ln|b0|), the sign in ss, cs
          const double sarg =
              fma(-r, F.sp_irs, fma(-fabs(pz), F.sp_ihs, kFast ? F.sp_crs_l : F.sp_crs));
          const double ay = kFast ? exp_tab(sarg) * y : F.sp_b0 * exp_tab(sarg) * y;
          bp_d = ay * fma(K1, d, K0);
          const float ayf = float(ay);
          bxr = ayf * (spf * xf - cpf * yf);
          byr = ayf * (spf * yf + cpf * xf);
        }
        if (fast_t) {
          if (kFast)  // n0 exp(a) = exp(a + ln n0), n0 > 0
            te_d = exp_tab(fma(-r, F.ex_irn, fma(-fabs(pz), F.ex_ihn, F.ex_ln0)));
          else
            te_d = F.ex_n0 * exp_tab(-fma(r, F.ex_irn, fabs(pz) * F.ex_ihn));
        }
      }
      if (slow_b) {
        const V3<double> Br = breg_model_x<kExt>(M, P.ext, px, py, pz, p3);
        bp_d = fma(Br.x, ux, fma(Br.y, uy, Br.z * uz));
        bxr = float(Br.x);
        byr = float(Br.y);
        bzr = float(Br.z);
      }
      if (slow_t) te_d = tereg_model_x<kExt>(M, P.ext, px, py, pz, p3);
      float bg[4] = {0.f, 0.f, 0.f, 0.f};
      if (kFast && NG == 1) {
        const DevGridGroup &G = P.groups[0];
        if ((unsigned)(i - ga) < (unsigned)(gb - ga)) {
          if (fx.inside(G.nx) && fy.inside(G.ny) && fz.inside(G.nz)) {
            int cx, cy, cz;
            float tx, ty, tz;
            fx.split(cx, tx);
            fy.split(cy, ty);
            fz.split(cz, tz);
            trilinear_f32(reinterpret_cast<const float4 *>(G.rec), G.ny, G.nz, cx, cy, cz,
                          tx, ty, tz, bg);
          }
          fx.next();
          fy.next();
          fz.next();
        }
      } else if (NG == 1) {
        const DevGridGroup &G = P.groups[0];
        const double gx = fma(gvx, d, g0x), gy = fma(gvy, d, g0y), gz = fma(gvz, d, g0z);
        if (gx > 0. && gx < G.gmax[0] && gy > 0. && gy < G.gmax[1] && gz > 0. &&
            gz < G.gmax[2]) {
          int cx, cy, cz;
          float fx, fy, fz;
          cell_split(gx, G.nx - 2, cx, fx);
          cell_split(gy, G.ny - 2, cy, fy);
          cell_split(gz, G.nz - 2, cz, fz);
          trilinear_f32(reinterpret_cast<const float4 *>(G.rec), G.ny, G.nz, cx, cy, cz,
                        fx, fy, fz, bg);
        }
      } else if (NG > 1) {
        float b3[3] = {0.f, 0.f, 0.f};
        CellCache<float> cc;
#pragma unroll 1
        for (int g = 0; g < P.ngroups; ++g) {
          cc.key = -1;
          sample_group<float, false>(P.groups[g], px, py, pz, cc, b3, bg[3]);
        }
        bg[0] = b3[0];
        bg[1] = b3[1];
        bg[2] = b3[2];
      }
      // n_e (clamped at 0, integrator.cc:201) and n_e B_par in FP64
      const double te = fmax(te_d + double(bg[3]), 0.);
      // B_par of the FP32 grid field projected in FP64 (the versor exact)
      const double bpg = fma(double(bg[0]), ux, fma(double(bg[1]), uy, double(bg[2]) * uz));
      sdm += te;
      sfd = fma(te, bp_d + bpg, sfd);
      if (P.do_sync) {
        const float bx = bxr + bg[0], by = byr + bg[1], bz = bzr + bg[2];
        // B_perp on the sky basis: |B_perp|^2 = xv^2 + yv^2, and the IAU
        // angle has cos 2ipa = (xv^2 - yv^2) / |B_perp|^2 and
        // sin 2ipa = 2 xv yv / |B_perp|^2 (integrator.cc:257-265)
        const float xv = -(epx * bx + epy * by);
        const float yv = -(etx * bx + ety * by + etz * bz);
        const float rr = fmaf(xv, xv, yv * yv);
        const float cc2 = fmaf(xv, xv, -yv * yv), ss2 = 2.f * xv * yv;
        // emissivity weights: frequency independent (one set for all passes)
        // except the variable-index form, whose A depends on the frequency
        // through a_s; the host fuses no CRE-grid pass (its spectral
        // integral depends on the frequency), so that branch reads pass 0
        float wt[NF], wpc[NF], wps[NF];
        bool shared_w = true;
        if (kExt && M.cre == kCreGrid) {
          // spectral integral over the CRE grid in FP64 (integrator.cc:288-330,
          // 357-400); scaled by 2^128 into FP32 range, k_t = k_p undo it
          double jt, jp;
          cre_grid_j(P.ext->cre, px, py, pz, double(sqrtf(rr)), jt, jp);
          wt[0] = float(jt * 0x1p128);
          const float wp = float(jp * 0x1p128);
          const float inv = rr > 0.f ? __frcp_rn(rr) : 0.f;
          wpc[0] = rr > 0.f ? wp * cc2 * inv : wp;
          wps[0] = wp * ss2 * inv;
        } else {
          float prof;
          if (kFast || M.cre == kCreAna) {
            // exp((R0 - r)/r0) sech^2(z/z0)
            //   = 4 exp((R0 - r)/r0 - 2|z|/z0) / (1 + exp(-2|z|/z0))^2
            //   = 2^(2 + (R0 - r) log2(e)/r0) t / (1 + t)^2, t = 2^(-2|z| log2(e)/z0)
            float rf = rcf;
            if (!(fast_b || fast_t)) {
              const float r2f = fmaf(xf, xf, yf * yf);
              rf = r2f * rsqrtf(fmaxf(r2f, 1e-30f));
            }
            prof = cre_ana_prof32(F, rf, zf);
          } else {
            prof = cre_profile<float>(M, xf, yf, zf, p3);
          }
          if (pe2) {
            wt[0] = prof * rr;
            wpc[0] = prof * cc2;
            wps[0] = prof * ss2;
          } else {
            float wp[NF];
            if (kFast || P.em_const) {
              const float bp = (pe == 1.f) ? sqrtf(rr) : powf(rr, 0.5f * pe);
              wt[0] = wp[0] = prof * bp;
            } else {
              shared_w = false;
              const float index = cre_index<float>(M, xf, yf, zf);
              if (index != last_index) {
                gt = tgammaf(-0.25f * index + 19.f / 12.f) * tgammaf(-0.25f * index - 1.f / 12.f);
                gp = tgammaf(-0.25f * index + 7.f / 12.f) * tgammaf(-0.25f * index - 1.f / 12.f);
                inv1mi = 1.f / (1.f - index);
                last_index = index;
              }
              const float bper = sqrtf(rr);
#pragma unroll
              for (int f = 0; f < NF; ++f) {
                const float Ae = exp2f(0.5f * (index + 1.f) * log2f(a_s[f] / bper));
                const float base = prof * bper * Ae;
                wt[f] = base * gt * inv1mi;
                wp[f] = base * gp;
              }
            }
            // ipa of a zero B_perp is 0 (atan2(0, 0)): cos 2ipa = 1
            const float inv = rr > 0.f ? __frcp_rn(rr) : 0.f;
#pragma unroll
            for (int f = 0; f < (NF > 1 ? NF : 1); ++f) {
              if (f > 0 && shared_w) break;
              wpc[f] = rr > 0.f ? wp[f] * cc2 * inv : wp[f];
              wps[f] = wp[f] * ss2 * inv;
            }
          }
        }
        if (shared_w) {
#pragma unroll
          for (int f = 1; f < NF; ++f) {
            wt[f] = wt[0];
            wpc[f] = wpc[0];
            wps[f] = wps[0];
          }
          ki[0].add(wt[0]);
        } else {
#pragma unroll
          for (int f = 0; f < NF; ++f) ki[f].add(wt[f]);
        }
        i_shared = shared_w;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          // Faraday phase: the turn count rev0 + rev_k * FD in FP64, its
          // fraction rounded to 2^-23 turn in [-1/2, 1/2) with integer ops
          const double rev = fma(rev_k[f], sfd, rev0[f]);
          const int q = __double2loint(rev) >> 9;
          const float ang =
              (__int_as_float(0x4B400000 + q) - 12582912.0f) * 7.490140565847857e-07f;
          float sf, cf;
          __sincosf(ang, &sf, &cf);
          kq[f].add(fmaf(wpc[f], cf, -wps[f] * sf));
          ku[f].add(fmaf(wpc[f], sf, wps[f] * cf));
        }
      }
     }
#pragma unroll
     for (int f = 0; f < NF; ++f) {
       if (f == 0 || !i_shared) ki[f].flush();
       kq[f].flush();
       ku[f].flush();
     }
    }
    dm = sdm * P.k_dm;
    fd = sfd * P.fd_fore;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      si[f] = (i_shared ? ki[0] : ki[f]).value() * Fq.k_t[f];
      sq[f] = kq[f].value() * Fq.k_p[f];
      su[f] = ku[f].value() * Fq.k_p[f];
    }
  }
  // adjoint checkpoint (one pass): the chunk's FD and local-frame Q, U
  // before the chunk combination, in the FP64 form's units
  if (NF == 1 && P.ck != nullptr && live) {
    const unsigned long long ci = nest * (unsigned long long)C + c;
    P.ck[3 * ci] = fd;
    P.ck[3 * ci + 1] = sq[0];
    P.ck[3 * ci + 2] = su[0];
  }
  combine_chunks_nf<NF>(P, Fq, c, dm, fd, si, sq, su);
  if (live && c == 0) {
    if (P.do_dm) P.out[0][ring] = dm;
    if (P.do_fd || P.do_sync) P.out[1][ring] = fd;
    if (P.do_sync) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        Fq.out[f][0][ring] = si[f] * Fq.tc_a[f] * Fq.tc_a[f] / Fq.tc_b[f];
        Fq.out[f][1][ring] = sq[f] * Fq.tc_a[f] * Fq.tc_a[f] / Fq.tc_b[f];
        Fq.out[f][2][ring] = su[f] * Fq.tc_a[f] * Fq.tc_a[f] / Fq.tc_b[f];
      }
    }
  } else if (valid && !live && c == 0) {
    if (P.do_dm) P.out[0][ring] = 0.;
    if (P.do_fd || P.do_sync) P.out[1][ring] = 0.;
    if (P.do_sync) {
#pragma unroll
      for (int f = 0; f < NF; ++f) Fq.out[f][0][ring] = Fq.out[f][1][ring] = Fq.out[f][2][ring] = 0.;
    }
  }
}

// One frequency pass: the pass's constants from its launch block.
template <int NG, bool kExt, bool kFast = false>
__device__ __forceinline__ void fp32c_tile(const ShellLaunch &P, long long gw, int lane) {
  FreqSet<1> Fq;
  Fq.lambda2[0] = P.lambda2;
  Fq.phase_k[0] = P.phase_k;
  Fq.k_t[0] = P.k_t;
  Fq.k_p[0] = P.k_p;
  Fq.tc_a[0] = P.tc_a;
  Fq.tc_b[0] = P.tc_b;
  Fq.a_s[0] = P.a_s;
  Fq.inner[0] = 1;
  Fq.out[0][0] = P.out[2];
  Fq.out[0][1] = P.out[3];
  Fq.out[0][2] = P.out[4];
  fp32c_tile<NG, kExt, 1, kFast>(P, Fq, gw, lane);
}

template <int NG, bool kExt, bool kFast>
__global__ void __launch_bounds__(HXG_FP32C_THREADS, HXG_FP32C_MIN_BLOCKS)
shell_fp32c_kernel(const ShellLaunch P) {
  fp32c_tile<NG, kExt, kFast>(P, ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                       threadIdx.x & 31);
}

// NF frequency passes in one traversal of the shell (launch shape
// HXG_FP32C_MULTI_THREADS x HXG_FP32C_MULTI_MIN_BLOCKS: the per-pass Q/U
// sums and phase constants take registers).
template <int NG, bool kExt, int NF, bool kFast>
__global__ void __launch_bounds__(HXG_FP32C_MULTI_THREADS,
                                  kFast ? HXG_FP32C_MULTI_MIN_BLOCKS_FAST
                                        : HXG_FP32C_MULTI_MIN_BLOCKS)
shell_fp32c_multi_kernel(const ShellLaunch P, const FreqSet<NF> Fq) {
  fp32c_tile<NG, kExt, NF, kFast>(P, Fq, ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                           threadIdx.x & 31);
}

}  // namespace hxg
