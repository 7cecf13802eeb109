// hxg_fields.cuh -- device field models and grid sampling of the
// line-of-sight integrator.
//
// Models are written once, templated on the working type T.  The FP64 form
// evaluates them in CGS (the reference's own units and operation order);
// the FP32 form evaluates them in kpc / 2^-20 G / cm^-3 so that no
// intermediate under- or overflows FP32.  All parameters arrive in a
// DevModels block already converted to the form's working units.
#pragma once

#include "hxg_common.cuh"
#include "hxg_models_ext.cuh"

namespace hxg {

enum : int {
  kBregNone = 0, kBregGrid = 1, kBregLsa = 2, kBregUnif = 3, kBregCart = 4,
  kBregHelix = 5, kBregJaffe = 6, kBregJf12 = 7, kBregSpiral = 8
};
enum : int {
  kTeregNone = 0, kTeregGrid = 1, kTeregUnif = 2, kTeregYmw16 = 3,
  kTeregExpdisk = 4
};
enum : int { kCreNone = 0, kCreAna = 1, kCreUnif = 2, kCreGrid = 3 };

// Model parameters in the working units of one precision form.
struct DevModels {
  int breg, tereg, cre, cre_const_index;
  double kpc;       // one kpc in working length units
  double obs[3];    // observer position (working length units)
  // Breg_lsa (source/field/b/breg_lsa.cc:9-26)
  double lsa_b0, lsa_psi0, lsa_psi1, lsa_chi0;
  // Breg_unif / Breg_cart: constant vector (breg_unif.cc:7-12, breg_cart.cc:7-11)
  double const_b[3];
  // Breg_helix (breg_helix.cc:13-30)
  double hx_bx, hx_by, hx_bz, hx_rmin, hx_rmax;
  // exponential-disk logarithmic spiral (include/hxg.h)
  double sp_b0, sp_sin, sp_cos, sp_rsun, sp_rs, sp_hs;
  // TEreg_unif (source/field/te/tereg_unif.cc:6-12)
  double teu_n0, teu_r0;
  // exponential electron disk (include/hxg.h)
  double tex_n0, tex_rs, tex_hs;
  // CRE_ana / CRE_unif (source/field/cre/cre_ana.cc, cre_unif.cc)
  double cre_alpha, cre_beta, cre_theta, cre_r0, cre_z0, cre_R0, cre_unif_r0;
};

template <typename T>
struct V3 {
  T x, y, z;
};

// Discontinuity decisions of the models.  The FP64 form takes them exactly
// as the reference does; the FP32 form takes them on the FP64 position p so
// that a sample next to a cutoff lands on the same side as in FP64.
template <typename T>
__device__ __forceinline__ bool outside_annulus(T r, const double p[3],
                                                double kpc, double lo_kpc,
                                                double hi_kpc) {
  if (sizeof(T) == 8) return r > (T(hi_kpc) * T(kpc)) || r < (T(lo_kpc) * T(kpc));
  const double r2 = p[0] * p[0] + p[1] * p[1];
  const double hi = hi_kpc * kpc, lo = lo_kpc * kpc;
  return r2 > hi * hi || r2 < lo * lo;
}

// |pos - observer| > r0 (tereg_unif.cc:8, cre_unif.cc:16)
template <typename T>
__device__ __forceinline__ bool beyond_observer(T x, T y, T z,
                                                const double p[3],
                                                const DevModels &m, double r0) {
  if (sizeof(T) == 8) {
    const T dx = x - T(m.obs[0]), dy = y - T(m.obs[1]), dz = z - T(m.obs[2]);
    return sqrt(dx * dx + dy * dy + dz * dz) > T(r0);
  }
  const double dx = p[0] - m.obs[0], dy = p[1] - m.obs[1], dz = p[2] - m.obs[2];
  return r0 < 0. || dx * dx + dy * dy + dz * dz > r0 * r0;
}

// ---- regular magnetic field models (Breg::write_field overrides) ---------
// The exponential-disk logarithmic spiral of the grid workloads (no
// reference class: amplitude b0 exp(-(r - r_sun)/r_s) exp(-|z|/h_s), pitch
// angle p, zero outside 3 kpc < r < 20 kpc).
template <typename T>
__device__ __forceinline__ V3<T> breg_spiral(const DevModels &m, T x, T y, T z,
                                             const double p[3]) {
  V3<T> b{T(0), T(0), T(0)};
  const T r = sqrt(x * x + y * y);
  if (outside_annulus<T>(r, p, m.kpc, 3., 20.)) return b;
  const T cos_p = x / r, sin_p = y / r;
  const T amp = T(m.sp_b0) * exp(-(r - T(m.sp_rsun)) / T(m.sp_rs)) *
                exp(-fabs(z) / T(m.sp_hs));
  const T sp = T(m.sp_sin), cp = T(m.sp_cos);
  b.x = amp * (sp * cos_p - cp * sin_p);
  b.y = amp * (sp * sin_p + cp * cos_p);
  return b;
}

template <typename T>
__device__ __forceinline__ V3<T> breg_model(const DevModels &m, T x, T y,
                                            T z, const double p[3]) {
  V3<T> b{T(0), T(0), T(0)};
  switch (m.breg) {
    case kBregLsa: {  // breg_lsa.cc:9-26
      const T kpc = T(m.kpc);
      const T r = sqrt(x * x + y * y);
      if (outside_annulus<T>(r, p, m.kpc, 3., 20.)) return b;
      const T cos_p = x / r, sin_p = y / r;
      const T psi = T(m.lsa_psi0) + T(m.lsa_psi1) * log(r / (T(8.) * kpc));
      const T chi = T(m.lsa_chi0) * tanh(z / (T(1.) * kpc));
      const T b0 = T(m.lsa_b0);
      const T sps = sin(psi), cps = cos(psi), cch = cos(chi);
      b.x = b0 * (sps * cch * cos_p - cps * cch * sin_p);
      b.y = b0 * (sps * cch * sin_p + cps * cch * cos_p);
      b.z = b0 * sin(chi);
      return b;
    }
    case kBregUnif:
    case kBregCart:
      b.x = T(m.const_b[0]);
      b.y = T(m.const_b[1]);
      b.z = T(m.const_b[2]);
      return b;
    case kBregHelix: {  // breg_helix.cc:13-30
      const T r = sqrt(x * x + y * y);
      const T phi = atan2(y, x) + T(cgs::pi / 2.0);
      bool inside;
      if (sizeof(T) == 8) {
        inside = (r > T(m.hx_rmin)) && (r < T(m.hx_rmax));
      } else {
        const double r2 = p[0] * p[0] + p[1] * p[1];
        inside = (m.hx_rmin < 0. || r2 > m.hx_rmin * m.hx_rmin) &&
                 (m.hx_rmax > 0. && r2 < m.hx_rmax * m.hx_rmax);
      }
      if (inside) {
        b.x = T(m.hx_bx) * cos(phi);
        b.y = T(m.hx_by) * sin(phi);
        b.z = T(m.hx_bz);
      }
      return b;
    }
    case kBregSpiral:
      return breg_spiral<T>(m, x, y, z, p);
    default:
      return b;
  }
}

// ---- regular thermal-electron models (TEreg::write_field overrides) ------
// Exponential disk of the grid workloads (no reference class):
// n0 exp(-r/r_s) exp(-|z|/h_s).
template <typename T>
__device__ __forceinline__ T tereg_expdisk(const DevModels &m, T x, T y, T z) {
  const T r = sqrt(x * x + y * y);
  return T(m.tex_n0) * exp(-r / T(m.tex_rs)) * exp(-fabs(z) / T(m.tex_hs));
}

template <typename T>
__device__ __forceinline__ T tereg_model(const DevModels &m, T x, T y, T z,
                                        const double p[3]) {
  switch (m.tereg) {
    case kTeregUnif:  // tereg_unif.cc:6-12
      return beyond_observer<T>(x, y, z, p, m, m.teu_r0) ? T(0) : T(m.teu_n0);
    case kTeregExpdisk:
      return tereg_expdisk<T>(m, x, y, z);
    default:
      return T(0);
  }
}

// Regular B and n_e including the models of hxg_models_ext.cuh (FP64).
// kExt = false instantiations compile to breg_model / tereg_model alone.
template <bool kExt>
__device__ __forceinline__ V3<double> breg_model_x(const DevModels &m, const ExtModels *ext,
                                                   double x, double y, double z,
                                                   const double p[3]) {
  if (kExt && (m.breg == kBregJaffe || m.breg == kBregJf12)) {
    double bb[3];
    if (m.breg == kBregJaffe)
      breg_jaffe(ext->jaffe, x, y, z, bb);
    else
      breg_jf12(ext->jf12, x, y, z, bb);
    return V3<double>{bb[0], bb[1], bb[2]};
  }
  return breg_model<double>(m, x, y, z, p);
}

template <bool kExt>
__device__ __forceinline__ double tereg_model_x(const DevModels &m, const ExtModels *ext,
                                                double x, double y, double z,
                                                const double p[3]) {
  if (kExt && m.tereg == kTeregYmw16) return tereg_ymw16(ext->ymw16, x, y, z);
  return tereg_model<double>(m, x, y, z, p);
}

// ---- CRE spectral index and spatial profile (cre_ana.cc:11-37,
//      cre_unif.cc:11-26) -------------------------------------------------
template <typename T>
__device__ __forceinline__ T cre_index(const DevModels &m, T x, T y, T z) {
  if (m.cre == kCreAna) {
    const T r = sqrt(x * x + y * y) / T(m.kpc);
    const T az = fabs(z) / T(m.kpc);
    return -T(m.cre_alpha) + T(m.cre_beta) * r + T(m.cre_theta) * az;
  }
  return -T(m.cre_alpha);
}

template <typename T>
__device__ __forceinline__ T cre_profile_ana(const DevModels &m, T x, T y, T z) {
  const T r = sqrt(x * x + y * y);
  const T ch = cosh(z / T(m.cre_z0));
  return exp((T(m.cre_R0) - r) / T(m.cre_r0)) * (T(1.) / (ch * ch));
}

template <typename T>
__device__ __forceinline__ T cre_profile(const DevModels &m, T x, T y, T z,
                                        const double p[3]) {
  if (m.cre == kCreAna) return cre_profile_ana<T>(m, x, y, z);
  return beyond_observer<T>(x, y, z, p, m, m.cre_unif_r0) ? T(0) : T(1);
}

// ---- packed grid groups --------------------------------------------------
// All gridded field slots that share one geometry are packed into a single
// array of 4-component voxel records {bx, by, bz, ne} (the sum of the B
// slots and of the n_e slots of that geometry), x-major with z fastest like
// the reference's Grid_* arrays (toolkit::index3d, include/toolkit.h:29-34).
// FP64 records are 32 B, FP32 records 16 B: a voxel is one (FP32) or two
// (FP64) 16-byte vector loads and the z-neighbour pair is contiguous.
struct DevGridGroup {
  const void *rec;
  int nx, ny, nz, has_b;
  double lo[3];     // box minimum (working length units)
  double scale[3];  // (n - 1) / (max - min)
  double gmax[3];   // n - 1: the grid coordinate of the upper box face
};

template <typename T>
struct Rec4 {
  T v[4];
};

__device__ __forceinline__ Rec4<double> load_rec(const double *base,
                                                 size_t idx) {
  const double2 *p = reinterpret_cast<const double2 *>(base + 4 * idx);
  const double2 a = __ldg(p), b = __ldg(p + 1);
  return Rec4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ Rec4<float> load_rec(const float *base,
                                                size_t idx) {
  const float4 a = __ldg(reinterpret_cast<const float4 *>(base) + idx);
  return Rec4<float>{{a.x, a.y, a.z, a.w}};
}

// Lerp in the reference's form a*(1-t) + b*t (breg.cc:64-96).
template <typename T>
__device__ __forceinline__ T lerp_ref(T a, T b, T t) {
  return a * (T(1.) - t) + b * t;
}

// The 8 corner records of one grid cell, cached in registers while a ray
// stays inside the cell.
template <typename T>
struct CellCache {
  long long key;  // x-major cell index, -1 = empty
  Rec4<T> c[8];   // (dx,dy,dz) corners: index dx*4 + dy*2 + dz
};

// Grid-space coordinates of p in group g; returns false on or outside the
// box surface (breg.cc:34-54: t <= 0 or t >= n-1 returns zero).
__device__ __forceinline__ bool grid_coords(const DevGridGroup &g, double px,
                                            double py, double pz, int &xl,
                                            int &yl, int &zl, double &xd,
                                            double &yd, double &zd) {
  const double tx = (px - g.lo[0]) * g.scale[0];
  if (!(tx > 0.) || tx >= g.gmax[0]) return false;
  const double ty = (py - g.lo[1]) * g.scale[1];
  if (!(ty > 0.) || ty >= g.gmax[1]) return false;
  const double tz = (pz - g.lo[2]) * g.scale[2];
  if (!(tz > 0.) || tz >= g.gmax[2]) return false;
  const double fx = floor(tx), fy = floor(ty), fz = floor(tz);
  xl = int(fx);
  yl = int(fy);
  zl = int(fz);
  xd = tx - fx;
  yd = ty - fy;
  zd = tz - fz;
  return true;
}

template <typename T>
__device__ __forceinline__ void fill_cell(const DevGridGroup &g, int xl,
                                          int yl, int zl, CellCache<T> &cc) {
  const T *base = reinterpret_cast<const T *>(g.rec);
  const size_t nyz = size_t(g.ny) * size_t(g.nz);
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const size_t i0 = size_t(xl + dx) * nyz + size_t(yl + dy) * g.nz + zl;
      cc.c[dx * 4 + dy * 2 + 0] = load_rec(base, i0);
      cc.c[dx * 4 + dy * 2 + 1] = load_rec(base, i0 + 1);
    }
}

// Trilinear interpolation of the cached cell: z, then y, then x
// (breg.cc:58-96, tereg.cc:65-73).  out[0..2] = B, out[3] = n_e.
template <typename T>
__device__ __forceinline__ void trilinear(const CellCache<T> &cc, T xd, T yd,
                                          T zd, T out[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const T i1 = lerp_ref(cc.c[0].v[k], cc.c[1].v[k], zd);
    const T i2 = lerp_ref(cc.c[2].v[k], cc.c[3].v[k], zd);
    const T j1 = lerp_ref(cc.c[4].v[k], cc.c[5].v[k], zd);
    const T j2 = lerp_ref(cc.c[6].v[k], cc.c[7].v[k], zd);
    const T w1 = lerp_ref(i1, i2, yd);
    const T w2 = lerp_ref(j1, j2, yd);
    out[k] = lerp_ref(w1, w2, xd);
  }
}

// Sample one grid group at p (working units); adds into b / te.  With a
// cache, the 8 corners are reloaded only when the cell changes.
template <typename T, bool kCache>
__device__ __forceinline__ void sample_group(const DevGridGroup &g, double px,
                                             double py, double pz,
                                             CellCache<T> &cc, T b[3], T &te) {
  int xl, yl, zl;
  double xd, yd, zd;
  if (!grid_coords(g, px, py, pz, xl, yl, zl, xd, yd, zd)) return;
  const long long key =
      (long long)xl * ((long long)g.ny * g.nz) + (long long)yl * g.nz + zl;
  if (!kCache || key != cc.key) {
    fill_cell<T>(g, xl, yl, zl, cc);
    cc.key = key;
  }
  T out[4];
  trilinear<T>(cc, T(xd), T(yd), T(zd), out);
  b[0] += out[0];
  b[1] += out[1];
  b[2] += out[2];
  te += out[3];
}

}  // namespace hxg
