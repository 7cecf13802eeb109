// hxg_common.cuh -- CGS constants and HEALPix RING geometry shared by the
// host glue and the sm_100a kernels of the line-of-sight integrator.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define HXG_HD __host__ __device__ __forceinline__
#else
#define HXG_HD inline
#endif

namespace hxg {

// ---- CGS constants: same expressions as include/hamunits.h:10-67 --------
namespace cgs {
constexpr double pi = 3.141592653589793238462643383279502884197;
constexpr double log2e = 1.4426950408889634;  // log2(e)
constexpr double halfpi = 1.570796326794896619231321691639751442099;
constexpr double twothirds = 0.666666666666666666666666666666666666667;
constexpr double twopi = 6.283185307179586476925286766559005768394;
constexpr double rad = (pi / 180.);
constexpr double erg = 1., cm = 1., sec = 1., Kelvin = 1.;
constexpr double m = (1.e2 * cm);
constexpr double pc = (3.0856775806e+18 * cm);
constexpr double kpc = (3.0856775806e+21 * cm);
constexpr double eV = (1.60217733e-12 * erg);
constexpr double GeV = (1.e9 * eV);
constexpr double GHz = 1.e9;
constexpr double muGauss = 1.e-6;  // 1e-6 * sqrt(erg/cm^3)
// Field unit of the FP32-compensated form (G).  A power of two, so that
// rescaling FP32 grid voxels into it is exact: a rounded voxel would carry
// the same error into every sample that reads it, which the Faraday phase
// then amplifies.
constexpr double fp32_bunit = 0x1p-20;
constexpr double ccm = (cm * cm * cm);
constexpr double c_light = (2.99792458e+10 * cm / sec);
constexpr double h_planck = (6.626075540e-27 * erg * sec);
constexpr double qe = (4.80320425e-10 * 1.0);  // * esu, esu = sqrt(erg*cm) = 1
constexpr double mec2 = (0.51099907e-3 * GeV);
constexpr double mec = (mec2 / c_light);
constexpr double kB = (1.380622e-16 * erg / Kelvin);
}  // namespace cgs

// HEALPix "undefined" marker (include/hamdis.h:95) and its test threshold
// (hamdis.h:689).
constexpr double kUndef = -1.6375e30;
constexpr double kUndefTest = -1.63749e30;

// ---- HEALPix RING scheme, after Hampix (include/hamdis.h:223-722) --------
struct Hpx {
  uint64_t nside, npix, npface, ncap;
  int order;
  double fact1, fact2;
};

// ilog2 (hamdis.h:261-284); the reference only supports power-of-two Nside.
HXG_HD int hpx_ilog2(uint64_t n) {
  int r = 0;
  while (n > 1) {
    n >>= 1;
    ++r;
  }
  return r;
}

// Hampix::prepare (hamdis.h:242-258)
HXG_HD Hpx hpx_make(uint64_t nside) {
  Hpx h;
  h.nside = nside;
  h.order = hpx_ilog2(nside);
  h.npface = nside * nside;
  h.npix = 12 * h.npface;
  h.ncap = (h.npface - nside) << 1;
  h.fact2 = 4. / (double)h.npix;
  h.fact1 = (double)(nside << 1) * h.fact2;
  return h;
}

// isqrt (hamdis.h:287-290)
HXG_HD uint64_t hpx_isqrt(uint64_t n) {
  return (uint64_t)floor(sqrt((double)n + 0.5));
}

// Hamp normalisation of (theta, phi) (include/hamp.h:93-98)
HXG_HD void hamp_norm(double &theta, double &phi) {
  theta = fmod(theta, cgs::pi);
  theta += (theta < 0) * cgs::pi;
  phi = fmod(phi, cgs::twopi);
  phi += (phi < 0) * cgs::twopi;
}

// Hampix::fillpoint = HEALPix RING pix2ang (hamdis.h:302-356)
HXG_HD void hpx_pix2ang(const Hpx &h, uint64_t idx, double &theta,
                        double &phi) {
  double z, ph, sth = 0.0;
  bool have_sth = false;
  if (idx < h.ncap) {
    const uint64_t iring = (1 + hpx_isqrt(1 + 2 * idx)) >> 1;
    const uint64_t iphi = (idx + 1) - 2 * iring * (iring - 1);
    const double tmp = (double)(iring * iring) * h.fact2;
    z = 1.0 - tmp;
    if (z > 0.99) {
      sth = sqrt(tmp * (2.0 - tmp));
      have_sth = true;
    }
    ph = ((double)iphi - 0.5) * cgs::halfpi / (double)iring;
  } else if (idx < (h.npix - h.ncap)) {
    const uint64_t nl4 = 4 * h.nside;
    const uint64_t ip = idx - h.ncap;
    const uint64_t tmp = ip >> (h.order + 2);
    const uint64_t iring = tmp + h.nside;
    const uint64_t iphi = ip - nl4 * tmp + 1;
    const double fodd = ((iring + h.nside) & 1) ? 1 : 0.5;
    z = ((double)(2 * h.nside) - (double)iring) * h.fact1;
    ph = ((double)iphi - fodd) * cgs::halfpi * 1.5 * h.fact1;
  } else {
    const uint64_t ip = h.npix - idx;
    const uint64_t iring = (1 + hpx_isqrt(2 * ip - 1)) >> 1;
    const uint64_t iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
    const double tmp = (double)(iring * iring) * h.fact2;
    z = tmp - 1.0;
    if (z < -0.99) {
      sth = sqrt(tmp * (2.0 - tmp));
      have_sth = true;
    }
    ph = ((double)iphi - 0.5) * cgs::halfpi / (double)iring;
  }
  theta = have_sth ? atan2(sth, z) : acos(z);
  phi = ph;
  hamp_norm(theta, phi);
}

// ring_above (hamdis.h:358-365)
HXG_HD uint64_t hpx_rabove(const Hpx &h, double z) {
  const double az = fabs(z);
  if (az <= cgs::twothirds) return (uint64_t)((double)h.nside * (2 - 1.5 * z));
  const uint64_t iring = (uint64_t)((double)h.nside * sqrt(3 * (1 - az)));
  return (z > 0) ? iring : 4 * h.nside - iring - 1;
}

// get_ring_info2 (hamdis.h:367-392)
HXG_HD void hpx_rinfo(const Hpx &h, uint64_t ring, uint64_t &startpix,
                      int64_t &ringpix, double &theta, bool &shifted) {
  const uint64_t northring = (ring > 2 * h.nside) ? 4 * h.nside - ring : ring;
  if (northring < h.nside) {
    const double tmp = (double)(northring * northring) * h.fact2;
    const double costheta = 1 - tmp;
    const double sintheta = sqrt(tmp * (2 - tmp));
    theta = atan2(sintheta, costheta);
    ringpix = (int64_t)(4 * northring);
    shifted = true;
    startpix = 2 * northring * (northring - 1);
  } else {
    theta = acos(((double)(2 * h.nside) - (double)northring) * h.fact1);
    ringpix = (int64_t)(4 * h.nside);
    shifted = ((northring - h.nside) & 1) == 0;
    startpix = h.ncap + (northring - h.nside) * (uint64_t)ringpix;
  }
  if (northring != ring) {
    theta = cgs::pi - theta;
    startpix = h.npix - startpix - (uint64_t)ringpix;
  }
}

// Pixel indices and weights of the 4-pixel bilinear interpolation
// (Hampix::interpolate, hamdis.h:609-682).
HXG_HD void hpx_interp_weights(const Hpx &h, double theta, double phi,
                               uint64_t pix[4], double wght[4]) {
  pix[0] = pix[1] = pix[2] = pix[3] = 0;
  wght[0] = wght[1] = wght[2] = wght[3] = 0.;
  const double z = cos(theta);
  const uint64_t ring1 = hpx_rabove(h, z);
  const uint64_t ring2 = ring1 + 1;
  double theta1 = 0.0, theta2 = 0.0;
  if (ring1 > 0) {
    uint64_t start;
    int64_t ringpix;
    bool shift;
    hpx_rinfo(h, ring1, start, ringpix, theta1, shift);
    const double dphi = 6.283185307179586476925286766559005768394 / (double)ringpix;
    const double tmp = (phi / dphi - 0.5 * shift);
    int64_t i1 = (int64_t)tmp - (int64_t)(tmp < 0);
    const double weight = (phi - ((double)i1 + 0.5 * shift) * dphi) / dphi;
    int64_t i2 = i1 + 1;
    i1 += ringpix * (i1 < 0);
    i2 -= ringpix * (i2 >= ringpix);
    pix[0] = start + (uint64_t)i1;
    pix[1] = start + (uint64_t)i2;
    wght[0] = 1.0 - weight;
    wght[1] = weight;
  }
  if (ring2 < (4 * h.nside)) {
    uint64_t start;
    int64_t ringpix;
    bool shift;
    hpx_rinfo(h, ring2, start, ringpix, theta2, shift);
    const double dphi = 6.283185307179586476925286766559005768394 / (double)ringpix;
    const double tmp = (phi / dphi - 0.5 * shift);
    int64_t i1 = (int64_t)tmp - (int64_t)(tmp < 0);
    const double weight = (phi - ((double)i1 + 0.5 * shift) * dphi) / dphi;
    int64_t i2 = i1 + 1;
    i1 += ringpix * (i1 < 0);
    i2 -= ringpix * (i2 >= ringpix);
    pix[2] = start + (uint64_t)i1;
    pix[3] = start + (uint64_t)i2;
    wght[2] = 1.0 - weight;
    wght[3] = weight;
  }
  if (ring1 == 0) {
    const double wtheta = theta / theta2;
    wght[2] *= wtheta;
    wght[3] *= wtheta;
    const double fac = (1.0 - wtheta) * 0.25;
    wght[0] = fac;
    wght[1] = fac;
    wght[2] += fac;
    wght[3] += fac;
    pix[0] = (pix[2] + 2) & 3;
    pix[1] = (pix[3] + 2) & 3;
  } else if (ring2 == (4 * h.nside)) {
    const double wtheta = (theta - theta1) / (cgs::pi - theta1);
    wght[0] *= (1.0 - wtheta);
    wght[1] *= (1.0 - wtheta);
    const double fac = wtheta * 0.25;
    wght[0] += fac;
    wght[1] += fac;
    wght[2] = fac;
    wght[3] = fac;
    pix[2] = ((pix[0] + 2) & 3) + h.npix - 4;
    pix[3] = ((pix[1] + 2) & 3) + h.npix - 4;
  } else {
    const double wtheta = (theta - theta1) / (theta2 - theta1);
    wght[0] *= (1.0 - wtheta);
    wght[1] *= (1.0 - wtheta);
    wght[2] *= wtheta;
    wght[3] *= wtheta;
  }
}

// Weighted sum over the 4 pixels, skipping undefined ones (hamdis.h:683-695)
HXG_HD double hpx_interp_apply(const double *map, const uint64_t pix[4],
                               const double wght[4]) {
  double wtot = 0.0, res = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double val = map[pix[i]];
    if (val > kUndefTest) {
      res += val * wght[i];
      wtot += wght[i];
    }
  }
  return (wtot == 0.0) ? kUndef : res / wtot;
}

HXG_HD double hpx_interpolate(const Hpx &h, const double *map, double theta,
                              double phi) {
  uint64_t pix[4];
  double w[4];
  hpx_interp_weights(h, theta, phi, pix, w);
  return hpx_interp_apply(map, pix, w);
}

// ---- (x, y, face) <-> ring index (hamdis.h:515-605) ---------------------
HXG_HD int64_t hpx_jrll(int64_t f) { return 2 + (f >> 2); }
HXG_HD int64_t hpx_jpll(int64_t f) {
  // {1,3,5,7,0,2,4,6,1,3,5,7}
  return ((f & 3) << 1) + 1 - ((f >> 2) & 1);
}

HXG_HD uint64_t hpx_xyf2ring(const Hpx &h, int64_t ix, int64_t iy,
                             int64_t face) {
  const uint64_t nl4 = 4 * h.nside;
  const uint64_t jr = (uint64_t)(hpx_jrll(face) * (int64_t)h.nside) -
                      (uint64_t)ix - (uint64_t)iy - 1;
  uint64_t nr, n_before;
  bool shifted;
  if (jr < h.nside) {
    shifted = true;
    nr = 4 * jr;
    n_before = 2 * jr * (jr - 1);
  } else if (jr < 3 * h.nside) {
    shifted = (((jr - h.nside) & 1) == 0);
    nr = 4 * h.nside;
    n_before = h.ncap + (jr - h.nside) * nr;
  } else {
    shifted = true;
    const uint64_t tmp = 4 * h.nside - jr;
    nr = 4 * tmp;
    n_before = h.npix - 2 * tmp * (tmp + 1);
  }
  nr >>= 2;
  const int64_t kshift = 1 - (int64_t)shifted;
  int64_t jp = (hpx_jpll(face) * (int64_t)nr + ix - iy + 1 + kshift) / 2;
  if (jp < 1) jp += (int64_t)nl4;
  return n_before + (uint64_t)jp - 1;
}

HXG_HD int64_t hpx_special_div(int64_t a, int64_t b) {
  int64_t p = a;
  const int64_t t = (p >= (b << 1));
  p -= t * (b << 1);
  return (t << 1) + (p >= b);
}

HXG_HD void hpx_ring2xyf(const Hpx &h, uint64_t pix, int64_t &ix,
                         int64_t &iy, int64_t &face) {
  int64_t iring, iphi, kshift, nr;
  const int64_t ns = (int64_t)h.nside;
  const int64_t nl2 = 2 * ns;
  if (pix < h.ncap) {
    iring = (int64_t)((1 + hpx_isqrt(1 + 2 * pix)) >> 1);
    iphi = (int64_t)(pix + 1) - 2 * iring * (iring - 1);
    kshift = 0;
    nr = iring;
    face = hpx_special_div(iphi - 1, nr);
  } else if (pix < (h.npix - h.ncap)) {
    const int64_t ip = (int64_t)(pix - h.ncap);
    const int64_t tmp = ip >> (h.order + 2);
    iring = tmp + ns;
    iphi = ip - tmp * 4 * ns + 1;
    kshift = (iring + ns) & 1;
    nr = ns;
    const int64_t ire = tmp + 1;
    const int64_t irm = nl2 + 1 - tmp;
    int64_t ifm = iphi - (ire >> 1) + ns - 1;
    int64_t ifp = iphi - (irm >> 1) + ns - 1;
    ifm >>= h.order;
    ifp >>= h.order;
    face = (ifp == ifm) ? (ifp | 4) : ((ifp < ifm) ? ifp : (ifm + 8));
  } else {
    const int64_t ip = (int64_t)(h.npix - pix);
    iring = (int64_t)((1 + hpx_isqrt((uint64_t)(2 * ip - 1))) >> 1);
    iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
    kshift = 0;
    nr = iring;
    iring = 2 * nl2 - iring;
    face = hpx_special_div(iphi - 1, nr) + 8;
  }
  const int64_t irt = iring - ((2 + (face >> 2)) * ns) + 1;
  int64_t ipt = 2 * iphi - hpx_jpll(face) * nr - kshift - 1;
  if (ipt >= nl2) ipt -= 8 * ns;
  ix = (ipt - irt) >> 1;
  iy = (-ipt - irt) >> 1;
}

// De-interleave the even bits of v (NESTED pixel -> x or y coordinate).
HXG_HD uint64_t hpx_compress_bits(uint64_t v) {
  v &= 0x5555555555555555ull;
  v = (v | (v >> 1)) & 0x3333333333333333ull;
  v = (v | (v >> 2)) & 0x0f0f0f0f0f0f0f0full;
  v = (v | (v >> 4)) & 0x00ff00ff00ff00ffull;
  v = (v | (v >> 8)) & 0x0000ffff0000ffffull;
  v = (v | (v >> 16)) & 0x00000000ffffffffull;
  return v;
}

// NESTED index -> RING index: used to walk the sky in compact NESTED
// patches while reading and writing RING-ordered maps.
HXG_HD uint64_t hpx_nest2ring(const Hpx &h, uint64_t nest) {
  const int64_t face = (int64_t)(nest >> (2 * h.order));
  const uint64_t ipf = nest & (h.npface - 1);
  const int64_t ix = (int64_t)hpx_compress_bits(ipf);
  const int64_t iy = (int64_t)hpx_compress_bits(ipf >> 1);
  return hpx_xyf2ring(h, ix, iy, face);
}

}  // namespace hxg
