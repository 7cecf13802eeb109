/*
 * hxo.c -- CPU oracle for hammurabiX's line-of-sight integrator.
 *
 * TEST INFRASTRUCTURE ONLY: the checker that tests/ and bench.py's CPU
 * baseline use.  It restates, in plain C and FP64, the reference algorithm
 * of Integrator::write_grid and everything it calls, keeping the
 * reference's operation order so that its results agree with the
 * reference to rounding.  Each function cites the reference file:line it
 * follows (paths relative to the hammurabiX source tree).  It is validated
 * against the reference's own unit-test fixtures (tests/golden) and against
 * the reference itself compiled by oracle/Makefile.
 */
#include "hxo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- CGS constants, include/hamunits.h:10-67 (same expressions) ------- */
static const double k_pi = 3.141592653589793238462643383279502884197;
static const double k_halfpi = 1.570796326794896619231321691639751442099;
static const double k_twothirds = 0.666666666666666666666666666666666666667;
static const double k_twopi = 6.283185307179586476925286766559005768394;
#define CGS_CM 1.
#define CGS_SEC 1.
#define CGS_ERG 1.
static double cgs_m(void) { return 1.e2 * CGS_CM; }
static double cgs_kpc(void) { return 3.0856775806e+21 * CGS_CM; }
static double cgs_GeV(void) { return 1.e9 * (1.60217733e-12 * CGS_ERG); }
static double cgs_c(void) { return 2.99792458e+10 * CGS_CM / CGS_SEC; }
static double cgs_h(void) { return 6.626075540e-27 * CGS_ERG * CGS_SEC; }
static double cgs_qe(void) { return 4.80320425e-10 * sqrt(CGS_ERG * CGS_CM); }
static double cgs_mec2(void) { return 0.51099907e-3 * cgs_GeV(); }
static double cgs_mec(void) { return cgs_mec2() / cgs_c(); }
static double cgs_kB(void) { return 1.380622e-16 * CGS_ERG / 1.; }

/* ======================================================================
 * HEALPix RING scheme: include/hamdis.h:223-722 (Hampix)
 * ====================================================================== */
typedef struct {
  uint64_t nside, npix, npface, ncap;
  int order;
  double fact1, fact2;
} hpx_t;

/* hamdis.h:261-284 */
static uint64_t hpx_ilog2(uint64_t n) {
  uint64_t tmp = n, res = 0;
  while (tmp > 0x0000FFFF) {
    res += 16;
    tmp >>= 16;
  }
  if (tmp > 0x000000FF) {
    res |= 8;
    tmp >>= 8;
  }
  if (tmp > 0x0000000F) {
    res |= 4;
    tmp >>= 4;
  }
  if (tmp > 0x00000003) {
    res |= 2;
    tmp >>= 2;
  }
  if (tmp > 0x00000001) res |= 1;
  return res;
}

/* hamdis.h:242-258 */
static hpx_t hpx_make(uint64_t nside) {
  hpx_t h;
  h.nside = nside;
  h.order = (int)hpx_ilog2(nside);
  h.npface = nside * nside;
  h.npix = 12 * h.npface;
  h.ncap = (h.npface - nside) << 1;
  h.fact2 = 4. / (double)h.npix;
  h.fact1 = (double)(nside << 1) * h.fact2;
  return h;
}

/* hamdis.h:287-290 */
static uint64_t hpx_isqrt(uint64_t n) {
  return (uint64_t)floor(sqrt((double)n + 0.5));
}

/* Hamp normalisation, include/hamp.h:93-98 */
static void hamp_norm(double *theta, double *phi) {
  *theta = fmod(*theta, k_pi);
  *theta += (*theta < 0) * k_pi;
  *phi = fmod(*phi, k_twopi);
  *phi += (*phi < 0) * k_twopi;
}

/* fillpoint = HEALPix pix2ang, hamdis.h:302-356 */
static void hpx_pix2ang(const hpx_t *h, uint64_t idx, double *theta,
                        double *phi) {
  double z = 0.0, ph = 0.0, sth = 0.0;
  int have_sth = 0;
  if (idx < h->ncap) {
    const uint64_t iring = (1 + hpx_isqrt(1 + 2 * idx)) >> 1;
    const uint64_t iphi = (idx + 1) - 2 * iring * (iring - 1);
    const double tmp = (double)(iring * iring) * h->fact2;
    z = 1.0 - tmp;
    if (z > 0.99) {
      sth = sqrt(tmp * (2.0 - tmp));
      have_sth = 1;
    }
    ph = ((double)iphi - 0.5) * k_halfpi / (double)iring;
  } else if (idx < (h->npix - h->ncap)) {
    const uint64_t nl4 = 4 * h->nside;
    const uint64_t ip = idx - h->ncap;
    const uint64_t tmp = (h->order >= 0) ? ip >> (h->order + 2) : ip / nl4;
    const uint64_t iring = tmp + h->nside;
    const uint64_t iphi = ip - nl4 * tmp + 1;
    const double fodd = ((iring + h->nside) & 1) ? 1 : 0.5;
    z = ((double)(2 * h->nside) - (double)iring) * h->fact1;
    ph = ((double)iphi - fodd) * k_halfpi * 1.5 * h->fact1;
  } else {
    const uint64_t ip = h->npix - idx;
    const uint64_t iring = (1 + hpx_isqrt(2 * ip - 1)) >> 1;
    const uint64_t iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
    const double tmp = (double)(iring * iring) * h->fact2;
    z = tmp - 1.0;
    if (z < -0.99) {
      sth = sqrt(tmp * (2.0 - tmp));
      have_sth = 1;
    }
    ph = ((double)iphi - 0.5) * k_halfpi / (double)iring;
  }
  *theta = have_sth ? atan2(sth, z) : acos(z);
  *phi = ph;
  hamp_norm(theta, phi);
}

/* hamdis.h:358-365 */
static uint64_t hpx_rabove(const hpx_t *h, double z) {
  const double az = fabs(z);
  if (az <= k_twothirds) return (uint64_t)((double)h->nside * (2 - 1.5 * z));
  const uint64_t iring = (uint64_t)((double)h->nside * sqrt(3 * (1 - az)));
  return (z > 0) ? iring : 4 * h->nside - iring - 1;
}

/* hamdis.h:367-392 */
static void hpx_rinfo(const hpx_t *h, uint64_t ring, uint64_t *startpix,
                      int64_t *ringpix, double *theta, int *shifted) {
  const uint64_t northring = (ring > 2 * h->nside) ? 4 * h->nside - ring : ring;
  if (northring < h->nside) {
    const double tmp = (double)(northring * northring) * h->fact2;
    const double costheta = 1 - tmp;
    const double sintheta = sqrt(tmp * (2 - tmp));
    *theta = atan2(sintheta, costheta);
    *ringpix = (int64_t)(4 * northring);
    *shifted = 1;
    *startpix = 2 * northring * (northring - 1);
  } else {
    *theta = acos(((double)(2 * h->nside) - (double)northring) * h->fact1);
    *ringpix = (int64_t)(4 * h->nside);
    *shifted = ((northring - h->nside) & 1) == 0;
    *startpix = h->ncap + (northring - h->nside) * (uint64_t)(*ringpix);
  }
  if (northring != ring) {
    *theta = k_pi - *theta;
    *startpix = h->npix - *startpix - (uint64_t)(*ringpix);
  }
}

/* Hampix::interpolate, hamdis.h:609-696 */
static double hpx_interpolate(const hpx_t *h, const double *map, double theta,
                              double phi) {
  uint64_t pix[4] = {0, 0, 0, 0};
  double wght[4] = {0, 0, 0, 0};
  const double z = cos(theta);
  const uint64_t ring1 = hpx_rabove(h, z);
  const uint64_t ring2 = ring1 + 1;
  double theta1 = 0.0, theta2 = 0.0;
  if (ring1 > 0) {
    uint64_t start;
    int64_t ringpix;
    int shift;
    hpx_rinfo(h, ring1, &start, &ringpix, &theta1, &shift);
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
  if (ring2 < (4 * h->nside)) {
    uint64_t start;
    int64_t ringpix;
    int shift;
    hpx_rinfo(h, ring2, &start, &ringpix, &theta2, &shift);
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
  } else if (ring2 == (4 * h->nside)) {
    const double wtheta = (theta - theta1) / (k_pi - theta1);
    wght[0] *= (1.0 - wtheta);
    wght[1] *= (1.0 - wtheta);
    const double fac = wtheta * 0.25;
    wght[0] += fac;
    wght[1] += fac;
    wght[2] = fac;
    wght[3] = fac;
    pix[2] = ((pix[0] + 2) & 3) + h->npix - 4;
    pix[3] = ((pix[1] + 2) & 3) + h->npix - 4;
  } else {
    const double wtheta = (theta - theta1) / (theta2 - theta1);
    wght[0] *= (1.0 - wtheta);
    wght[1] *= (1.0 - wtheta);
    wght[2] *= wtheta;
    wght[3] *= wtheta;
  }
  double wtot = 0.0, res = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double val = map[pix[i]];
    if (val > -1.63749e30) {
      res += val * wght[i];
      wtot += wght[i];
    }
  }
  return (wtot == 0.0) ? -1.6375e30 : res / wtot;
}

/* Hampix::accumulate, hamdis.h:698-721 */
void hxo_accumulate(uint32_t nside_dst, double *dst, uint32_t nside_src,
                    const double *src) {
  const hpx_t hd = hpx_make(nside_dst);
  const hpx_t hs = hpx_make(nside_src);
  if (hd.npix == hs.npix) {
    for (uint64_t i = 0; i < hd.npix; ++i) dst[i] = dst[i] + src[i];
  } else {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)hd.npix; ++i) {
      double th, ph;
      hpx_pix2ang(&hd, (uint64_t)i, &th, &ph);
      dst[i] = dst[i] + hpx_interpolate(&hs, src, th, ph);
    }
  }
}

void hxo_pix2ang(uint32_t nside, uint64_t npix, double *theta, double *phi) {
  const hpx_t h = hpx_make(nside);
  for (uint64_t i = 0; i < npix && i < h.npix; ++i)
    hpx_pix2ang(&h, i, &theta[i], &phi[i]);
}

void hxo_interpolate(uint32_t nside, const double *map, uint64_t n,
                     const double *theta, const double *phi, double *out) {
  const hpx_t h = hpx_make(nside);
  for (uint64_t i = 0; i < n; ++i) {
    double th = theta[i], ph = phi[i];
    hamp_norm(&th, &ph);
    out[i] = hpx_interpolate(&h, map, th, ph);
  }
}

/* ---- ring <-> (x,y,face), hamdis.h:515-605 --------------------------- */
static const int64_t k_jrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
static const int64_t k_jpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

static int64_t special_div(int64_t a, int64_t b) {
  int64_t p = a, q = b;
  const int64_t t = (p >= (q << 1));
  p -= t * (q << 1);
  return (t << 1) + (p >= q);
}

static void hpx_ring2xyf(const hpx_t *h, uint64_t pix, int64_t *ix,
                         int64_t *iy, int64_t *face) {
  int64_t iring, iphi, kshift, nr;
  const int64_t ns = (int64_t)h->nside;
  const int64_t nl2 = 2 * ns;
  if (pix < h->ncap) {
    iring = (int64_t)((1 + hpx_isqrt(1 + 2 * pix)) >> 1);
    iphi = (int64_t)(pix + 1) - 2 * iring * (iring - 1);
    kshift = 0;
    nr = iring;
    *face = special_div(iphi - 1, nr);
  } else if (pix < (h->npix - h->ncap)) {
    const int64_t ip = (int64_t)(pix - h->ncap);
    const int64_t tmp = (h->order >= 0) ? ip >> (h->order + 2) : ip / (4 * ns);
    iring = tmp + ns;
    iphi = ip - tmp * 4 * ns + 1;
    kshift = (iring + ns) & 1;
    nr = ns;
    const int64_t ire = tmp + 1;
    const int64_t irm = nl2 + 1 - tmp;
    int64_t ifm = iphi - (ire >> 1) + ns - 1;
    int64_t ifp = iphi - (irm >> 1) + ns - 1;
    if (h->order >= 0) {
      ifm >>= h->order;
      ifp >>= h->order;
    } else {
      ifm /= ns;
      ifp /= ns;
    }
    *face = (ifp == ifm) ? (ifp | 4) : ((ifp < ifm) ? ifp : (ifm + 8));
  } else {
    const int64_t ip = (int64_t)(h->npix - pix);
    iring = (int64_t)((1 + hpx_isqrt((uint64_t)(2 * ip - 1))) >> 1);
    iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
    kshift = 0;
    nr = iring;
    iring = 2 * nl2 - iring;
    *face = special_div(iphi - 1, nr) + 8;
  }
  const int64_t irt = iring - ((2 + (*face >> 2)) * ns) + 1;
  int64_t ipt = 2 * iphi - k_jpll[*face] * nr - kshift - 1;
  if (ipt >= nl2) ipt -= 8 * ns;
  *ix = (ipt - irt) >> 1;
  *iy = (-ipt - irt) >> 1;
}

static uint64_t hpx_xyf2ring(const hpx_t *h, int64_t ix, int64_t iy,
                             int64_t face) {
  const uint64_t nl4 = 4 * h->nside;
  const uint64_t jr = (uint64_t)(k_jrll[face] * (int64_t)h->nside) - (uint64_t)ix -
                      (uint64_t)iy - 1;
  uint64_t nr, n_before;
  int shifted;
  if (jr < h->nside) {
    shifted = 1;
    nr = 4 * jr;
    n_before = 2 * jr * (jr - 1);
  } else if (jr < 3 * h->nside) {
    shifted = (((jr - h->nside) & 1) == 0);
    nr = 4 * h->nside;
    n_before = h->ncap + (jr - h->nside) * nr;
  } else {
    shifted = 1;
    const uint64_t tmp = 4 * h->nside - jr;
    nr = 4 * tmp;
    n_before = h->npix - 2 * tmp * (tmp + 1);
  }
  nr >>= 2;
  const int64_t kshift = 1 - shifted;
  int64_t jp = (k_jpll[face] * (int64_t)nr + ix - iy + 1 + kshift) / 2;
  if (jp < 1) jp += (int64_t)nl4;
  return n_before + (uint64_t)jp - 1;
}

/* Hampisk::duplicate, include/hamsk.h:55-103 */
int hxo_mask_duplicate(uint32_t pivot_nside, const double *pivot_mask,
                       uint32_t nside, double *out) {
  const hpx_t hp = hpx_make(pivot_nside);
  const hpx_t ht = hpx_make(nside);
  if (pivot_nside == nside) {
    memcpy(out, pivot_mask, sizeof(double) * hp.npix);
    return 0;
  }
  for (uint64_t i = 0; i < ht.npix; ++i) out[i] = 0.0;
  if (pivot_nside > nside) {
    const uint64_t fact = pivot_nside / nside;
    for (uint64_t mp = 0; mp < ht.npix; ++mp) {
      int64_t x, y, f;
      hpx_ring2xyf(&ht, mp, &x, &y, &f);
      int hit = 0;
      for (uint64_t j = fact * (uint64_t)y; j < fact * (uint64_t)(y + 1); ++j) {
        for (uint64_t i = fact * (uint64_t)x; i < fact * (uint64_t)(x + 1); ++i) {
          const uint64_t opix = hpx_xyf2ring(&hp, (int64_t)i, (int64_t)j, f);
          hit = (pivot_mask[opix] > 0);
          if (hit) break;
        }
        if (hit) break;
      }
      out[mp] = (double)hit;
    }
  } else {
    const uint64_t fact = nside / pivot_nside;
    for (uint64_t mp = 0; mp < hp.npix; ++mp) {
      const double val = pivot_mask[mp];
      int64_t x, y, f;
      hpx_ring2xyf(&hp, mp, &x, &y, &f);
      for (uint64_t j = fact * (uint64_t)y; j < fact * (uint64_t)(y + 1); ++j)
        for (uint64_t i = fact * (uint64_t)x; i < fact * (uint64_t)(x + 1); ++i)
          out[hpx_xyf2ring(&ht, (int64_t)i, (int64_t)j, f)] = val;
    }
  }
  return 0;
}

/* ======================================================================
 * Field sampling
 * ====================================================================== */

/* Vertex-grid trilinear read: Breg::read_grid (source/field/b/breg.cc:28-97),
 * TEreg::read_grid (source/field/te/tereg.cc:27-74).  Lerp along z, then y,
 * then x; exactly zero on and outside the box surface.                     */
static int tri_setup(const hxg_grid_desc_t *g, const double pos[3],
                     uint64_t *xl, uint64_t *yl, uint64_t *zl, double *xd,
                     double *yd, double *zd) {
  double tmp = (double)(g->nx - 1) * (pos[0] - g->x_min) / (g->x_max - g->x_min);
  if (tmp <= 0 || tmp >= (double)(g->nx - 1)) return 0;
  *xl = (uint64_t)floor(tmp);
  *xd = tmp - (double)*xl;
  tmp = (double)(g->ny - 1) * (pos[1] - g->y_min) / (g->y_max - g->y_min);
  if (tmp <= 0 || tmp >= (double)(g->ny - 1)) return 0;
  *yl = (uint64_t)floor(tmp);
  *yd = tmp - (double)*yl;
  tmp = (double)(g->nz - 1) * (pos[2] - g->z_min) / (g->z_max - g->z_min);
  if (tmp <= 0 || tmp >= (double)(g->nz - 1)) return 0;
  *zl = (uint64_t)floor(tmp);
  *zd = tmp - (double)*zl;
  return 1;
}

static inline uint64_t idx3(const hxg_grid_desc_t *g, uint64_t i, uint64_t j,
                            uint64_t l) {
  return i * g->ny * g->nz + j * g->nz + l; /* toolkit.h:29-34 */
}

static double tri_scalar(const hxo_grid_t *gr, int c, uint64_t xl, uint64_t yl,
                         uint64_t zl, double xd, double yd, double zd) {
  const hxg_grid_desc_t *g = &gr->desc;
  const double *a = gr->c[c];
  uint64_t i1 = idx3(g, xl, yl, zl), i2 = idx3(g, xl, yl, zl + 1);
  const double v1 = a[i1] * (1. - zd) + a[i2] * zd;
  i1 = idx3(g, xl, yl + 1, zl);
  i2 = idx3(g, xl, yl + 1, zl + 1);
  const double v2 = a[i1] * (1. - zd) + a[i2] * zd;
  i1 = idx3(g, xl + 1, yl, zl);
  i2 = idx3(g, xl + 1, yl, zl + 1);
  const double v3 = a[i1] * (1. - zd) + a[i2] * zd;
  i1 = idx3(g, xl + 1, yl + 1, zl);
  i2 = idx3(g, xl + 1, yl + 1, zl + 1);
  const double v4 = a[i1] * (1. - zd) + a[i2] * zd;
  const double w1 = v1 * (1. - yd) + v2 * yd;
  const double w2 = v3 * (1. - yd) + v4 * yd;
  return w1 * (1. - xd) + w2 * xd;
}

static void read_grid_vec(const hxo_grid_t *gr, const double pos[3],
                          double out[3]) {
  uint64_t xl, yl, zl;
  double xd, yd, zd;
  out[0] = out[1] = out[2] = 0.;
  if (!tri_setup(&gr->desc, pos, &xl, &yl, &zl, &xd, &yd, &zd)) return;
  for (int c = 0; c < 3; ++c) out[c] = tri_scalar(gr, c, xl, yl, zl, xd, yd, zd);
}

static double read_grid_scalar(const hxo_grid_t *gr, const double pos[3]) {
  uint64_t xl, yl, zl;
  double xd, yd, zd;
  if (!tri_setup(&gr->desc, pos, &xl, &yl, &zl, &xd, &yd, &zd)) return 0.;
  return tri_scalar(gr, 0, xl, yl, zl, xd, yd, zd);
}

int hxo_read_grid(const hxo_grid_t *g, int ncomp, uint64_t n,
                  const double *pos, double *out) {
  for (uint64_t i = 0; i < n; ++i) {
    if (ncomp == 3)
      read_grid_vec(g, &pos[3 * i], &out[3 * i]);
    else
      out[i] = read_grid_scalar(g, &pos[3 * i]);
  }
  return 0;
}

/* ---- analytic models ------------------------------------------------ */
void hxo_breg_field(const hxg_models_t *m, const double obs[3],
                    const double pos[3], double out[3]) {
  out[0] = out[1] = out[2] = 0.;
  const double kpc = cgs_kpc();
  switch (m->breg) {
    case HXG_BREG_LSA: { /* source/field/b/breg_lsa.cc:9-26 */
      const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
      if (r > (20. * kpc) || r < (3. * kpc)) return;
      const double cos_p = pos[0] / r, sin_p = pos[1] / r;
      const double psi = m->lsa.psi0 + m->lsa.psi1 * log(r / (8. * kpc));
      const double chi = m->lsa.chi0 * tanh(pos[2] / (1. * kpc));
      out[0] = m->lsa.b0 * (sin(psi) * cos(chi) * cos_p - cos(psi) * cos(chi) * sin_p);
      out[1] = m->lsa.b0 * (sin(psi) * cos(chi) * sin_p + cos(psi) * cos(chi) * cos_p);
      out[2] = m->lsa.b0 * sin(chi);
      return;
    }
    case HXG_BREG_UNIF: /* breg_unif.cc:7-12 */
      out[0] = m->unif.bp * cos(m->unif.l0);
      out[1] = m->unif.bp * sin(m->unif.l0);
      out[2] = m->unif.bv;
      return;
    case HXG_BREG_CART: /* breg_cart.cc:7-11 */
      out[0] = m->cart.bx;
      out[1] = m->cart.by;
      out[2] = m->cart.bz;
      return;
    case HXG_BREG_HELIX: { /* breg_helix.cc:13-30 */
      const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
      const double phi = atan2(pos[1], pos[0]) + M_PI / 2.0;
      if ((r > m->helix.r_min) && (r < m->helix.r_max)) {
        out[0] = m->helix.bx * cos(phi);
        out[1] = m->helix.by * sin(phi);
        out[2] = m->helix.bz;
      }
      return;
    }
    case HXG_BREG_SPIRAL: { /* hxg_breg_spiral_t definition (include/hxg.h) */
      const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
      if (r > (20. * kpc) || r < (3. * kpc)) return;
      const double rsun = sqrt(obs[0] * obs[0] + obs[1] * obs[1]);
      const double cos_p = pos[0] / r, sin_p = pos[1] / r;
      const double amp = m->spiral.b0 * exp(-(r - rsun) / m->spiral.r_scale) *
                         exp(-fabs(pos[2]) / m->spiral.h_scale);
      const double sp = sin(m->spiral.pitch), cp = cos(m->spiral.pitch);
      out[0] = amp * (sp * cos_p - cp * sin_p);
      out[1] = amp * (sp * sin_p + cp * cos_p);
      out[2] = 0.;
      return;
    }
    default:
      return;
  }
}

double hxo_tereg_field(const hxg_models_t *m, const double obs[3],
                       const double pos[3]) {
  switch (m->tereg) {
    case HXG_TEREG_UNIF: { /* source/field/te/tereg_unif.cc:6-12 */
      const double d[3] = {pos[0] - obs[0], pos[1] - obs[1], pos[2] - obs[2]};
      double l = 0.;
      for (int i = 0; i < 3; ++i) l += d[i] * d[i];
      if (sqrt(l) > m->te_unif.r0) return 0.;
      return m->te_unif.n0;
    }
    case HXG_TEREG_EXPDISK: { /* hxg_tereg_expdisk_t definition */
      const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
      return m->te_exp.n0 * exp(-r / m->te_exp.r_scale) *
             exp(-fabs(pos[2]) / m->te_exp.h_scale);
    }
    default:
      return 0.;
  }
}

/* ---- CRE models: source/field/cre/cre_ana.cc:11-63, cre_unif.cc:11-59 -- */
static double cre_flux_idx(const hxg_models_t *m, const double pos[3]) {
  if (m->cre == HXG_CRE_ANA) {
    const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]) / cgs_kpc();
    const double z = fabs(pos[2]) / cgs_kpc();
    return -m->cre_ana.alpha + m->cre_ana.beta * r + m->cre_ana.theta * z;
  }
  return -(m->cre_unif.alpha);
}

static double cre_spatial_profile(const hxg_models_t *m, const double obs[3],
                                  const double pos[3]) {
  if (m->cre == HXG_CRE_ANA) {
    const double R0 = sqrt(obs[0] * obs[0] + obs[1] * obs[1]);
    const double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    return exp((R0 - r) / m->cre_ana.r0) *
           (1. / (cosh(pos[2] / m->cre_ana.z0) * cosh(pos[2] / m->cre_ana.z0)));
  }
  const double d[3] = {pos[0] - obs[0], pos[1] - obs[1], pos[2] - obs[2]};
  double l = 0.;
  for (int i = 0; i < 3; ++i) l += d[i] * d[i];
  return (sqrt(l) > m->cre_unif.r0) ? 0 : 1;
}

static double cre_flux_norm(const hxg_models_t *m, const double obs[3],
                            const double pos[3]) {
  const double E0 = (m->cre == HXG_CRE_ANA) ? m->cre_ana.E0 : m->cre_unif.E0;
  const double j0 = (m->cre == HXG_CRE_ANA) ? m->cre_ana.j0 : m->cre_unif.j0;
  const double gamma0 = E0 / cgs_mec2();
  const double beta0 = sqrt(1. - 1. / gamma0);
  const double unit = 4. * k_pi * cgs_mec() /
                      (cgs_GeV() * cgs_m() * cgs_m() * CGS_SEC * beta0);
  const double norm = j0 * pow(gamma0, -cre_flux_idx(m, obs));
  return norm * unit * cre_spatial_profile(m, obs, pos);
}

/* Integrator::sync_emissivity_t / _p, analytic branch
 * (source/integrator/integrator.cc:332-346, 401-415).                      */
void hxo_sync_emissivity(const hxg_models_t *m, const double obs[3],
                         double freq, const double pos[3], double b_per,
                         double *jt, double *jp) {
  const double qe = cgs_qe(), mec2 = cgs_mec2(), mec = cgs_mec();
  const double index = cre_flux_idx(m, pos);
  const double fn = cre_flux_norm(m, obs, pos);
  const double A = 2. * k_pi * freq * mec / (3. * qe * fabs(b_per));
  {
    const double norm = fn * 1.73205081 * (qe * qe * qe) * fabs(b_per) /
                        (4. * k_pi * mec2 * (1. - index));
    *jt = norm * (pow(A, 0.5 * (index + 1)) * tgamma(-0.25 * index + 19. / 12.) *
                  tgamma(-0.25 * index - 1. / 12.));
  }
  {
    const double norm = fn * 1.73205081 * (qe * qe * qe) * fabs(b_per) /
                        (16. * k_pi * mec2);
    *jp = norm * (pow(A, 0.5 * (index + 1)) * tgamma(-0.25 * index + 7. / 12.) *
                  tgamma(-0.25 * index - 1. / 12.));
  }
}

/* Integrator::temp_convert, integrator.cc:275-279 */
double hxo_temp_convert(double temp_br, double freq) {
  const double p = cgs_h() * freq / (cgs_kB() * 2.725);
  return temp_br * (exp(p) - 1.) * (exp(p) - 1.) / (p * p * exp(p));
}

/* los_versor (integrator.cc:268-272), los_parproj / los_perproj
 * (integrator.h:39-49), sync_ipa (integrator.cc:257-265).                  */
static void los_versor(double the, double phi, double u[3]) {
  u[0] = cos(phi) * sin(the);
  u[1] = sin(phi) * sin(the);
  u[2] = cos(the);
}

static double sync_ipa(const double b[3], double the, double phi) {
  const double vt[3] = {cos(the) * cos(phi), cos(the) * sin(phi), -sin(the)};
  const double vp[3] = {-sin(phi), cos(phi), 0.};
  double dt = 0., dp = 0.;
  for (int i = 0; i < 3; ++i) dt += vt[i] * b[i];
  for (int i = 0; i < 3; ++i) dp += vp[i] * b[i];
  return atan2(-dt, -dp);
}

static double los_perproj(const double b[3], const double u[3]) {
  double c[3];
  for (int i = 0; i < 3; ++i)
    c[i] = b[(i + 1) % 3] * u[(i + 2) % 3] - b[(i + 2) % 3] * u[(i + 1) % 3];
  double l = 0.;
  for (int i = 0; i < 3; ++i) l += c[i] * c[i];
  return sqrt(l);
}

static double los_parproj(const double b[3], const double u[3]) {
  double d = 0.;
  for (int i = 0; i < 3; ++i) d += b[i] * u[i];
  return d;
}

void hxo_los_geometry(uint64_t n, const double *theta, const double *phi,
                      const double *b, double *versor, double *b_par,
                      double *b_per, double *ipa) {
  for (uint64_t i = 0; i < n; ++i) {
    double u[3];
    los_versor(theta[i], phi[i], u);
    for (int c = 0; c < 3; ++c) versor[3 * i + c] = u[c];
    b_par[i] = los_parproj(&b[3 * i], u);
    b_per[i] = los_perproj(&b[3 * i], u);
    ipa[i] = sync_ipa(&b[3 * i], theta[i], phi[i]);
  }
}

/* Integrator::assemble_shell_ref, integrator.cc:231-254 */
int hxo_shell_ref(const hxg_obs_t *obs, uint32_t shell, double *d_start,
                  double *delta_d, uint64_t *step) {
  if (shell >= obs->total_shell) return HXG_ERR_INVALID;
  const double ds = obs->radii_shell[shell];
  const double de = obs->radii_shell[shell + 1];
  double dd = obs->oc_r_res;
  const uint64_t st = (uint64_t)floor((de / dd - ds / dd));
  dd = (de - ds) / (double)st;
  *d_start = ds;
  *delta_d = dd;
  *step = st;
  return 0;
}

/* ======================================================================
 * Integrator::write_grid + radial_integration (integrator.cc:23-228)
 * ====================================================================== */
typedef struct {
  const hxg_obs_t *obs;
  const hxg_models_t *m;
  const hxo_grids_t *g;
} ctx_t;

typedef struct {
  double is, qs, us, fd, dm;
} pixobs_t;

static void radial_integration(const ctx_t *c, double d_start, double delta_d,
                               uint64_t step, double THE, double PHI,
                               pixobs_t *po) {
  const hxg_obs_t *obs = c->obs;
  const hxg_models_t *m = c->m;
  const int do_sync = obs->do_sync;
  double inner_shells_fd = 0.;
  if (obs->do_fd || do_sync) inner_shells_fd = po->fd;
  po->dm = po->fd = po->is = po->us = po->qs = 0.;
  double u[3];
  los_versor(THE, PHI, u);
  double lambda_square = 0, i2bt_sync = 0.;
  const double qe = cgs_qe(), mec2 = cgs_mec2(), c_l = cgs_c();
  const double fd_forefactor = -(qe * qe * qe) / (2. * k_pi * mec2 * mec2);
  if (do_sync) {
    const double f = obs->sync_freq;
    lambda_square = (c_l / f) * (c_l / f);
    i2bt_sync = c_l * c_l / (2. * cgs_kB() * f * f);
  }
  for (uint64_t looper = 0; looper < step; ++looper) {
    const double dist = d_start + ((double)looper + 0.5) * delta_d;
    double pos[3];
    for (int i = 0; i < 3; ++i) pos[i] = u[i] * dist + obs->observer[i];
    double len = 0.;
    for (int i = 0; i < 3; ++i) len += pos[i] * pos[i];
    len = sqrt(len);
    if (len < obs->gc_r_min) continue;
    if (len > obs->gc_r_max) continue;
    if (pos[2] < obs->gc_z_min) continue;
    if (pos[2] > obs->gc_z_max) continue;
    double B[3] = {0., 0., 0.}, Br[3] = {0., 0., 0.};
    if (m->breg == HXG_BREG_GRID)
      read_grid_vec(&c->g->slot[HXG_FIELD_BREG], pos, B);
    else
      hxo_breg_field(m, obs->observer, pos, B);
    if (m->brnd == HXG_BRND_GRID) read_grid_vec(&c->g->slot[HXG_FIELD_BRND], pos, Br);
    for (int i = 0; i < 3; ++i) B[i] += Br[i];
    const double B_par = los_parproj(B, u);
    const double B_per = los_perproj(B, u);
    double te;
    if (m->tereg == HXG_TEREG_GRID)
      te = read_grid_scalar(&c->g->slot[HXG_FIELD_TEREG], pos);
    else
      te = hxo_tereg_field(m, obs->observer, pos);
    if (m->ternd == HXG_TERND_GRID)
      te += read_grid_scalar(&c->g->slot[HXG_FIELD_TERND], pos);
    te *= (double)(te > 0.);
    if (obs->do_dm) po->dm += te * delta_d;
    if (obs->do_fd || do_sync) po->fd += te * B_par * fd_forefactor * delta_d;
    if (do_sync) {
      double jt, jp;
      hxo_sync_emissivity(m, obs->observer, obs->sync_freq, pos, B_per, &jt, &jp);
      const double Jtot = jt * delta_d * i2bt_sync;
      const double Jpol = jp * delta_d * i2bt_sync;
      po->is += Jtot;
      const double qui = (inner_shells_fd + po->fd) * lambda_square + sync_ipa(B, THE, PHI);
      po->qs += cos(2. * qui) * Jpol;
      po->us += sin(2. * qui) * Jpol;
    }
  }
}

static int models_supported(const hxg_models_t *m) {
  switch (m->breg) {
    case HXG_BREG_NONE: case HXG_BREG_GRID: case HXG_BREG_LSA:
    case HXG_BREG_UNIF: case HXG_BREG_CART: case HXG_BREG_HELIX:
    case HXG_BREG_SPIRAL:
      break;
    default:
      return 0;
  }
  switch (m->tereg) {
    case HXG_TEREG_NONE: case HXG_TEREG_GRID: case HXG_TEREG_UNIF:
    case HXG_TEREG_EXPDISK:
      break;
    default:
      return 0;
  }
  return 1;
}

int hxo_write_grid(const hxg_obs_t *obs, const hxg_models_t *m,
                   const hxo_grids_t *grids, uint32_t mask_nside,
                   const double *mask, double *dm, double *fd, double *is,
                   double *qs, double *us) {
  if (!models_supported(m)) return HXG_ERR_UNSUPPORTED;
  if (obs->do_sync && m->cre != HXG_CRE_ANA && m->cre != HXG_CRE_UNIF)
    return HXG_ERR_UNSUPPORTED;
  ctx_t c = {obs, m, grids};
  /* Grid_obs::build_grid (source/grid/grid_obs.cc:21-43): the FD map read
   * for the inner-shell cache is the do_fd output map when requested, else
   * a zero map at nside_sync that is never accumulated.                    */
  const uint32_t nside_fdmap = obs->do_fd ? obs->nside_fd : obs->nside_sync;
  double *fdmap = NULL;
  if (obs->do_fd || obs->do_sync) {
    if (obs->do_fd) {
      fdmap = fd;
    } else {
      fdmap = (double *)calloc(12ull * nside_fdmap * nside_fdmap, sizeof(double));
    }
    if (obs->do_fd)
      for (uint64_t i = 0; i < 12ull * obs->nside_fd * obs->nside_fd; ++i) fd[i] = 0.;
  }
  if (obs->do_dm)
    for (uint64_t i = 0; i < 12ull * obs->nside_dm * obs->nside_dm; ++i) dm[i] = 0.;
  if (obs->do_sync) {
    const uint64_t n = 12ull * obs->nside_sync * obs->nside_sync;
    for (uint64_t i = 0; i < n; ++i) is[i] = qs[i] = us[i] = 0.;
  }
  const hpx_t hfd = hpx_make(nside_fdmap ? nside_fdmap : 1);
  for (uint32_t s = 0; s < obs->total_shell; ++s) {
    const uint32_t ns = obs->nside_shell[s];
    const hpx_t hs = hpx_make(ns);
    const uint64_t npix = hs.npix;
    double *smask = NULL;
    if (obs->do_mask) {
      smask = (double *)malloc(sizeof(double) * npix);
      hxo_mask_duplicate(mask_nside, mask, ns, smask);
    }
    double *t_dm = (double *)calloc(npix, sizeof(double));
    double *t_fd = (double *)calloc(npix, sizeof(double));
    double *t_is = (double *)calloc(npix, sizeof(double));
    double *t_qs = (double *)calloc(npix, sizeof(double));
    double *t_us = (double *)calloc(npix, sizeof(double));
    double d_start, delta_d;
    uint64_t step;
    hxo_shell_ref(obs, s, &d_start, &delta_d, &step);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t ip = 0; ip < (int64_t)npix; ++ip) {
      pixobs_t po = {0., 0., 0., 0., 0.};
      if (!obs->do_mask || smask[ip] == 1.0) {
        double the, phi;
        hpx_pix2ang(&hs, (uint64_t)ip, &the, &phi);
        if (obs->do_fd || obs->do_sync) po.fd = hpx_interpolate(&hfd, fdmap, the, phi);
        radial_integration(&c, d_start, delta_d, step, the, phi, &po);
      }
      if (obs->do_dm) t_dm[ip] = po.dm;
      if (obs->do_sync) {
        t_is[ip] = hxo_temp_convert(po.is, obs->sync_freq);
        t_qs[ip] = hxo_temp_convert(po.qs, obs->sync_freq);
        t_us[ip] = hxo_temp_convert(po.us, obs->sync_freq);
      }
      if (obs->do_fd || obs->do_sync) t_fd[ip] = po.fd;
    }
    if (obs->do_dm) hxo_accumulate(obs->nside_dm, dm, ns, t_dm);
    if (obs->do_sync) {
      hxo_accumulate(obs->nside_sync, is, ns, t_is);
      hxo_accumulate(obs->nside_sync, qs, ns, t_qs);
      hxo_accumulate(obs->nside_sync, us, ns, t_us);
    }
    if (obs->do_fd) hxo_accumulate(obs->nside_fd, fd, ns, t_fd);
    free(t_dm);
    free(t_fd);
    free(t_is);
    free(t_qs);
    free(t_us);
    free(smask);
  }
  if (fdmap && !obs->do_fd) free(fdmap);
  return 0;
}
