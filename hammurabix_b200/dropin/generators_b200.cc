// generators_b200.cc -- link-time drop-in for hammurabiX's random-field
// generators Brnd_es and TErnd_dft.
//
// Defines the reference's own
//   void Brnd_es::write_grid(const Param*, const Breg*, const Grid_breg*,
//                            Grid_brnd*) const;          (include/bfield.h:269-316)
//   void TErnd_dft::write_grid(const Param*, const TEreg*, const Grid_tereg*,
//                              Grid_ternd*) const;       (include/tefield.h:150-166)
// and the virtual helpers the two classes declare, on top of
// hxg_generate_brnd_es / hxg_generate_ternd_dft (include/hxg.h).  Compiled in
// place of source/field/b/brnd_es.cc and source/field/te/ternd_dft.cc.  The
// field is made in the device slot the drop-in integrator reads (one handle
// per process, dropin_common.h) and copied into the Grid_brnd / Grid_ternd
// arrays, so export_grid and any host reader see it.  The Gaussian deviates
// are the library's Philox stream, not GSL's taus: a seed gives another
// realisation than the reference with the same statistics.
#include <cmath>

#include <bfield.h>
#include <grid.h>
#include <hamunits.h>
#include <hamvec.h>
#include <param.h>
#include <tefield.h>

#include "../../include/hxg.h"
#include "dropin_common.h"

using namespace hxg_dropin;

void Brnd_es::write_grid(const Param *par, const Breg *breg, const Grid_breg *gbreg,
                         Grid_brnd *grid) const {
  DeviceState &s = state();
  // the anisotropy direction follows the regular field (brnd_es.cc:18-22)
  hxg_models_t m{};
  map_breg(s, breg, gbreg, par, m);
  check(hxg_set_models(s.h, &m), s.h, "hxg_set_models");
  const auto &e = par->brnd_es;
  const hxg_brnd_es_t p{e.rms, e.k0, e.k1, e.a0, e.a1, e.rho, e.r0, e.z0};
  const double obs[3] = {par->observer[0], par->observer[1], par->observer[2]};
  const hxg_grid_desc_t d = desc_of(par->grid_brnd);
  check(hxg_generate_brnd_es(s.h, &d, &p, obs, par->brnd_seed), s.h, "hxg_generate_brnd_es");
  check(hxg_download_grid(s.h, HXG_FIELD_BRND, grid->bx.get(), grid->by.get(), grid->bz.get()),
        s.h, "hxg_download_grid");
  mark_resident(s, HXG_FIELD_BRND, d, grid->bx.get(), grid->by.get(), grid->bz.get());
}

// Brnd_es::spectrum (brnd_es.cc:34-49): broken power law in k (1/kpc)
ham_float Brnd_es::spectrum(const ham_float &k, const Param *par) const {
  const auto &e = par->brnd_es;
  const ham_float below_k1 = k < e.k1 ? 1. : 0.;
  const ham_float mid = (k > e.k1 && k < e.k0) ? 1. : 0.;
  const ham_float above_k0 = k > e.k0 ? 1. : 0.;
  const ham_float shape = below_k1 * std::pow(e.k0 / e.k1, e.a1) * std::pow(k / e.k1, 6.) +
                          mid / std::pow(k / e.k0, e.a1) + above_k0 / std::pow(k / e.k0, e.a0);
  return shape * e.rms * e.rms / (4. * cgs::pi * k * k);
}

// Brnd_es::spatial_profile (brnd_es.cc:53-59): 1 at the observer
ham_float Brnd_es::spatial_profile(const Hamvec<3, ham_float> &pos, const Param *par) const {
  const ham_float r_cyl = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1]) -
                          std::fabs(par->observer[0]);
  const ham_float z = std::fabs(pos[2]) - std::fabs(par->observer[2]);
  return std::exp(-r_cyl / par->brnd_es.r0) * std::exp(-z / par->brnd_es.z0);
}

void TErnd_dft::write_grid(const Param *par, const TEreg *, const Grid_tereg *,
                           Grid_ternd *grid) const {
  DeviceState &s = state();
  const auto &t = par->ternd_dft;
  const hxg_ternd_dft_t p{t.rms, t.k0, t.a0, t.r0, t.z0};
  const double obs[3] = {par->observer[0], par->observer[1], par->observer[2]};
  const hxg_grid_desc_t d = desc_of(par->grid_ternd);
  // the reference seeds this generator from brnd_seed (ternd_dft.cc:42-49)
  check(hxg_generate_ternd_dft(s.h, &d, &p, obs, par->brnd_seed), s.h,
        "hxg_generate_ternd_dft");
  check(hxg_download_grid(s.h, HXG_FIELD_TERND, grid->te.get(), nullptr, nullptr), s.h,
        "hxg_download_grid");
  mark_resident(s, HXG_FIELD_TERND, d, grid->te.get(), nullptr, nullptr);
}

// TErnd_dft::spectrum (ternd_dft.cc:17-24): zero below k0
ham_float TErnd_dft::spectrum(const ham_float &k, const Param *par) const {
  const auto &t = par->ternd_dft;
  if (k < t.k0) return 0.;
  return t.rms * std::pow(k / t.k0, t.a0) / (4 * cgs::pi * k * k);
}

// TErnd_dft::spatial_profile (ternd_dft.cc:26-33)
ham_float TErnd_dft::spatial_profile(const Hamvec<3, ham_float> &pos, const Param *par) const {
  const ham_float r_cyl = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1]) -
                          std::fabs(par->observer[0]);
  const ham_float z = std::fabs(pos[2]) - std::fabs(par->observer[2]);
  return std::exp(-r_cyl / par->ternd_dft.r0) * std::exp(-z / par->ternd_dft.z0);
}
