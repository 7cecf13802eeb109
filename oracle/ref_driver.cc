/*
 * ref_driver.cc -- drives the reference hammurabiX integrator from the
 * hxg_* structs, for validation and CPU-baseline timing.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
 * reference's own, unmodified sources (read in place from the hammurabiX
 * tree) into oracle/_ref/libhxref.so.  It fills the reference's public
 * Param / Grid_* members directly (no XML, no file I/O), instantiates the
 * reference's field classes, and times Integrator::write_grid alone with
 * std::chrono, as the reference's own loop runs it (OpenMP over pixels).
 *
 * This translation unit is built without NDEBUG so that the reference's
 * NDEBUG-only access specifiers (include/integrator.h:29-31, 81-83) do not
 * hide the helpers it exposes for known-answer checks.
 */
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <omp.h>
#include <vector>

#include <bfield.h>
#include <crefield.h>
#include <grid.h>
#include <hamdis.h>
#include <hamsk.h>
#include <hamunits.h>
#include <integrator.h>
#include <param.h>
#include <tefield.h>
#include <gsl/gsl_rng.h>

#include "hxo.h"

namespace {

// Exponential-disk logarithmic spiral: the hxg_breg_spiral_t definition
// (include/hxg.h), written as a Breg subclass through the reference's own
// extension point (include/bfield.h:63-64).
class BregSpiral final : public Breg {
 public:
  explicit BregSpiral(const hxg_breg_spiral_t &p) : p_(p) {}
  Hamvec<3, ham_float> write_field(const Hamvec<3, ham_float> &pos,
                                   const Param *par) const override {
    const ham_float r{std::sqrt(pos[0] * pos[0] + pos[1] * pos[1])};
    if (r > (20. * cgs::kpc) or r < (3. * cgs::kpc)) {
      return Hamvec<3, ham_float>{0., 0., 0.};
    }
    const ham_float rsun{std::sqrt(par->observer[0] * par->observer[0] +
                                   par->observer[1] * par->observer[1])};
    const ham_float cos_p{pos[0] / r};
    const ham_float sin_p{pos[1] / r};
    const ham_float amp{p_.b0 * std::exp(-(r - rsun) / p_.r_scale) *
                        std::exp(-std::fabs(pos[2]) / p_.h_scale)};
    const ham_float sp{std::sin(p_.pitch)}, cp{std::cos(p_.pitch)};
    return Hamvec<3, ham_float>{amp * (sp * cos_p - cp * sin_p),
                                amp * (sp * sin_p + cp * cos_p), 0.};
  }

 private:
  hxg_breg_spiral_t p_;
};

// Exponential electron disk: the hxg_tereg_expdisk_t definition.
class TEregExpdisk final : public TEreg {
 public:
  explicit TEregExpdisk(const hxg_tereg_expdisk_t &p) : p_(p) {}
  ham_float write_field(const Hamvec<3, ham_float> &pos,
                        const Param *) const override {
    const ham_float r{std::sqrt(pos[0] * pos[0] + pos[1] * pos[1])};
    return p_.n0 * std::exp(-r / p_.r_scale) *
           std::exp(-std::fabs(pos[2]) / p_.h_scale);
  }

 private:
  hxg_tereg_expdisk_t p_;
};

// Exposes the reference's protected helpers.
class IntegratorProbe : public Integrator {
 public:
  using Integrator::assemble_shell_ref;
  using Integrator::los_parproj;
  using Integrator::los_perproj;
  using Integrator::los_versor;
  using Integrator::sync_emissivity_p;
  using Integrator::sync_emissivity_t;
  using Integrator::sync_ipa;
  using Integrator::temp_convert;
  using Integrator::struct_shell;
};

template <typename P>
void set_box(P &g, const hxg_grid_desc_t &d) {
  g.nx = d.nx;
  g.ny = d.ny;
  g.nz = d.nz;
  g.full_size = static_cast<ham_uint>(d.nx) * d.ny * d.nz;
  g.x_min = d.x_min;
  g.x_max = d.x_max;
  g.y_min = d.y_min;
  g.y_max = d.y_max;
  g.z_min = d.z_min;
  g.z_max = d.z_max;
}

std::unique_ptr<ham_float[]> copy_array(const double *src, size_t n) {
  auto a = std::make_unique<ham_float[]>(n);
  std::memcpy(a.get(), src, n * sizeof(double));
  return a;
}

void fill_obs(Param *par, const hxg_obs_t *obs) {
  par->observer =
      Hamvec<3, ham_float>{obs->observer[0], obs->observer[1], obs->observer[2]};
  auto &go = par->grid_obs;
  go.total_shell = obs->total_shell;
  go.nside_shell.assign(obs->nside_shell, obs->nside_shell + obs->total_shell);
  go.radii_shell.assign(obs->radii_shell,
                        obs->radii_shell + obs->total_shell + 1);
  go.oc_r_res = obs->oc_r_res;
  go.gc_r_min = obs->gc_r_min;
  go.gc_r_max = obs->gc_r_max;
  go.gc_z_min = obs->gc_z_min;
  go.gc_z_max = obs->gc_z_max;
  go.do_dm = obs->do_dm != 0;
  go.do_fd = obs->do_fd != 0;
  go.do_sync.assign(1, obs->do_sync != 0);
  go.sim_sync_freq.assign(1, obs->sync_freq);
  go.nside_sync.assign(1, obs->nside_sync);
  go.nside_dm = obs->nside_dm;
  go.nside_fd = obs->nside_fd;
  go.do_mask = false;
  go.write_permission = true;
}

struct Fields {
  std::unique_ptr<Breg> breg;
  std::unique_ptr<Brnd> brnd;
  std::unique_ptr<TEreg> tereg;
  std::unique_ptr<TErnd> ternd;
  std::unique_ptr<CREfield> cre;
  std::unique_ptr<Grid_breg> gbreg;
  std::unique_ptr<Grid_brnd> gbrnd;
  std::unique_ptr<Grid_tereg> gtereg;
  std::unique_ptr<Grid_ternd> gternd;
  std::unique_ptr<Grid_cre> gcre;
};

// Reproduces the reference's model selection (Pipeline::assemble_*,
// source/pipeline/pipeline.cc:33-162) for an hxg_models_t.
int build_fields(Param *par, const hxg_models_t *m, const hxo_grids_t *g,
                 Fields *f) {
  f->gbreg = std::make_unique<Grid_breg>();
  f->gbrnd = std::make_unique<Grid_brnd>();
  f->gtereg = std::make_unique<Grid_tereg>();
  f->gternd = std::make_unique<Grid_ternd>();
  f->gcre = std::make_unique<Grid_cre>();
  par->grid_breg.read_permission = par->grid_breg.build_permission = false;
  switch (m->breg) {
    case HXG_BREG_NONE:
      f->breg = std::make_unique<Breg>();
      break;
    case HXG_BREG_GRID: {
      const hxo_grid_t &s = g->slot[HXG_FIELD_BREG];
      set_box(par->grid_breg, s.desc);
      par->grid_breg.read_permission = true;
      par->grid_breg.build_permission = true;
      const size_t n = par->grid_breg.full_size;
      f->gbreg->bx = copy_array(s.c[0], n);
      f->gbreg->by = copy_array(s.c[1], n);
      f->gbreg->bz = copy_array(s.c[2], n);
      f->breg = std::make_unique<Breg>();
      break;
    }
    case HXG_BREG_LSA:
      par->grid_breg.build_permission = true;
      par->breg_lsa.b0 = m->lsa.b0;
      par->breg_lsa.psi0 = m->lsa.psi0;
      par->breg_lsa.psi1 = m->lsa.psi1;
      par->breg_lsa.chi0 = m->lsa.chi0;
      f->breg = std::make_unique<Breg_lsa>();
      break;
    case HXG_BREG_UNIF:
      par->grid_breg.build_permission = true;
      par->breg_unif.bp = m->unif.bp;
      par->breg_unif.bv = m->unif.bv;
      par->breg_unif.l0 = m->unif.l0;
      f->breg = std::make_unique<Breg_unif>();
      break;
    case HXG_BREG_CART:
      par->grid_breg.build_permission = true;
      par->breg_cart.bx = m->cart.bx;
      par->breg_cart.by = m->cart.by;
      par->breg_cart.bz = m->cart.bz;
      f->breg = std::make_unique<Breg_cart>();
      break;
    case HXG_BREG_HELIX:
      par->grid_breg.build_permission = true;
      par->breg_helix.bx = m->helix.bx;
      par->breg_helix.by = m->helix.by;
      par->breg_helix.bz = m->helix.bz;
      par->breg_helix.r_min = m->helix.r_min;
      par->breg_helix.r_max = m->helix.r_max;
      f->breg = std::make_unique<Breg_helix>();
      break;
    case HXG_BREG_JAFFE: {
      par->grid_breg.build_permission = true;
      auto &j = par->breg_jaffe;
      const auto &s = m->jaffe;
      j.quadruple = s.quadruple;
      j.bss = s.bss;
      j.ring = s.ring;
      j.bar = s.bar;
      j.disk_amp = s.disk_amp;
      j.disk_z0 = s.disk_z0;
      j.halo_amp = s.halo_amp;
      j.halo_z0 = s.halo_z0;
      j.r_inner = s.r_inner;
      j.r_scale = s.r_scale;
      j.r_peak = s.r_peak;
      j.ring_amp = s.ring_amp;
      j.bar_amp = s.bar_amp;
      j.ring_r = s.ring_r;
      j.bar_a = s.bar_a;
      j.bar_b = s.bar_b;
      j.bar_phi0 = s.bar_phi0;
      j.arm_num = s.arm_num;
      j.arm_amp.assign(s.arm_amp, s.arm_amp + 4);
      j.arm_phi0.assign(s.arm_phi0, s.arm_phi0 + 4);
      j.arm_pitch = s.arm_pitch;
      j.arm_r0 = s.arm_r0;
      j.arm_z0 = s.arm_z0;
      j.comp_r = s.comp_r;
      j.comp_c = s.comp_c;
      j.comp_d = s.comp_d;
      j.comp_p = s.comp_p;
      f->breg = std::make_unique<Breg_jaffe>();
      break;
    }
    case HXG_BREG_JF12: {
      par->grid_breg.build_permission = true;
      auto &j = par->breg_jf12;
      const auto &s = m->jf12;
      j.b_arm1 = s.b_arm1;
      j.b_arm2 = s.b_arm2;
      j.b_arm3 = s.b_arm3;
      j.b_arm4 = s.b_arm4;
      j.b_arm5 = s.b_arm5;
      j.b_arm6 = s.b_arm6;
      j.b_arm7 = s.b_arm7;
      j.b_ring = s.b_ring;
      j.h_disk = s.h_disk;
      j.w_disk = s.w_disk;
      j.Bn = s.Bn;
      j.Bs = s.Bs;
      j.rn = s.rn;
      j.rs = s.rs;
      j.wh = s.wh;
      j.z0 = s.z0;
      j.B0_X = s.B0_X;
      j.Xtheta = s.Xtheta;
      j.rpc_X = s.rpc_X;
      j.r0_X = s.r0_X;
      f->breg = std::make_unique<Breg_jf12>();
      break;
    }
    case HXG_BREG_SPIRAL:
      par->grid_breg.build_permission = true;
      f->breg = std::make_unique<BregSpiral>(m->spiral);
      break;
    default:
      return HXG_ERR_UNSUPPORTED;
  }
  par->grid_brnd.read_permission = par->grid_brnd.build_permission = false;
  f->brnd = std::make_unique<Brnd>();
  if (m->brnd == HXG_BRND_GRID) {
    const hxo_grid_t &s = g->slot[HXG_FIELD_BRND];
    set_box(par->grid_brnd, s.desc);
    par->grid_brnd.read_permission = true;
    const size_t n = par->grid_brnd.full_size;
    f->gbrnd->bx = copy_array(s.c[0], n);
    f->gbrnd->by = copy_array(s.c[1], n);
    f->gbrnd->bz = copy_array(s.c[2], n);
  } else if (m->brnd != HXG_BRND_NONE) {
    return HXG_ERR_UNSUPPORTED;
  }
  par->grid_tereg.read_permission = par->grid_tereg.build_permission = false;
  switch (m->tereg) {
    case HXG_TEREG_NONE:
      f->tereg = std::make_unique<TEreg>();
      break;
    case HXG_TEREG_GRID: {
      const hxo_grid_t &s = g->slot[HXG_FIELD_TEREG];
      set_box(par->grid_tereg, s.desc);
      par->grid_tereg.read_permission = true;
      par->grid_tereg.build_permission = true;
      f->gtereg->te = copy_array(s.c[0], par->grid_tereg.full_size);
      f->tereg = std::make_unique<TEreg>();
      break;
    }
    case HXG_TEREG_UNIF:
      par->grid_tereg.build_permission = true;
      par->tereg_unif.n0 = m->te_unif.n0;
      par->tereg_unif.r0 = m->te_unif.r0;
      f->tereg = std::make_unique<TEreg_unif>();
      break;
    case HXG_TEREG_YMW16: {
      par->grid_tereg.build_permission = true;
      static_assert(sizeof(par->tereg_ymw16) == sizeof(m->ymw16),
                    "ymw16 parameter block layout");
      std::memcpy(&par->tereg_ymw16, &m->ymw16, sizeof(m->ymw16));
      f->tereg = std::make_unique<TEreg_ymw16>();
      break;
    }
    case HXG_TEREG_EXPDISK:
      par->grid_tereg.build_permission = true;
      f->tereg = std::make_unique<TEregExpdisk>(m->te_exp);
      break;
    default:
      return HXG_ERR_UNSUPPORTED;
  }
  par->grid_ternd.read_permission = par->grid_ternd.build_permission = false;
  f->ternd = std::make_unique<TErnd>();
  if (m->ternd == HXG_TERND_GRID) {
    const hxo_grid_t &s = g->slot[HXG_FIELD_TERND];
    set_box(par->grid_ternd, s.desc);
    par->grid_ternd.read_permission = true;
    f->gternd->te = copy_array(s.c[0], par->grid_ternd.full_size);
  } else if (m->ternd != HXG_TERND_NONE) {
    return HXG_ERR_UNSUPPORTED;
  }
  par->grid_cre.read_permission = par->grid_cre.build_permission = false;
  switch (m->cre) {
    case HXG_CRE_NONE:
      break;
    case HXG_CRE_ANA:
      par->grid_cre.build_permission = true;
      par->cre_ana.alpha = m->cre_ana.alpha;
      par->cre_ana.beta = m->cre_ana.beta;
      par->cre_ana.theta = m->cre_ana.theta;
      par->cre_ana.r0 = m->cre_ana.r0;
      par->cre_ana.z0 = m->cre_ana.z0;
      par->cre_ana.E0 = m->cre_ana.E0;
      par->cre_ana.j0 = m->cre_ana.j0;
      f->cre = std::make_unique<CRE_ana>();
      break;
    case HXG_CRE_UNIF:
      par->grid_cre.build_permission = true;
      par->cre_unif.alpha = m->cre_unif.alpha;
      par->cre_unif.r0 = m->cre_unif.r0;
      par->cre_unif.E0 = m->cre_unif.E0;
      par->cre_unif.j0 = m->cre_unif.j0;
      f->cre = std::make_unique<CRE_unif>();
      break;
    case HXG_CRE_GRID: {
      const hxo_grid_t &s = g->slot[HXG_FIELD_CRE];
      auto &gc = par->grid_cre;
      gc.read_permission = true;
      gc.nx = s.desc.nx;
      gc.ny = s.desc.ny;
      gc.nz = s.desc.nz;
      gc.nE = s.desc.nE;
      gc.x_min = s.desc.x_min;
      gc.x_max = s.desc.x_max;
      gc.y_min = s.desc.y_min;
      gc.y_max = s.desc.y_max;
      gc.z_min = s.desc.z_min;
      gc.z_max = s.desc.z_max;
      gc.E_min = s.desc.E_min;
      gc.E_max = s.desc.E_max;
      gc.E_fact = s.desc.E_fact;
      gc.cre_size = static_cast<ham_uint>(gc.nE) * gc.nx * gc.ny * gc.nz;
      f->gcre->cre_flux = copy_array(s.c[0], gc.cre_size);
      f->cre = std::make_unique<CRE_num>();
      break;
    }
    default:
      return HXG_ERR_UNSUPPORTED;
  }
  return HXG_OK;
}

void copy_map(const Hampix<ham_float> &m, double *out) {
  for (ham_uint i = 0; i < m.npix(); ++i) out[i] = m.data(i);
}

}  // namespace

extern "C" {

/* Integrator::write_grid on the reference, timed alone. */
int hxref_write_grid(const hxg_obs_t *obs, const hxg_models_t *m,
                     const hxo_grids_t *grids, uint32_t mask_nside,
                     const double *mask, double *dm, double *fd, double *is,
                     double *qs, double *us, int nthreads, double *seconds) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  auto par = std::make_unique<Param>();
  fill_obs(par.get(), obs);
  Fields f;
  const int st = build_fields(par.get(), m, grids, &f);
  if (st != HXG_OK) return st;
  if (obs->do_sync and not f.cre) return HXG_ERR_INVALID;
  auto gobs = std::make_unique<Grid_obs>(par.get());
  if (obs->do_mask) {
    Hampix<ham_float> pivot(mask_nside);
    for (ham_uint i = 0; i < pivot.npix(); ++i) pivot.data(i, mask[i]);
    gobs->mask_map = std::make_unique<Hampisk<ham_float>>(pivot);
    par->grid_obs.do_mask = true;
    par->grid_obs.nside_mask = mask_nside;
  }
  Integrator integ;
  const auto t0 = std::chrono::steady_clock::now();
  integ.write_grid(f.breg.get(), f.brnd.get(), f.tereg.get(), f.ternd.get(),
                   f.cre.get(), f.gbreg.get(), f.gbrnd.get(), f.gtereg.get(),
                   f.gternd.get(), f.gcre.get(), gobs.get(), par.get());
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (obs->do_dm and dm) copy_map(*gobs->dm_map, dm);
  if (obs->do_fd and fd) copy_map(*gobs->fd_map, fd);
  if (obs->do_sync) {
    if (is) copy_map(*gobs->is_map, is);
    if (qs) copy_map(*gobs->qs_map, qs);
    if (us) copy_map(*gobs->us_map, us);
  }
  return HXG_OK;
}

int hxref_max_threads(void) { return omp_get_max_threads(); }

/* ---- known-answer helpers on the reference's own code ---------------- */
void hxref_pix2ang(uint32_t nside, double *theta, double *phi) {
  Hampix<ham_float> m(nside);
  for (ham_uint i = 0; i < m.npix(); ++i) {
    theta[i] = m.pointing(i).theta();
    phi[i] = m.pointing(i).phi();
  }
}

void hxref_interpolate(uint32_t nside, const double *map, uint64_t n,
                       const double *theta, const double *phi, double *out) {
  std::vector<ham_float> v(map, map + 12ull * nside * nside);
  Hampix<ham_float> m(nside, v);
  for (uint64_t i = 0; i < n; ++i) out[i] = m.interpolate(Hamp(theta[i], phi[i]));
}

void hxref_accumulate(uint32_t nside_dst, double *dst, uint32_t nside_src,
                      const double *src) {
  std::vector<ham_float> vd(dst, dst + 12ull * nside_dst * nside_dst);
  std::vector<ham_float> vs(src, src + 12ull * nside_src * nside_src);
  Hampix<ham_float> md(nside_dst, vd), ms(nside_src, vs);
  md.accumulate(ms);
  copy_map(md, dst);
}

void hxref_mask_duplicate(uint32_t pivot_nside, const double *pivot_mask,
                          uint32_t nside, double *out) {
  std::vector<ham_float> v(pivot_mask, pivot_mask + 12ull * pivot_nside * pivot_nside);
  Hampix<ham_float> pm(pivot_nside, v);
  Hampisk<ham_float> mk(pm);
  mk.duplicate(nside);
  for (ham_uint i = 0; i < 12ull * nside * nside; ++i) out[i] = mk.data(nside, i);
}

void hxref_shell_ref(const hxg_obs_t *obs, uint32_t shell, double *d_start,
                     double *delta_d, uint64_t *step, double *dist) {
  auto par = std::make_unique<Param>();
  fill_obs(par.get(), obs);
  IntegratorProbe p;
  IntegratorProbe::struct_shell s;
  p.assemble_shell_ref(&s, par.get(), shell);
  *d_start = s.d_start;
  *delta_d = s.delta_d;
  *step = s.step;
  if (dist)
    for (ham_uint i = 0; i < s.step; ++i) dist[i] = s.dist[i];
}

void hxref_los_geometry(uint64_t n, const double *theta, const double *phi,
                        const double *b, double *versor, double *b_par,
                        double *b_per, double *ipa) {
  IntegratorProbe p;
  for (uint64_t i = 0; i < n; ++i) {
    const Hamvec<3, ham_float> u = p.los_versor(theta[i], phi[i]);
    const Hamvec<3, ham_float> B{b[3 * i], b[3 * i + 1], b[3 * i + 2]};
    for (int c = 0; c < 3; ++c) versor[3 * i + c] = u[c];
    b_par[i] = p.los_parproj(B, u);
    b_per[i] = p.los_perproj(B, u);
    ipa[i] = p.sync_ipa(B, theta[i], phi[i]);
  }
}

double hxref_temp_convert(double temp_br, double freq) {
  IntegratorProbe p;
  return p.temp_convert(temp_br, freq);
}

/* Breg / TEreg read_grid and analytic write_field through the reference. */
int hxref_read_field(int field, const hxg_models_t *m, const hxo_grids_t *g,
                     const double observer[3], uint64_t n, const double *pos,
                     double *out) {
  auto par = std::make_unique<Param>();
  par->observer = Hamvec<3, ham_float>{observer[0], observer[1], observer[2]};
  Fields f;
  const int st = build_fields(par.get(), m, g, &f);
  if (st != HXG_OK) return st;
  for (uint64_t i = 0; i < n; ++i) {
    const Hamvec<3, ham_float> p{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    if (field == HXG_FIELD_BREG or field == HXG_FIELD_BRND) {
      const Hamvec<3, ham_float> v =
          field == HXG_FIELD_BREG ? f.breg->read_field(p, par.get(), f.gbreg.get())
                                  : f.brnd->read_field(p, par.get(), f.gbrnd.get());
      for (int c = 0; c < 3; ++c) out[3 * i + c] = v[c];
    } else if (field == HXG_FIELD_TEREG) {
      out[i] = f.tereg->read_field(p, par.get(), f.gtereg.get());
    } else if (field == HXG_FIELD_TERND) {
      out[i] = f.ternd->read_field(p, par.get(), f.gternd.get());
    } else {
      return HXG_ERR_INVALID;
    }
  }
  return HXG_OK;
}

/* sync_emissivity_t / _p (integrator.cc:282-420) through the reference. */
int hxref_sync_emissivity(const hxg_models_t *m, const hxo_grids_t *g,
                          const double observer[3], double freq, uint64_t n,
                          const double *pos, const double *b_per, double *jt,
                          double *jp) {
  auto par = std::make_unique<Param>();
  par->observer = Hamvec<3, ham_float>{observer[0], observer[1], observer[2]};
  par->grid_obs.sim_sync_freq.assign(1, freq);
  par->grid_obs.do_sync.assign(1, true);
  Fields f;
  const int st = build_fields(par.get(), m, g, &f);
  if (st != HXG_OK) return st;
  if (not f.cre) return HXG_ERR_INVALID;
  IntegratorProbe p;
  for (uint64_t i = 0; i < n; ++i) {
    const Hamvec<3, ham_float> q{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    jt[i] = p.sync_emissivity_t(q, par.get(), f.cre.get(), f.gcre.get(), b_per[i]);
    jp[i] = p.sync_emissivity_p(q, par.get(), f.cre.get(), f.gcre.get(), b_per[i]);
  }
  return HXG_OK;
}

/* Brnd_es::write_grid / TErnd_dft::write_grid through the reference, run on
 * one thread with the shim's cell-indexed deviates (shim/gsl/gsl_rng.h), so
 * that draw t is deviate t % k of k-space cell 1 + t / k: the deviates the
 * device generators use.  The FFTs are the shim's direct-sum DFT. */
int hxref_generate_brnd_es(const hxg_models_t *m, const hxo_grids_t *g,
                           const double observer[3], const hxg_grid_desc_t *d,
                           const hxg_brnd_es_t *p, uint64_t seed, double *bx,
                           double *by, double *bz) {
  const int threads = omp_get_max_threads();
  omp_set_num_threads(1);
  hxo_shim_cell_stream(4);
  auto par = std::make_unique<Param>();
  par->observer = Hamvec<3, ham_float>{observer[0], observer[1], observer[2]};
  hxg_models_t mm = *m;
  mm.brnd = HXG_BRND_NONE;
  mm.tereg = HXG_TEREG_NONE;
  mm.ternd = HXG_TERND_NONE;
  mm.cre = HXG_CRE_NONE;
  Fields f;
  int st = build_fields(par.get(), &mm, g, &f);
  if (st == HXG_OK) {
    set_box(par->grid_brnd, *d);
    par->grid_brnd.build_permission = true;
    par->grid_brnd.read_permission = false;
    par->brnd_seed = seed;
    par->brnd_es.rms = p->rms;
    par->brnd_es.k0 = p->k0;
    par->brnd_es.k1 = p->k1;
    par->brnd_es.a0 = p->a0;
    par->brnd_es.a1 = p->a1;
    par->brnd_es.rho = p->rho;
    par->brnd_es.r0 = p->r0;
    par->brnd_es.z0 = p->z0;
    Grid_brnd grid(par.get());
    Brnd_es gen;
    gen.write_grid(par.get(), f.breg.get(), f.gbreg.get(), &grid);
    const size_t n = par->grid_brnd.full_size;
    std::memcpy(bx, grid.bx.get(), n * sizeof(double));
    std::memcpy(by, grid.by.get(), n * sizeof(double));
    std::memcpy(bz, grid.bz.get(), n * sizeof(double));
  }
  hxo_shim_cell_stream(0);
  omp_set_num_threads(threads);
  return st;
}

int hxref_generate_ternd_dft(const double observer[3], const hxg_grid_desc_t *d,
                             const hxg_ternd_dft_t *p, uint64_t seed, double *te) {
  const int threads = omp_get_max_threads();
  omp_set_num_threads(1);
  hxo_shim_cell_stream(2);
  auto par = std::make_unique<Param>();
  par->observer = Hamvec<3, ham_float>{observer[0], observer[1], observer[2]};
  set_box(par->grid_ternd, *d);
  par->grid_ternd.build_permission = true;
  par->grid_ternd.read_permission = false;
  // TErnd_dft seeds from brnd_seed (ternd_dft.cc:42-49)
  par->brnd_seed = seed;
  par->ternd_dft.rms = p->rms;
  par->ternd_dft.k0 = p->k0;
  par->ternd_dft.a0 = p->a0;
  par->ternd_dft.r0 = p->r0;
  par->ternd_dft.z0 = p->z0;
  {
    Grid_ternd grid(par.get());
    TErnd_dft gen;
    gen.write_grid(par.get(), nullptr, nullptr, &grid);
    std::memcpy(te, grid.te.get(), par->grid_ternd.full_size * sizeof(double));
  }
  hxo_shim_cell_stream(0);
  omp_set_num_threads(threads);
  return HXG_OK;
}

}  // extern "C"
