// dropin_common.h -- state and model mapping shared by the drop-in
// translation units (integrator_b200.cc, generators_b200.cc): one device
// handle per process, so a grid made by a generator stays in its slot for
// the integrator.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <typeinfo>

#include <bfield.h>
#include <grid.h>
#include <param.h>

#include "../../include/hxg.h"

namespace hxg_dropin {

inline void check(int st, hxg_handle *h, const char *what) {
  if (st != HXG_OK) {
    std::string msg = std::string("hammurabiX-B200: ") + what + " failed (status " +
                      std::to_string(st) + ")";
    if (h) msg += std::string(": ") + hxg_last_error(h);
    throw std::runtime_error(msg);
  }
}

// One device handle per process, re-used across frequency passes
// (Pipeline::assemble_obs calls write_grid once per <sync> entry).
struct DeviceState {
  hxg_handle *h = nullptr;
  int precision = HXG_FP64;
  const void *uploaded[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  ~DeviceState() {
    if (h) hxg_destroy(h);
  }
};

inline DeviceState &state() {
  static DeviceState s;
  if (!s.h) {
    const char *p = std::getenv("HAMMURABIX_PRECISION");
    const int prec = (p && std::string(p) == "fp32c") ? HXG_FP32C : HXG_FP64;
    const char *d = std::getenv("HAMMURABIX_DEVICE");
    check(hxg_create(d ? std::atoi(d) : 0, prec, &s.h), nullptr, "hxg_create");
    s.precision = prec;
  }
  return s;
}

template <typename P>
inline hxg_grid_desc_t desc_of(const P &g) {
  hxg_grid_desc_t d{};
  d.nx = static_cast<uint32_t>(g.nx);
  d.ny = static_cast<uint32_t>(g.ny);
  d.nz = static_cast<uint32_t>(g.nz);
  d.x_min = g.x_min;
  d.x_max = g.x_max;
  d.y_min = g.y_min;
  d.y_max = g.y_max;
  d.z_min = g.z_min;
  d.z_max = g.z_max;
  return d;
}

inline void upload_vec(DeviceState &s, int slot, const hxg_grid_desc_t &d,
                       const double *x, const double *y, const double *z) {
  if (s.uploaded[slot] == x) return;
  check(hxg_upload_grid(s.h, slot, &d, x, y, z), s.h, "hxg_upload_grid");
  s.uploaded[slot] = x;
}

// The regular-field part of the reference's model selection
// (pipeline.cc:33-84, breg.cc:11-26): m.breg and its parameter block, the
// BREG grid uploaded when it is read from a file.
inline void map_breg(DeviceState &s, const Breg *breg, const Grid_breg *gbreg,
                     const Param *par, hxg_models_t &m) {
  if (par->grid_breg.read_permission) {
    m.breg = HXG_BREG_GRID;
    upload_vec(s, HXG_FIELD_BREG, desc_of(par->grid_breg), gbreg->bx.get(),
               gbreg->by.get(), gbreg->bz.get());
  } else if (par->grid_breg.build_permission) {
    if (dynamic_cast<const Breg_lsa *>(breg)) {
      m.breg = HXG_BREG_LSA;
      m.lsa = {par->breg_lsa.b0, par->breg_lsa.psi0, par->breg_lsa.psi1,
               par->breg_lsa.chi0};
    } else if (dynamic_cast<const Breg_unif *>(breg)) {
      m.breg = HXG_BREG_UNIF;
      m.unif = {par->breg_unif.bp, par->breg_unif.bv, par->breg_unif.l0};
    } else if (dynamic_cast<const Breg_cart *>(breg)) {
      m.breg = HXG_BREG_CART;
      m.cart = {par->breg_cart.bx, par->breg_cart.by, par->breg_cart.bz};
    } else if (dynamic_cast<const Breg_helix *>(breg)) {
      m.breg = HXG_BREG_HELIX;
      m.helix = {par->breg_helix.bx, par->breg_helix.by, par->breg_helix.bz,
                 par->breg_helix.r_min, par->breg_helix.r_max};
    } else if (dynamic_cast<const Breg_jaffe *>(breg)) {
      m.breg = HXG_BREG_JAFFE;
      const auto &j = par->breg_jaffe;
      auto &d = m.jaffe;
      d.quadruple = j.quadruple;
      d.bss = j.bss;
      d.ring = j.ring;
      d.bar = j.bar;
      d.arm_num = (uint32_t)std::min<std::size_t>(j.arm_num, 8);
      d.disk_amp = j.disk_amp;
      d.disk_z0 = j.disk_z0;
      d.halo_amp = j.halo_amp;
      d.halo_z0 = j.halo_z0;
      d.r_inner = j.r_inner;
      d.r_scale = j.r_scale;
      d.r_peak = j.r_peak;
      d.ring_amp = j.ring_amp;
      d.bar_amp = j.bar_amp;
      d.ring_r = j.ring_r;
      d.bar_a = j.bar_a;
      d.bar_b = j.bar_b;
      d.bar_phi0 = j.bar_phi0;
      for (std::size_t k = 0; k < j.arm_amp.size() && k < 8; ++k) d.arm_amp[k] = j.arm_amp[k];
      for (std::size_t k = 0; k < j.arm_phi0.size() && k < 8; ++k) d.arm_phi0[k] = j.arm_phi0[k];
      d.arm_pitch = j.arm_pitch;
      d.arm_r0 = j.arm_r0;
      d.arm_z0 = j.arm_z0;
      d.comp_r = j.comp_r;
      d.comp_c = j.comp_c;
      d.comp_d = j.comp_d;
      d.comp_p = j.comp_p;
    } else if (dynamic_cast<const Breg_jf12 *>(breg)) {
      m.breg = HXG_BREG_JF12;
      const auto &j = par->breg_jf12;
      m.jf12 = {j.b_arm1, j.b_arm2, j.b_arm3, j.b_arm4, j.b_arm5, j.b_arm6, j.b_arm7,
                j.b_ring, j.h_disk, j.w_disk, j.Bn, j.Bs, j.rn, j.rs, j.wh, j.z0,
                j.B0_X, j.Xtheta, j.rpc_X, j.r0_X};
    } else if (typeid(*breg) == typeid(Breg)) {
      m.breg = HXG_BREG_NONE;
    } else {
      throw std::runtime_error("hammurabiX-B200: unsupported breg model");
    }
  } else {
    m.breg = HXG_BREG_NONE;
  }
}

}  // namespace hxg_dropin
