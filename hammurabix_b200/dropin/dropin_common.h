// dropin_common.h -- state and model mapping shared by the drop-in
// translation units (integrator_b200.cc, generators_b200.cc): one device
// handle per process, so a grid made by a generator stays in its slot for
// the integrator.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
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

// What a device slot holds: the host arrays it was uploaded from (or
// downloaded into), their geometry and a fingerprint of their contents.  A
// host address alone does not identify a grid: a second Pipeline in the
// same process can get a recycled address for a new Grid_* array, and a
// caller can rewrite an array in place between runs (a sampling loop), so
// an upload is skipped only when all three match.
struct SlotKey {
  bool valid = false;
  const void *ptr[3] = {nullptr, nullptr, nullptr};
  hxg_grid_desc_t desc{};
  uint64_t fp[3] = {0, 0, 0};
};

inline bool same_desc(const hxg_grid_desc_t &a, const hxg_grid_desc_t &b) {
  return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.nE == b.nE && a.x_min == b.x_min &&
         a.x_max == b.x_max && a.y_min == b.y_min && a.y_max == b.y_max &&
         a.z_min == b.z_min && a.z_max == b.z_max && a.E_min == b.E_min &&
         a.E_max == b.E_max && a.E_fact == b.E_fact;
}

inline bool same_key(const SlotKey &a, const SlotKey &b) {
  if (!a.valid || !b.valid || !same_desc(a.desc, b.desc)) return false;
  for (int k = 0; k < 3; ++k)
    if (a.ptr[k] != b.ptr[k] || a.fp[k] != b.fp[k]) return false;
  return true;
}

// Content fingerprint of n doubles: the sum over 8-byte words of a mixed
// hash of (word, index) -- the splitmix64 finaliser (Steele, Lea & Flood,
// OOPSLA 2014) -- so a change of any word or a swap of two words changes
// it.  Summed by all host threads: bound by host memory bandwidth.
inline uint64_t fingerprint(const double *p, size_t n) {
  if (p == nullptr) return 0;
  uint64_t acc = 0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
  for (long long i = 0; i < (long long)n; ++i) {
    uint64_t x;
    std::memcpy(&x, p + i, sizeof(x));
    x ^= 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    acc += x ^ (x >> 31);
  }
  return acc ^ (uint64_t)n;
}

inline size_t values_per_component(const hxg_grid_desc_t &d) {
  return (size_t)d.nx * d.ny * d.nz * (d.nE ? d.nE : 1);
}

inline SlotKey key_of(const hxg_grid_desc_t &d, const double *x, const double *y,
                      const double *z) {
  SlotKey k;
  k.valid = true;
  k.desc = d;
  const double *c[3] = {x, y, z};
  const size_t n = values_per_component(d);
  for (int j = 0; j < 3; ++j) {
    k.ptr[j] = c[j];
    k.fp[j] = fingerprint(c[j], n);
  }
  return k;
}

// One device handle per process, re-used across frequency passes
// (Pipeline::assemble_obs calls write_grid once per <sync> entry).
struct DeviceState {
  hxg_handle *h = nullptr;
  int precision = HXG_FP64;
  SlotKey slots[5];
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

// Uploads the host arrays into the slot unless it already holds exactly
// these contents at this geometry.
inline void upload_vec(DeviceState &s, int slot, const hxg_grid_desc_t &d,
                       const double *x, const double *y, const double *z) {
  const SlotKey k = key_of(d, x, y, z);
  if (same_key(k, s.slots[slot])) return;
  s.slots[slot].valid = false;
  check(hxg_upload_grid(s.h, slot, &d, x, y, z), s.h, "hxg_upload_grid");
  s.slots[slot] = k;
}

// Records that the slot's device contents were copied into these host
// arrays (a device generator's output).
inline void mark_resident(DeviceState &s, int slot, const hxg_grid_desc_t &d,
                          const double *x, const double *y, const double *z) {
  s.slots[slot] = key_of(d, x, y, z);
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
      // Param reads a phase and an amplitude for four arms
      // (param.cc:207-227); more arms than it holds, or than the device
      // block holds, would be read past the end (the reference reads past
      // its vectors): refused
      if (j.arm_num > j.arm_amp.size() || j.arm_num > j.arm_phi0.size() || j.arm_num > 8)
        throw std::runtime_error("hammurabiX-B200: Breg_jaffe arm_num " +
                                 std::to_string(j.arm_num) + " exceeds the " +
                                 std::to_string(std::min<std::size_t>(
                                     8, std::min(j.arm_amp.size(), j.arm_phi0.size()))) +
                                 " arms given");
      d.arm_num = static_cast<uint32_t>(j.arm_num);
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
