// hxg_api.cu -- host glue of the C ABI (include/hxg.h): the B200
// replacement of Integrator::write_grid (source/integrator/integrator.cc:23-134).
//
// The shell loop, shell geometry, mask duplication and all per-launch
// constants run here in FP64 on the host; the per-pixel radial integration
// (hxg_integrate.cuh) and the shell merge (hxg_kernels.cu) run on the GPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <functional>
#include <thread>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/hxg.h"
#include "hxg_adjoint.cuh"
#include "hxg_adjoint32.cuh"
#include "hxg_batch.cuh"
#include "hxg_integrate.cuh"
#include "hxg_internal.h"

using namespace hxg;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct Slot {
  bool present = false;
  hxg_grid_desc_t desc{};
  double *d[3] = {nullptr, nullptr, nullptr};
  size_t n = 0;
};

struct Group {
  hxg_grid_desc_t desc{};
  int b_slots[2] = {-1, -1};
  int t_slots[2] = {-1, -1};
  void *rec = nullptr;
  size_t n = 0;
};

}  // namespace

struct hxg_handle {
  int device = 0;
  int precision = HXG_FP64;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  hxg_models_t models{};
  bool have_models = false;
  Slot slots[5];
  std::vector<Group> groups;
  bool groups_dirty = true;
  // bumped whenever a grid slot or a group's record array moves to new
  // device memory; a batch made before that refuses to run
  uint64_t layout_gen = 0;
  bool have_mask = false;
  uint32_t mask_nside = 0;
  std::vector<double> mask_host;
  std::map<uint32_t, unsigned char *> mask_dev;
  DevBuf tmp_fd;        // the shell FD map, merged after each shell
  DevBuf stage32;       // staged chunk of an FP32 host grid
  // FP32 host uploads: copies and widening on a stream of the greatest
  // priority, so that the widening is not queued behind the blocks of an
  // integration running on another stream
  cudaStream_t up_stream = nullptr;
  cudaEvent_t up_event = nullptr;
  cudaEvent_t switch_event = nullptr;  // hxg_set_stream's hand-over
  DevBuf shell_all;     // every shell's DM and Stokes maps of a pass
  // interpolation tables by (output Nside << 32 | shell Nside)
  std::map<uint64_t, DevBuf> interp;
  size_t interp_bytes = 0;
  size_t interp_limit = 8ull << 30;
  DevBuf out[5];
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  std::vector<int64_t> event_samples;
  double acc_ms = 0.;
  int64_t acc_launches = 0, acc_samples = 0;
  double waves = 4.0;
  int64_t launch_count = 0;
  // adjoint checkpoint of the last forward pass (FP64 form)
  bool checkpoint = false;
  bool ck_valid = false;
  hxg_obs_t ck_obs{};
  hxg_models_t ck_models{};
  std::vector<DevBuf> ck, ck_inner;
  std::vector<int> ck_chunks;
  // checkpoints of per-shell forward calls (hxg_shell_integrate_device):
  // which shells of pass ck_sobs, models ck_smodels and shard ck_shard of
  // ck_nshards hold one, and the sharded adjoint's next shell (-1: none open)
  std::vector<char> ck_shell;
  hxg_obs_t ck_sobs{};
  hxg_models_t ck_smodels{};
  uint32_t ck_shard = 0, ck_nshards = 1;
  int adj_next = -1;
  bool adj_open = false;
  DevBuf grad_rec, grad_par, g_shell[5], g_fdmap;
  DevBuf ext;  // ExtModels block of the current launches
  DevBuf cre_tab;  // synchrotron tables + CRE energy tables
  hxg::RfgWork *rfg = nullptr;  // random-field generator workspace
};

namespace {

int fail(hxg_handle *h, int code, const char *fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->err = buf;
  }
  return code;
}

int cuda_fail(hxg_handle *h, cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation)
    return fail(h, HXG_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return fail(h, HXG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define HXG_CK(call)                                       \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
  } while (0)

int ensure(hxg_handle *h, DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes) return HXG_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc");
  b.bytes = bytes;
  return HXG_OK;
}

bool is_pow2(uint32_t n) { return n > 0 && (n & (n - 1)) == 0; }

uint64_t npix_of(uint32_t nside) { return 12ull * nside * nside; }

bool same_geometry(const hxg_grid_desc_t &a, const hxg_grid_desc_t &b) {
  return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.x_min == b.x_min &&
         a.x_max == b.x_max && a.y_min == b.y_min && a.y_max == b.y_max &&
         a.z_min == b.z_min && a.z_max == b.z_max;
}

bool models_supported(const hxg_models_t &m, std::string *why) {
  switch (m.breg) {
    case HXG_BREG_NONE: case HXG_BREG_GRID: case HXG_BREG_LSA:
    case HXG_BREG_UNIF: case HXG_BREG_CART: case HXG_BREG_HELIX:
    case HXG_BREG_SPIRAL: case HXG_BREG_JAFFE: case HXG_BREG_JF12:
      break;
    default:
      *why = "regular B model not supported on the device";
      return false;
  }
  if (m.breg == HXG_BREG_JAFFE && m.jaffe.arm_num > 8) {
    *why = "Breg_jaffe with more than 8 spiral arms";
    return false;
  }
  if (m.brnd != HXG_BRND_NONE && m.brnd != HXG_BRND_GRID) {
    *why = "random B model must be NONE or GRID";
    return false;
  }
  switch (m.tereg) {
    case HXG_TEREG_NONE: case HXG_TEREG_GRID: case HXG_TEREG_UNIF:
    case HXG_TEREG_EXPDISK: case HXG_TEREG_YMW16:
      break;
    default:
      *why = "regular n_e model not supported on the device";
      return false;
  }
  if (m.ternd != HXG_TERND_NONE && m.ternd != HXG_TERND_GRID) {
    *why = "random n_e model must be NONE or GRID";
    return false;
  }
  if (m.cre != HXG_CRE_NONE && m.cre != HXG_CRE_ANA && m.cre != HXG_CRE_UNIF &&
      m.cre != HXG_CRE_GRID) {
    *why = "CRE model not supported on the device";
    return false;
  }
  return true;
}

// The slots whose grids the models read (Breg/Brnd/TEreg/TErnd::read_field,
// breg.cc:11-26, brnd.cc:12-23, tereg.cc:11-25, ternd.cc:12-19).
void active_slots(const hxg_models_t &m, bool act[4]) {
  act[HXG_FIELD_BREG] = m.breg == HXG_BREG_GRID;
  act[HXG_FIELD_BRND] = m.brnd == HXG_BRND_GRID;
  act[HXG_FIELD_TEREG] = m.tereg == HXG_TEREG_GRID;
  act[HXG_FIELD_TERND] = m.ternd == HXG_TERND_GRID;
}

void free_groups(hxg_handle *h) {
  for (auto &g : h->groups)
    if (g.rec) cudaFree(g.rec);
  h->groups.clear();
}

// Pack every active grid slot into per-geometry 4-component record arrays.
// New values in the same slots and geometries are packed into the record
// arrays already there, so plans that hold their addresses stay valid.
int build_groups(hxg_handle *h) {
  if (!h->groups_dirty) return HXG_OK;
  bool act[4];
  active_slots(h->models, act);
  std::vector<Group> next;
  for (int s = 0; s < 4; ++s) {
    if (!act[s]) continue;
    if (!h->slots[s].present)
      return fail(h, HXG_ERR_STATE, "model reads grid slot %d but no grid was uploaded", s);
    Group *grp = nullptr;
    for (auto &g : next)
      if (same_geometry(g.desc, h->slots[s].desc)) grp = &g;
    if (!grp) {
      next.emplace_back();
      grp = &next.back();
      grp->desc = h->slots[s].desc;
      grp->n = h->slots[s].n;
    }
    const bool is_b = (s == HXG_FIELD_BREG || s == HXG_FIELD_BRND);
    int *list = is_b ? grp->b_slots : grp->t_slots;
    if (list[0] < 0)
      list[0] = s;
    else
      list[1] = s;
  }
  if (next.size() > (size_t)kMaxGroups)
    return fail(h, HXG_ERR_UNSUPPORTED, "more than %d grid geometries", kMaxGroups);
  bool same = next.size() == h->groups.size();
  for (size_t i = 0; same && i < next.size(); ++i) {
    const Group &a = next[i], &b = h->groups[i];
    same = b.rec && a.n == b.n && same_geometry(a.desc, b.desc) &&
           std::memcmp(a.b_slots, b.b_slots, sizeof(a.b_slots)) == 0 &&
           std::memcmp(a.t_slots, b.t_slots, sizeof(a.t_slots)) == 0;
  }
  if (same) {
    for (size_t i = 0; i < next.size(); ++i) next[i].rec = h->groups[i].rec;
    h->groups.clear();
  } else {
    free_groups(h);
    ++h->layout_gen;
  }
  h->groups = std::move(next);
  const bool fp32 = h->precision == HXG_FP32C;
  const size_t esz = fp32 ? sizeof(float) : sizeof(double);
  for (auto &g : h->groups) {
    if (!g.rec) {
      cudaError_t e = cudaMalloc(&g.rec, g.n * 4 * esz);
      if (e != cudaSuccess) {
        free_groups(h);
        return cuda_fail(h, e, "cudaMalloc(grid records)");
      }
    }
    const double *b0[3] = {nullptr, nullptr, nullptr};
    const double *b1[3] = {nullptr, nullptr, nullptr};
    if (g.b_slots[0] >= 0)
      for (int k = 0; k < 3; ++k) b0[k] = h->slots[g.b_slots[0]].d[k];
    if (g.b_slots[1] >= 0)
      for (int k = 0; k < 3; ++k) b1[k] = h->slots[g.b_slots[1]].d[k];
    const double *t0 = g.t_slots[0] >= 0 ? h->slots[g.t_slots[0]].d[0] : nullptr;
    const double *t1 = g.t_slots[1] >= 0 ? h->slots[g.t_slots[1]].d[0] : nullptr;
    const double bscale = fp32 ? 1.0 / cgs::fp32_bunit : 1.0;
    HXG_CK(launch_pack(h->stream, fp32, g.n, g.rec, b0, b1, t0, t1, bscale, 1.0));
    ++h->launch_count;
  }
  h->groups_dirty = false;
  return HXG_OK;
}

// Hampisk::duplicate (include/hamsk.h:55-103).
void mask_duplicate_host(uint32_t pivot_nside, const double *pm,
                         uint32_t nside, double *out) {
  const Hpx hp = hpx_make(pivot_nside), ht = hpx_make(nside);
  if (pivot_nside == nside) {
    std::memcpy(out, pm, sizeof(double) * hp.npix);
    return;
  }
  for (uint64_t i = 0; i < ht.npix; ++i) out[i] = 0.;
  if (pivot_nside > nside) {
    const uint64_t fact = pivot_nside / nside;
    for (uint64_t m = 0; m < ht.npix; ++m) {
      int64_t x, y, f;
      hpx_ring2xyf(ht, m, x, y, f);
      bool hit = false;
      for (uint64_t j = fact * (uint64_t)y; j < fact * (uint64_t)(y + 1) && !hit; ++j)
        for (uint64_t i = fact * (uint64_t)x; i < fact * (uint64_t)(x + 1); ++i) {
          hit = pm[hpx_xyf2ring(hp, (int64_t)i, (int64_t)j, f)] > 0;
          if (hit) break;
        }
      out[m] = (double)hit;
    }
  } else {
    const uint64_t fact = nside / pivot_nside;
    for (uint64_t m = 0; m < hp.npix; ++m) {
      const double val = pm[m];
      int64_t x, y, f;
      hpx_ring2xyf(hp, m, x, y, f);
      for (uint64_t j = fact * (uint64_t)y; j < fact * (uint64_t)(y + 1); ++j)
        for (uint64_t i = fact * (uint64_t)x; i < fact * (uint64_t)(x + 1); ++i)
          out[hpx_xyf2ring(ht, (int64_t)i, (int64_t)j, f)] = val;
    }
  }
}

int device_mask(hxg_handle *h, uint32_t nside, const unsigned char **out) {
  auto it = h->mask_dev.find(nside);
  if (it != h->mask_dev.end()) {
    *out = it->second;
    return HXG_OK;
  }
  const uint64_t n = npix_of(nside);
  std::vector<double> dup(n);
  mask_duplicate_host(h->mask_nside, h->mask_host.data(), nside, dup.data());
  std::vector<unsigned char> flags(n);
  for (uint64_t i = 0; i < n; ++i) flags[i] = dup[i] == 1.0 ? 1 : 0;
  unsigned char *d = nullptr;
  HXG_CK(cudaMalloc(&d, n));
  HXG_CK(cudaMemcpyAsync(d, flags.data(), n, cudaMemcpyHostToDevice, h->stream));
  HXG_CK(cudaStreamSynchronize(h->stream));
  h->mask_dev[nside] = d;
  *out = d;
  return HXG_OK;
}

void clear_masks(hxg_handle *h) {
  for (auto &kv : h->mask_dev) cudaFree(kv.second);
  h->mask_dev.clear();
}

// Integrator::assemble_shell_ref (integrator.cc:231-254)
void shell_ref(const hxg_obs_t &o, uint32_t s, double &d_start,
               double &delta_d, uint64_t &step) {
  const double ds = o.radii_shell[s], de = o.radii_shell[s + 1];
  double dd = o.oc_r_res;
  step = (uint64_t)std::floor((de / dd - ds / dd));
  dd = (de - ds) / (double)step;
  d_start = ds;
  delta_d = dd;
}

// CRE spectral index at the observer (cre_ana.cc:114-119, cre_unif.cc:175-178)
double cre_index_at(const hxg_models_t &m, const double p[3]) {
  if (m.cre == HXG_CRE_ANA) {
    const double r = std::sqrt(p[0] * p[0] + p[1] * p[1]) / cgs::kpc;
    const double z = std::fabs(p[2]) / cgs::kpc;
    return -m.cre_ana.alpha + m.cre_ana.beta * r + m.cre_ana.theta * z;
  }
  return -(m.cre_unif.alpha);
}

// Fill the model block in the working units of the form: CGS for FP64,
// kpc / 2^-20 G for FP32C (L = length scale, Bu = field scale).
DevModels dev_models(const hxg_models_t &m, const double obs[3], double L,
                     double Bu) {
  DevModels d{};
  d.breg = m.breg == HXG_BREG_GRID ? kBregNone : m.breg;
  d.tereg = m.tereg == HXG_TEREG_GRID ? kTeregNone : m.tereg;
  d.cre = m.cre;
  d.cre_const_index =
      (m.cre == HXG_CRE_UNIF) ||
      (m.cre == HXG_CRE_ANA && m.cre_ana.beta == 0. && m.cre_ana.theta == 0.);
  d.kpc = cgs::kpc * L;
  for (int i = 0; i < 3; ++i) d.obs[i] = obs[i] * L;
  d.lsa_b0 = m.lsa.b0 * Bu;
  d.lsa_psi0 = m.lsa.psi0;
  d.lsa_psi1 = m.lsa.psi1;
  d.lsa_chi0 = m.lsa.chi0;
  if (m.breg == HXG_BREG_UNIF) {
    d.const_b[0] = m.unif.bp * std::cos(m.unif.l0) * Bu;
    d.const_b[1] = m.unif.bp * std::sin(m.unif.l0) * Bu;
    d.const_b[2] = m.unif.bv * Bu;
  } else if (m.breg == HXG_BREG_CART) {
    d.const_b[0] = m.cart.bx * Bu;
    d.const_b[1] = m.cart.by * Bu;
    d.const_b[2] = m.cart.bz * Bu;
  }
  d.hx_bx = m.helix.bx * Bu;
  d.hx_by = m.helix.by * Bu;
  d.hx_bz = m.helix.bz * Bu;
  d.hx_rmin = m.helix.r_min * L;
  d.hx_rmax = m.helix.r_max * L;
  const double rsun = std::sqrt(obs[0] * obs[0] + obs[1] * obs[1]);
  d.sp_b0 = m.spiral.b0 * Bu;
  d.sp_sin = std::sin(m.spiral.pitch);
  d.sp_cos = std::cos(m.spiral.pitch);
  d.sp_rsun = rsun * L;
  d.sp_rs = m.spiral.r_scale * L;
  d.sp_hs = m.spiral.h_scale * L;
  d.teu_n0 = m.te_unif.n0;
  d.teu_r0 = m.te_unif.r0 * L;
  d.tex_n0 = m.te_exp.n0;
  d.tex_rs = m.te_exp.r_scale * L;
  d.tex_hs = m.te_exp.h_scale * L;
  if (m.cre == HXG_CRE_ANA) {
    d.cre_alpha = m.cre_ana.alpha;
    d.cre_beta = m.cre_ana.beta;
    d.cre_theta = m.cre_ana.theta;
    d.cre_r0 = m.cre_ana.r0 * L;
    d.cre_z0 = m.cre_ana.z0 * L;
  } else if (m.cre == HXG_CRE_UNIF) {
    d.cre_alpha = m.cre_unif.alpha;
    d.cre_unif_r0 = m.cre_unif.r0 * L;
  }
  d.cre_R0 = rsun * L;
  return d;
}

// Models whose blocks live in ExtModels (separate kernel instantiations).
bool uses_ext(const hxg_models_t &m) {
  return m.breg == HXG_BREG_JAFFE || m.breg == HXG_BREG_JF12 ||
         m.tereg == HXG_TEREG_YMW16 || m.cre == HXG_CRE_GRID;
}

// ---- synchrotron functions for the CRE-grid emissivity ------------------
// F(x) = x Int_x^inf K_{5/3}(t) dt and G(x) = x K_{2/3}(x) (the functions
// gsl_sf_synchrotron_1/2 evaluate, integrator.cc:320, 396), tabulated as
// ln(F/x^(1/3)), ln(G/x^(1/3)) on 32768 points of u = ln x in
// [ln 1e-24, ln 128].
// The integral runs down from x = 128 by 10-point Gauss-Legendre panels
// between consecutive table points (Int_128^inf K_{5/3} below 1e-54).
constexpr int kSynchroN = 32768;
constexpr double kSynchroU0 = -55.262042231857095;  // ln 1e-24
constexpr double kSynchroU1 = 4.852030263919617;    // ln 128

const std::vector<double> &synchro_tables() {
  static std::vector<double> tab;
  static std::once_flag once;
  std::call_once(once, [] {
    const double gx[10] = {-0.9739065285171717, -0.8650633666889845, -0.6794095682990244,
                           -0.4333953941292472, -0.1488743389816312, 0.1488743389816312,
                           0.4333953941292472,  0.6794095682990244,  0.8650633666889845,
                           0.9739065285171717};
    const double gw[10] = {0.0666713443086881, 0.1494513491505806, 0.2190863625159820,
                           0.2692667193099963, 0.2955242247147529, 0.2955242247147529,
                           0.2692667193099963, 0.2190863625159820, 0.1494513491505806,
                           0.0666713443086881};
    const int n = kSynchroN;
    const double du = (kSynchroU1 - kSynchroU0) / (n - 1);
    tab.assign(2 * n, 0.);
    // Int_{x_k}^{x_{k+1}} K_{5/3}(t) dt with t = e^u, dt = t du
    double acc = 0.;
    for (int k = n - 1; k >= 0; --k) {
      const double u = kSynchroU0 + k * du;
      const double x = std::exp(u);
      if (k < n - 1) {
        double seg = 0.;
        for (int q = 0; q < 10; ++q) {
          const double uq = u + 0.5 * du * (gx[q] + 1.);
          const double t = std::exp(uq);
          seg += gw[q] * std::cyl_bessel_k(5. / 3., t) * t;
        }
        acc += 0.5 * du * seg;
      }
      tab[k] = std::log(x * acc / std::cbrt(x));                          // ln F/x^(1/3)
      tab[n + k] = std::log(x * std::cyl_bessel_k(2. / 3., x) / std::cbrt(x));  // ln G/x^(1/3)
    }
  });
  return tab;
}

// Device copies of the CRE grid's energy tables and the synchrotron tables,
// and the CreGridDev block in working units (L, Bu of the form).
int cre_grid_block(hxg_handle *h, double L, double Bu, double freq, CreGridDev &c);


// Jaffe / JF12 / YMW16 blocks in the working units of the form.
void ext_models(const hxg_models_t &m, double L, double Bu, ExtModels &x) {
  std::memset(&x, 0, sizeof(x));
  // Breg_jaffe: the Param block in working units and its parameter-only
  // constants (breg_jaffe.cc:14-17, 42-46, 107-108, 183-187)
  {
    JaffeDev &J = x.jaffe;
    J.p = m.jaffe;
    for (double *v : {&J.p.disk_amp, &J.p.halo_amp, &J.p.ring_amp, &J.p.bar_amp}) *v *= Bu;
    for (int k = 0; k < 8; ++k) J.p.arm_amp[k] *= Bu;
    for (double *v : {&J.p.disk_z0, &J.p.halo_z0, &J.p.r_inner, &J.p.r_scale, &J.p.r_peak,
                      &J.p.ring_r, &J.p.bar_a, &J.p.bar_b, &J.p.arm_r0, &J.p.arm_z0,
                      &J.p.comp_r, &J.p.comp_d})
      *v *= L;
    J.cos_p = std::cos(m.jaffe.arm_pitch);
    J.sin_p = std::sin(m.jaffe.arm_pitch);
    J.beta_inv = -J.sin_p / J.cos_p;
    J.cos_b = std::cos(m.jaffe.bar_phi0);
    J.sin_b = std::sin(m.jaffe.bar_phi0);
    J.bar_lim = J.p.bar_a + 0.5 * J.p.comp_d;
    J.c0 = 1. / m.jaffe.comp_c - 1.;
    J.r_forbid = 0.5 * cgs::kpc * L;
  }
  // Breg_jf12 (breg_jf12.cc:10-62, 96-104)
  {
    Jf12Dev &F = x.jf12;
    F.p = m.jf12;
    for (double *v : {&F.p.b_arm1, &F.p.b_arm2, &F.p.b_arm3, &F.p.b_arm4, &F.p.b_arm5,
                      &F.p.b_arm6, &F.p.b_arm7, &F.p.b_ring, &F.p.Bn, &F.p.Bs, &F.p.B0_X})
      *v *= Bu;
    for (double *v : {&F.p.h_disk, &F.p.w_disk, &F.p.rn, &F.p.rs, &F.p.wh, &F.p.z0,
                      &F.p.rpc_X, &F.p.r0_X})
      *v *= L;
    // fractions of the circumference of each arm and the arm boundaries on
    // the negative x axis (kpc), fixed in the model (breg_jf12.cc:49-58)
    const double f[8] = {0.130, 0.165, 0.094, 0.122, 0.13, 0.118, 0.084, 0.156};
    const double rc[8] = {5.1, 6.3, 7.1, 8.3, 9.8, 11.4, 12.7, 15.5};
    const double bv[8] = {F.p.b_arm1, F.p.b_arm2, F.p.b_arm3, F.p.b_arm4,
                          F.p.b_arm5, F.p.b_arm6, F.p.b_arm7, 0.};
    double b8 = 0.;
    for (int i = 0; i < 7; i++) b8 -= f[i] * bv[i] / f[7];
    for (int i = 0; i < 7; i++) F.bv[i] = bv[i];
    F.bv[7] = b8;
    for (int i = 0; i < 8; i++) F.rc_b[i] = rc[i] * cgs::kpc * L;
    const double inc = 11.5;  // degrees
    F.cot_inc = 1 / std::tan(cgs::pi / 180. * (90 - inc));
    F.sin_inc = std::sin(cgs::pi / 180. * inc);
    F.cos_inc = std::cos(cgs::pi / 180. * inc);
    F.tan_x = std::tan(m.jf12.Xtheta);
    F.r_max = 20 * cgs::kpc * L;
    F.rho_gc = 1. * cgs::kpc * L;
    F.r_min = 5. * cgs::kpc * L;
    F.r_cent = 3. * cgs::kpc * L;
    F.tiny = 1.e-12 * Bu;
  }
  // TEreg_ymw16 (tereg_ymw16.cc:233-240, 305-307)
  {
    Ymw16Dev &Y = x.ymw16;
    Y.p = m.ymw16;
    hxg_tereg_ymw16_t &q = Y.p;
    for (double *v : {&q.r_warp, &q.r0, &q.t1_ad, &q.t1_bd, &q.t1_h1, &q.t2_a2, &q.t2_b2,
                      &q.t3_b2s, &q.t3_aa, &q.t4_agc, &q.t4_hgc, &q.t5_wgn, &q.t5_agn,
                      &q.t6_wlb1, &q.t6_hlb1, &q.t6_wlb2, &q.t6_hlb2, &q.t7_rli, &q.t7_wli})
      *v *= L;
    for (int k = 0; k < 5; ++k) {
      q.t3_warm[k] *= L;
      q.t3_rmin[k] *= L;
    }
    Y.pc = cgs::pc * L;
    Y.kpc = cgs::kpc * L;
    const double lc = 264. * cgs::rad, bc = -4. * cgs::rad, dc = 450. * cgs::pc * L;
    Y.gum_xc = dc * std::cos(bc) * std::sin(lc);
    Y.gum_yc = q.r0 - dc * std::cos(bc) * std::cos(lc);
    Y.gum_zc = dc * std::sin(bc);
    Y.cos_li = std::cos((m.ymw16.t7_thetali) * cgs::rad);
    Y.sin_li = std::sin((m.ymw16.t7_thetali) * cgs::rad);
  }
}

// Upload the handle's ExtModels block for models m; *dev = its device
// address, or null when m uses none of the three models.
int upload_ext(hxg_handle *h, const hxg_models_t &m, double freq, const ExtModels **dev) {
  *dev = nullptr;
  if (!uses_ext(m)) return HXG_OK;
  const bool fp32 = h->precision == HXG_FP32C;
  ExtModels x;
  const double L = fp32 ? 1.0 / cgs::kpc : 1.0, Bu = fp32 ? 1.0 / cgs::fp32_bunit : 1.0;
  ext_models(m, L, Bu, x);
  if (m.cre == HXG_CRE_GRID) {
    const int st = cre_grid_block(h, L, Bu, freq, x.cre);
    if (st != HXG_OK) return st;
  }
  int st = ensure(h, h->ext, sizeof(ExtModels));
  if (st != HXG_OK) return st;
  // pageable source: the call returns once the bytes are staged
  HXG_CK(cudaMemcpyAsync(h->ext.p, &x, sizeof(x), cudaMemcpyHostToDevice, h->stream));
  *dev = static_cast<const ExtModels *>(h->ext.p);
  return HXG_OK;
}

int cre_grid_block(hxg_handle *h, double L, double Bu, double freq, CreGridDev &c) {
  const Slot &S = h->slots[HXG_FIELD_CRE];
  if (!S.present) return fail(h, HXG_ERR_STATE, "CRE grid model without an uploaded CRE grid");
  const hxg_grid_desc_t &g = S.desc;
  const int nE = (int)g.nE;
  const std::vector<double> &tab = synchro_tables();
  // device layout: tab_f | tab_g | inv_ke2[nE] | beta[nE] | dke[nE-1]
  std::vector<double> host(tab);
  std::vector<double> ke(nE);
  for (int i = 0; i < nE; ++i) ke[i] = g.E_min * std::exp(i * g.E_fact);  // integrator.cc:300-304
  for (int i = 0; i < nE; ++i) host.push_back(1. / (ke[i] * ke[i]));
  for (int i = 0; i < nE; ++i) host.push_back(std::sqrt(1 - cgs::mec2 / ke[i]));
  for (int i = 0; i + 1 < nE; ++i) host.push_back(std::fabs(ke[i + 1] - ke[i]));
  int st = ensure(h, h->cre_tab, host.size() * sizeof(double));
  if (st != HXG_OK) return st;
  HXG_CK(cudaMemcpy(h->cre_tab.p, host.data(), host.size() * sizeof(double),
                    cudaMemcpyHostToDevice));
  const double *d = static_cast<const double *>(h->cre_tab.p);
  c.flux = S.d[0];
  c.nx = (int)g.nx;
  c.ny = (int)g.ny;
  c.nz = (int)g.nz;
  c.nE = nE;
  c.lo[0] = g.x_min * L;
  c.lo[1] = g.y_min * L;
  c.lo[2] = g.z_min * L;
  c.hi[0] = g.x_max * L;
  c.hi[1] = g.y_max * L;
  c.hi[2] = g.z_max * L;
  c.tab_f = d;
  c.tab_g = d + kSynchroN;
  c.inv_ke2 = d + 2 * kSynchroN;
  c.beta = c.inv_ke2 + nE;
  c.dke = c.beta + nE;
  c.u0 = kSynchroU0;
  c.inv_du = (kSynchroN - 1) / (kSynchroU1 - kSynchroU0);
  c.ntab = kSynchroN;
  // x_fact numerators and fore factor in the reference's order
  // (integrator.cc:297-299, 319-325, 367-369, 382-385)
  c.xnum_t = 4. * cgs::pi * freq * cgs::mec * cgs::mec2 * cgs::mec2;
  c.xnum_p = (2. * cgs::mec * cgs::mec2 * cgs::mec2 * 2. * cgs::pi * freq);
  c.fore_num = 1.73205081 * cgs::qe * cgs::qe * cgs::qe;
  c.fore_den = cgs::mec2 * cgs::c_light * cgs::GeV * cgs::m * cgs::m * cgs::sec;
  c.bunit = 1. / Bu;
  return HXG_OK;
}

int choose_chunks(const hxg_handle *h, uint64_t npix, uint64_t step) {
  const double target = h->waves * h->sm_count * 2048.0;
  int c = 1;
  while (c < 32 && (double)npix * c < target && step / (2ull * c) >= 16) c *= 2;
  return c;
}

// All launch constants of one shell (integrator.cc:136-228 semantics).
int build_launch(hxg_handle *h, const hxg_models_t &m, const hxg_obs_t &o,
                 uint32_t s, ShellLaunch &P, uint64_t &step_out) {
  const bool fp32 = h->precision == HXG_FP32C;
  const double L = fp32 ? 1.0 / cgs::kpc : 1.0;
  const double Bu = fp32 ? 1.0 / cgs::fp32_bunit : 1.0;
  std::memset(&P, 0, sizeof(P));
  double d_start, delta;
  uint64_t step;
  shell_ref(o, s, d_start, delta, step);
  step_out = step;
  for (int i = 0; i < 3; ++i) P.obs[i] = o.observer[i] * L;
  P.d_start = d_start * L;
  P.delta = delta * L;
  P.step = (long long)step;
  P.gc_r_min = o.gc_r_min * L;
  P.gc_r_max = o.gc_r_max * L;
  P.gc_z_min = o.gc_z_min * L;
  P.gc_z_max = o.gc_z_max * L;
  P.nside = (int)o.nside_shell[s];
  P.shard = 0;
  P.nshards = 1;
  P.shard_log2 = 5;
  P.do_dm = o.do_dm != 0;
  P.do_fd = o.do_fd != 0;
  P.do_sync = o.do_sync != 0;
  const double qe = cgs::qe, mec2 = cgs::mec2, c_l = cgs::c_light;
  const double fdfore = -(qe * qe * qe) / (2. * cgs::pi * mec2 * mec2);
  const double freq = o.sync_freq;
  if (P.do_sync) {
    P.lambda2 = (c_l / freq) * (c_l / freq);
    P.i2bt = c_l * c_l / (2. * cgs::kB * freq * freq);
    const double p = cgs::h_planck * freq / (cgs::kB * 2.725);
    P.tc_a = std::exp(p) - 1.;
    P.tc_b = p * p * std::exp(p);
  } else {
    P.tc_a = 1.;
    P.tc_b = 1.;
  }
  P.models = dev_models(m, o.observer, L, Bu);
  // CRE grid: the emissivity is integrated per sample (cre_grid_j); the
  // FP32C form scales it by 2^128 into FP32 range and k_t = k_p undo that
  if (P.do_sync && m.cre == HXG_CRE_GRID) {
    P.k_t = P.k_p = delta * P.i2bt * 0x1p-128;
  }
  // analytic synchrotron emissivity constants (integrator.cc:332-346, 401-415)
  if (P.do_sync && m.cre != HXG_CRE_GRID) {
    const double E0 = m.cre == HXG_CRE_ANA ? m.cre_ana.E0 : m.cre_unif.E0;
    const double j0 = m.cre == HXG_CRE_ANA ? m.cre_ana.j0 : m.cre_unif.j0;
    const double gamma0 = E0 / cgs::mec2;
    const double beta0 = std::sqrt(1. - 1. / gamma0);
    const double unit = 4. * cgs::pi * cgs::mec /
                        (cgs::GeV * cgs::m * cgs::m * cgs::sec * beta0);
    const double norm = j0 * std::pow(gamma0, -cre_index_at(m, o.observer));
    P.em_n0u = norm * unit;
    P.em_qe3 = qe * qe * qe;
    P.em_anum = 2. * cgs::pi * freq * cgs::mec;
    P.em_3qe = 3. * qe;
    P.em_den_p = 16. * cgs::pi * mec2;
    P.em_const = P.models.cre_const_index;
    const double a_s = P.em_anum / (P.em_3qe * cgs::fp32_bunit);
    P.a_s = a_s;
    const double kbase = P.em_n0u * 1.73205081 * P.em_qe3 * cgs::fp32_bunit;
    if (P.em_const) {
      const double idx =
          m.cre == HXG_CRE_ANA ? -m.cre_ana.alpha : -(m.cre_unif.alpha);
      P.em_index = idx;
      P.em_gt = std::tgamma(-0.25 * idx + 19. / 12.) * std::tgamma(-0.25 * idx - 1. / 12.);
      P.em_gp = std::tgamma(-0.25 * idx + 7. / 12.) * std::tgamma(-0.25 * idx - 1. / 12.);
      P.em_den_t = 4. * cgs::pi * mec2 * (1. - idx);
      const double e = 0.5 * (idx + 1);
      P.em_pow_kind = (e == -1.) ? 1 : (e == 0. ? 2 : 0);
      P.em_pe = 1. - e;
      const double ae = std::pow(a_s, e);
      P.k_t = kbase / P.em_den_t * ae * P.em_gt * delta * P.i2bt;
      P.k_p = kbase / P.em_den_p * ae * P.em_gp * delta * P.i2bt;
    } else {
      P.k_t = kbase / (4. * cgs::pi * mec2) * delta * P.i2bt;
      P.k_p = kbase / P.em_den_p * delta * P.i2bt;
    }
  }
  if (fp32) {
    P.fd_fore = fdfore * delta * cgs::fp32_bunit;
    P.k_dm = delta;
    P.phase_k = 2. * P.lambda2 * P.fd_fore;
    const DevModels &D = P.models;
    FastModels &F = P.fast;
    F.sp_b0 = D.sp_b0;
    F.sp_irs = 1. / D.sp_rs;
    F.sp_crs = D.sp_rsun / D.sp_rs;
    F.sp_ihs = 1. / D.sp_hs;
    F.sp_sin = D.sp_sin;
    F.sp_cos = D.sp_cos;
    const double sgn = D.sp_b0 < 0. ? -1. : 1.;
    F.sp_crs_l = F.sp_crs + (D.sp_b0 != 0. ? std::log(std::fabs(D.sp_b0)) : 0.);
    F.sp_sin_s = sgn * D.sp_sin;
    F.sp_cos_s = sgn * D.sp_cos;
    F.sp_sinf_s = float(F.sp_sin_s);
    F.sp_cosf_s = float(F.sp_cos_s);
    F.ex_ln0 = D.tex_n0 > 0. ? std::log(D.tex_n0) : 0.;
    F.ex_n0 = D.tex_n0;
    F.ex_irn = 1. / D.tex_rs;
    F.ex_ihn = 1. / D.tex_hs;
    F.r2min = P.gc_r_min * P.gc_r_min;
    F.r2max = P.gc_r_max * P.gc_r_max;
    F.rc2_hi = 400. * D.kpc * D.kpc;
    F.rc2_lo = 9. * D.kpc * D.kpc;
    F.sp_sinf = float(D.sp_sin);
    F.sp_cosf = float(D.sp_cos);
    F.cre_ir0 = float(1. / D.cre_r0);
    F.cre_2iz0 = float(2. / D.cre_z0);
    F.cre_R0 = float(D.cre_R0);
    F.cre_ir0_l2 = float(cgs::log2e / D.cre_r0);
    F.cre_2iz0_l2 = float(2. * cgs::log2e / D.cre_z0);
    F.cre_R0_l2 = float(2. + D.cre_R0 * cgs::log2e / D.cre_r0);
    F.pe = float(P.em_pe);
  } else {
    P.fd_fore = fdfore;
  }
  // grid groups
  P.ngroups = (int)h->groups.size();
  for (size_t g = 0; g < h->groups.size(); ++g) {
    const Group &G = h->groups[g];
    DevGridGroup &D = P.groups[g];
    D.rec = G.rec;
    D.nx = (int)G.desc.nx;
    D.ny = (int)G.desc.ny;
    D.nz = (int)G.desc.nz;
    D.has_b = G.b_slots[0] >= 0;
    D.gmax[0] = (double)(G.desc.nx - 1);
    D.gmax[1] = (double)(G.desc.ny - 1);
    D.gmax[2] = (double)(G.desc.nz - 1);
    D.lo[0] = G.desc.x_min * L;
    D.lo[1] = G.desc.y_min * L;
    D.lo[2] = G.desc.z_min * L;
    D.scale[0] = (double)(G.desc.nx - 1) / ((G.desc.x_max - G.desc.x_min) * L);
    D.scale[1] = (double)(G.desc.ny - 1) / ((G.desc.y_max - G.desc.y_min) * L);
    D.scale[2] = (double)(G.desc.nz - 1) / ((G.desc.z_max - G.desc.z_min) * L);
  }
  return HXG_OK;
}

int validate_obs(hxg_handle *h, const hxg_obs_t *o) {
  if (!o) return fail(h, HXG_ERR_INVALID, "obs is NULL");
  if (o->total_shell < 1 || o->total_shell > HXG_MAX_SHELLS)
    return fail(h, HXG_ERR_INVALID, "total_shell %u out of [1,%d]", o->total_shell,
                HXG_MAX_SHELLS);
  for (uint32_t s = 0; s < o->total_shell; ++s) {
    if (!is_pow2(o->nside_shell[s]) || o->nside_shell[s] > 8192)
      return fail(h, HXG_ERR_INVALID, "nside_shell[%u]=%u is not a power of two <= 8192",
                  s, o->nside_shell[s]);
    if (!(o->radii_shell[s + 1] > o->radii_shell[s]))
      return fail(h, HXG_ERR_INVALID, "shell %u has non-increasing radii", s);
    double ds, dd;
    uint64_t st;
    shell_ref(*o, s, ds, dd, st);
    // the shell kernels index a ray's samples with 32-bit integers
    if (st < 1 || st > (1ull << 30))
      return fail(h, HXG_ERR_INVALID, "shell %u has %llu radial steps", s,
                  (unsigned long long)st);
  }
  if (!(o->oc_r_res > 0.)) return fail(h, HXG_ERR_INVALID, "oc_r_res must be > 0");
  if (o->do_dm && (!is_pow2(o->nside_dm) || o->nside_dm > 8192))
    return fail(h, HXG_ERR_INVALID, "bad nside_dm %u", o->nside_dm);
  if (o->do_fd && (!is_pow2(o->nside_fd) || o->nside_fd > 8192))
    return fail(h, HXG_ERR_INVALID, "bad nside_fd %u", o->nside_fd);
  if (o->do_sync) {
    if (!is_pow2(o->nside_sync) || o->nside_sync > 8192)
      return fail(h, HXG_ERR_INVALID, "bad nside_sync %u", o->nside_sync);
    if (!(o->sync_freq > 0.)) return fail(h, HXG_ERR_INVALID, "sync_freq must be > 0");
  }
  if (o->do_mask && !h->have_mask)
    return fail(h, HXG_ERR_STATE, "do_mask set but no mask uploaded");
  return HXG_OK;
}

// Validate a grid descriptor for slot `field` and (re)allocate the slot's
// device arrays: 3 components for the B slots, 1 otherwise; the CRE slot
// holds nx*ny*nz*nE values.  The slot is marked present by the caller once
// its data are in place.
int slot_prepare(hxg_handle *h, int field, const hxg_grid_desc_t *g, size_t *n_out,
                 int *ncomp_out) {
  if (field < 0 || field > HXG_FIELD_CRE || !g)
    return fail(h, HXG_ERR_INVALID, "bad field slot %d", field);
  if (field == HXG_FIELD_CRE && (g->nE < 2 || !(g->E_fact > 0.) || !(g->E_min > 0.)))
    return fail(h, HXG_ERR_INVALID, "CRE grid needs nE >= 2, E_min > 0, E_fact > 0");
  if (g->nx < 2 || g->ny < 2 || g->nz < 2)
    return fail(h, HXG_ERR_INVALID, "grid needs at least 2 vertices per axis");
  // the FP32C kernels step grid coordinates in 64-bit fixed point with 44
  // fraction bits
  if (g->nx > (1u << 19) || g->ny > (1u << 19) || g->nz > (1u << 19))
    return fail(h, HXG_ERR_INVALID, "grid has more than 2^19 vertices on an axis");
  // and index voxel records with 32-bit integers
  if ((uint64_t)g->nx * g->ny * g->nz > 0xFFFFFFFFull)
    return fail(h, HXG_ERR_INVALID, "grid has more than 2^32 - 1 vertices");
  if (!(g->x_max > g->x_min) || !(g->y_max > g->y_min) || !(g->z_max > g->z_min))
    return fail(h, HXG_ERR_INVALID, "grid box has non-positive extent");
  const int ncomp = (field == HXG_FIELD_BREG || field == HXG_FIELD_BRND) ? 3 : 1;
  Slot &S = h->slots[field];
  const size_t n = (size_t)g->nx * g->ny * g->nz * (field == HXG_FIELD_CRE ? g->nE : 1);
  if (S.n != n && (S.d[0] || S.d[1] || S.d[2])) {
    for (auto &p : S.d)
      if (p) cudaFree(p);
    S.d[0] = S.d[1] = S.d[2] = nullptr;
    ++h->layout_gen;
  }
  S.present = false;
  for (int k = 0; k < ncomp; ++k) {
    if (!S.d[k]) {
      cudaError_t e = cudaMalloc(&S.d[k], n * sizeof(double));
      if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc(grid)");
    }
  }
  S.n = n;
  S.desc = *g;
  *n_out = n;
  *ncomp_out = ncomp;
  return HXG_OK;
}

int upload_common(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                  const double *c0, const double *c1, const double *c2,
                  cudaMemcpyKind kind) {
  if (!h) return HXG_ERR_INVALID;
  const bool vec = field == HXG_FIELD_BREG || field == HXG_FIELD_BRND;
  const double *src[3] = {c0, c1, c2};
  for (int k = 0; k < (vec ? 3 : 1); ++k)
    if (!src[k]) return fail(h, HXG_ERR_INVALID, "grid component %d is NULL", k);
  size_t n;
  int ncomp;
  int st = slot_prepare(h, field, g, &n, &ncomp);
  if (st != HXG_OK) return st;
  Slot &S = h->slots[field];
  for (int k = 0; k < ncomp; ++k)
    HXG_CK(cudaMemcpyAsync(S.d[k], src[k], n * sizeof(double), kind, h->stream));
  S.present = true;
  h->groups_dirty = true;
  return HXG_OK;
}

}  // namespace


namespace hxg {
// Launch constants of shell s for the FP64 form from plain inputs (one
// caller-packed grid group of FP64 records, or none), without a live handle
// and without any allocation.  Used by the allocation-free entry point.
int noalloc_shell_launch(const hxg_obs_t *o, const hxg_models_t *m,
                         const hxg_grid_desc_t *g, const double *rec,
                         uint32_t s, ShellLaunch *P, uint64_t *step) {
  hxg_handle h;
  h.precision = HXG_FP64;
  h.models = *m;
  h.have_models = true;
  h.groups_dirty = false;
  if (rec != nullptr) {
    h.groups.emplace_back();
    Group &G = h.groups.back();
    G.desc = *g;
    G.rec = const_cast<double *>(rec);
    G.n = (size_t)g->nx * g->ny * g->nz;
    G.b_slots[0] = (m->breg == HXG_BREG_GRID || m->brnd == HXG_BRND_GRID) ? 0 : -1;
    G.t_slots[0] = (m->tereg == HXG_TEREG_GRID || m->ternd == HXG_TERND_GRID) ? 2 : -1;
  }
  const int st = build_launch(&h, h.models, *o, s, *P, *step);
  h.groups.clear();  // the records belong to the caller
  return st;
}

bool noalloc_models_supported(const hxg_models_t *m) {
  std::string why;
  // the Jaffe / JF12 / YMW16 blocks would need a device allocation
  return models_supported(*m, &why) && !uses_ext(*m);
}

bool noalloc_obs_valid(const hxg_obs_t *o) {
  hxg_handle h;
  return validate_obs(&h, o) == HXG_OK;
}
}  // namespace hxg

// ============================================================ C ABI ======
extern "C" {

int hxg_abi_version(void) { return HXG_ABI_VERSION; }

int hxg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int hxg_create(int device, int precision, hxg_handle **out) {
  if (!out) return HXG_ERR_INVALID;
  *out = nullptr;
  if (precision != HXG_FP64 && precision != HXG_FP32C) return HXG_ERR_INVALID;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return HXG_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return HXG_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return HXG_ERR_CUDA;
  hxg_handle *h = new hxg_handle();
  h->device = device;
  h->precision = precision;
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return HXG_ERR_CUDA;
  }
  h->stream = h->own_stream;
  *out = h;
  return HXG_OK;
}

int hxg_destroy(hxg_handle *h) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_groups(h);
  clear_masks(h);
  for (auto &s : h->slots)
    for (auto &p : s.d)
      if (p) cudaFree(p);
  if (h->tmp_fd.p) cudaFree(h->tmp_fd.p);
  if (h->stage32.p) cudaFree(h->stage32.p);
  if (h->up_event) cudaEventDestroy(h->up_event);
  if (h->switch_event) cudaEventDestroy(h->switch_event);
  if (h->up_stream) cudaStreamDestroy(h->up_stream);
  if (h->shell_all.p) cudaFree(h->shell_all.p);
  for (auto &kv : h->interp) cudaFree(kv.second.p);
  for (auto &b : h->out)
    if (b.p) cudaFree(b.p);
  for (auto &b : h->ck)
    if (b.p) cudaFree(b.p);
  for (auto &b : h->ck_inner)
    if (b.p) cudaFree(b.p);
  for (auto *b : {&h->grad_rec, &h->grad_par, &h->g_fdmap, &h->ext, &h->cre_tab})
    if (b->p) cudaFree(b->p);
  for (auto &b : h->g_shell)
    if (b.p) cudaFree(b.p);
  rfg_release(h->rfg);
  for (auto &e : h->events) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return HXG_OK;
}

const char *hxg_last_error(const hxg_handle *h) {
  return h ? h->err.c_str() : "null handle";
}

int hxg_set_stream(hxg_handle *h, void *stream) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  cudaStream_t next = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
  if (next != h->stream) {
    // the handle's device state (packed grids, interpolation tables, maps)
    // may still be written by work queued on the previous stream: the new
    // stream waits for it
    if (!h->switch_event)
      HXG_CK(cudaEventCreateWithFlags(&h->switch_event, cudaEventDisableTiming));
    HXG_CK(cudaEventRecord(h->switch_event, h->stream));
    HXG_CK(cudaStreamWaitEvent(next, h->switch_event, 0));
  }
  h->stream = next;
  return HXG_OK;
}

int hxg_set_models(hxg_handle *h, const hxg_models_t *m) {
  if (!h || !m) return HXG_ERR_INVALID;
  std::string why;
  if (!models_supported(*m, &why)) return fail(h, HXG_ERR_UNSUPPORTED, "%s", why.c_str());
  bool a0[4], a1[4];
  active_slots(h->models, a0);
  active_slots(*m, a1);
  if (!h->have_models || std::memcmp(a0, a1, sizeof(a0)) != 0) h->groups_dirty = true;
  h->models = *m;
  h->have_models = true;
  return HXG_OK;
}

int hxg_upload_grid(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                    const double *c0, const double *c1, const double *c2) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  const int st = upload_common(h, field, g, c0, c1, c2, cudaMemcpyHostToDevice);
  if (st != HXG_OK) return st;
  HXG_CK(cudaStreamSynchronize(h->stream));
  return HXG_OK;
}

int hxg_upload_grid_f32(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                        const float *c0, const float *c1, const float *c2) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  const bool vec = field == HXG_FIELD_BREG || field == HXG_FIELD_BRND;
  const float *src[3] = {c0, c1, c2};
  for (int k = 0; k < (vec ? 3 : 1); ++k)
    if (!src[k]) return fail(h, HXG_ERR_INVALID, "grid component %d is NULL", k);
  size_t n;
  int ncomp;
  int st = slot_prepare(h, field, g, &n, &ncomp);
  if (st != HXG_OK) return st;
  // chunks of 2^26 values (256 MiB) staged on the device and widened into
  // the slot, in order on the upload stream (the widening of a chunk takes
  // about 1/40 of its copy), after the work already queued on the handle's
  // stream (which may still read the slot); the handle's stream then waits
  // for the upload
  const size_t chunk = (size_t)1 << 26;
  if ((st = ensure(h, h->stage32, std::min(chunk, n) * sizeof(float))) != HXG_OK) return st;
  if (!h->up_stream) {
    int least = 0, greatest = 0;
    HXG_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    HXG_CK(cudaStreamCreateWithPriority(&h->up_stream, cudaStreamNonBlocking, greatest));
    HXG_CK(cudaEventCreateWithFlags(&h->up_event, cudaEventDisableTiming));
  }
  HXG_CK(cudaEventRecord(h->up_event, h->stream));
  HXG_CK(cudaStreamWaitEvent(h->up_stream, h->up_event, 0));
  float *stage = static_cast<float *>(h->stage32.p);
  Slot &S = h->slots[field];
  for (int k = 0; k < ncomp; ++k)
    for (size_t off = 0; off < n; off += chunk) {
      const size_t m = std::min(chunk, n - off);
      HXG_CK(cudaMemcpyAsync(stage, src[k] + off, m * sizeof(float), cudaMemcpyHostToDevice,
                             h->up_stream));
      HXG_CK(launch_widen(h->up_stream, m, stage, S.d[k] + off));
      ++h->launch_count;
    }
  HXG_CK(cudaEventRecord(h->up_event, h->up_stream));
  HXG_CK(cudaStreamWaitEvent(h->stream, h->up_event, 0));
  S.present = true;
  h->groups_dirty = true;
  HXG_CK(cudaEventSynchronize(h->up_event));
  return HXG_OK;
}

int hxg_upload_grid_device(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                           const double *d_c0, const double *d_c1,
                           const double *d_c2) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  return upload_common(h, field, g, d_c0, d_c1, d_c2, cudaMemcpyDeviceToDevice);
}

int hxg_upload_grid_file(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                         const char *path) {
  if (!h) return HXG_ERR_INVALID;
  if (!path) return fail(h, HXG_ERR_INVALID, "path is NULL");
  cudaSetDevice(h->device);
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return fail(h, HXG_ERR_INVALID, "cannot open %s", path);
  struct Closer {
    std::FILE *f;
    ~Closer() { std::fclose(f); }
  } closer{f};
  size_t n;
  int ncomp;
  int st = slot_prepare(h, field, g, &n, &ncomp);
  if (st != HXG_OK) return st;
  const size_t total = n * (size_t)ncomp;  // doubles in the file
  if (std::fseek(f, 0, SEEK_END) != 0) return fail(h, HXG_ERR_INVALID, "cannot seek %s", path);
  const long bytes = std::ftell(f);
  if (bytes < 0 || (size_t)bytes != total * sizeof(double))
    return fail(h, HXG_ERR_INVALID, "%s holds %ld bytes, the grid needs %zu", path, bytes,
                total * sizeof(double));
  std::rewind(f);
  // double-buffered chunks of 3 * 2^20 doubles (24 MiB, whole voxels for
  // 3 components): read chunk k while chunk k-1 is copied and split
  const size_t chunk = 3ull << 20;
  struct Bufs {
    void *pin[2] = {nullptr, nullptr};
    double *stage[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Bufs() {
      for (int k = 0; k < 2; ++k) {
        if (ev[k]) cudaEventSynchronize(ev[k]), cudaEventDestroy(ev[k]);
        if (pin[k]) cudaFreeHost(pin[k]);
        if (stage[k]) cudaFree(stage[k]);
      }
    }
  } B;
  for (int k = 0; k < 2; ++k) {
    HXG_CK(cudaHostAlloc(&B.pin[k], chunk * sizeof(double), cudaHostAllocDefault));
    if (ncomp == 3) HXG_CK(cudaMalloc(&B.stage[k], chunk * sizeof(double)));
    HXG_CK(cudaEventCreateWithFlags(&B.ev[k], cudaEventDisableTiming));
    HXG_CK(cudaEventRecord(B.ev[k], h->stream));
  }
  Slot &S = h->slots[field];
  int k = 0;
  for (size_t off = 0; off < total; off += chunk, k ^= 1) {
    const size_t cnt = std::min(chunk, total - off);
    HXG_CK(cudaEventSynchronize(B.ev[k]));  // pin[k] free again
    if (std::fread(B.pin[k], sizeof(double), cnt, f) != cnt)
      return fail(h, HXG_ERR_INVALID, "short read from %s", path);
    if (ncomp == 1) {
      HXG_CK(cudaMemcpyAsync(S.d[0] + off, B.pin[k], cnt * sizeof(double),
                             cudaMemcpyHostToDevice, h->stream));
    } else {
      HXG_CK(cudaMemcpyAsync(B.stage[k], B.pin[k], cnt * sizeof(double),
                             cudaMemcpyHostToDevice, h->stream));
      const size_t v0 = off / 3;
      HXG_CK(launch_deinterleave3(h->stream, cnt / 3, B.stage[k], S.d[0] + v0, S.d[1] + v0,
                                  S.d[2] + v0));
      ++h->launch_count;
    }
    HXG_CK(cudaEventRecord(B.ev[k], h->stream));
  }
  HXG_CK(cudaStreamSynchronize(h->stream));
  S.present = true;
  h->groups_dirty = true;
  return HXG_OK;
}

int hxg_download_grid(hxg_handle *h, int field, double *c0, double *c1, double *c2) {
  if (!h) return HXG_ERR_INVALID;
  if (field < 0 || field > HXG_FIELD_CRE) return fail(h, HXG_ERR_INVALID, "bad field slot %d", field);
  cudaSetDevice(h->device);
  const Slot &S = h->slots[field];
  if (!S.present) return fail(h, HXG_ERR_STATE, "grid slot %d is empty", field);
  const int ncomp = (field == HXG_FIELD_BREG || field == HXG_FIELD_BRND) ? 3 : 1;
  double *dst[3] = {c0, c1, c2};
  for (int k = 0; k < ncomp; ++k)
    if (!dst[k]) return fail(h, HXG_ERR_INVALID, "grid component %d is NULL", k);
  for (int k = 0; k < ncomp; ++k)
    HXG_CK(cudaMemcpyAsync(dst[k], S.d[k], S.n * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
  HXG_CK(cudaStreamSynchronize(h->stream));
  return HXG_OK;
}

int hxg_export_grid_file(hxg_handle *h, int field, const char *path) {
  if (!h) return HXG_ERR_INVALID;
  if (!path) return fail(h, HXG_ERR_INVALID, "path is NULL");
  if (field < 0 || field > HXG_FIELD_CRE) return fail(h, HXG_ERR_INVALID, "bad field slot %d", field);
  cudaSetDevice(h->device);
  const Slot &S = h->slots[field];
  if (!S.present) return fail(h, HXG_ERR_STATE, "grid slot %d is empty", field);
  const int ncomp = (field == HXG_FIELD_BREG || field == HXG_FIELD_BRND) ? 3 : 1;
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return fail(h, HXG_ERR_INVALID, "cannot create %s", path);
  struct Closer {
    std::FILE *f;
    ~Closer() {
      if (f) std::fclose(f);
    }
  } closer{f};
  const size_t total = S.n * (size_t)ncomp;
  // double-buffered chunks of 3 * 2^20 doubles: chunk k is interleaved and
  // copied to pinned memory while chunk k-1 is written
  const size_t chunk = 3ull << 20;
  struct Bufs {
    void *pin[2] = {nullptr, nullptr};
    double *stage[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~Bufs() {
      for (int k = 0; k < 2; ++k) {
        if (ev[k]) cudaEventSynchronize(ev[k]), cudaEventDestroy(ev[k]);
        if (pin[k]) cudaFreeHost(pin[k]);
        if (stage[k]) cudaFree(stage[k]);
      }
    }
  } B;
  for (int k = 0; k < 2; ++k) {
    HXG_CK(cudaHostAlloc(&B.pin[k], chunk * sizeof(double), cudaHostAllocDefault));
    if (ncomp == 3) HXG_CK(cudaMalloc(&B.stage[k], chunk * sizeof(double)));
    HXG_CK(cudaEventCreateWithFlags(&B.ev[k], cudaEventDisableTiming));
  }
  size_t cnt[2] = {0, 0};
  auto flush = [&](int k) -> int {
    HXG_CK(cudaEventSynchronize(B.ev[k]));
    if (std::fwrite(B.pin[k], sizeof(double), cnt[k], f) != cnt[k])
      return fail(h, HXG_ERR_INVALID, "short write to %s", path);
    cnt[k] = 0;
    return HXG_OK;
  };
  int k = 0;
  for (size_t off = 0; off < total; off += chunk, k ^= 1) {
    if (cnt[k]) {
      const int st = flush(k);
      if (st != HXG_OK) return st;
    }
    const size_t c = std::min(chunk, total - off);
    if (ncomp == 1) {
      HXG_CK(cudaMemcpyAsync(B.pin[k], S.d[0] + off, c * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream));
    } else {
      const size_t v0 = off / 3;
      HXG_CK(launch_interleave3(h->stream, c / 3, S.d[0] + v0, S.d[1] + v0, S.d[2] + v0,
                                B.stage[k]));
      ++h->launch_count;
      HXG_CK(cudaMemcpyAsync(B.pin[k], B.stage[k], c * sizeof(double), cudaMemcpyDeviceToHost,
                             h->stream));
    }
    HXG_CK(cudaEventRecord(B.ev[k], h->stream));
    cnt[k] = c;
  }
  for (int j = 0; j < 2; ++j, k ^= 1)
    if (cnt[k]) {
      const int st = flush(k);
      if (st != HXG_OK) return st;
    }
  if (std::fclose(f) != 0) {
    closer.f = nullptr;
    return fail(h, HXG_ERR_INVALID, "cannot close %s", path);
  }
  closer.f = nullptr;
  return HXG_OK;
}

// ---- random-field generators ---------------------------------------------
namespace {

// toolkit::random_seed (include/toolkit.h:122-136): a given seed, or one
// from the clock and the calling thread for 0.
uint64_t rfg_seed(uint64_t seed) {
  if (seed) return seed;
  const auto now = std::chrono::system_clock::now();
  const uint64_t t = (uint64_t)std::chrono::system_clock::to_time_t(now);
  return t + (uint64_t)std::hash<std::thread::id>{}(std::this_thread::get_id());
}

bool finite_pos(double v) { return std::isfinite(v) && v > 0.; }

int rfg_result(hxg_handle *h, int st, const char *what) {
  if (st == HXG_OK) return st;
  if (st == HXG_ERR_INVALID) return fail(h, st, "%s: the spectrum has no power on this grid", what);
  if (st == HXG_ERR_OOM) return fail(h, st, "%s: out of device memory", what);
  return fail(h, st, "%s: a CUDA or cuFFT call failed", what);
}

}  // namespace

int hxg_generate_ternd_dft(hxg_handle *h, const hxg_grid_desc_t *g,
                           const hxg_ternd_dft_t *p, const double observer[3],
                           uint64_t seed) {
  if (!h) return HXG_ERR_INVALID;
  if (!g || !p || !observer) return fail(h, HXG_ERR_INVALID, "NULL argument");
  if (!(std::isfinite(p->rms) && p->rms >= 0.) || !finite_pos(p->k0) ||
      !std::isfinite(p->a0) || !finite_pos(p->r0) || !finite_pos(p->z0))
    return fail(h, HXG_ERR_INVALID, "ternd_dft needs rms >= 0 and k0, r0, z0 > 0");
  cudaSetDevice(h->device);
  size_t n;
  int ncomp;
  int st = slot_prepare(h, HXG_FIELD_TERND, g, &n, &ncomp);
  if (st != HXG_OK) return st;
  Slot &S = h->slots[HXG_FIELD_TERND];
  st = generate_ternd_dft(h->stream, h->rfg, *g, *p, observer, rfg_seed(seed), S.d[0]);
  h->launch_count += 4;  // fill, two reduction passes, rescale
  if (st != HXG_OK) return rfg_result(h, st, "ternd_dft");
  S.present = true;
  h->groups_dirty = true;
  return HXG_OK;
}

int hxg_generate_brnd_es(hxg_handle *h, const hxg_grid_desc_t *g, const hxg_brnd_es_t *p,
                         const double observer[3], uint64_t seed) {
  if (!h) return HXG_ERR_INVALID;
  if (!g || !p || !observer) return fail(h, HXG_ERR_INVALID, "NULL argument");
  if (!(std::isfinite(p->rms) && p->rms >= 0.) || !finite_pos(p->k0) || !finite_pos(p->k1) ||
      !std::isfinite(p->a0) || !std::isfinite(p->a1) || !finite_pos(p->rho) ||
      !finite_pos(p->r0) || !finite_pos(p->z0))
    return fail(h, HXG_ERR_INVALID, "brnd_es needs rms >= 0 and k0, k1, rho, r0, z0 > 0");
  if (!h->have_models)
    return fail(h, HXG_ERR_STATE, "models not set: the anisotropy follows the regular field");
  cudaSetDevice(h->device);
  const hxg_models_t &m = h->models;
  RfgBregGrid bg{};
  if (m.breg == HXG_BREG_GRID) {
    const Slot &B = h->slots[HXG_FIELD_BREG];
    if (!B.present) return fail(h, HXG_ERR_STATE, "BREG grid not uploaded");
    bg.bx = B.d[0];
    bg.by = B.d[1];
    bg.bz = B.d[2];
    bg.nx = (int)B.desc.nx;
    bg.ny = (int)B.desc.ny;
    bg.nz = (int)B.desc.nz;
    bg.x_min = B.desc.x_min;
    bg.x_max = B.desc.x_max;
    bg.y_min = B.desc.y_min;
    bg.y_max = B.desc.y_max;
    bg.z_min = B.desc.z_min;
    bg.z_max = B.desc.z_max;
  }
  const DevModels M = dev_models(m, observer, 1.0, 1.0);
  // Jaffe / JF12 blocks in CGS for the anisotropy direction
  struct ExtBuf {
    ExtModels *p = nullptr;
    ~ExtBuf() {
      if (p) cudaFree(p);
    }
  } xb;
  if (m.breg == HXG_BREG_JAFFE || m.breg == HXG_BREG_JF12) {
    ExtModels x;
    ext_models(m, 1.0, 1.0, x);
    HXG_CK(cudaMalloc(&xb.p, sizeof(ExtModels)));
    HXG_CK(cudaMemcpy(xb.p, &x, sizeof(x), cudaMemcpyHostToDevice));
  }
  size_t n;
  int ncomp;
  int st = slot_prepare(h, HXG_FIELD_BRND, g, &n, &ncomp);
  if (st != HXG_OK) return st;
  Slot &S = h->slots[HXG_FIELD_BRND];
  st = generate_brnd_es(h->stream, h->rfg, *g, *p, M, xb.p, bg, rfg_seed(seed), S.d[0], S.d[1],
                        S.d[2]);
  h->launch_count += 7;  // fill, two reductions, rescale, project, repack, final
  if (st != HXG_OK) return rfg_result(h, st, "brnd_es");
  S.present = true;
  h->groups_dirty = true;
  return HXG_OK;
}

int hxg_set_mask(hxg_handle *h, uint32_t nside, const double *mask) {
  if (!h) return HXG_ERR_INVALID;
  clear_masks(h);
  if (!mask) {
    h->have_mask = false;
    h->mask_host.clear();
    return HXG_OK;
  }
  if (!is_pow2(nside) || nside > 8192) return fail(h, HXG_ERR_INVALID, "bad mask nside %u", nside);
  h->mask_host.assign(mask, mask + npix_of(nside));
  h->mask_nside = nside;
  h->have_mask = true;
  return HXG_OK;
}

}  // extern "C"

namespace {

// Checks shared by the pass entry points: obs, models, requested outputs.
int check_pass(hxg_handle *h, const hxg_obs_t *o, bool dm, bool fd, bool sync3) {
  int st = validate_obs(h, o);
  if (st != HXG_OK) return st;
  if (!h->have_models) return fail(h, HXG_ERR_STATE, "models not set");
  if (o->do_sync && h->models.cre == HXG_CRE_NONE)
    return fail(h, HXG_ERR_INVALID, "synchrotron output needs a CRE model");
  if (o->do_sync && h->models.cre == HXG_CRE_GRID && !h->slots[HXG_FIELD_CRE].present)
    return fail(h, HXG_ERR_STATE, "CRE grid model without an uploaded CRE grid");
  if ((o->do_dm && !dm) || (o->do_fd && !fd) || (o->do_sync && !sync3))
    return fail(h, HXG_ERR_INVALID, "an output requested by obs is NULL");
  return build_groups(h);
}

// Block size (log2 pixels) of the shard interleave: 2048-pixel NESTED
// patches keep neighbouring warps of a shard on neighbouring rays (grid
// cache reuse; measured on config 3 with 8 shards: 4 % less work than
// 32-pixel blocks), shrunk to keep at least 8 blocks per shard for balance,
// never below one warp's 32 pixels.
unsigned shard_block_log2(uint64_t npix, uint32_t nshards) {
  unsigned L = 11;
  while (L > 5 && (npix >> L) < 8ull * nshards) --L;
  return L;
}

// Shell s of pass o over the pixels of shard `shard` of `nshards` (the
// 32-pixel NESTED blocks b with b % nshards == shard) into the shell maps tmp (radial_integration for every pixel of the shell,
// integrator.cc:60-100); fdmap = the accumulated FD output of the inner
// shells, or null.
int run_shell(hxg_handle *h, const hxg_obs_t &o, uint32_t s, const ExtModels *ext_dev,
              const double *fdmap, double *const tmp[5], uint32_t shard, uint32_t nshards,
              bool checkpoint) {
  const bool fp32 = h->precision == HXG_FP32C;
  ShellLaunch P;
  uint64_t step;
  int st = build_launch(h, h->models, o, s, P, step);
  if (st != HXG_OK) return st;
  P.ext = ext_dev;
  // inner-shell Faraday depth: the accumulated FD output map when it is
  // requested, otherwise an all-zero map (integrator.cc:78-86, 130-132)
  P.fdmap = o.do_fd ? fdmap : nullptr;
  P.nside_fdmap = o.do_fd ? (int)o.nside_fd : 0;
  P.mask = nullptr;
  if (o.do_mask) {
    const unsigned char *dm = nullptr;
    if ((st = device_mask(h, o.nside_shell[s], &dm)) != HXG_OK) return st;
    P.mask = dm;
  }
  for (int k = 0; k < 5; ++k) P.out[k] = tmp[k];
  const uint64_t npix = npix_of(o.nside_shell[s]);
  P.shard = shard;
  P.nshards = nshards;
  P.shard_log2 = shard_block_log2(npix, nshards);
  // pixels of this shard, counted in whole blocks (the kernel drops the
  // ones past npix)
  const uint64_t bsz = 1ull << P.shard_log2;
  const uint64_t nblk = (npix + bsz - 1) / bsz;
  const uint64_t local = nshards == 1 ? npix : (nblk + nshards - 1 - shard) / nshards * bsz;
  const int C = choose_chunks(h, local, step);
  P.chunks = C;
  P.log2_chunks = hpx_ilog2((uint64_t)C);
  if (checkpoint) {
    if (h->ck.size() < o.total_shell) {
      h->ck.resize(o.total_shell);
      h->ck_inner.resize(o.total_shell);
      h->ck_chunks.resize(o.total_shell);
    }
    if ((st = ensure(h, h->ck[s], npix * C * 3 * sizeof(double))) != HXG_OK) return st;
    if ((st = ensure(h, h->ck_inner[s], npix * sizeof(double))) != HXG_OK) return st;
    HXG_CK(cudaMemsetAsync(h->ck_inner[s].p, 0, npix * sizeof(double), h->stream));
    P.ck = static_cast<double *>(h->ck[s].p);
    P.ck_inner = static_cast<double *>(h->ck_inner[s].p);
    h->ck_chunks[s] = C;
  }
  if (local == 0) return HXG_OK;
  const uint64_t warps = (local + (32 / C) - 1) / (32 / C);
  const unsigned threads = fp32 ? HXG_FP32C_THREADS : HXG_FP64_THREADS;
  const unsigned blocks = (unsigned)((warps * 32 + threads - 1) / threads);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->timing) {
    HXG_CK(cudaEventCreate(&e0));
    HXG_CK(cudaEventCreate(&e1));
    HXG_CK(cudaEventRecord(e0, h->stream));
  }
  HXG_CK(launch_shell(h->stream, fp32, P, blocks, threads));
  ++h->launch_count;
  if (h->timing) {
    HXG_CK(cudaEventRecord(e1, h->stream));
    h->events.emplace_back(e0, e1);
    h->event_samples.push_back((int64_t)(std::min(local, npix) * step));
  }
  return HXG_OK;
}

// The interpolation table of an Nside pair, made on first use on the
// handle's stream.  Null members (the kernels then find the weights in
// place) when the Nsides agree, the shell map has more than 2^32 pixels,
// the tables would pass the handle's bound (hxg_set_interp_cache) or the
// allocation fails.
int interp_tab(hxg_handle *h, uint32_t nside_dst, uint32_t nside_src, InterpTab *t) {
  *t = InterpTab{};
  if (nside_dst == nside_src || npix_of(nside_src) > 0xffffffffull) return HXG_OK;
  const uint64_t key = (uint64_t)nside_dst << 32 | nside_src;
  auto it = h->interp.find(key);
  if (it == h->interp.end()) {
    const size_t n = npix_of(nside_dst);
    const size_t bytes = n * (sizeof(uint4) + 2 * sizeof(double2));
    if (h->interp_bytes + bytes > h->interp_limit) return HXG_OK;
    DevBuf b;
    if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      return HXG_OK;
    }
    b.bytes = bytes;
    const cudaError_t e = launch_interp_table(h->stream, (int)nside_dst, (int)nside_src,
                                              static_cast<uint4 *>(b.p),
                                              reinterpret_cast<double2 *>(
                                                  static_cast<char *>(b.p) + n * sizeof(uint4)));
    if (e != cudaSuccess) {
      cudaFree(b.p);
      return cuda_fail(h, e, "launch_interp_table");
    }
    ++h->launch_count;
    h->interp_bytes += bytes;
    it = h->interp.emplace(key, b).first;
  }
  const size_t n = npix_of(nside_dst);
  t->pix = static_cast<const uint4 *>(it->second.p);
  t->w = reinterpret_cast<const double2 *>(static_cast<const char *>(it->second.p) +
                                           n * sizeof(uint4));
  return HXG_OK;
}

// Accumulate the shell maps of shell s into the pass outputs
// (Hampix::accumulate, integrator.cc:121-132).
int merge_shell(hxg_handle *h, const hxg_obs_t &o, uint32_t s, const double *const tmp[5],
                double *d_dm, double *d_fd, double *d_is, double *d_qs, double *d_us) {
  const int ns = (int)o.nside_shell[s];
  // one merge launch per output Nside (DM, FD and I/Q/U usually share one)
  const bool want[5] = {o.do_dm != 0, o.do_fd != 0, o.do_sync != 0, o.do_sync != 0,
                        o.do_sync != 0};
  const uint32_t nside[5] = {o.nside_dm, o.nside_fd, o.nside_sync, o.nside_sync,
                             o.nside_sync};
  double *const out[5] = {d_dm, d_fd, d_is, d_qs, d_us};
  bool done[5] = {false, false, false, false, false};
  for (int a = 0; a < 5; ++a) {
    if (!want[a] || done[a]) continue;
    double *d[5];
    const double *sr[5];
    int n = 0;
    for (int b = a; b < 5; ++b)
      if (want[b] && !done[b] && nside[b] == nside[a]) {
        d[n] = out[b];
        sr[n] = tmp[b];
        ++n;
        done[b] = true;
      }
    InterpTab tab;
    int st = interp_tab(h, nside[a], (uint32_t)ns, &tab);
    if (st != HXG_OK) return st;
    HXG_CK(launch_accumulate(h->stream, (int)nside[a], ns, n, d, sr, &tab));
    ++h->launch_count;
  }
  return HXG_OK;
}

// One block of nm shell maps per shell in h->shell_all, for a pass whose DM
// and Stokes maps are merged at its end: base[s] = shell s's block.
int shell_blocks(hxg_handle *h, const hxg_obs_t &o, int nm, double **base) {
  size_t off[HXG_MAX_SHELLS], total = 0;
  for (uint32_t s = 0; s < o.total_shell; ++s) {
    off[s] = total;
    total += (size_t)nm * npix_of(o.nside_shell[s]);
  }
  const int st = ensure(h, h->shell_all, total * sizeof(double));
  if (st != HXG_OK) return st;
  for (uint32_t s = 0; s < o.total_shell; ++s)
    base[s] = static_cast<double *>(h->shell_all.p) + off[s];
  return HXG_OK;
}

// An output of the pass-end merge: the map idx of every shell's block summed
// into dst at Nside nside.
struct PassOut {
  uint32_t nside;
  int idx;
  double *dst;
};

// The pass-end merge of the DM and Stokes maps (Hampix::accumulate of every
// shell, integrator.cc:121-132, in shell order into the zeroed outputs): one
// launch per output Nside.
int merge_pass(hxg_handle *h, const hxg_obs_t &o, double *const *base,
               const std::vector<PassOut> &outs) {
  int nside[HXG_MAX_SHELLS];
  const double *b[HXG_MAX_SHELLS];
  InterpTab tab[HXG_MAX_SHELLS];
  for (uint32_t s = 0; s < o.total_shell; ++s) {
    nside[s] = (int)o.nside_shell[s];
    b[s] = base[s];
  }
  std::vector<bool> done(outs.size(), false);
  for (size_t a = 0; a < outs.size(); ++a) {
    if (done[a]) continue;
    std::vector<int> idx;
    std::vector<double *> dst;
    for (size_t c = a; c < outs.size(); ++c)
      if (!done[c] && outs[c].nside == outs[a].nside) {
        idx.push_back(outs[c].idx);
        dst.push_back(outs[c].dst);
        done[c] = true;
      }
    for (uint32_t s = 0; s < o.total_shell; ++s) {
      const int st = interp_tab(h, outs[a].nside, o.nside_shell[s], &tab[s]);
      if (st != HXG_OK) return st;
    }
    HXG_CK(launch_merge_all(h->stream, (int)outs[a].nside, (int)idx.size(), idx.data(),
                            dst.data(), (int)o.total_shell, nside, b, tab));
    h->launch_count += ((int64_t)idx.size() + kMaxMergeOuts - 1) / kMaxMergeOuts;
  }
  return HXG_OK;
}

}  // namespace

extern "C" {

int hxg_write_grid_device(hxg_handle *h, const hxg_obs_t *o, double *d_dm,
                          double *d_fd, double *d_is, double *d_qs,
                          double *d_us) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  int st = check_pass(h, o, d_dm, d_fd, d_is && d_qs && d_us);
  if (st != HXG_OK) return st;
  uint32_t max_nside = 0;
  for (uint32_t s = 0; s < o->total_shell; ++s)
    max_nside = std::max(max_nside, o->nside_shell[s]);
  const size_t tbytes = npix_of(max_nside) * sizeof(double);
  // the shell FD map is merged after each shell (the next one reads the
  // accumulated FD); DM, I, Q, U of every shell are kept and merged at the end
  if ((st = ensure(h, h->tmp_fd, tbytes)) != HXG_OK) return st;
  double *const tmp_fd = static_cast<double *>(h->tmp_fd.p);
  double *base[HXG_MAX_SHELLS];
  if ((st = shell_blocks(h, *o, 4, base)) != HXG_OK) return st;
  // Grid_obs maps start at zero (Grid_obs::build_grid, grid_obs.cc:21-43)
  if (o->do_dm) HXG_CK(cudaMemsetAsync(d_dm, 0, npix_of(o->nside_dm) * 8, h->stream));
  if (o->do_fd) HXG_CK(cudaMemsetAsync(d_fd, 0, npix_of(o->nside_fd) * 8, h->stream));
  if (o->do_sync) {
    const size_t b = npix_of(o->nside_sync) * 8;
    HXG_CK(cudaMemsetAsync(d_is, 0, b, h->stream));
    HXG_CK(cudaMemsetAsync(d_qs, 0, b, h->stream));
    HXG_CK(cudaMemsetAsync(d_us, 0, b, h->stream));
  }
  const ExtModels *ext_dev = nullptr;
  if ((st = upload_ext(h, h->models, o->sync_freq, &ext_dev)) != HXG_OK) return st;
  const bool ck = h->checkpoint;
  for (uint32_t s = 0; s < o->total_shell; ++s) {
    const size_t np = npix_of(o->nside_shell[s]);
    double *const tmp[5] = {base[s], tmp_fd, base[s] + np, base[s] + 2 * np, base[s] + 3 * np};
    st = run_shell(h, *o, s, ext_dev, d_fd, tmp, 0, 1, ck);
    if (st != HXG_OK) return st;
    if (o->do_fd) {
      const double *src = tmp_fd;
      InterpTab tab;
      if ((st = interp_tab(h, o->nside_fd, o->nside_shell[s], &tab)) != HXG_OK) return st;
      HXG_CK(launch_accumulate(h->stream, (int)o->nside_fd, (int)o->nside_shell[s], 1, &d_fd,
                               &src, &tab));
      ++h->launch_count;
    }
  }
  std::vector<PassOut> outs;
  if (o->do_dm) outs.push_back({o->nside_dm, 0, d_dm});
  if (o->do_sync) {
    outs.push_back({o->nside_sync, 1, d_is});
    outs.push_back({o->nside_sync, 2, d_qs});
    outs.push_back({o->nside_sync, 3, d_us});
  }
  if ((st = merge_pass(h, *o, base, outs)) != HXG_OK) return st;
  if (ck) {
    // the per-shell checkpoints were overwritten
    h->ck_shell.clear();
    h->adj_open = false;
    h->ck_valid = true;
    h->ck_obs = *o;
    h->ck_models = h->models;
  } else {
    h->ck_valid = false;
  }
  return HXG_OK;
}

}  // extern "C"

namespace {

// Whether passes o[0..n) can share one shell traversal: FP32C form, the
// same observer, shells, radial step, limits and mask switch, synchrotron on
// in every pass, and no CRE grid (its emissivity depends on the frequency).
// Passes o[0..n) with synchrotron output and the same observer, shells,
// radial step, limits and mask switch: one traversal can serve them all.
bool same_traversal(const hxg_obs_t *o, int n) {
  for (int k = 0; k < n; ++k) {
    const hxg_obs_t &a = o[0], &b = o[k];
    if (!b.do_sync) return false;
    if (std::memcmp(a.observer, b.observer, sizeof(a.observer)) != 0 ||
        a.total_shell != b.total_shell || a.oc_r_res != b.oc_r_res ||
        a.gc_r_min != b.gc_r_min || a.gc_r_max != b.gc_r_max || a.gc_z_min != b.gc_z_min ||
        a.gc_z_max != b.gc_z_max || a.do_mask != b.do_mask)
      return false;
    for (uint32_t s = 0; s < a.total_shell; ++s)
      if (a.nside_shell[s] != b.nside_shell[s]) return false;
    for (uint32_t s = 0; s <= a.total_shell; ++s)
      if (a.radii_shell[s] != b.radii_shell[s]) return false;
  }
  return true;
}

// Whether passes o[0..n) of the handle's models can share one traversal:
// FP32C form, no CRE grid (its emissivity depends on the frequency).
bool fusable(const hxg_handle *h, const hxg_obs_t *o, int n) {
  if (h->precision != HXG_FP32C || n < 2 || h->models.cre == HXG_CRE_GRID) return false;
  return same_traversal(o, n);
}

// One shell of NF fusable passes o[0..NF) over shard `shard` of `nshards`
// into the shell maps tmp_dm, tmp_fd (shared) and tmp_iqu[f] (per pass);
// fdmap = the accumulated FD output that passes with do_fd read.
template <int NF>
int fused_shell(hxg_handle *h, const hxg_obs_t *o, uint32_t s, uint32_t shard, uint32_t nshards,
                const double *fdmap, int nside_fdmap, const ExtModels *ext_dev, double *tmp_dm,
                double *tmp_fd, double *const (*tmp_iqu)[3]) {
  const hxg_obs_t &o0 = o[0];
  bool any_dm = false, any_fd = false;
  for (int f = 0; f < NF; ++f) {
    any_dm = any_dm || o[f].do_dm;
    any_fd = any_fd || o[f].do_fd;
  }
  ShellLaunch P, Pf;
  uint64_t step;
  FreqSet<NF> Fq;
  int st;
  for (int f = NF - 1; f >= 0; --f) {  // P ends as pass 0's launch block
    if ((st = build_launch(h, h->models, o[f], s, f == 0 ? P : Pf, step)) != HXG_OK) return st;
    const ShellLaunch &L = f == 0 ? P : Pf;
    Fq.lambda2[f] = L.lambda2;
    Fq.phase_k[f] = L.phase_k;
    Fq.k_t[f] = L.k_t;
    Fq.k_p[f] = L.k_p;
    Fq.tc_a[f] = L.tc_a;
    Fq.tc_b[f] = L.tc_b;
    Fq.a_s[f] = L.a_s;
    Fq.inner[f] = o[f].do_fd ? 1 : 0;
    for (int j = 0; j < 3; ++j) Fq.out[f][j] = tmp_iqu[f][j];
  }
  P.ext = ext_dev;
  P.do_dm = any_dm;
  P.do_fd = any_fd;
  P.do_sync = 1;
  P.fdmap = any_fd ? fdmap : nullptr;
  P.nside_fdmap = any_fd ? nside_fdmap : 0;
  P.mask = nullptr;
  if (o0.do_mask) {
    const unsigned char *dm = nullptr;
    if ((st = device_mask(h, o0.nside_shell[s], &dm)) != HXG_OK) return st;
    P.mask = dm;
  }
  P.out[0] = tmp_dm;
  P.out[1] = tmp_fd;
  P.out[2] = P.out[3] = P.out[4] = nullptr;
  const uint64_t npix = npix_of(o0.nside_shell[s]);
  P.shard = shard;
  P.nshards = nshards;
  P.shard_log2 = shard_block_log2(npix, nshards);
  const uint64_t bsz = 1ull << P.shard_log2;
  const uint64_t nblk = (npix + bsz - 1) / bsz;
  const uint64_t local = nshards == 1 ? npix : (nblk + nshards - 1 - shard) / nshards * bsz;
  const int C = choose_chunks(h, local, step);
  P.chunks = C;
  P.log2_chunks = hpx_ilog2((uint64_t)C);
  if (local == 0) return HXG_OK;
  const uint64_t warps = (local + (32 / C) - 1) / (32 / C);
  const unsigned threads = HXG_FP32C_MULTI_THREADS;
  const unsigned blocks = (unsigned)((warps * 32 + threads - 1) / threads);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->timing) {
    HXG_CK(cudaEventCreate(&e0));
    HXG_CK(cudaEventCreate(&e1));
    HXG_CK(cudaEventRecord(e0, h->stream));
  }
  HXG_CK(launch_shell_multi(h->stream, P, NF, &Fq, blocks, threads));
  ++h->launch_count;
  if (h->timing) {
    HXG_CK(cudaEventRecord(e1, h->stream));
    h->events.emplace_back(e0, e1);
    h->event_samples.push_back((int64_t)(std::min(local, npix) * step * NF));
  }
  return HXG_OK;
}

// nf (2 or 3) fusable passes in one traversal per shell; outs[5 k + j] =
// map j (dm, fd, is, qs, us) of pass k.
template <int NF>
int write_fused(hxg_handle *h, const hxg_obs_t *o, double *const *outs) {
  const hxg_obs_t &o0 = o[0];
  uint32_t max_nside = 0;
  for (uint32_t s = 0; s < o0.total_shell; ++s) max_nside = std::max(max_nside, o0.nside_shell[s]);
  const size_t tbytes = npix_of(max_nside) * sizeof(double);
  int st;
  // the shell FD map is merged after each shell (the next one reads the
  // accumulated FD); the shared DM and each pass's I, Q, U of every shell
  // (map 0 and maps 1 + 3 f + j of the shell's block) are merged at the end
  if ((st = ensure(h, h->tmp_fd, tbytes)) != HXG_OK) return st;
  double *const tmp_fd = static_cast<double *>(h->tmp_fd.p);
  double *base[HXG_MAX_SHELLS];
  if ((st = shell_blocks(h, o0, 1 + 3 * NF, base)) != HXG_OK) return st;
  // the pass outputs start at zero (Grid_obs::build_grid, grid_obs.cc:21-43);
  // the inner-shell FD is read from the first pass that accumulates FD
  bool any_fd = false;
  int fd_pass = -1;
  for (int f = 0; f < NF; ++f) {
    double *const *m = outs + 5 * f;
    if (o[f].do_dm) HXG_CK(cudaMemsetAsync(m[0], 0, npix_of(o[f].nside_dm) * 8, h->stream));
    if (o[f].do_fd) HXG_CK(cudaMemsetAsync(m[1], 0, npix_of(o[f].nside_fd) * 8, h->stream));
    const size_t b = npix_of(o[f].nside_sync) * 8;
    for (int j = 2; j < 5; ++j) HXG_CK(cudaMemsetAsync(m[j], 0, b, h->stream));
    any_fd = any_fd || o[f].do_fd;
    if (o[f].do_fd && fd_pass < 0) fd_pass = f;
  }
  const ExtModels *ext_dev = nullptr;
  if ((st = upload_ext(h, h->models, o0.sync_freq, &ext_dev)) != HXG_OK) return st;
  for (uint32_t s = 0; s < o0.total_shell; ++s) {
    const size_t np = npix_of(o0.nside_shell[s]);
    double *tmp_iqu[NF][3];
    for (int f = 0; f < NF; ++f)
      for (int j = 0; j < 3; ++j) tmp_iqu[f][j] = base[s] + (size_t)(1 + 3 * f + j) * np;
    st = fused_shell<NF>(h, o, s, 0, 1, any_fd ? outs[5 * fd_pass + 1] : nullptr,
                         any_fd ? (int)o[fd_pass].nside_fd : 0, ext_dev, base[s], tmp_fd,
                         tmp_iqu);
    if (st != HXG_OK) return st;
    // every pass that asks for FD merges the shell FD map: one launch per
    // FD output Nside
    std::vector<bool> done(NF, false);
    for (int a = 0; a < NF; ++a) {
      if (!o[a].do_fd || done[a]) continue;
      std::vector<double *> d;
      std::vector<const double *> sr;
      for (int c = a; c < NF; ++c)
        if (o[c].do_fd && !done[c] && o[c].nside_fd == o[a].nside_fd) {
          d.push_back(outs[5 * c + 1]);
          sr.push_back(tmp_fd);
          done[c] = true;
        }
      InterpTab tab;
      if ((st = interp_tab(h, o[a].nside_fd, o0.nside_shell[s], &tab)) != HXG_OK) return st;
      HXG_CK(launch_accumulate(h->stream, (int)o[a].nside_fd, (int)o0.nside_shell[s],
                               (int)d.size(), d.data(), sr.data(), &tab));
      ++h->launch_count;
    }
  }
  std::vector<PassOut> pouts;
  for (int f = 0; f < NF; ++f) {
    double *const *m = outs + 5 * f;
    if (o[f].do_dm) pouts.push_back({o[f].nside_dm, 0, m[0]});
    for (int j = 0; j < 3; ++j) pouts.push_back({o[f].nside_sync, 1 + 3 * f + j, m[2 + j]});
  }
  if ((st = merge_pass(h, o0, base, pouts)) != HXG_OK) return st;
  h->ck_valid = false;
  return HXG_OK;
}

}  // namespace

extern "C" {

int hxg_write_grid_multi(hxg_handle *h, int npass, const hxg_obs_t *obs, double *const *d_outs) {
  if (!h) return HXG_ERR_INVALID;
  if (npass < 1 || !obs || !d_outs) return fail(h, HXG_ERR_INVALID, "bad pass list");
  cudaSetDevice(h->device);
  int st;
  for (int k = 0; k < npass; ++k) {
    double *const *m = d_outs + 5 * k;
    if ((st = check_pass(h, obs + k, m[0], m[1], m[2] && m[3] && m[4])) != HXG_OK) return st;
  }
  int k = 0;
  while (k < npass) {
    const int left = npass - k;
    const int nf = left >= 3 && fusable(h, obs + k, 3) ? 3 : (left >= 2 && fusable(h, obs + k, 2) ? 2 : 1);
    if (nf == 3)
      st = write_fused<3>(h, obs + k, d_outs + 5 * k);
    else if (nf == 2)
      st = write_fused<2>(h, obs + k, d_outs + 5 * k);
    else {
      double *const *m = d_outs + 5 * k;
      st = hxg_write_grid_device(h, obs + k, m[0], m[1], m[2], m[3], m[4]);
    }
    if (st != HXG_OK) return st;
    k += nf;
  }
  return HXG_OK;
}

int hxg_write_grid_multi_host(hxg_handle *h, int npass, const hxg_obs_t *obs,
                              double *const *outs) {
  if (!h) return HXG_ERR_INVALID;
  if (npass < 1 || !obs || !outs) return fail(h, HXG_ERR_INVALID, "bad pass list");
  cudaSetDevice(h->device);
  // device maps for every requested output, one allocation
  const auto count = [](const hxg_obs_t &o, int j) -> size_t {
    const bool on[5] = {o.do_dm != 0, o.do_fd != 0, o.do_sync != 0, o.do_sync != 0,
                        o.do_sync != 0};
    const uint32_t ns[5] = {o.nside_dm, o.nside_fd, o.nside_sync, o.nside_sync, o.nside_sync};
    return on[j] ? npix_of(ns[j]) : 0;
  };
  size_t total = 0;
  for (int k = 0; k < npass; ++k)
    for (int j = 0; j < 5; ++j) {
      if (count(obs[k], j) && !outs[5 * k + j])
        return fail(h, HXG_ERR_INVALID, "pass %d: output %d requested but NULL", k, j);
      total += count(obs[k], j);
    }
  int st = ensure(h, h->out[0], std::max<size_t>(total, 1) * sizeof(double));
  if (st != HXG_OK) return st;
  std::vector<double *> dev(5 * npass, nullptr);
  double *base = static_cast<double *>(h->out[0].p);
  for (int k = 0, off = 0; k < npass; ++k)
    for (int j = 0; j < 5; ++j)
      if (const size_t c = count(obs[k], j)) {
        dev[5 * k + j] = base + off;
        off += (int)c;
      }
  if ((st = hxg_write_grid_multi(h, npass, obs, dev.data())) != HXG_OK) return st;
  for (int k = 0; k < npass; ++k)
    for (int j = 0; j < 5; ++j)
      if (const size_t c = count(obs[k], j))
        HXG_CK(cudaMemcpyAsync(outs[5 * k + j], dev[5 * k + j], c * sizeof(double),
                               cudaMemcpyDeviceToHost, h->stream));
  HXG_CK(cudaStreamSynchronize(h->stream));
  return HXG_OK;
}

int hxg_shell_integrate_device(hxg_handle *h, const hxg_obs_t *o, uint32_t shell,
                               uint32_t shard, uint32_t nshards, const double *d_fd,
                               double *d_tmp_dm, double *d_tmp_fd, double *d_tmp_is,
                               double *d_tmp_qs, double *d_tmp_us) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!o || shell >= o->total_shell || nshards == 0 || shard >= nshards)
    return fail(h, HXG_ERR_INVALID, "bad shell %u or shard %u of %u", shell, shard, nshards);
  const bool sync3 = d_tmp_is && d_tmp_qs && d_tmp_us;
  int st = check_pass(h, o, d_tmp_dm, d_tmp_fd && (d_fd || !o->do_fd), sync3);
  if (st != HXG_OK) return st;
  if ((o->do_fd || o->do_sync) && !d_tmp_fd)
    return fail(h, HXG_ERR_INVALID, "the shell FD map is written whenever FD or sync is on");
  const uint64_t npix = npix_of(o->nside_shell[shell]);
  double *tmp[5] = {d_tmp_dm, d_tmp_fd, d_tmp_is, d_tmp_qs, d_tmp_us};
  if (nshards > 1) {  // pixels of other shards stay zero: shard maps add up
    for (int k = 0; k < 5; ++k)
      if (tmp[k]) HXG_CK(cudaMemsetAsync(tmp[k], 0, npix * sizeof(double), h->stream));
  }
  const ExtModels *ext_dev = nullptr;
  if ((st = upload_ext(h, h->models, o->sync_freq, &ext_dev)) != HXG_OK) return st;
  h->ck_valid = false;
  const bool ck = h->checkpoint;
  if (ck && (shell == 0 || h->ck_shell.size() != o->total_shell ||
             std::memcmp(&h->ck_sobs, o, sizeof(*o)) != 0 ||
             std::memcmp(&h->ck_smodels, &h->models, sizeof(h->models)) != 0 ||
             h->ck_shard != shard || h->ck_nshards != nshards)) {
    h->ck_shell.assign(o->total_shell, 0);
    h->ck_sobs = *o;
    h->ck_smodels = h->models;
    h->ck_shard = shard;
    h->ck_nshards = nshards;
  }
  h->adj_next = -1;
  h->adj_open = false;
  st = run_shell(h, *o, shell, ext_dev, d_fd, tmp, shard, nshards, ck);
  if (st == HXG_OK && ck) h->ck_shell[shell] = 1;
  return st;
}

int hxg_shell_integrate_multi_device(hxg_handle *h, int npass, const hxg_obs_t *o,
                                     uint32_t shell, uint32_t shard, uint32_t nshards,
                                     const double *d_fd, double *d_tmp_dm, double *d_tmp_fd,
                                     double *const *d_tmp_iqu) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!o || !d_tmp_iqu || npass < 2 || npass > 3 || shell >= o[0].total_shell ||
      nshards == 0 || shard >= nshards)
    return fail(h, HXG_ERR_INVALID, "bad pass count %d, shell %u or shard %u of %u", npass,
                shell, shard, nshards);
  int st;
  bool any_fd = false;
  int fd_pass = -1;
  for (int f = 0; f < npass; ++f) {
    const double *const *t = d_tmp_iqu + 3 * f;
    if ((st = check_pass(h, o + f, d_tmp_dm, d_tmp_fd && (d_fd || !o[f].do_fd),
                         t[0] && t[1] && t[2])) != HXG_OK)
      return st;
    any_fd = any_fd || o[f].do_fd;
    if (o[f].do_fd && fd_pass < 0) fd_pass = f;
  }
  if (!d_tmp_fd) return fail(h, HXG_ERR_INVALID, "the shell FD map is always written");
  if (!fusable(h, o, npass))
    return fail(h, HXG_ERR_UNSUPPORTED, "these passes cannot share a traversal");
  const uint64_t npix = npix_of(o[0].nside_shell[shell]);
  double *tmp_iqu[3][3];
  for (int f = 0; f < npass; ++f)
    for (int j = 0; j < 3; ++j) tmp_iqu[f][j] = d_tmp_iqu[3 * f + j];
  if (nshards > 1) {  // pixels of other shards stay zero: shard maps add up
    std::vector<double *> all = {d_tmp_dm, d_tmp_fd};
    for (int f = 0; f < npass; ++f)
      for (int j = 0; j < 3; ++j) all.push_back(tmp_iqu[f][j]);
    for (double *t : all)
      if (t) HXG_CK(cudaMemsetAsync(t, 0, npix * sizeof(double), h->stream));
  }
  const ExtModels *ext_dev = nullptr;
  if ((st = upload_ext(h, h->models, o[0].sync_freq, &ext_dev)) != HXG_OK) return st;
  h->ck_valid = false;
  const int nfd = any_fd ? (int)o[fd_pass].nside_fd : 0;
  if (npass == 2)
    return fused_shell<2>(h, o, shell, shard, nshards, d_fd, nfd, ext_dev, d_tmp_dm, d_tmp_fd,
                          tmp_iqu);
  return fused_shell<3>(h, o, shell, shard, nshards, d_fd, nfd, ext_dev, d_tmp_dm, d_tmp_fd,
                        tmp_iqu);
}

int hxg_shell_merge_device(hxg_handle *h, const hxg_obs_t *o, uint32_t shell,
                           const double *d_tmp_dm, const double *d_tmp_fd,
                           const double *d_tmp_is, const double *d_tmp_qs,
                           const double *d_tmp_us, double *d_dm, double *d_fd,
                           double *d_is, double *d_qs, double *d_us) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!o || shell >= o->total_shell) return fail(h, HXG_ERR_INVALID, "bad shell %u", shell);
  int st = validate_obs(h, o);
  if (st != HXG_OK) return st;
  if ((o->do_dm && (!d_dm || !d_tmp_dm)) || (o->do_fd && (!d_fd || !d_tmp_fd)) ||
      (o->do_sync && (!d_is || !d_qs || !d_us || !d_tmp_is || !d_tmp_qs || !d_tmp_us)))
    return fail(h, HXG_ERR_INVALID, "a map requested by obs is NULL");
  const double *tmp[5] = {d_tmp_dm, d_tmp_fd, d_tmp_is, d_tmp_qs, d_tmp_us};
  return merge_shell(h, *o, shell, tmp, d_dm, d_fd, d_is, d_qs, d_us);
}

}  // extern "C"

namespace {

// The adjoint of shell s for the pixels of shard `shard` of `nshards`
// (integrator.cc:60-133 differentiated): the transposes of the shell merges
// (integrator.cc:121-132) take dL/d(outputs) to dL/d(shell maps), with
// g_fdmap the complete dL/d(accumulated FD map) of the shells outside s;
// the kernel adds the shell's inner-FD gradients into gfd_target and the
// grid-record and parameter gradients into the handle's accumulators.
int adjoint_shell(hxg_handle *h, const hxg_obs_t &o, uint32_t s, uint32_t shard,
                  uint32_t nshards, const ExtModels *ext_dev, const double *g_dm,
                  const double *g_fdmap, const double *g_is, const double *g_qs,
                  const double *g_us, double *gfd_target) {
  const bool fp32 = h->precision == HXG_FP32C;
  ShellLaunch F;
  uint64_t step;
  int st = build_launch(h, h->models, o, s, F, step);
  if (st != HXG_OK) return st;
  F.ext = ext_dev;
  const int ns = (int)o.nside_shell[s];
  const uint64_t npix = npix_of((uint32_t)ns);
  double *gs[5];
  for (int k = 0; k < 5; ++k) gs[k] = static_cast<double *>(h->g_shell[k].p);
  for (int k = 0; k < 5; ++k)
    HXG_CK(cudaMemsetAsync(gs[k], 0, npix * sizeof(double), h->stream));
  // transposes of the shell merges (integrator.cc:121-132)
  if (o.do_dm && g_dm)
    HXG_CK(launch_accumulate_transpose(h->stream, (int)o.nside_dm, ns, g_dm, gs[0], 1.));
  if (o.do_fd)
    HXG_CK(launch_accumulate_transpose(h->stream, (int)o.nside_fd, ns, g_fdmap, gs[1], 1.));
  if (o.do_sync) {
    const double tc = F.tc_a * F.tc_a / F.tc_b;
    const double *gsy[3] = {g_is, g_qs, g_us};
    for (int k = 0; k < 3; ++k)
      if (gsy[k])
        HXG_CK(launch_accumulate_transpose(h->stream, (int)o.nside_sync, ns, gsy[k], gs[2 + k],
                                           tc));
  }
  F.fdmap = o.do_fd ? g_fdmap : nullptr;  // non-null marks inner-FD use
  F.nside_fdmap = o.do_fd ? (int)o.nside_fd : 0;
  F.mask = nullptr;
  if (o.do_mask) {
    const unsigned char *dmk = nullptr;
    if ((st = device_mask(h, o.nside_shell[s], &dmk)) != HXG_OK) return st;
    F.mask = dmk;
  }
  const int C = h->ck_chunks[s];
  F.chunks = C;
  F.log2_chunks = hpx_ilog2((uint64_t)C);
  F.shard = shard;
  F.nshards = nshards;
  F.shard_log2 = shard_block_log2(npix, nshards);
  const uint64_t bsz = 1ull << F.shard_log2;
  const uint64_t nblk = (npix + bsz - 1) / bsz;
  const uint64_t local = nshards == 1 ? npix : (nblk + nshards - 1 - shard) / nshards * bsz;
  if (fp32 && !fast_models(F))
    return fail(h, HXG_ERR_UNSUPPORTED,
                "the FP32C adjoint covers the grid workloads' models (spiral or no regular "
                "B, exponential disk or no regular n_e, CRE_ana with a constant index, no "
                "inner radius cut); run the FP64 form");
  AdjointLaunch A{};
  A.F = F;
  A.ck = static_cast<const double *>(h->ck[s].p);
  A.ck_inner = static_cast<const double *>(h->ck_inner[s].p);
  for (int k = 0; k < 5; ++k) A.g[k] = gs[k];
  const size_t ngrid = h->groups.empty() ? 0 : h->groups[0].n;
  A.grad_rec = ngrid ? static_cast<double *>(h->grad_rec.p) : nullptr;
  A.grad_par = static_cast<double *>(h->grad_par.p);
  A.g_fdmap = o.do_fd ? gfd_target : nullptr;
  A.want_j0 = (h->models.cre == HXG_CRE_ANA || h->models.cre == HXG_CRE_UNIF) ? 1 : 0;
  if (local == 0) return HXG_OK;
  const uint64_t warps = (local + (32 / C) - 1) / (32 / C);
  const unsigned threads = fp32 ? HXG_ADJ32_THREADS : HXG_ADJ_THREADS;
  const unsigned blocks = (unsigned)((warps * 32 + threads - 1) / threads);
  HXG_CK(fp32 ? launch_adjoint32(h->stream, A, blocks, threads)
              : launch_adjoint(h->stream, A, blocks, threads));
  ++h->launch_count;
  return HXG_OK;
}

// Checks and zeroed accumulators of a reverse-mode pass: the grid-record
// and parameter gradients and the per-shell gradient maps.
int adjoint_prepare(hxg_handle *h, const hxg_obs_t &o) {
  if (h->groups.size() > 1)
    return fail(h, HXG_ERR_UNSUPPORTED, "the adjoint supports one grid geometry");
  if (h->models.cre == HXG_CRE_GRID)
    return fail(h, HXG_ERR_UNSUPPORTED, "the adjoint does not cover the CRE-grid emissivity");
  int st;
  const size_t ngrid = h->groups.empty() ? 0 : h->groups[0].n;
  if (ngrid) {
    if ((st = ensure(h, h->grad_rec, ngrid * 4 * sizeof(double))) != HXG_OK) return st;
    HXG_CK(cudaMemsetAsync(h->grad_rec.p, 0, ngrid * 4 * sizeof(double), h->stream));
  }
  if ((st = ensure(h, h->grad_par, kNumParams * sizeof(double))) != HXG_OK) return st;
  HXG_CK(cudaMemsetAsync(h->grad_par.p, 0, kNumParams * sizeof(double), h->stream));
  uint32_t max_nside = 0;
  for (uint32_t s = 0; s < o.total_shell; ++s) max_nside = std::max(max_nside, o.nside_shell[s]);
  for (int k = 0; k < 5; ++k)
    if ((st = ensure(h, h->g_shell[k], npix_of(max_nside) * sizeof(double))) != HXG_OK)
      return st;
  return HXG_OK;
}

// dL/d(parameters) and dL/d(grid values) from the handle's accumulators
// (the grid records unpacked into the slots' SoA layout and units).
int adjoint_finish(hxg_handle *h, double *d_grad_params, double *d_grad_bx, double *d_grad_by,
                   double *d_grad_bz, double *d_grad_ne) {
  const bool fp32 = h->precision == HXG_FP32C;
  const size_t ngrid = h->groups.empty() ? 0 : h->groups[0].n;
  // parameter gradients: j0 slot holds sum (dL/dJ) J, divide by j0
  double gp[kNumParams];
  HXG_CK(cudaMemcpyAsync(gp, h->grad_par.p, sizeof(gp), cudaMemcpyDeviceToHost, h->stream));
  HXG_CK(cudaStreamSynchronize(h->stream));
  const double j0 = h->models.cre == HXG_CRE_ANA ? h->models.cre_ana.j0
                                                 : h->models.cre_unif.j0;
  gp[7] = (j0 != 0.) ? gp[7] / j0 : 0.;
  if (fp32) {
    // the FP32C kernel sums log-derivatives for the amplitudes and
    // per-kpc derivatives for the lengths (hxg_adjoint32.cuh)
    const auto &sp = h->models.spiral;
    const auto &ex = h->models.te_exp;
    gp[0] = sp.b0 != 0. ? gp[0] / sp.b0 : 0.;
    gp[4] = ex.n0 != 0. ? gp[4] / ex.n0 : 0.;
    for (int k : {2, 3, 5, 6}) gp[k] /= cgs::kpc;
  }
  if (d_grad_params)
    HXG_CK(cudaMemcpyAsync(d_grad_params, gp, sizeof(gp), cudaMemcpyHostToDevice, h->stream));
  if (ngrid && (d_grad_bx || d_grad_ne)) {
    const Group &G = h->groups[0];
    const bool has_b = G.b_slots[0] >= 0, has_t = G.t_slots[0] >= 0;
    HXG_CK(launch_unpack_grad(h->stream, ngrid, static_cast<const double *>(h->grad_rec.p),
                              has_b ? d_grad_bx : nullptr, has_b ? d_grad_by : nullptr,
                              has_b ? d_grad_bz : nullptr, has_t ? d_grad_ne : nullptr,
                              fp32 ? 1.0 / cgs::fp32_bunit : 1.0));
  }
  HXG_CK(cudaStreamSynchronize(h->stream));
  return HXG_OK;
}

}  // namespace

extern "C" {

int hxg_set_checkpointing(hxg_handle *h, int enable) {
  if (!h) return HXG_ERR_INVALID;
  h->checkpoint = enable != 0;
  h->ck_valid = false;
  h->ck_shell.clear();
  h->adj_next = -1;
  h->adj_open = false;
  return HXG_OK;
}

int hxg_adjoint_shard_begin(hxg_handle *h, const hxg_obs_t *o, uint32_t shard,
                            uint32_t nshards) {
  if (!h || !o) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  bool all = h->ck_shell.size() == o->total_shell && o->total_shell > 0;
  for (char c : h->ck_shell) all = all && c;
  if (!all || std::memcmp(&h->ck_sobs, o, sizeof(*o)) != 0 ||
      std::memcmp(&h->ck_smodels, &h->models, sizeof(h->models)) != 0 ||
      h->ck_shard != shard || h->ck_nshards != nshards)
    return fail(h, HXG_ERR_STATE,
                "no checkpointed per-shell forward pass of shard %u of %u for these obs/models "
                "(enable hxg_set_checkpointing and call hxg_shell_integrate_device for every "
                "shell first)", shard, nshards);
  const int st = adjoint_prepare(h, *o);
  if (st != HXG_OK) return st;
  h->adj_next = (int)o->total_shell - 1;
  h->adj_open = true;
  return HXG_OK;
}

int hxg_adjoint_shard_shell(hxg_handle *h, const hxg_obs_t *o, uint32_t shell,
                            const double *g_dm, const double *g_fdmap, const double *g_is,
                            const double *g_qs, const double *g_us, double *d_gfd_inc) {
  if (!h || !o) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!h->adj_open || std::memcmp(&h->ck_sobs, o, sizeof(*o)) != 0)
    return fail(h, HXG_ERR_STATE, "no sharded adjoint open for these obs (hxg_adjoint_shard_begin)");
  if (shell >= o->total_shell || (int)shell != h->adj_next)
    return fail(h, HXG_ERR_INVALID, "shell %u out of order: the adjoint runs shell %d next "
                "(outermost first)", shell, h->adj_next);
  if (o->do_fd && (!g_fdmap || !d_gfd_inc))
    return fail(h, HXG_ERR_INVALID, "an FD pass needs g_fdmap and the increment map");
  if (o->do_fd)
    HXG_CK(cudaMemsetAsync(d_gfd_inc, 0, npix_of(o->nside_fd) * sizeof(double), h->stream));
  const ExtModels *ext_dev = nullptr;
  int st = upload_ext(h, h->models, o->sync_freq, &ext_dev);
  if (st != HXG_OK) return st;
  st = adjoint_shell(h, *o, shell, h->ck_shard, h->ck_nshards, ext_dev, g_dm,
                     o->do_fd ? g_fdmap : nullptr, g_is, g_qs, g_us,
                     o->do_fd ? d_gfd_inc : nullptr);
  if (st != HXG_OK) return st;
  --h->adj_next;
  return HXG_OK;
}

int hxg_adjoint_shard_finish(hxg_handle *h, double *d_grad_params, double *d_grad_bx,
                             double *d_grad_by, double *d_grad_bz, double *d_grad_ne) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!h->adj_open || h->adj_next != -1)
    return fail(h, HXG_ERR_STATE, "the sharded adjoint has shells left or was not begun");
  h->adj_open = false;
  h->ck_shell.clear();  // one reverse pass per forward pass
  return adjoint_finish(h, d_grad_params, d_grad_bx, d_grad_by, d_grad_bz, d_grad_ne);
}

// Reverse-mode pass over the shells of the last checkpointed forward call
// (integrator.cc:23-228 differentiated): outer shells first, so that the
// inner-shell Faraday-depth gradients of shell s reach shells < s.
int hxg_adjoint_device(hxg_handle *h, const hxg_obs_t *o, const double *g_dm,
                       const double *g_fd, const double *g_is,
                       const double *g_qs, const double *g_us,
                       double *d_grad_params, double *d_grad_bx,
                       double *d_grad_by, double *d_grad_bz,
                       double *d_grad_ne) {
  if (!h || !o) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!h->ck_valid || std::memcmp(&h->ck_obs, o, sizeof(*o)) != 0 ||
      std::memcmp(&h->ck_models, &h->models, sizeof(h->models)) != 0)
    return fail(h, HXG_ERR_STATE,
                "no checkpointed forward pass for these obs/models (enable "
                "hxg_set_checkpointing and call hxg_write_grid_device first)");
  int st = adjoint_prepare(h, *o);
  if (st != HXG_OK) return st;
  double *gfdmap = nullptr;
  if (o->do_fd) {
    const size_t b = npix_of(o->nside_fd) * sizeof(double);
    if ((st = ensure(h, h->g_fdmap, b)) != HXG_OK) return st;
    gfdmap = static_cast<double *>(h->g_fdmap.p);
    if (g_fd)
      HXG_CK(cudaMemcpyAsync(gfdmap, g_fd, b, cudaMemcpyDeviceToDevice, h->stream));
    else
      HXG_CK(cudaMemsetAsync(gfdmap, 0, b, h->stream));
  }
  const ExtModels *ext_dev = nullptr;
  if ((st = upload_ext(h, h->models, o->sync_freq, &ext_dev)) != HXG_OK) return st;
  for (int s = (int)o->total_shell - 1; s >= 0; --s) {
    st = adjoint_shell(h, *o, (uint32_t)s, 0, 1, ext_dev, g_dm, gfdmap, g_is, g_qs, g_us,
                       gfdmap);
    if (st != HXG_OK) return st;
  }
  return adjoint_finish(h, d_grad_params, d_grad_bx, d_grad_by, d_grad_bz, d_grad_ne);
}

int hxg_write_grid(hxg_handle *h, const hxg_obs_t *o, double *dm, double *fd,
                   double *is, double *qs, double *us) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  int st = validate_obs(h, o);
  if (st != HXG_OK) return st;
  if ((o->do_dm && !dm) || (o->do_fd && !fd) || (o->do_sync && (!is || !qs || !us)))
    return fail(h, HXG_ERR_INVALID, "an output requested by obs is NULL");
  const size_t b_dm = o->do_dm ? npix_of(o->nside_dm) * 8 : 8;
  const size_t b_fd = o->do_fd ? npix_of(o->nside_fd) * 8 : 8;
  const size_t b_sy = o->do_sync ? npix_of(o->nside_sync) * 8 : 8;
  const size_t bytes[5] = {b_dm, b_fd, b_sy, b_sy, b_sy};
  for (int k = 0; k < 5; ++k)
    if ((st = ensure(h, h->out[k], bytes[k])) != HXG_OK) return st;
  double *d[5];
  for (int k = 0; k < 5; ++k) d[k] = static_cast<double *>(h->out[k].p);
  st = hxg_write_grid_device(h, o, d[0], d[1], d[2], d[3], d[4]);
  if (st != HXG_OK) return st;
  double *host[5] = {dm, fd, is, qs, us};
  const bool want[5] = {o->do_dm != 0, o->do_fd != 0, o->do_sync != 0,
                        o->do_sync != 0, o->do_sync != 0};
  for (int k = 0; k < 5; ++k)
    if (want[k])
      HXG_CK(cudaMemcpyAsync(host[k], d[k], bytes[k], cudaMemcpyDeviceToHost, h->stream));
  HXG_CK(cudaStreamSynchronize(h->stream));
  return HXG_OK;
}

int hxg_sync(hxg_handle *h) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  HXG_CK(cudaStreamSynchronize(h->stream));
  HXG_CK(cudaGetLastError());
  return HXG_OK;
}

int hxg_set_interp_cache(hxg_handle *h, uint64_t bytes) {
  if (!h) return HXG_ERR_INVALID;
  h->interp_limit = (size_t)bytes;
  return HXG_OK;
}

int hxg_set_timing(hxg_handle *h, int enable) {
  if (!h) return HXG_ERR_INVALID;
  h->timing = enable != 0;
  h->acc_ms = 0.;
  h->acc_launches = h->acc_samples = 0;
  for (auto &e : h->events) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  h->events.clear();
  h->event_samples.clear();
  return HXG_OK;
}

int hxg_get_timing(hxg_handle *h, double *kernel_ms, int64_t *launches,
                   int64_t *samples) {
  if (!h) return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  HXG_CK(cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < h->events.size(); ++i) {
    float ms = 0.f;
    HXG_CK(cudaEventElapsedTime(&ms, h->events[i].first, h->events[i].second));
    h->acc_ms += ms;
    h->acc_launches += 1;
    h->acc_samples += h->event_samples[i];
    cudaEventDestroy(h->events[i].first);
    cudaEventDestroy(h->events[i].second);
  }
  h->events.clear();
  h->event_samples.clear();
  if (kernel_ms) *kernel_ms = h->acc_ms;
  if (launches) *launches = h->acc_launches;
  if (samples) *samples = h->acc_samples;
  return HXG_OK;
}

int hxg_get_launch_count(hxg_handle *h, int64_t *count) {
  if (!h || !count) return HXG_ERR_INVALID;
  *count = h->launch_count;
  return HXG_OK;
}

int hxg_shell_ref(const hxg_obs_t *obs, uint32_t shell, double *d_start,
                  double *delta_d, uint64_t *step) {
  if (!obs || !d_start || !delta_d || !step || shell >= obs->total_shell ||
      obs->total_shell > HXG_MAX_SHELLS)
    return HXG_ERR_INVALID;
  shell_ref(*obs, shell, *d_start, *delta_d, *step);
  return HXG_OK;
}

int hxg_mask_duplicate(uint32_t pivot_nside, const double *pivot_mask,
                       uint32_t nside, double *out) {
  if (!pivot_mask || !out || !is_pow2(pivot_nside) || !is_pow2(nside) ||
      pivot_nside > 8192 || nside > 8192)
    return HXG_ERR_INVALID;
  mask_duplicate_host(pivot_nside, pivot_mask, nside, out);
  return HXG_OK;
}

// ---- device known-answer helpers ----------------------------------------
namespace {
struct Scratch {
  std::vector<void *> ptrs;
  ~Scratch() {
    for (void *p : ptrs) cudaFree(p);
  }
  double *alloc(size_t n) {
    void *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(double) + 8) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<double *>(p);
  }
};

int kat_status(cudaError_t e) {
  if (e == cudaSuccess) return HXG_OK;
  return e == cudaErrorMemoryAllocation ? HXG_ERR_OOM : HXG_ERR_CUDA;
}

#define KAT_ALLOC(var, n) \
  double *var = S.alloc(n); \
  if (!var) return HXG_ERR_OOM;
#define KAT_CK(call)                          \
  do {                                        \
    const int s_ = kat_status(call);          \
    if (s_ != HXG_OK) return s_;              \
  } while (0)

int kat_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return HXG_ERR_NO_DEVICE;
  return HXG_OK;
}
}  // namespace

int hxg_pix2ang(uint32_t nside, uint64_t npix, double *theta, double *phi) {
  if (!theta || !phi || !is_pow2(nside) || nside > 8192 || npix > npix_of(nside))
    return HXG_ERR_INVALID;
  if (kat_device() != HXG_OK) return HXG_ERR_NO_DEVICE;
  Scratch S;
  KAT_ALLOC(dt, npix);
  KAT_ALLOC(dp, npix);
  KAT_CK(launch_pix2ang(0, (int)nside, npix, dt, dp));
  KAT_CK(cudaMemcpy(theta, dt, npix * 8, cudaMemcpyDeviceToHost));
  KAT_CK(cudaMemcpy(phi, dp, npix * 8, cudaMemcpyDeviceToHost));
  return HXG_OK;
}

int hxg_interpolate(uint32_t nside, const double *map, uint64_t n,
                    const double *theta, const double *phi, double *out) {
  if (!map || !theta || !phi || !out || !is_pow2(nside) || nside > 8192)
    return HXG_ERR_INVALID;
  if (kat_device() != HXG_OK) return HXG_ERR_NO_DEVICE;
  Scratch S;
  const uint64_t np = npix_of(nside);
  KAT_ALLOC(dm, np);
  KAT_ALLOC(dt, n);
  KAT_ALLOC(dp, n);
  KAT_ALLOC(dout, n);
  KAT_CK(cudaMemcpy(dm, map, np * 8, cudaMemcpyHostToDevice));
  KAT_CK(cudaMemcpy(dt, theta, n * 8, cudaMemcpyHostToDevice));
  KAT_CK(cudaMemcpy(dp, phi, n * 8, cudaMemcpyHostToDevice));
  KAT_CK(launch_interpolate(0, (int)nside, dm, n, dt, dp, dout));
  KAT_CK(cudaMemcpy(out, dout, n * 8, cudaMemcpyDeviceToHost));
  return HXG_OK;
}

int hxg_accumulate(uint32_t nside_dst, double *dst, uint32_t nside_src,
                   const double *src) {
  if (!dst || !src || !is_pow2(nside_dst) || !is_pow2(nside_src) ||
      nside_dst > 8192 || nside_src > 8192)
    return HXG_ERR_INVALID;
  if (kat_device() != HXG_OK) return HXG_ERR_NO_DEVICE;
  Scratch S;
  const uint64_t nd = npix_of(nside_dst), ns = npix_of(nside_src);
  KAT_ALLOC(dd, nd);
  KAT_ALLOC(ds, ns);
  KAT_CK(cudaMemcpy(dd, dst, nd * 8, cudaMemcpyHostToDevice));
  KAT_CK(cudaMemcpy(ds, src, ns * 8, cudaMemcpyHostToDevice));
  double *d[1] = {dd};
  const double *s[1] = {ds};
  KAT_CK(launch_accumulate(0, (int)nside_dst, (int)nside_src, 1, d, s));
  KAT_CK(cudaMemcpy(dst, dd, nd * 8, cudaMemcpyDeviceToHost));
  return HXG_OK;
}

int hxg_los_geometry(uint64_t n, const double *theta, const double *phi,
                     const double *b, double *versor, double *b_par,
                     double *b_per, double *cos2ipa, double *sin2ipa) {
  if (!theta || !phi || !b || !versor || !b_par || !b_per || !cos2ipa || !sin2ipa)
    return HXG_ERR_INVALID;
  if (kat_device() != HXG_OK) return HXG_ERR_NO_DEVICE;
  Scratch S;
  KAT_ALLOC(dt, n);
  KAT_ALLOC(dp, n);
  KAT_ALLOC(db, 3 * n);
  KAT_ALLOC(dv, 3 * n);
  KAT_ALLOC(dpar, n);
  KAT_ALLOC(dper, n);
  KAT_ALLOC(dc, n);
  KAT_ALLOC(ds, n);
  KAT_CK(cudaMemcpy(dt, theta, n * 8, cudaMemcpyHostToDevice));
  KAT_CK(cudaMemcpy(dp, phi, n * 8, cudaMemcpyHostToDevice));
  KAT_CK(cudaMemcpy(db, b, 3 * n * 8, cudaMemcpyHostToDevice));
  KAT_CK(launch_los_geometry(0, n, dt, dp, db, dv, dpar, dper, dc, ds));
  KAT_CK(cudaMemcpy(versor, dv, 3 * n * 8, cudaMemcpyDeviceToHost));
  KAT_CK(cudaMemcpy(b_par, dpar, n * 8, cudaMemcpyDeviceToHost));
  KAT_CK(cudaMemcpy(b_per, dper, n * 8, cudaMemcpyDeviceToHost));
  KAT_CK(cudaMemcpy(cos2ipa, dc, n * 8, cudaMemcpyDeviceToHost));
  KAT_CK(cudaMemcpy(sin2ipa, ds, n * 8, cudaMemcpyDeviceToHost));
  return HXG_OK;
}

int hxg_synchrotron(int which, uint64_t n, const double *x, double *out) {
  if ((which != 1 && which != 2) || (n > 0 && (!x || !out))) return HXG_ERR_INVALID;
  const std::vector<double> &tab = synchro_tables();
  const double *t = tab.data() + (which == 1 ? 0 : kSynchroN);
  const double inv_du = (kSynchroN - 1) / (kSynchroU1 - kSynchroU0);
  for (uint64_t i = 0; i < n; ++i)
    out[i] = x[i] > 0. ? synchro_fn(t, kSynchroU0, inv_du, kSynchroN, x[i]) : 0.;
  return HXG_OK;
}

int hxg_read_grid(hxg_handle *h, int field, uint64_t n, const double *pos,
                  double *out) {
  if (!h || !pos || !out || field < 0 || field > HXG_FIELD_TERND)
    return HXG_ERR_INVALID;
  cudaSetDevice(h->device);
  if (!h->have_models) return fail(h, HXG_ERR_STATE, "models not set");
  int st = build_groups(h);
  if (st != HXG_OK) return st;
  const Group *G = nullptr;
  for (const auto &g : h->groups)
    for (int k = 0; k < 2; ++k)
      if (g.b_slots[k] == field || g.t_slots[k] == field) G = &g;
  if (!G) return fail(h, HXG_ERR_STATE, "grid slot %d is not read by the models", field);
  const bool fp32 = h->precision == HXG_FP32C;
  const double L = fp32 ? 1.0 / cgs::kpc : 1.0;
  DevGridGroup D{};
  D.rec = G->rec;
  D.nx = (int)G->desc.nx;
  D.ny = (int)G->desc.ny;
  D.nz = (int)G->desc.nz;
  D.gmax[0] = (double)(G->desc.nx - 1);
  D.gmax[1] = (double)(G->desc.ny - 1);
  D.gmax[2] = (double)(G->desc.nz - 1);
  D.lo[0] = G->desc.x_min * L;
  D.lo[1] = G->desc.y_min * L;
  D.lo[2] = G->desc.z_min * L;
  D.scale[0] = (double)(G->desc.nx - 1) / ((G->desc.x_max - G->desc.x_min) * L);
  D.scale[1] = (double)(G->desc.ny - 1) / ((G->desc.y_max - G->desc.y_min) * L);
  D.scale[2] = (double)(G->desc.nz - 1) / ((G->desc.z_max - G->desc.z_min) * L);
  std::vector<double> p(3 * n), res(4 * n);
  for (uint64_t i = 0; i < 3 * n; ++i) p[i] = pos[i] * L;
  Scratch S;
  double *dpos = S.alloc(3 * n), *dout = S.alloc(4 * n);
  if (!dpos || !dout) return fail(h, HXG_ERR_OOM, "scratch");
  HXG_CK(cudaMemcpy(dpos, p.data(), 3 * n * 8, cudaMemcpyHostToDevice));
  HXG_CK(launch_read_group(0, fp32, D, n, dpos, dout));
  HXG_CK(cudaMemcpy(res.data(), dout, 4 * n * 8, cudaMemcpyDeviceToHost));
  const double bu = fp32 ? cgs::fp32_bunit : 1.0;
  const bool vec = field == HXG_FIELD_BREG || field == HXG_FIELD_BRND;
  for (uint64_t i = 0; i < n; ++i) {
    if (vec)
      for (int k = 0; k < 3; ++k) out[3 * i + k] = res[4 * i + k] * bu;
    else
      out[i] = res[4 * i + 3];
  }
  return HXG_OK;
}

}  // extern "C"

// ===================================================================
// batched forward
// ===================================================================
struct hxg_batch {
  hxg_handle *h = nullptr;
  std::vector<hxg_batch_entry_t> e;
  int levels = 0;
  bool fp32 = false;
  int ngroups = 0;
  int lanes = 1, grain = 4, tried = 0;
  double best_ms = 0.;
  int64_t samples = 0;
  std::vector<size_t> tmp_off;  // per entry, doubles into tmp
  std::vector<size_t> tmp_n;    // per entry, doubles per map
  DevBuf tmp, zeros, zblocks, counters;
  DevBuf ext;               // ExtModels per entry (entries that use them)
  bool ext_any = false;
  // plan tables per (level, class): class c holds plans of c + 1 fused
  // frequency passes, at index 3 * level + c
  std::vector<DevBuf> plans, tiles, merges, mblocks;
  std::vector<int> nplans, nmerge;
  std::vector<unsigned long long> merge_blocks;
  std::vector<int> group;  // passes fused with entry i (0: inside a group)
  int nzero = 0;
  unsigned long long zero_blocks = 0;
  unsigned level_blocks[3] = {0, 0, 0};
  int graph_kernels = 0;  // kernels one run of the graph launches
  uint64_t layout_gen = 0;  // the handle's layout_gen the graph was made for
  bool fast = false;        // every entry's models satisfy fast_models
  cudaGraphExec_t exec = nullptr;
};

namespace {

using hxg::BatchLevel;
using hxg::MergeJob;
using hxg::ShellLaunch;
using hxg::ZeroJob;

bool reads_grid(const hxg_models_t &m, int which) {
  switch (which) {
    case 0: return m.breg == HXG_BREG_GRID;
    case 1: return m.brnd == HXG_BRND_GRID;
    case 2: return m.tereg == HXG_TEREG_GRID;
    case 3: return m.ternd == HXG_TERND_GRID;
    default: return m.cre == HXG_CRE_GRID;
  }
}

template <typename T>
int upload_vec(hxg_handle *h, DevBuf &b, const std::vector<T> &v) {
  const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
  int st = ensure(h, b, bytes);
  if (st != HXG_OK) return st;
  if (!v.empty()) HXG_CK(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return HXG_OK;
}

// Device tables of a batch for one launch shape.
int batch_tables(hxg_batch *b, int lanes, int grain) {
  hxg_handle *h = b->h;
  int st;
  b->lanes = lanes;
  b->grain = grain;
  b->samples = 0;
  double *tmp = static_cast<double *>(b->tmp.p);
  const auto map = [&](size_t i, int k) { return tmp + b->tmp_off[i] + k * b->tmp_n[i]; };
  for (int s = 0; s < b->levels; ++s) {
    std::vector<ShellLaunch> P1;
    std::vector<hxg::FusedPlan<2>> P2;
    std::vector<hxg::FusedPlan<3>> P3;
    std::vector<unsigned long long> t0[3];
    for (auto &t : t0) t.assign(1, 0ull);
    std::vector<MergeJob> mj;
    std::vector<unsigned long long> m0(1, 0ull);
    int tab_st = HXG_OK;
    const auto job = [&](int nmaps, double *const *d, const double *const *src, uint32_t nd,
                         int ns) {
      MergeJob J{};
      for (int q = 0; q < nmaps; ++q) {
        J.dst[q] = d[q];
        J.src[q] = src[q];
      }
      J.nmaps = nmaps;
      J.nside_dst = (int)nd;
      J.nside_src = ns;
      const int ts = interp_tab(h, nd, (uint32_t)ns, &J.tab);
      if (ts != HXG_OK) tab_st = ts;
      mj.push_back(J);
      m0.push_back(m0.back() + (npix_of(nd) + 255) / 256);
    };
    for (size_t i = 0; i < b->e.size(); i += (size_t)b->group[i]) {
      const int nf = b->group[i];
      const hxg_batch_entry_t &E = b->e[i];
      const hxg_obs_t &o = E.obs;
      if ((uint32_t)s >= o.total_shell) continue;
      ShellLaunch L;
      uint64_t step;
      if ((st = build_launch(h, E.models, o, (uint32_t)s, L, step)) != HXG_OK) return st;
      L.mask = nullptr;
      L.ext = uses_ext(E.models) ? static_cast<const ExtModels *>(b->ext.p) + i : nullptr;
      int C = std::min(lanes, 32);
      while (C > 1 && step / (uint64_t)C < 16) C >>= 1;
      L.chunks = C;
      L.log2_chunks = hxg::hpx_ilog2((uint64_t)C);
      const uint64_t npix = npix_of(o.nside_shell[s]);
      const int ns = (int)o.nside_shell[s];
      const unsigned long long tiles = (npix * C + 31) / 32;
      b->samples += (int64_t)(npix * step * nf);
      // inner-shell FD and the shared DM / FD shell maps: the first pass of
      // the group that accumulates FD; DM / FD shell maps live in the
      // group's first entry
      size_t fd_entry = i;
      bool any_dm = false, any_fd = false;
      for (int f = nf - 1; f >= 0; --f) {
        any_dm = any_dm || b->e[i + f].obs.do_dm;
        if (b->e[i + f].obs.do_fd) {
          any_fd = true;
          fd_entry = i + f;
        }
      }
      L.fdmap = any_fd ? b->e[fd_entry].d_fd : nullptr;
      L.nside_fdmap = any_fd ? (int)b->e[fd_entry].obs.nside_fd : 0;
      for (int k = 0; k < 5; ++k) L.out[k] = map(i, k);
      if (nf > 1) {
        L.do_dm = any_dm;
        L.do_fd = any_fd;
        L.do_sync = 1;
        L.out[2] = L.out[3] = L.out[4] = nullptr;
      }
      const auto freqs = [&](auto &F) -> int {
        for (int f = 0; f < nf; ++f) {
          ShellLaunch Lf;
          uint64_t sf;
          const int r = build_launch(h, b->e[i + f].models, b->e[i + f].obs, (uint32_t)s, Lf, sf);
          if (r != HXG_OK) return r;
          F.lambda2[f] = Lf.lambda2;
          F.phase_k[f] = Lf.phase_k;
          F.k_t[f] = Lf.k_t;
          F.k_p[f] = Lf.k_p;
          F.tc_a[f] = Lf.tc_a;
          F.tc_b[f] = Lf.tc_b;
          F.a_s[f] = Lf.a_s;
          F.inner[f] = b->e[i + f].obs.do_fd ? 1 : 0;
          for (int j = 0; j < 3; ++j) F.out[f][j] = map(i + f, 2 + j);
        }
        return HXG_OK;
      };
      if (nf == 1) {
        P1.push_back(L);
      } else if (nf == 2) {
        hxg::FusedPlan<2> FP;
        FP.P = L;
        if ((st = freqs(FP.F)) != HXG_OK) return st;
        P2.push_back(FP);
      } else {
        hxg::FusedPlan<3> FP;
        FP.P = L;
        if ((st = freqs(FP.F)) != HXG_OK) return st;
        P3.push_back(FP);
      }
      t0[nf - 1].push_back(t0[nf - 1].back() + tiles);
      for (int f = 0; f < nf; ++f) {
        const hxg_batch_entry_t &Ef = b->e[i + f];
        const hxg_obs_t &of = Ef.obs;
        if (of.do_dm) {
          double *d[1] = {Ef.d_dm};
          const double *sr[1] = {map(i, 0)};
          job(1, d, sr, of.nside_dm, ns);
        }
        if (of.do_sync) {
          double *d[3] = {Ef.d_is, Ef.d_qs, Ef.d_us};
          const double *sr[3] = {map(i + f, 2), map(i + f, 3), map(i + f, 4)};
          job(3, d, sr, of.nside_sync, ns);
        }
        if (of.do_fd) {
          double *d[1] = {Ef.d_fd};
          const double *sr[1] = {map(i, 1)};
          job(1, d, sr, of.nside_fd, ns);
        }
      }
    }
    const int c0 = 3 * s;
    b->nplans[c0] = (int)P1.size();
    b->nplans[c0 + 1] = (int)P2.size();
    b->nplans[c0 + 2] = (int)P3.size();
    if (tab_st != HXG_OK) return tab_st;
    b->nmerge[s] = (int)mj.size();
    b->merge_blocks[s] = m0.back();
    if ((st = upload_vec(h, b->plans[c0], P1)) != HXG_OK) return st;
    if ((st = upload_vec(h, b->plans[c0 + 1], P2)) != HXG_OK) return st;
    if ((st = upload_vec(h, b->plans[c0 + 2], P3)) != HXG_OK) return st;
    for (int c = 0; c < 3; ++c)
      if ((st = upload_vec(h, b->tiles[c0 + c], t0[c])) != HXG_OK) return st;
    if ((st = upload_vec(h, b->merges[s], mj)) != HXG_OK) return st;
    if ((st = upload_vec(h, b->mblocks[s], m0)) != HXG_OK) return st;
  }
  return HXG_OK;
}

void batch_drop_graph(hxg_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

int batch_capture(hxg_batch *b) {
  hxg_handle *h = b->h;
  batch_drop_graph(b);
  cudaStream_t s = h->stream;
  HXG_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = hxg::launch_batch_zero(s, static_cast<const ZeroJob *>(b->zeros.p),
                                         static_cast<const unsigned long long *>(b->zblocks.p),
                                         b->nzero, b->zero_blocks);
  unsigned long long *ctr = static_cast<unsigned long long *>(b->counters.p);
  b->graph_kernels = 1 + b->levels;  // zeroing, one merge per level
  for (int l = 0; l < b->levels && e == cudaSuccess; ++l) {
    for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
      const int k = 3 * l + c;
      if (b->nplans[k] == 0) continue;
      ++b->graph_kernels;
      e = cudaMemsetAsync(ctr + k, 0, sizeof(unsigned long long), s);
      if (e != cudaSuccess) break;
      const auto *tiles = static_cast<const unsigned long long *>(b->tiles[k].p);
      if (c == 0) {
        BatchLevel B;
        B.plans = static_cast<const ShellLaunch *>(b->plans[k].p);
        B.tile_start = tiles;
        B.nplans = b->nplans[k];
        B.grain = b->grain;
        B.counter = ctr + k;
        e = hxg::launch_batch_level(s, b->fp32, b->ngroups, b->ext_any, b->fast, B,
                                    b->level_blocks[0]);
      } else if (c == 1) {
        hxg::BatchLevelMulti<2> B{static_cast<const hxg::FusedPlan<2> *>(b->plans[k].p), tiles,
                                  b->nplans[k], b->grain, ctr + k};
        e = hxg::launch_batch_level_multi(s, b->ngroups, b->ext_any, b->fast, 2, &B,
                                          b->level_blocks[1]);
      } else {
        hxg::BatchLevelMulti<3> B{static_cast<const hxg::FusedPlan<3> *>(b->plans[k].p), tiles,
                                  b->nplans[k], b->grain, ctr + k};
        e = hxg::launch_batch_level_multi(s, b->ngroups, b->ext_any, b->fast, 3, &B,
                                          b->level_blocks[2]);
      }
    }
    if (e != cudaSuccess) break;
    e = hxg::launch_batch_merge(s, static_cast<const MergeJob *>(b->merges[l].p),
                                static_cast<const unsigned long long *>(b->mblocks[l].p),
                                b->nmerge[l], b->merge_blocks[l]);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_fail(h, e != cudaSuccess ? e : e2, "batch graph capture");
  }
  const cudaError_t e3 = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) {
    b->exec = nullptr;
    return cuda_fail(h, e3, "cudaGraphInstantiate");
  }
  return HXG_OK;
}

int batch_time(hxg_batch *b, double *ms) {
  hxg_handle *h = b->h;
  cudaEvent_t e0, e1;
  HXG_CK(cudaEventCreate(&e0));
  HXG_CK(cudaEventCreate(&e1));
  cudaError_t e = cudaGraphLaunch(b->exec, h->stream);  // warm-up
  if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
  if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, h->stream);
  if (e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float f = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(h, e, "batch timing run");
  *ms = f;
  return HXG_OK;
}

void batch_free(hxg_batch *b) {
  batch_drop_graph(b);
  DevBuf *bufs[] = {&b->tmp, &b->zeros, &b->zblocks, &b->counters, &b->ext};
  for (DevBuf *d : bufs)
    if (d->p) cudaFree(d->p);
  for (auto *v : {&b->plans, &b->tiles, &b->merges, &b->mblocks})
    for (DevBuf &d : *v)
      if (d.p) cudaFree(d.p);
}

}  // namespace

extern "C" {

int hxg_batch_create(hxg_handle *h, int n, const hxg_batch_entry_t *entries,
                     int tune, hxg_batch **out) {
  if (!h || !out || n < 1 || !entries) return HXG_ERR_INVALID;
  *out = nullptr;
  cudaSetDevice(h->device);
  if (!h->have_models) return fail(h, HXG_ERR_STATE, "models not set");
  int st;
  for (int i = 0; i < n; ++i) {
    const hxg_batch_entry_t &E = entries[i];
    if (E.obs.do_mask) return fail(h, HXG_ERR_UNSUPPORTED, "entry %d: masks are not batched", i);
    if ((st = validate_obs(h, &E.obs)) != HXG_OK) return st;
    for (int w = 0; w < 5; ++w)
      if (reads_grid(E.models, w) != reads_grid(h->models, w))
        return fail(h, HXG_ERR_INVALID,
                    "entry %d reads other fields from grids than the handle's models", i);
    if (E.obs.do_sync && E.models.cre == HXG_CRE_NONE)
      return fail(h, HXG_ERR_INVALID, "entry %d: synchrotron output needs a CRE model", i);
    if ((E.obs.do_dm && !E.d_dm) || (E.obs.do_fd && !E.d_fd) ||
        (E.obs.do_sync && (!E.d_is || !E.d_qs || !E.d_us)))
      return fail(h, HXG_ERR_INVALID, "entry %d: an output requested by obs is NULL", i);
    std::string why;
    if (!models_supported(E.models, &why))
      return fail(h, HXG_ERR_UNSUPPORTED, "entry %d: %s", i, why.c_str());
  }
  if ((st = build_groups(h)) != HXG_OK) return st;
  hxg_batch *b = new hxg_batch();
  b->h = h;
  b->layout_gen = h->layout_gen;
  b->e.assign(entries, entries + n);
  b->fp32 = h->precision == HXG_FP32C;
  b->ngroups = (int)h->groups.size();
  size_t total = 0;
  std::vector<ZeroJob> zj;
  std::vector<unsigned long long> z0(1, 0ull);
  for (const hxg_batch_entry_t &E : b->e) {
    uint32_t mx = 0;
    for (uint32_t s = 0; s < E.obs.total_shell; ++s) mx = std::max(mx, E.obs.nside_shell[s]);
    b->levels = std::max(b->levels, (int)E.obs.total_shell);
    b->tmp_off.push_back(total);
    b->tmp_n.push_back(npix_of(mx));
    total += 5 * npix_of(mx);
    const auto zero = [&](double *p, uint32_t ns) {
      zj.push_back(ZeroJob{p, npix_of(ns)});
      z0.push_back(z0.back() + (npix_of(ns) + 255) / 256);
    };
    if (E.obs.do_dm) zero(E.d_dm, E.obs.nside_dm);
    if (E.obs.do_fd) zero(E.d_fd, E.obs.nside_fd);
    if (E.obs.do_sync) {
      zero(E.d_is, E.obs.nside_sync);
      zero(E.d_qs, E.obs.nside_sync);
      zero(E.d_us, E.obs.nside_sync);
    }
  }
  b->nzero = (int)zj.size();
  b->zero_blocks = z0.back();
  b->plans.resize(3 * b->levels);
  b->tiles.resize(3 * b->levels);
  b->merges.resize(b->levels);
  b->mblocks.resize(b->levels);
  b->nplans.assign(3 * b->levels, 0);
  b->nmerge.assign(b->levels, 0);
  b->merge_blocks.assign(b->levels, 0ull);
  const auto bail = [&](int code) {
    batch_free(b);
    delete b;
    return code;
  };
  if ((st = ensure(h, b->tmp, total * sizeof(double))) != HXG_OK) return bail(st);
  if ((st = ensure(h, b->counters, 3 * b->levels * sizeof(unsigned long long))) != HXG_OK)
    return bail(st);
  // frequency passes of one parameter set that can share a traversal: up to
  // three consecutive entries with the same models and geometry (FP32C form,
  // synchrotron in every pass, no CRE grid)
  b->group.assign(b->e.size(), 0);
  for (size_t i = 0; i < b->e.size();) {
    int nf = 1;
    for (int cand = 3; b->fp32 && cand >= 2 && nf == 1; --cand) {
      if (i + cand > b->e.size() || b->e[i].models.cre == HXG_CRE_GRID) continue;
      hxg_obs_t o[3];
      bool same = true;
      for (int f = 0; f < cand; ++f) {
        o[f] = b->e[i + f].obs;
        same = same && std::memcmp(&b->e[i].models, &b->e[i + f].models,
                                   sizeof(hxg_models_t)) == 0;
      }
      if (same && same_traversal(o, cand)) nf = cand;
    }
    b->group[i] = nf;
    i += nf;
  }
  if ((st = upload_vec(h, b->zeros, zj)) != HXG_OK) return bail(st);
  if ((st = upload_vec(h, b->zblocks, z0)) != HXG_OK) return bail(st);
  {
    std::vector<ExtModels> ext(b->e.size());
    for (size_t i = 0; i < b->e.size(); ++i) {
      if (!uses_ext(b->e[i].models)) continue;
      b->ext_any = true;
      const double L = b->fp32 ? 1.0 / cgs::kpc : 1.0;
      const double Bu = b->fp32 ? 1.0 / cgs::fp32_bunit : 1.0;
      ext_models(b->e[i].models, L, Bu, ext[i]);
      if (b->e[i].models.cre == HXG_CRE_GRID &&
          (st = cre_grid_block(h, L, Bu, b->e[i].obs.sync_freq, ext[i].cre)) != HXG_OK)
        return bail(st);
    }
    if (b->ext_any && (st = upload_vec(h, b->ext, ext)) != HXG_OK) return bail(st);
  }
  // the kFast kernels when every entry's models are among the grid workloads'
  b->fast = true;
  for (const hxg_batch_entry_t &E : b->e) {
    ShellLaunch L;
    uint64_t step;
    if ((st = build_launch(h, E.models, E.obs, 0, L, step)) != HXG_OK) return bail(st);
    L.ext = uses_ext(E.models) ? static_cast<const ExtModels *>(b->ext.p) : nullptr;
    b->fast = b->fast && hxg::fast_models(L);
  }
  int per_sm = 0;
  cudaError_t ce = hxg::batch_level_occupancy(b->fp32, b->ngroups, b->ext_any, b->fast, &per_sm);
  if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "occupancy"));
  b->level_blocks[0] = (unsigned)std::max(1, per_sm) * (unsigned)h->sm_count;
  for (int nf = 2; nf <= 3 && b->fp32; ++nf) {
    ce = hxg::batch_multi_occupancy(b->ngroups, b->ext_any, b->fast, nf, &per_sm);
    if (ce != cudaSuccess) return bail(cuda_fail(h, ce, "occupancy"));
    b->level_blocks[nf - 1] = (unsigned)std::max(1, per_sm) * (unsigned)h->sm_count;
  }
  // launch shapes: lanes per pixel x tiles per work fetch
  const int shapes[][2] = {{1, 4}, {2, 4}, {4, 4}, {8, 4}, {1, 16}, {2, 1}};
  int best = 0;
  if (tune) {
    double best_ms = 1e300;
    for (int k = 0; k < (int)(sizeof(shapes) / sizeof(shapes[0])); ++k) {
      if ((st = batch_tables(b, shapes[k][0], shapes[k][1])) != HXG_OK) return bail(st);
      if ((st = batch_capture(b)) != HXG_OK) return bail(st);
      double ms;
      if ((st = batch_time(b, &ms)) != HXG_OK) return bail(st);
      ++b->tried;
      if (ms < best_ms) {
        best_ms = ms;
        best = k;
      }
    }
    b->best_ms = best_ms;
  }
  if ((st = batch_tables(b, shapes[best][0], shapes[best][1])) != HXG_OK) return bail(st);
  if ((st = batch_capture(b)) != HXG_OK) return bail(st);
  *out = b;
  return HXG_OK;
}

int hxg_batch_run(hxg_batch *b) {
  if (!b || !b->exec) return HXG_ERR_INVALID;
  hxg_handle *h = b->h;
  cudaSetDevice(h->device);
  // grids uploaded since the last run are packed into the same record
  // arrays; a new geometry or set of grid fields moves them
  const int st = build_groups(h);
  if (st != HXG_OK) return st;
  if (b->layout_gen != h->layout_gen)
    return fail(h, HXG_ERR_STATE,
                "the handle's grids changed geometry or fields since hxg_batch_create; "
                "create the batch again");
  HXG_CK(cudaGraphLaunch(b->exec, h->stream));
  h->launch_count += b->graph_kernels;
  return HXG_OK;
}

int hxg_batch_info(const hxg_batch *b, int *lanes_per_pixel, int *grain,
                   int *tried, double *best_ms, int64_t *samples) {
  if (!b) return HXG_ERR_INVALID;
  if (lanes_per_pixel) *lanes_per_pixel = b->lanes;
  if (grain) *grain = b->grain;
  if (tried) *tried = b->tried;
  if (best_ms) *best_ms = b->best_ms;
  if (samples) *samples = b->samples;
  return HXG_OK;
}

int hxg_batch_destroy(hxg_batch *b) {
  if (!b) return HXG_ERR_INVALID;
  cudaSetDevice(b->h->device);
  batch_free(b);
  delete b;
  return HXG_OK;
}

}  // extern "C"
