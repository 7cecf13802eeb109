// hxg_rfg.cu -- Gaussian random-field generators on the device:
//   TErnd_dft::write_grid (source/field/te/ternd_dft.cc:35-128): isotropic
//     n_e fluctuations with a power-law spectrum, rescaled by a spatial
//     profile;
//   Brnd_es::write_grid (source/field/b/brnd_es.cc:76-308): a random B field
//     with a broken power-law spectrum, the local anisotropy along the
//     regular field, and the divergence-free projection.
// The steps, their order and the reference's in-place complex packing are
// the reference's; the FFTs are cuFFT Z2Z transforms (FFTW_BACKWARD is
// CUFFT_INVERSE, both unnormalised), and the Gaussian deviates come from a
// counter-based generator (Philox4x32-10, Salmon et al., "Parallel random
// numbers: as easy as 1, 2, 3", SC 2011) with Box-Muller, indexed by the
// k-space cell, so a field depends only on the seed and not on the launch
// shape.  GSL's taus streams are not reproduced, so a seed gives another
// realisation than the reference's; fed the same deviates, the reference's
// generator gives the same field to rounding.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdint>

#include "hxg_fields.cuh"
#include "hxg_internal.h"

namespace hxg {

// ---- Philox4x32-10 ----------------------------------------------------
__host__ __device__ inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;  // round multipliers
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;  // key schedule (Weyl)
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)M0 * ctr[0], p1 = (uint64_t)M1 * ctr[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t c0 = hi1 ^ ctr[1] ^ k0, c2 = hi0 ^ ctr[3] ^ k1;
    ctr[0] = c0;
    ctr[1] = lo1;
    ctr[2] = c2;
    ctr[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

// Four standard normal deviates for cell idx: two Philox blocks give four
// 53-bit uniforms in (0, 1), two Box-Muller pairs turn them into normals;
// nb = 1: the first pair only (from the first block), the same two values.
template <int nb = 2>
__device__ inline void gauss4(uint64_t seed, uint64_t idx, double g[4]) {
  double u[4];
#pragma unroll
  for (int b = 0; b < nb; ++b) {
    uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), (uint32_t)b, 0x52464721u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    for (int q = 0; q < 2; ++q) {
      const uint64_t w = ((uint64_t)c[2 * q] << 21) ^ (uint64_t)(c[2 * q + 1] >> 11);
      u[2 * b + q] = ((double)(w & ((1ull << 53) - 1)) + 0.5) * 0x1p-53;
    }
  }
#pragma unroll
  for (int q = 0; q < nb; ++q) {
    const double r = sqrt(-2. * log(u[2 * q]));
    double s, c;
    sincospi(2. * u[2 * q + 1], &s, &c);
    g[2 * q] = r * c;
    g[2 * q + 1] = r * s;
  }
}

// k of FFT index i in 1/kpc (ternd_dft.cc:60-62): i / L, wrapped for the
// upper half
__device__ inline double kcomp(int i, int n, double L) {
  double k = cgs::kpc * i / L;
  if (i >= (n + 1) / 2) k -= cgs::kpc * n / L;
  return k;
}

// TErnd_dft::spectrum (ternd_dft.cc:17-24)
__device__ inline double spec_dft(double k, const hxg_ternd_dft_t &p) {
  if (k < p.k0) return 0.;
  return p.rms * pow(k / p.k0, p.a0) / (4 * cgs::pi * k * k);
}

// Brnd_es::spectrum (brnd_es.cc:30-44)
__device__ inline double spec_es(double k, const hxg_brnd_es_t &p) {
  const double p0 = p.rms * p.rms;
  const double unit = 1. / (4. * cgs::pi * k * k);
  const double band1 = double(k < p.k1);
  const double band2 = double(k > p.k1) * double(k < p.k0);
  const double band3 = double(k > p.k0);
  // the band that holds k, the others adding exact zeros: the value of
  // band1 * A * B + band2 / C + band3 / D with one or none of its terms
  // evaluated
  double P = 0.;
  if (band1 != 0.)
    P = band1 * pow(p.k0 / p.k1, p.a1) * pow(k / p.k1, 6.);
  else if (band2 != 0.)
    P = band2 / pow(k / p.k0, p.a1);
  else if (band3 != 0.)
    P = band3 / pow(k / p.k0, p.a0);
  return P * p0 * unit;
}

// The square root of spatial_profile (ternd_dft.cc:26-33, brnd_es.cc:46-52),
// exp(-r_cyl / r0) exp(-zz / z0), that both rescales take: one exponential
// of half the summed exponent (equal to rounding).
__device__ inline double sqrt_profile(double x, double y, double z, const double obs[3],
                                      double r0, double z0) {
  const double r_cyl = sqrt(x * x + y * y) - fabs(obs[0]);
  const double zz = fabs(z) - fabs(obs[2]);
  return exp(-0.5 * (r_cyl / r0 + zz / z0));
}

struct RfgGrid {
  int nx, ny, nz;
  double lx, ly, lz, xmin, ymin, zmin;  // cm
  double dk3;                           // kpc^3 / (lx ly lz)
};

__device__ inline void unflat(const RfgGrid &G, uint64_t idx, int &i, int &j, int &l) {
  l = (int)(idx % G.nz);
  const uint64_t t = idx / G.nz;
  j = (int)(t % G.ny);
  i = (int)(t / G.ny);
}

// ---- STEP I: Gaussian k-space fill ---------------------------------------
__global__ void rfg_fill_kernel(RfgGrid G, int kind, hxg_ternd_dft_t pt, hxg_brnd_es_t pb,
                                uint64_t seed, double2 *c0, double2 *c1) {
  const uint64_t n = (uint64_t)G.nx * G.ny * G.nz;
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  if (idx == 0) {  // the k = 0 cell is skipped: no mean field
    c0[0] = make_double2(0., 0.);
    if (kind) c1[0] = make_double2(0., 0.);
    return;
  }
  int i, j, l;
  unflat(G, idx, i, j, l);
  const double kx = kcomp(i, G.nx, G.lx), ky = kcomp(j, G.ny, G.ly), kz = kcomp(l, G.nz, G.lz);
  const double ks = sqrt(kx * kx + ky * ky + kz * kz);
  double g[4];
  if (kind == 0)
    gauss4<1>(seed, idx, g);
  else
    gauss4<2>(seed, idx, g);
  if (kind == 0) {
    const double sigma = sqrt(spec_dft(ks, pt) * G.dk3);
    c0[idx] = make_double2(sigma * g[0], sigma * g[1]);
  } else {
    const double sigma = sqrt(0.333333333333333333 * spec_es(ks, pb) * G.dk3);
    c0[idx] = make_double2(sigma * g[0], sigma * g[1]);
    c1[idx] = make_double2(sigma * g[2], sigma * g[3]);
  }
}

// ---- per-block partial sums of a double array (for mean and variance) ----
__global__ void rfg_sum_kernel(const double *x, uint64_t n, double mean, int squared,
                               double *partial) {
  __shared__ double sh[256];
  double acc = 0.;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double v = x[i] - mean;
    acc += squared ? v * v : x[i];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// ---- STEP II (TErnd_dft): real part times the profile ratio ---------------
__global__ void ternd_rescale_kernel(RfgGrid G, hxg_ternd_dft_t p, double obs0, double obs1,
                                     double obs2, double var_invsq, const double2 *c,
                                     double *te) {
  const uint64_t n = (uint64_t)G.nx * G.ny * G.nz;
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int i, j, l;
  unflat(G, idx, i, j, l);
  const double obs[3] = {obs0, obs1, obs2};
  const double x = i * G.lx / (G.nx - 1) + G.xmin;
  const double y = j * G.ly / (G.ny - 1) + G.ymin;
  const double z = l * G.lz / (G.nz - 1) + G.zmin;
  const double ratio = sqrt_profile(x, y, z, obs, p.r0, p.z0) * p.rms * var_invsq;
  te[idx] = c[idx].x * ratio;
}

// Breg::read_grid (source/field/b/breg.cc:28-97): zero on or outside the
// box surface, else trilinear in the order z, then y, then x.
__device__ inline V3<double> breg_grid_at(const RfgBregGrid &g, double x, double y, double z) {
  const V3<double> zero{0., 0., 0.};
  double t = (g.nx - 1) * (x - g.x_min) / (g.x_max - g.x_min);
  if (t <= 0 || t >= g.nx - 1) return zero;
  const int xl = (int)floor(t);
  const double xd = t - xl;
  t = (g.ny - 1) * (y - g.y_min) / (g.y_max - g.y_min);
  if (t <= 0 || t >= g.ny - 1) return zero;
  const int yl = (int)floor(t);
  const double yd = t - yl;
  t = (g.nz - 1) * (z - g.z_min) / (g.z_max - g.z_min);
  if (t <= 0 || t >= g.nz - 1) return zero;
  const int zl = (int)floor(t);
  const double zd = t - zl;
  const double *c[3] = {g.bx, g.by, g.bz};
  double out[3];
  for (int a = 0; a < 3; ++a) {
    const double *v = c[a];
    auto at = [&](int i, int j, int l) {
      return v[((size_t)i * g.ny + j) * g.nz + l];
    };
    const double i1 = at(xl, yl, zl) * (1. - zd) + at(xl, yl, zl + 1) * zd;
    const double i2 = at(xl, yl + 1, zl) * (1. - zd) + at(xl, yl + 1, zl + 1) * zd;
    const double j1 = at(xl + 1, yl, zl) * (1. - zd) + at(xl + 1, yl, zl + 1) * zd;
    const double j2 = at(xl + 1, yl + 1, zl) * (1. - zd) + at(xl + 1, yl + 1, zl + 1) * zd;
    const double w1 = i1 * (1. - yd) + i2 * yd;
    const double w2 = j1 * (1. - yd) + j2 * yd;
    out[a] = w1 * (1. - xd) + w2 * xd;
  }
  return V3<double>{out[0], out[1], out[2]};
}

// ---- Brnd_es STEP II: profile and anisotropy in real space ---------------
// (brnd_es.cc:157-204).  A vertex where the regular field is zero (versor
// length^2 below 1e-10) keeps the unscaled value of the first transform,
// as in the reference.
template <bool kExt>
__global__ void brnd_rescale_kernel(RfgGrid G, hxg_brnd_es_t p, DevModels M,
                                    const ExtModels *ext, RfgBregGrid bg, double var_invsq,
                                    double2 *c0, double2 *c1) {
  const uint64_t n = (uint64_t)G.nx * G.ny * G.nz;
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int i, j, l;
  unflat(G, idx, i, j, l);
  const double x = i * G.lx / (G.nx - 1) + G.xmin;
  const double y = j * G.ly / (G.ny - 1) + G.ymin;
  const double z = l * G.lz / (G.nz - 1) + G.zmin;
  const double ratio = sqrt_profile(x, y, z, M.obs, p.r0, p.z0) * p.rms * var_invsq;
  const double2 a0 = c0[idx], a1 = c1[idx];
  const double b[3] = {a0.x * ratio, a0.y * ratio, a1.y * ratio};
  const double p3[3] = {x, y, z};
  const V3<double> H = bg.bx ? breg_grid_at(bg, x, y, z) : breg_model_x<kExt>(M, ext, x, y, z, p3);
  // Hamvec::versor (include/hamvec.h:176-186)
  const double l2 = H.x * H.x + H.y * H.y + H.z * H.z;
  double h[3] = {0., 0., 0.};
  if (l2 != 0.) {
    const double inv = 1. / sqrt(l2);
    h[0] = H.x * inv;
    h[1] = H.y * inv;
    h[2] = H.z * inv;
  }
  if (h[0] * h[0] + h[1] * h[1] + h[2] * h[2] < 1e-10) return;
  const double rho = p.rho;
  const double rho2 = rho * rho;
  const double rhonorm = 1. / sqrt(0.333333333333333333 * rho2 + 0.666666666666666667 / rho2);
  const double hb = h[0] * b[0] + h[1] * b[1] + h[2] * b[2];
  double o[3];
  for (int a = 0; a < 3; ++a) {
    const double par = h[a] * hb;
    const double perp = b[a] - par;
    o[a] = (par * rho + perp / rho) * rhonorm;
  }
  c0[idx] = make_double2(o[0], o[1]);
  c1[idx] = make_double2(o[1], o[2]);
}

// index of -k for FFT index idx (brnd_es.cc:200-225)
__device__ inline uint64_t sym_index(const RfgGrid &G, int i, int j, int l) {
  const int is = i == 0 ? 0 : G.nx - i, js = j == 0 ? 0 : G.ny - j, ls = l == 0 ? 0 : G.nz - l;
  return ((uint64_t)is * G.ny + js) * G.nz + ls;
}

// ---- Brnd_es STEP III: Hermitian part and divergence-free projection ------
// (brnd_es.cc:196-245): gramschmidt() with the sqrt(3) factor, times sqrt(2)
__global__ void brnd_project_kernel(RfgGrid G, const double2 *c0, const double2 *c1,
                                    double *bx, double *by, double *bz) {
  const uint64_t n = (uint64_t)G.nx * G.ny * G.nz;
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int i, j, l;
  unflat(G, idx, i, j, l);
  const uint64_t s = sym_index(G, i, j, l);
  const double k[3] = {kcomp(i, G.nx, G.lx), kcomp(j, G.ny, G.ly), kcomp(l, G.nz, G.lz)};
  const double b[3] = {0.5 * (c0[idx].x + c0[s].x), 0.5 * (c1[idx].x + c1[s].x),
                       0.5 * (c1[idx].y + c1[s].y)};
  const double kk = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  const double bb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  double f[3] = {b[0], b[1], b[2]};
  if (kk != 0. && bb != 0.) {
    const double inv_k_mod = 1. / kk;
    const double kb = k[0] * b[0] + k[1] * b[1] + k[2] * b[2];
    for (int a = 0; a < 3; ++a) f[a] = 1.7320508075688772935 * (b[a] - k[a] * kb * inv_k_mod);
  }
  bx[idx] = 1.4142135623730950488 * f[0];
  by[idx] = 1.4142135623730950488 * f[1];
  bz[idx] = 1.4142135623730950488 * f[2];
}

// c0 = (bx, by), c1 = (by, bz)  (brnd_es.cc:247-256)
__global__ void brnd_repack_kernel(uint64_t n, const double *bx, const double *by,
                                   const double *bz, double2 *c0, double2 *c1) {
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  c0[idx] = make_double2(bx[idx], by[idx]);
  c1[idx] = make_double2(by[idx], bz[idx]);
}

// final Hermitian part over N (brnd_es.cc:259-300)
__global__ void brnd_final_kernel(RfgGrid G, const double2 *c0, const double2 *c1, double *bx,
                                  double *by, double *bz) {
  const uint64_t n = (uint64_t)G.nx * G.ny * G.nz;
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int i, j, l;
  unflat(G, idx, i, j, l);
  const uint64_t s = sym_index(G, i, j, l);
  const double inv = 1. / (double)n;
  bx[idx] = 0.5 * (c0[idx].x + c0[s].x) * inv;
  by[idx] = 0.5 * (c1[idx].x + c1[s].x) * inv;
  bz[idx] = 0.5 * (c1[idx].y + c1[s].y) * inv;
}

// ---- host side ---------------------------------------------------------

static unsigned nblk(uint64_t n) { return (unsigned)((n + 255) / 256); }

// variance of the first n doubles of x (toolkit::variance, include/toolkit.h:70-78)
static cudaError_t variance(cudaStream_t s, const double *x, uint64_t n, double *part,
                            int nparts, double *out) {
  double h[1024];
  double sum = 0.;
  rfg_sum_kernel<<<nparts, 256, 0, s>>>(x, n, 0., 0, part);
  cudaError_t e = cudaMemcpyAsync(h, part, nparts * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  for (int k = 0; k < nparts; ++k) sum += h[k];
  const double mean = sum / (double)n;
  rfg_sum_kernel<<<nparts, 256, 0, s>>>(x, n, mean, 1, part);
  e = cudaMemcpyAsync(h, part, nparts * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  double var = 0.;
  for (int k = 0; k < nparts; ++k) var += h[k];
  *out = var / (double)n;
  return cudaSuccess;
}

static RfgGrid rfg_grid(const hxg_grid_desc_t &g) {
  RfgGrid G;
  G.nx = (int)g.nx;
  G.ny = (int)g.ny;
  G.nz = (int)g.nz;
  G.lx = g.x_max - g.x_min;
  G.ly = g.y_max - g.y_min;
  G.lz = g.z_max - g.z_min;
  G.xmin = g.x_min;
  G.ymin = g.y_min;
  G.zmin = g.z_min;
  G.dk3 = cgs::kpc * cgs::kpc * cgs::kpc / (G.lx * G.ly * G.lz);
  return G;
}

// Workspace of the generators, kept on the handle between calls: the k-space
// arrays, the reduction partials and the cuFFT plan of the last grid shape.
struct RfgWork {
  uint32_t nx = 0, ny = 0, nz = 0;
  double2 *c0 = nullptr, *c1 = nullptr;
  double *part = nullptr;
  cufftHandle plan = 0;
  bool have_plan = false;
  void release() {
    if (have_plan) cufftDestroy(plan);
    if (c0) cudaFree(c0);
    if (c1) cudaFree(c1);
    if (part) cudaFree(part);
    *this = RfgWork{};
  }
};

void rfg_release(RfgWork *w) {
  if (!w) return;
  w->release();
  delete w;
}

static int rfg_status(cudaError_t e) {
  if (e == cudaSuccess) return HXG_OK;
  return e == cudaErrorMemoryAllocation ? HXG_ERR_OOM : HXG_ERR_CUDA;
}

static int fft_status(cufftResult r) {
  if (r == CUFFT_SUCCESS) return HXG_OK;
  return r == CUFFT_ALLOC_FAILED ? HXG_ERR_OOM : HXG_ERR_CUDA;
}

#define RFG_CK(call)                              \
  do {                                            \
    const int st_ = rfg_status(call);             \
    if (st_ != HXG_OK) return st_;                \
  } while (0)
#define RFG_FFT(call)                             \
  do {                                            \
    const int st_ = fft_status(call);             \
    if (st_ != HXG_OK) return st_;                \
  } while (0)

// Make the workspace fit grid g (two k-space arrays for Brnd_es); reuses
// the previous buffers and plan when the shape is unchanged.
static int rfg_setup(cudaStream_t s, const hxg_grid_desc_t &g, bool two, RfgWork *&pw) {
  if (!pw) pw = new RfgWork;
  RfgWork &W = *pw;
  const uint64_t n = (uint64_t)g.nx * g.ny * g.nz;
  if (W.nx != g.nx || W.ny != g.ny || W.nz != g.nz) {
    W.release();
    RFG_CK(cudaMalloc(&W.c0, n * sizeof(double2)));
    RFG_CK(cudaMalloc(&W.part, 1024 * sizeof(double)));
    RFG_FFT(cufftPlan3d(&W.plan, (int)g.nx, (int)g.ny, (int)g.nz, CUFFT_Z2Z));
    W.have_plan = true;
    W.nx = g.nx;
    W.ny = g.ny;
    W.nz = g.nz;
  }
  if (two && !W.c1) RFG_CK(cudaMalloc(&W.c1, n * sizeof(double2)));
  RFG_FFT(cufftSetStream(W.plan, s));
  return HXG_OK;
}

int generate_ternd_dft(cudaStream_t s, RfgWork *&work, const hxg_grid_desc_t &g,
                       const hxg_ternd_dft_t &p, const double obs[3], uint64_t seed,
                       double *te) {
  int st = rfg_setup(s, g, false, work);
  if (st != HXG_OK) return st;
  RfgWork &W = *work;
  const RfgGrid G = rfg_grid(g);
  const uint64_t n = (uint64_t)g.nx * g.ny * g.nz;
  const hxg_brnd_es_t none{};
  rfg_fill_kernel<<<nblk(n), 256, 0, s>>>(G, 0, p, none, seed, W.c0, nullptr);
  RFG_CK(cudaGetLastError());
  RFG_FFT(cufftExecZ2Z(W.plan, W.c0, W.c0, CUFFT_INVERSE));
  // the reference's variance runs over the first n doubles of the complex
  // array, i.e. the interleaved (Re, Im) of its first n/2 cells
  double var = 0.;
  RFG_CK(variance(s, reinterpret_cast<const double *>(W.c0), n, W.part, 1024, &var));
  if (!(var > 0.) || !std::isfinite(var)) return HXG_ERR_INVALID;
  const double var_invsq = 1. / sqrt(var);
  ternd_rescale_kernel<<<nblk(n), 256, 0, s>>>(G, p, obs[0], obs[1], obs[2], var_invsq, W.c0, te);
  RFG_CK(cudaGetLastError());
  RFG_CK(cudaStreamSynchronize(s));
  return HXG_OK;
}

int generate_brnd_es(cudaStream_t s, RfgWork *&work, const hxg_grid_desc_t &g,
                     const hxg_brnd_es_t &p, const DevModels &M, const ExtModels *ext,
                     const RfgBregGrid &breg, uint64_t seed, double *bx, double *by,
                     double *bz) {
  int st = rfg_setup(s, g, true, work);
  if (st != HXG_OK) return st;
  RfgWork &W = *work;
  const RfgGrid G = rfg_grid(g);
  const uint64_t n = (uint64_t)g.nx * g.ny * g.nz;
  const hxg_ternd_dft_t none{};
  rfg_fill_kernel<<<nblk(n), 256, 0, s>>>(G, 1, none, p, seed, W.c0, W.c1);
  RFG_CK(cudaGetLastError());
  RFG_FFT(cufftExecZ2Z(W.plan, W.c0, W.c0, CUFFT_INVERSE));
  RFG_FFT(cufftExecZ2Z(W.plan, W.c1, W.c1, CUFFT_INVERSE));
  double var = 0.;
  RFG_CK(variance(s, reinterpret_cast<const double *>(W.c0), n, W.part, 1024, &var));
  if (!(var > 0.) || !std::isfinite(var)) return HXG_ERR_INVALID;
  const double var_invsq = 1. / sqrt(3. * var);
  if (ext)
    brnd_rescale_kernel<true><<<nblk(n), 256, 0, s>>>(G, p, M, ext, breg, var_invsq, W.c0, W.c1);
  else
    brnd_rescale_kernel<false><<<nblk(n), 256, 0, s>>>(G, p, M, ext, breg, var_invsq, W.c0,
                                                       W.c1);
  RFG_CK(cudaGetLastError());
  RFG_FFT(cufftExecZ2Z(W.plan, W.c0, W.c0, CUFFT_FORWARD));
  RFG_FFT(cufftExecZ2Z(W.plan, W.c1, W.c1, CUFFT_FORWARD));
  brnd_project_kernel<<<nblk(n), 256, 0, s>>>(G, W.c0, W.c1, bx, by, bz);
  RFG_CK(cudaGetLastError());
  brnd_repack_kernel<<<nblk(n), 256, 0, s>>>(n, bx, by, bz, W.c0, W.c1);
  RFG_CK(cudaGetLastError());
  RFG_FFT(cufftExecZ2Z(W.plan, W.c0, W.c0, CUFFT_INVERSE));
  RFG_FFT(cufftExecZ2Z(W.plan, W.c1, W.c1, CUFFT_INVERSE));
  brnd_final_kernel<<<nblk(n), 256, 0, s>>>(G, W.c0, W.c1, bx, by, bz);
  RFG_CK(cudaGetLastError());
  RFG_CK(cudaStreamSynchronize(s));
  return HXG_OK;
}

}  // namespace hxg
