// hxg_kernels.cu -- map kernels (shell merge, HEALPix helpers), grid
// packing, and the instantiations of the shell-integration kernels.
#include <cuda_runtime.h>

#include <type_traits>

#include "hxg_adjoint.cuh"
#include "hxg_adjoint32.cuh"
#include "hxg_batch.cuh"
#include "hxg_fp32c.cuh"
#include "hxg_integrate.cuh"
#include "hxg_internal.h"

namespace hxg {

// ---- Hampix::accumulate (include/hamdis.h:698-721) ----------------------
// dst_k += src_k for up to kMaxMergeMaps map pairs sharing one (nside_dst,
// nside_src); when the Nsides differ, src is interpolated at each dst
// pixel's pointing (the pointing and the 4 weights once for all maps).
constexpr int kMaxMergeMaps = kMaxMergeOuts;
struct MergeMaps {
  int n;
  double *dst[kMaxMergeMaps];
  const double *src[kMaxMergeMaps];
};

// hpx_interp_apply (Hampix::interpolate's weighted sum, hamdis.h:683-695)
// with the map values read through the read-only path: the shell maps are
// not written while a merge runs.  The same operations in the same order.
__device__ __forceinline__ double interp_apply_nc(const double *map, const unsigned pix[4],
                                                  const double wght[4]) {
  double wtot = 0.0, res = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double val = __ldg(map + pix[c]);
    if (val > kUndefTest) {
      res += val * wght[c];
      wtot += wght[c];
    }
  }
  return (wtot == 0.0) ? kUndef : res / wtot;
}

// The 4 source pixels and weights of output pixel i: from the table when
// there is one, else from the output pixel's pointing.
__device__ __forceinline__ void interp_at(const InterpTab &T, const Hpx &hd, const Hpx &hs,
                                          uint64_t i, uint64_t pix[4], double w[4]) {
  if (T.pix) {
    const uint4 p = __ldg(T.pix + i);
    const double2 a = __ldg(T.w + 2 * i), b = __ldg(T.w + 2 * i + 1);
    pix[0] = p.x;
    pix[1] = p.y;
    pix[2] = p.z;
    pix[3] = p.w;
    w[0] = a.x;
    w[1] = a.y;
    w[2] = b.x;
    w[3] = b.y;
    return;
  }
  double th, ph;
  hpx_pix2ang(hd, i, th, ph);
  hpx_interp_weights(hs, th, ph, pix, w);
}

__global__ void interp_table_kernel(int nside_dst, int nside_src, uint4 *tp, double2 *tw) {
  const Hpx hd = hpx_make((uint64_t)nside_dst), hs = hpx_make((uint64_t)nside_src);
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hd.npix) return;
  uint64_t pix[4];
  double w[4];
  interp_at(InterpTab{}, hd, hs, i, pix, w);
  tp[i] = make_uint4((unsigned)pix[0], (unsigned)pix[1], (unsigned)pix[2], (unsigned)pix[3]);
  tw[2 * i] = make_double2(w[0], w[1]);
  tw[2 * i + 1] = make_double2(w[2], w[3]);
}

__global__ void accumulate_kernel(int nside_dst, int nside_src, MergeMaps M, InterpTab T) {
  const Hpx hd = hpx_make((uint64_t)nside_dst);
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hd.npix) return;
  if (nside_dst == nside_src) {
    for (int k = 0; k < M.n; ++k) M.dst[k][i] = M.dst[k][i] + M.src[k][i];
    return;
  }
  const Hpx hs = hpx_make((uint64_t)nside_src);
  uint64_t pix[4];
  double w[4];
  interp_at(T, hd, hs, i, pix, w);
  const unsigned p32[4] = {(unsigned)pix[0], (unsigned)pix[1], (unsigned)pix[2],
                           (unsigned)pix[3]};
  for (int k = 0; k < M.n; ++k)
    M.dst[k][i] = M.dst[k][i] + interp_apply_nc(M.src[k], p32, w);
}

// All shells' maps merged into the pass outputs at once (the DM and Stokes
// maps, whose merges no later shell waits for).  Shell s holds its maps in
// one block at base[s], map j at base[s] + j npix(nside[s]); output k sums
// map idx[k] of every shell, in shell order, at its pixel: directly where the
// Nsides agree, else by HEALPix interpolation (Hampix::accumulate,
// hamdis.h:698-721).  These are the additions of one accumulate per shell into
// zeroed outputs, in the same order, with each output written once instead
// of read and written per shell.
struct MergeAll {
  int n;        // outputs
  int nshells;
  int idx[kMaxMergeMaps];
  int nside[HXG_MAX_SHELLS];
  const double *base[HXG_MAX_SHELLS];
  double *dst[kMaxMergeMaps];
  InterpTab tab[HXG_MAX_SHELLS];
};

// One thread per output pixel walks the shells in order and keeps the
// running sums in the outputs themselves (a thread's output lines stay in
// cache from one shell to the next, so DRAM sees each output written about
// once).  A shell's source pixels and weights come from its Nside pair's
// interpolation table, or are found in place -- the same values: one
// function makes both.  kTab: every interpolated shell has its table.
template <bool kTab>
__global__ void __launch_bounds__(256, 4) merge_all_kernel(int nside_dst, MergeAll M) {
  const Hpx hd = hpx_make((uint64_t)nside_dst);
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hd.npix) return;
  for (int s = 0; s < M.nshells; ++s) {
    const uint64_t ns = (uint64_t)M.nside[s];
    const uint64_t npix = 12ull * ns * ns;
    if (M.nside[s] == nside_dst) {
      for (int k = 0; k < M.n; ++k) {
        const double v = __ldg(M.base[s] + (uint64_t)M.idx[k] * npix + i);
        M.dst[k][i] = (s == 0 ? 0. : M.dst[k][i]) + v;
      }
      continue;
    }
    unsigned pix[4];
    double w[4];
    if (kTab) {
      const uint4 q = __ldg(M.tab[s].pix + i);
      const double2 a = __ldg(M.tab[s].w + 2 * i), b = __ldg(M.tab[s].w + 2 * i + 1);
      pix[0] = q.x;
      pix[1] = q.y;
      pix[2] = q.z;
      pix[3] = q.w;
      w[0] = a.x;
      w[1] = a.y;
      w[2] = b.x;
      w[3] = b.y;
    } else {
      uint64_t p[4];
      interp_at(InterpTab{}, hd, hpx_make(ns), i, p, w);
      for (int c = 0; c < 4; ++c) pix[c] = (unsigned)p[c];
    }
    for (int k = 0; k < M.n; ++k) {
      const double v = interp_apply_nc(M.base[s] + (uint64_t)M.idx[k] * npix, pix, w);
      M.dst[k][i] = (s == 0 ? 0. : M.dst[k][i]) + v;
    }
  }
}

__global__ void pix2ang_kernel(int nside, uint64_t n, double *theta,
                               double *phi) {
  const Hpx h = hpx_make((uint64_t)nside);
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || i >= h.npix) return;
  hpx_pix2ang(h, i, theta[i], phi[i]);
}

__global__ void interpolate_kernel(int nside, const double *map, uint64_t n,
                                   const double *theta, const double *phi,
                                   double *out) {
  const Hpx h = hpx_make((uint64_t)nside);
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double th = theta[i], ph = phi[i];
  hamp_norm(th, ph);
  out[i] = hpx_interpolate(h, map, th, ph);
}

// LOS geometry of the FP64 shell kernel, exposed for known-answer tests.
__global__ void los_geometry_kernel(uint64_t n, const double *theta,
                                    const double *phi, const double *b,
                                    double *versor, double *b_par,
                                    double *b_per, double *c2ipa,
                                    double *s2ipa) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double th = theta[i], ph = phi[i];
  const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
  const double ux = cp * st, uy = sp * st, uz = ct;
  const double bx = b[3 * i], by = b[3 * i + 1], bz = b[3 * i + 2];
  versor[3 * i] = ux;
  versor[3 * i + 1] = uy;
  versor[3 * i + 2] = uz;
  b_par[i] = bx * ux + by * uy + bz * uz;
  const double cx = by * uz - bz * uy, cy = bz * ux - bx * uz,
               cz = bx * uy - by * ux;
  b_per[i] = sqrt(cx * cx + cy * cy + cz * cz);
  double c2, s2;
  ipa2<double>(-(-sp * bx + cp * by), -(ct * cp * bx + ct * sp * by - st * bz),
               c2, s2);
  c2ipa[i] = c2;
  s2ipa[i] = s2;
}

// Trilinear read of one packed group at n positions (working units in,
// working units out: 3 B components then n_e per position).
template <typename T>
__global__ void read_group_kernel(DevGridGroup g, uint64_t n,
                                  const double *pos, double *out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  CellCache<T> cc;
  cc.key = -1;
  T b[3] = {T(0), T(0), T(0)};
  T te = T(0);
  sample_group<T, false>(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], cc, b,
                         te);
  out[4 * i] = b[0];
  out[4 * i + 1] = b[1];
  out[4 * i + 2] = b[2];
  out[4 * i + 3] = te;
}

// Pack the FP64 SoA slots of one geometry into 4-component voxel records:
// rec = {sum of B slots (x,y,z), sum of n_e slots}, scaled by bscale / tscale.
template <typename T>
__global__ void pack_kernel(uint64_t n, T *rec, const double *bx0,
                            const double *by0, const double *bz0,
                            const double *bx1, const double *by1,
                            const double *bz1, const double *t0,
                            const double *t1, double bscale, double tscale) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double bx = 0., by = 0., bz = 0., te = 0.;
  if (bx0) {
    bx = bx0[i];
    by = by0[i];
    bz = bz0[i];
  }
  if (bx1) {
    bx += bx1[i];
    by += by1[i];
    bz += bz1[i];
  }
  if (t0) te = t0[i];
  if (t1) te += t1[i];
  rec[4 * i] = T(bx * bscale);
  rec[4 * i + 1] = T(by * bscale);
  rec[4 * i + 2] = T(bz * bscale);
  rec[4 * i + 3] = T(te * tscale);
}

// dL/d(shell map) from dL/d(output map): the transpose of Hampix::accumulate
// (include/hamdis.h:698-721).  Same Nside: g_shell += scale * g_out; else
// each output pixel scatters its gradient to the 4 interpolation pixels.
__global__ void accumulate_transpose_kernel(int nside_out, int nside_shell,
                                            const double *g_out,
                                            double *g_shell, double scale) {
  const Hpx ho = hpx_make((uint64_t)nside_out);
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ho.npix) return;
  const double g = g_out[i] * scale;
  if (g == 0.) return;
  if (nside_out == nside_shell) {
    g_shell[i] += g;
    return;
  }
  const Hpx hs = hpx_make((uint64_t)nside_shell);
  double th, ph;
  hpx_pix2ang(ho, i, th, ph);
  uint64_t pix[4];
  double w[4];
  hpx_interp_weights(hs, th, ph, pix, w);
  const double wtot = w[0] + w[1] + w[2] + w[3];
  for (int k = 0; k < 4; ++k) atomicAdd(g_shell + pix[k], g * w[k] / wtot);
}

// Split the group-record gradient [N][4] into B (3 SoA arrays) and n_e.
// Record gradient -> per-slot gradients; bscale converts the B gradient
// from the records' field unit to the slots' (1 in the FP64 form, 2^20 per
// Gauss in the FP32C form, whose records hold B in 2^-20 G).
__global__ void unpack_grad_kernel(uint64_t n, const double *rec, double *gbx,
                                   double *gby, double *gbz, double *gne, double bscale) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (gbx) {
    gbx[i] = rec[4 * i] * bscale;
    gby[i] = rec[4 * i + 1] * bscale;
    gbz[i] = rec[4 * i + 2] * bscale;
  }
  if (gne) gne[i] = rec[4 * i + 3];
}

// ---- launch wrappers -----------------------------------------------------
// Block b of a job-table kernel belongs to the last job j with
// block0[j] <= b (block0 has njobs + 1 entries).
__device__ __forceinline__ int job_of_block(const unsigned long long *block0,
                                            int njobs) {
  __shared__ int sj;
  if (threadIdx.x == 0) {
    const unsigned long long b = blockIdx.x;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (block0[mid] <= b) lo = mid; else hi = mid - 1;
    }
    sj = lo;
  }
  __syncthreads();
  return sj;
}

__global__ void batch_merge_kernel(const MergeJob *jobs,
                                   const unsigned long long *block0,
                                   int njobs) {
  const int j = job_of_block(block0, njobs);
  const MergeJob &J = jobs[j];
  const Hpx hd = hpx_make((uint64_t)J.nside_dst);
  const uint64_t i = (blockIdx.x - block0[j]) * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= hd.npix) return;
  if (J.nside_dst == J.nside_src) {
    for (int k = 0; k < J.nmaps; ++k) J.dst[k][i] = J.dst[k][i] + J.src[k][i];
    return;
  }
  const Hpx hs = hpx_make((uint64_t)J.nside_src);
  uint64_t pix[4];
  double w[4];
  interp_at(J.tab, hd, hs, i, pix, w);
  const unsigned p32[4] = {(unsigned)pix[0], (unsigned)pix[1], (unsigned)pix[2],
                           (unsigned)pix[3]};
  for (int k = 0; k < J.nmaps; ++k)
    J.dst[k][i] = J.dst[k][i] + interp_apply_nc(J.src[k], p32, w);
}

__global__ void batch_zero_kernel(const ZeroJob *jobs,
                                  const unsigned long long *block0, int njobs) {
  const int j = job_of_block(block0, njobs);
  const uint64_t i = (blockIdx.x - block0[j]) * (uint64_t)blockDim.x + threadIdx.x;
  if (i < jobs[j].n) jobs[j].p[i] = 0.;
}

static inline unsigned blocks_for(uint64_t n, unsigned tpb) {
  return (unsigned)((n + tpb - 1) / tpb);
}

cudaError_t launch_interp_table(cudaStream_t s, int nside_dst, int nside_src, uint4 *pix,
                                double2 *w) {
  const uint64_t n = 12ull * nside_dst * nside_dst;
  if (12ull * nside_src * nside_src > 0xffffffffull) return cudaErrorInvalidValue;
  interp_table_kernel<<<blocks_for(n, 256), 256, 0, s>>>(nside_dst, nside_src, pix, w);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(cudaStream_t s, int nside_dst, int nside_src,
                              int nmaps, double *const *dst,
                              const double *const *src, const InterpTab *tab) {
  const uint64_t n = 12ull * nside_dst * nside_dst;
  for (int k0 = 0; k0 < nmaps; k0 += kMaxMergeMaps) {
    MergeMaps M{};
    M.n = nmaps - k0 < kMaxMergeMaps ? nmaps - k0 : kMaxMergeMaps;
    for (int k = 0; k < M.n; ++k) {
      M.dst[k] = dst[k0 + k];
      M.src[k] = src[k0 + k];
    }
    accumulate_kernel<<<blocks_for(n, 256), 256, 0, s>>>(nside_dst, nside_src, M,
                                                         tab ? *tab : InterpTab{});
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_merge_all(cudaStream_t s, int nside_dst, int nout, const int *idx,
                             double *const *dst, int nshells, const int *nside,
                             const double *const *base, const InterpTab *tab) {
  if (nshells < 1 || nshells > HXG_MAX_SHELLS) return cudaErrorInvalidValue;
  const uint64_t n = 12ull * nside_dst * nside_dst;
  for (int k0 = 0; k0 < nout; k0 += kMaxMergeMaps) {
    MergeAll M{};
    M.n = nout - k0 < kMaxMergeMaps ? nout - k0 : kMaxMergeMaps;
    M.nshells = nshells;
    bool all_tab = true;
    for (int sh = 0; sh < nshells; ++sh) {
      M.nside[sh] = nside[sh];
      M.base[sh] = base[sh];
      if (tab) M.tab[sh] = tab[sh];
      if (nside[sh] != nside_dst && !M.tab[sh].pix) all_tab = false;
    }
    for (int k = 0; k < M.n; ++k) {
      M.idx[k] = idx[k0 + k];
      M.dst[k] = dst[k0 + k];
    }
    if (all_tab)
      merge_all_kernel<true><<<blocks_for(n, 256), 256, 0, s>>>(nside_dst, M);
    else
      merge_all_kernel<false><<<blocks_for(n, 256), 256, 0, s>>>(nside_dst, M);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_pix2ang(cudaStream_t s, int nside, uint64_t n,
                           double *theta, double *phi) {
  pix2ang_kernel<<<blocks_for(n, 256), 256, 0, s>>>(nside, n, theta, phi);
  return cudaGetLastError();
}

cudaError_t launch_interpolate(cudaStream_t s, int nside, const double *map,
                               uint64_t n, const double *theta,
                               const double *phi, double *out) {
  interpolate_kernel<<<blocks_for(n, 256), 256, 0, s>>>(nside, map, n, theta,
                                                        phi, out);
  return cudaGetLastError();
}

cudaError_t launch_los_geometry(cudaStream_t s, uint64_t n,
                                const double *theta, const double *phi,
                                const double *b, double *versor, double *bpar,
                                double *bper, double *c2, double *s2) {
  los_geometry_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      n, theta, phi, b, versor, bpar, bper, c2, s2);
  return cudaGetLastError();
}

cudaError_t launch_read_group(cudaStream_t s, bool fp32,
                              const DevGridGroup &g, uint64_t n,
                              const double *pos, double *out) {
  if (fp32)
    read_group_kernel<float><<<blocks_for(n, 256), 256, 0, s>>>(g, n, pos, out);
  else
    read_group_kernel<double><<<blocks_for(n, 256), 256, 0, s>>>(g, n, pos, out);
  return cudaGetLastError();
}

cudaError_t launch_pack(cudaStream_t s, bool fp32, uint64_t n, void *rec,
                        const double *const b0[3], const double *const b1[3],
                        const double *t0, const double *t1, double bscale,
                        double tscale) {
  if (fp32)
    pack_kernel<float><<<blocks_for(n, 256), 256, 0, s>>>(
        n, static_cast<float *>(rec), b0[0], b0[1], b0[2], b1[0], b1[1], b1[2],
        t0, t1, bscale, tscale);
  else
    pack_kernel<double><<<blocks_for(n, 256), 256, 0, s>>>(
        n, static_cast<double *>(rec), b0[0], b0[1], b0[2], b1[0], b1[1],
        b1[2], t0, t1, bscale, tscale);
  return cudaGetLastError();
}

// The kernels are instantiated per grid-group count (0, 1, up to
// kMaxGroups) and per use of the Jaffe / JF12 / YMW16 blocks.
template <typename F>
static cudaError_t by_shape(int ngroups, bool ext, F &&f) {
  const auto g = [&](auto ng) {
    if (ext)
      f(ng, std::true_type{});
    else
      f(ng, std::false_type{});
  };
  if (ngroups == 0)
    g(std::integral_constant<int, 0>{});
  else if (ngroups == 1)
    g(std::integral_constant<int, 1>{});
  else
    g(std::integral_constant<int, 4>{});
  return cudaGetLastError();
}

cudaError_t launch_shell(cudaStream_t s, bool fp32, const ShellLaunch &P,
                         unsigned blocks, unsigned threads) {
  const bool fast = fast_models(P);
  return by_shape(P.ngroups, P.ext != nullptr, [&](auto ng, auto ext) {
    constexpr int NG = decltype(ng)::value;
    constexpr bool E = decltype(ext)::value;
    if (fp32 && fast)
      shell_fp32c_kernel<NG, false, true><<<blocks, threads, 0, s>>>(P);
    else if (fp32)
      shell_fp32c_kernel<NG, E, false><<<blocks, threads, 0, s>>>(P);
    else if (fast)
      shell_fp64_kernel<NG, false, false, true><<<blocks, threads, 0, s>>>(P);
    else
      shell_fp64_kernel<decltype(ng)::value, false, decltype(ext)::value>
          <<<blocks, threads, 0, s>>>(P);
  });
}

cudaError_t launch_shell_multi(cudaStream_t s, const ShellLaunch &P, int nf, const void *fq,
                               unsigned blocks, unsigned threads) {
  const bool fast = fast_models(P);
  return by_shape(P.ngroups, P.ext != nullptr, [&](auto ng, auto ext) {
    constexpr int NG = decltype(ng)::value;
    constexpr bool E = decltype(ext)::value;
    const FreqSet<2> &F2 = *static_cast<const FreqSet<2> *>(fq);
    const FreqSet<3> &F3 = *static_cast<const FreqSet<3> *>(fq);
    if (fast && nf == 2)
      shell_fp32c_multi_kernel<NG, false, 2, true><<<blocks, threads, 0, s>>>(P, F2);
    else if (fast)
      shell_fp32c_multi_kernel<NG, false, 3, true><<<blocks, threads, 0, s>>>(P, F3);
    else if (nf == 2)
      shell_fp32c_multi_kernel<NG, E, 2, false><<<blocks, threads, 0, s>>>(P, F2);
    else
      shell_fp32c_multi_kernel<NG, E, 3, false><<<blocks, threads, 0, s>>>(P, F3);
  });
}

cudaError_t launch_batch_level(cudaStream_t s, bool fp32, int ngroups, bool ext, bool fast,
                               const BatchLevel &B, unsigned blocks) {
  return by_shape(ngroups, ext, [&](auto ng, auto ex) {
    constexpr int NG = decltype(ng)::value;
    constexpr bool E = decltype(ex)::value;
    if (fp32 && fast)
      batch_fp32c_kernel<NG, false, true><<<blocks, 256, 0, s>>>(B);
    else if (fp32)
      batch_fp32c_kernel<NG, E, false><<<blocks, 256, 0, s>>>(B);
    else if (fast)
      batch_fp64_kernel<NG, false, true><<<blocks, 256, 0, s>>>(B);
    else
      batch_fp64_kernel<NG, E, false><<<blocks, 256, 0, s>>>(B);
  });
}

cudaError_t launch_batch_level_multi(cudaStream_t s, int ngroups, bool ext, bool fast, int nf,
                                     const void *B, unsigned blocks) {
  return by_shape(ngroups, ext, [&](auto ng, auto ex) {
    constexpr int NG = decltype(ng)::value;
    constexpr bool E = decltype(ex)::value;
    const auto &B2 = *static_cast<const BatchLevelMulti<2> *>(B);
    const auto &B3 = *static_cast<const BatchLevelMulti<3> *>(B);
    if (fast && nf == 2)
      batch_fp32c_multi_kernel<NG, false, 2, true><<<blocks, HXG_BATCH_MULTI_THREADS, 0, s>>>(B2);
    else if (fast)
      batch_fp32c_multi_kernel<NG, false, 3, true><<<blocks, HXG_BATCH_MULTI_THREADS, 0, s>>>(B3);
    else if (nf == 2)
      batch_fp32c_multi_kernel<NG, E, 2, false><<<blocks, HXG_BATCH_MULTI_THREADS, 0, s>>>(B2);
    else
      batch_fp32c_multi_kernel<NG, E, 3, false><<<blocks, HXG_BATCH_MULTI_THREADS, 0, s>>>(B3);
  });
}

cudaError_t batch_multi_occupancy(int ngroups, bool ext, bool fast, int nf, int *blocks_per_sm) {
  const void *f = nullptr;
  by_shape(ngroups, ext, [&](auto ng, auto ex) {
    constexpr int NG = decltype(ng)::value;
    constexpr bool E = decltype(ex)::value;
    if (fast && nf == 2)
      f = (const void *)batch_fp32c_multi_kernel<NG, false, 2, true>;
    else if (fast)
      f = (const void *)batch_fp32c_multi_kernel<NG, false, 3, true>;
    else if (nf == 2)
      f = (const void *)batch_fp32c_multi_kernel<NG, E, 2, false>;
    else
      f = (const void *)batch_fp32c_multi_kernel<NG, E, 3, false>;
  });
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, HXG_BATCH_MULTI_THREADS, 0);
}

cudaError_t batch_level_occupancy(bool fp32, int ngroups, bool ext, bool fast,
                                  int *blocks_per_sm) {
  const void *f = nullptr;
  by_shape(ngroups, ext, [&](auto ng, auto ex) {
    constexpr int NG = decltype(ng)::value;
    constexpr bool E = decltype(ex)::value;
    if (fp32 && fast)
      f = (const void *)batch_fp32c_kernel<NG, false, true>;
    else if (fp32)
      f = (const void *)batch_fp32c_kernel<NG, E, false>;
    else if (fast)
      f = (const void *)batch_fp64_kernel<NG, false, true>;
    else
      f = (const void *)batch_fp64_kernel<NG, E, false>;
  });
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, 256, 0);
}

// Split interleaved (x, y, z) voxel triples into three SoA arrays
// (the on-disk layout of Grid_breg / Grid_brnd, grid_breg.cc:48-66).
__global__ void deinterleave3_kernel(uint64_t n, const double *src, double *x, double *y,
                                     double *z) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = src[3 * i];
  y[i] = src[3 * i + 1];
  z[i] = src[3 * i + 2];
}

cudaError_t launch_deinterleave3(cudaStream_t s, uint64_t n, const double *src, double *x,
                                 double *y, double *z) {
  if (n == 0) return cudaSuccess;
  deinterleave3_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, src, x, y, z);
  return cudaGetLastError();
}

// The inverse: three SoA arrays into (x, y, z) triples (Grid_brnd::export_grid,
// grid_brnd.cc:57-73).
__global__ void interleave3_kernel(uint64_t n, const double *x, const double *y,
                                   const double *z, double *dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dst[3 * i] = x[i];
  dst[3 * i + 1] = y[i];
  dst[3 * i + 2] = z[i];
}

cudaError_t launch_interleave3(cudaStream_t s, uint64_t n, const double *x, const double *y,
                               const double *z, double *dst) {
  if (n == 0) return cudaSuccess;
  interleave3_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, x, y, z, dst);
  return cudaGetLastError();
}

// FP32 values widened to FP64 (exact): an FP32 host grid's staged chunk
// into its FP64 slot.
__global__ void widen_kernel(uint64_t n, const float *src, double *dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dst[i] = (double)src[i];
}

cudaError_t launch_widen(cudaStream_t s, uint64_t n, const float *src, double *dst) {
  if (n == 0) return cudaSuccess;
  widen_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, src, dst);
  return cudaGetLastError();
}

cudaError_t launch_batch_merge(cudaStream_t s, const MergeJob *jobs,
                               const unsigned long long *block0, int njobs,
                               unsigned long long nblocks) {
  if (njobs == 0 || nblocks == 0) return cudaSuccess;
  batch_merge_kernel<<<(unsigned)nblocks, 256, 0, s>>>(jobs, block0, njobs);
  return cudaGetLastError();
}

cudaError_t launch_batch_zero(cudaStream_t s, const ZeroJob *jobs,
                              const unsigned long long *block0, int njobs,
                              unsigned long long nblocks) {
  if (njobs == 0 || nblocks == 0) return cudaSuccess;
  batch_zero_kernel<<<(unsigned)nblocks, 256, 0, s>>>(jobs, block0, njobs);
  return cudaGetLastError();
}

cudaError_t launch_accumulate_transpose(cudaStream_t s, int nside_out,
                                        int nside_shell, const double *g_out,
                                        double *g_shell, double scale) {
  const uint64_t n = 12ull * nside_out * nside_out;
  accumulate_transpose_kernel<<<blocks_for(n, 256), 256, 0, s>>>(
      nside_out, nside_shell, g_out, g_shell, scale);
  return cudaGetLastError();
}

cudaError_t launch_adjoint(cudaStream_t s, const AdjointLaunch &A,
                           unsigned blocks, unsigned threads) {
  const bool ext = A.F.ext != nullptr;
  const bool fast = fast_models(A.F);
  if (A.F.ngroups == 0) {
    if (fast)
      shell_fp64_adjoint_kernel<0, false, true><<<blocks, threads, 0, s>>>(A);
    else if (ext)
      shell_fp64_adjoint_kernel<0, true, false><<<blocks, threads, 0, s>>>(A);
    else
      shell_fp64_adjoint_kernel<0, false, false><<<blocks, threads, 0, s>>>(A);
  } else {
    if (fast)
      shell_fp64_adjoint_kernel<1, false, true><<<blocks, threads, 0, s>>>(A);
    else if (ext)
      shell_fp64_adjoint_kernel<1, true, false><<<blocks, threads, 0, s>>>(A);
    else
      shell_fp64_adjoint_kernel<1, false, false><<<blocks, threads, 0, s>>>(A);
  }
  return cudaGetLastError();
}

cudaError_t launch_adjoint32(cudaStream_t s, const AdjointLaunch &A, unsigned blocks,
                             unsigned threads) {
  if (A.F.ngroups == 0)
    shell_fp32c_adjoint_kernel<0><<<blocks, threads, 0, s>>>(A);
  else
    shell_fp32c_adjoint_kernel<1><<<blocks, threads, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_unpack_grad(cudaStream_t s, uint64_t n, const double *rec,
                               double *gbx, double *gby, double *gbz,
                               double *gne, double bscale) {
  unpack_grad_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, rec, gbx, gby, gbz, gne, bscale);
  return cudaGetLastError();
}

}  // namespace hxg
