// hxg_internal.h -- declarations shared by the host glue (hxg_api.cu) and
// the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/hxg.h"

namespace hxg {

struct ShellLaunch;
struct DevGridGroup;
struct AdjointLaunch;
struct BatchLevel;
struct MergeJob;
struct ZeroJob;
struct DevModels;
struct ExtModels;

// The BREG slot as the Brnd_es anisotropy reads it (Breg::read_grid,
// source/field/b/breg.cc:28-97): FP64 SoA vertex arrays in CGS.
struct RfgBregGrid {
  const double *bx, *by, *bz;  // null: the regular field is analytic
  int nx, ny, nz;
  double x_min, x_max, y_min, y_max, z_min, z_max;
};

// The bilinear interpolation of an Nside-nside_src map at every pixel of an
// Nside-nside_dst map (hpx_interp_weights), made once per Nside pair: pix[i]
// = the 4 source pixels of output pixel i, w[2 i] and w[2 i + 1] = weights
// 0-1 and 2-3.  Source maps of up to 2^32 pixels.
struct InterpTab {
  const uint4 *pix = nullptr;
  const double2 *w = nullptr;
};
cudaError_t launch_interp_table(cudaStream_t s, int nside_dst, int nside_src, uint4 *pix,
                                double2 *w);
// dst_k += src_k (interpolated when the Nsides differ, from tab when given)
cudaError_t launch_accumulate(cudaStream_t s, int nside_dst, int nside_src,
                              int nmaps, double *const *dst,
                              const double *const *src, const InterpTab *tab = nullptr);
cudaError_t launch_pix2ang(cudaStream_t s, int nside, uint64_t n,
                           double *theta, double *phi);
cudaError_t launch_interpolate(cudaStream_t s, int nside, const double *map,
                               uint64_t n, const double *theta,
                               const double *phi, double *out);
cudaError_t launch_los_geometry(cudaStream_t s, uint64_t n,
                                const double *theta, const double *phi,
                                const double *b, double *versor, double *bpar,
                                double *bper, double *c2, double *s2);
cudaError_t launch_read_group(cudaStream_t s, bool fp32,
                              const DevGridGroup &g, uint64_t n,
                              const double *pos, double *out);
cudaError_t launch_pack(cudaStream_t s, bool fp32, uint64_t n, void *rec,
                        const double *const b0[3], const double *const b1[3],
                        const double *t0, const double *t1, double bscale,
                        double tscale);
cudaError_t launch_shell(cudaStream_t s, bool fp32, const ShellLaunch &P,
                         unsigned blocks, unsigned threads);
// nf = 2 or 3 frequency passes in one FP32C shell traversal; fq points to a
// FreqSet<nf> (hxg_integrate.cuh).
cudaError_t launch_shell_multi(cudaStream_t s, const ShellLaunch &P, int nf, const void *fq,
                               unsigned blocks, unsigned threads);
cudaError_t launch_accumulate_transpose(cudaStream_t s, int nside_out,
                                        int nside_shell, const double *g_out,
                                        double *g_shell, double scale);
cudaError_t launch_adjoint(cudaStream_t s, const AdjointLaunch &A,
                           unsigned blocks, unsigned threads);
// The FP32C form's adjoint (the grid workloads' models, at most one grid).
cudaError_t launch_adjoint32(cudaStream_t s, const AdjointLaunch &A, unsigned blocks,
                             unsigned threads);
// fast: every plan's models satisfy fast_models (the kFast instantiations).
cudaError_t launch_batch_level(cudaStream_t s, bool fp32, int ngroups, bool ext, bool fast,
                               const BatchLevel &B, unsigned blocks);
cudaError_t batch_level_occupancy(bool fp32, int ngroups, bool ext, bool fast,
                                  int *blocks_per_sm);
// Fused-frequency plans (nf = 2 or 3): B points to a BatchLevelMulti<nf>.
cudaError_t launch_batch_level_multi(cudaStream_t s, int ngroups, bool ext, bool fast, int nf,
                                     const void *B, unsigned blocks);
cudaError_t batch_multi_occupancy(int ngroups, bool ext, bool fast, int nf,
                                  int *blocks_per_sm);
cudaError_t launch_batch_merge(cudaStream_t s, const MergeJob *jobs,
                               const unsigned long long *block0, int njobs,
                               unsigned long long nblocks);
cudaError_t launch_batch_zero(cudaStream_t s, const ZeroJob *jobs,
                              const unsigned long long *block0, int njobs,
                              unsigned long long nblocks);
cudaError_t launch_deinterleave3(cudaStream_t s, uint64_t n, const double *src, double *x,
                                 double *y, double *z);
cudaError_t launch_widen(cudaStream_t s, uint64_t n, const float *src, double *dst);
cudaError_t launch_interleave3(cudaStream_t s, uint64_t n, const double *x, const double *y,
                               const double *z, double *dst);
// Outputs per merge launch (launch_accumulate, launch_merge_all).
constexpr int kMaxMergeOuts = 12;
// Merges the shell maps of a whole pass into nout outputs at one Nside:
// shell s holds its maps in one block at base[s] (map j at
// base[s] + j npix(nside[s])); dst[k] = the shell-ordered sum of map idx[k].
// tab[s]: shell s's interpolation table (null members: computed in place).
cudaError_t launch_merge_all(cudaStream_t s, int nside_dst, int nout, const int *idx,
                             double *const *dst, int nshells, const int *nside,
                             const double *const *base, const InterpTab *tab);
cudaError_t launch_unpack_grad(cudaStream_t s, uint64_t n, const double *rec,
                               double *gbx, double *gby, double *gbz,
                               double *gne, double bscale);

// Random-field generators (hxg_rfg.cu); synchronous on s, HXG_* status.
// `work` is the caller's workspace (created on first use, kept for the next
// call of the same grid shape, freed by rfg_release).
struct RfgWork;
void rfg_release(RfgWork *work);
int generate_ternd_dft(cudaStream_t s, RfgWork *&work, const hxg_grid_desc_t &g,
                       const hxg_ternd_dft_t &p, const double obs[3], uint64_t seed,
                       double *te);
int generate_brnd_es(cudaStream_t s, RfgWork *&work, const hxg_grid_desc_t &g,
                     const hxg_brnd_es_t &p, const DevModels &M, const ExtModels *ext,
                     const RfgBregGrid &breg, uint64_t seed, double *bx, double *by,
                     double *bz);

}  // namespace hxg
