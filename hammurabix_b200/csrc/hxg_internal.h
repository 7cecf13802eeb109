// hxg_internal.h -- declarations shared by the host glue (hxg_api.cu) and
// the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hxg {

struct ShellLaunch;
struct DevGridGroup;
struct AdjointLaunch;
struct BatchLevel;
struct MergeJob;
struct ZeroJob;

cudaError_t launch_accumulate(cudaStream_t s, int nside_dst, int nside_src,
                              int nmaps, double *const *dst,
                              const double *const *src);
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
cudaError_t launch_accumulate_transpose(cudaStream_t s, int nside_out,
                                        int nside_shell, const double *g_out,
                                        double *g_shell, double scale);
cudaError_t launch_adjoint(cudaStream_t s, const AdjointLaunch &A,
                           unsigned blocks, unsigned threads);
cudaError_t launch_batch_level(cudaStream_t s, bool fp32, int ngroups, bool ext,
                               const BatchLevel &B, unsigned blocks);
cudaError_t batch_level_occupancy(bool fp32, int ngroups, bool ext, int *blocks_per_sm);
cudaError_t launch_batch_merge(cudaStream_t s, const MergeJob *jobs,
                               const unsigned long long *block0, int njobs,
                               unsigned long long nblocks);
cudaError_t launch_batch_zero(cudaStream_t s, const ZeroJob *jobs,
                              const unsigned long long *block0, int njobs,
                              unsigned long long nblocks);
cudaError_t launch_deinterleave3(cudaStream_t s, uint64_t n, const double *src, double *x,
                                 double *y, double *z);
cudaError_t launch_unpack_grad(cudaStream_t s, uint64_t n, const double *rec,
                               double *gbx, double *gby, double *gbz,
                               double *gne);

}  // namespace hxg
