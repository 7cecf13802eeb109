// hxg_batch.cuh -- batched forward: many independent passes (parameter
// sets x frequencies) of Integrator::write_grid (integrator.cc:23-134) in
// one CUDA graph.  Per shell level the graph holds one persistent shell
// kernel over every entry that has that shell and one kernel that merges
// the shell maps into each entry's outputs (Hampix::accumulate,
// hamdis.h:698-721); the outer-shell levels read the inner Faraday depth
// the earlier levels accumulated (integrator.cc:78-86).
#pragma once

#include "hxg_fp32c.cuh"
#include "hxg_integrate.cuh"
#include "hxg_internal.h"

namespace hxg {

// One shell level of a batch: plan k (one entry's shell launch block) owns
// the warp tiles [tile_start[k], tile_start[k + 1]).  Warps take `grain`
// tiles at a time from the work counter (zeroed before the launch).
struct BatchLevel {
  const ShellLaunch *plans;
  const unsigned long long *tile_start;  // nplans + 1 entries
  int nplans;
  int grain;
  unsigned long long *counter;
};

// A plan of NF frequency passes of one parameter set fused into one
// traversal (the FP32C form; fp32c_tile<NG, kExt, NF>).
template <int NF>
struct FusedPlan {
  ShellLaunch P;
  FreqSet<NF> F;
};

// The same work distribution over fused plans.
template <int NF>
struct BatchLevelMulti {
  const FusedPlan<NF> *plans;
  const unsigned long long *tile_start;
  int nplans;
  int grain;
  unsigned long long *counter;
};

// Plan index of tile t0: the last plan whose first tile is <= t0.
__device__ __forceinline__ int batch_plan_of(const unsigned long long *tile_start, int nplans,
                                             unsigned long long t0) {
  int lo = 0, hi = nplans - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_start[mid] <= t0) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int NG, bool kExt, int NF, bool kFast>
__device__ __forceinline__ void batch_multi_body(const BatchLevelMulti<NF> &B) {
  const int lane = threadIdx.x & 31;
  const unsigned long long total = B.tile_start[B.nplans];
  for (;;) {
    unsigned long long t0 = 0;
    if (lane == 0) t0 = atomicAdd(B.counter, (unsigned long long)B.grain);
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= total) return;
    const unsigned long long t1 = min(t0 + (unsigned long long)B.grain, total);
    int k = batch_plan_of(B.tile_start, B.nplans, t0);
    for (unsigned long long t = t0; t < t1; ++t) {
      while (t >= B.tile_start[k + 1]) ++k;
      const FusedPlan<NF> &FP = B.plans[k];
      fp32c_tile<NG, kExt, NF, kFast>(FP.P, FP.F, (long long)(t - B.tile_start[k]), lane);
    }
  }
}

// Launch shape of the fused batch kernel (threads per block, resident
// blocks per SM its register allocation must allow).  256 x 2 (128
// registers) runs config 5 in 927 ms against 943 ms at 128 x 5, 968 ms at
// 256 x 3 and 988 ms at 128 x 7 (the smaller budgets spill 300-460 bytes).
#ifndef HXG_BATCH_MULTI_THREADS
#define HXG_BATCH_MULTI_THREADS 256
#endif
#ifndef HXG_BATCH_MULTI_MIN_BLOCKS
#define HXG_BATCH_MULTI_MIN_BLOCKS 2
#endif

// kFast: every plan's models satisfy fast_models.
template <int NG, bool kExt, int NF, bool kFast>
__global__ void __launch_bounds__(HXG_BATCH_MULTI_THREADS, HXG_BATCH_MULTI_MIN_BLOCKS)
batch_fp32c_multi_kernel(const BatchLevelMulti<NF> B) {
  batch_multi_body<NG, kExt, NF, kFast>(B);
}

template <int NG, bool kFp32, bool kExt, bool kFast>
__device__ __forceinline__ void batch_level_body(const BatchLevel &B) {
  const int lane = threadIdx.x & 31;
  const unsigned long long total = B.tile_start[B.nplans];
  for (;;) {
    unsigned long long t0 = 0;
    if (lane == 0) t0 = atomicAdd(B.counter, (unsigned long long)B.grain);
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= total) return;
    const unsigned long long t1 = min(t0 + (unsigned long long)B.grain, total);
    // last plan whose first tile is <= t0
    int lo = 0, hi = B.nplans - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (B.tile_start[mid] <= t0) lo = mid; else hi = mid - 1;
    }
    int k = lo;
    for (unsigned long long t = t0; t < t1; ++t) {
      while (t >= B.tile_start[k + 1]) ++k;
      const ShellLaunch &P = B.plans[k];
      const long long gw = (long long)(t - B.tile_start[k]);
      if (kFp32)
        fp32c_tile<NG, kExt, kFast>(P, gw, lane);
      else
        fp64_tile<NG, false, kExt, kFast>(P, gw, lane);
    }
  }
}

// The launch blocks are read from global memory, which needs more live
// registers than the single-launch kernel: 2 resident blocks per SM.
template <int NG, bool kExt, bool kFast>
__global__ void __launch_bounds__(256, 2)
batch_fp32c_kernel(const BatchLevel B) {
  batch_level_body<NG, true, kExt, kFast>(B);
}

template <int NG, bool kExt, bool kFast>
__global__ void __launch_bounds__(256)
batch_fp64_kernel(const BatchLevel B) {
  batch_level_body<NG, false, kExt, kFast>(B);
}

// Map merges of one level: job j adds nmaps shell maps at nside_src into
// outputs at nside_dst (directly when the Nsides agree, else by HEALPix
// interpolation at each output pixel); it owns blocks
// [block0[j], block0[j + 1]).
struct MergeJob {
  double *dst[3];
  const double *src[3];
  int nmaps, nside_dst, nside_src, _pad;
  InterpTab tab;  // the Nside pair's interpolation table (null: in place)
};

// Zeroing of every output map of the batch (Grid_obs maps start at zero,
// grid_obs.cc:21-43): job j clears n doubles at p with blocks
// [block0[j], block0[j + 1]).
struct ZeroJob {
  double *p;
  unsigned long long n;
};

}  // namespace hxg
