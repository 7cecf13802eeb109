// hxg_noalloc.cu -- the allocation-free variant of the FP64 integrator.
//
// Some callers cannot call cudaMalloc: plugins that live inside a host
// application which owns every device allocation through its own pool, and
// real-time pipelines whose memory is fixed at start-up and which must not
// touch the allocator afterwards.  hxg_write_grid_noalloc serves them: it takes device inputs and
// device outputs from the caller and keeps its only scratch -- the five
// per-shell HEALPix maps -- in the fixed-size array below.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds it until the process exits.  Host code never uses its name
// as an address (in host code the name is only a stand-in symbol); the
// device address is looked up with cudaGetSymbolAddress once per CUDA
// context, with that context current.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/hxg.h"
#include "hxg_integrate.cuh"
#include "hxg_internal.h"

namespace hxg {
int noalloc_shell_launch(const hxg_obs_t *o, const hxg_models_t *m,
                         const hxg_grid_desc_t *g, const double *rec,
                         uint32_t s, ShellLaunch *P, uint64_t *step);
bool noalloc_models_supported(const hxg_models_t *m);
bool noalloc_obs_valid(const hxg_obs_t *o);
}  // namespace hxg

namespace {

constexpr uint64_t kMaxShellPix = 12ull * HXG_NOALLOC_MAX_NSIDE * HXG_NOALLOC_MAX_NSIDE;

// Five shell maps (dm, fd, I, Q, U) at the largest allowed shell Nside.
static __device__ __align__(256) double g_noalloc_scratch[5 * kMaxShellPix];

// Device addresses of the scratch array, one per CUDA context that has
// called in.  A context is named by its driver-assigned ID (cuCtxGetId),
// which is never reused within the process: after cudaDeviceReset the
// module is loaded again into a new context, the array may move, and the
// new context's ID misses this table, so the address is looked up again.
// Only successful lookups are stored; a failed one is retried next call.
struct ScratchEntry {
  unsigned long long ctx_id;
  double *ptr;
};
constexpr int kMaxContexts = 64;
std::mutex g_mu;
ScratchEntry g_entries[kMaxContexts] = {};
int g_next_entry = 0;  // slot reused next when the table is full

using CtxGetCurrentFn = int (*)(void **ctx);
using CtxGetIdFn = int (*)(void *ctx, unsigned long long *id);

// ID of the context current on this thread; 0 when there is none yet.
// The driver functions are fetched through the runtime, so the library
// needs no link-time libcuda.
bool current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  if (get_current == nullptr || get_id == nullptr) return false;
  void *ctx = nullptr;
  if (get_current(&ctx) != 0) return false;
  if (ctx == nullptr) {
    *id = 0;
    return true;
  }
  return get_id(ctx, id) == 0;
}

// Device address of the scratch array in the current context (the
// current device's primary context for runtime-API callers).  The first
// call in a context looks it up with cudaGetSymbolAddress, which also
// creates the primary context when none is current yet.
int scratch_for_current_context(double **out) {
  unsigned long long id = 0;
  if (!current_context_id(&id)) return HXG_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  if (id != 0)
    for (const ScratchEntry &e : g_entries)
      if (e.ctx_id == id && e.ptr != nullptr) {
        *out = e.ptr;
        return HXG_OK;
      }
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
    (void)cudaGetLastError();  // the failure is reported by the status
    return HXG_ERR_CUDA;
  }
  // the lookup made a context current if none was
  if (id == 0 && (!current_context_id(&id) || id == 0)) return HXG_ERR_CUDA;
  g_entries[g_next_entry] = ScratchEntry{id, static_cast<double *>(p)};
  g_next_entry = (g_next_entry + 1) % kMaxContexts;
  *out = static_cast<double *>(p);
  return HXG_OK;
}

}  // namespace

extern "C" int hxg_write_grid_noalloc(const hxg_obs_t *obs,
                                      const hxg_models_t *models,
                                      const hxg_grid_desc_t *grid,
                                      const double *d_records, double *d_dm,
                                      double *d_fd, double *d_is,
                                      double *d_qs, double *d_us,
                                      void *stream) {
  using namespace hxg;
  if (!obs || !models) return HXG_ERR_INVALID;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return HXG_ERR_NO_DEVICE;
  // the per-shell mask duplicates would need device storage of their own
  if (obs->do_mask) return HXG_ERR_UNSUPPORTED;
  if (!noalloc_obs_valid(obs)) return HXG_ERR_INVALID;
  if (!noalloc_models_supported(models)) return HXG_ERR_UNSUPPORTED;
  if (obs->do_sync && models->cre == HXG_CRE_NONE) return HXG_ERR_INVALID;
  const bool uses_grid = models->breg == HXG_BREG_GRID || models->brnd == HXG_BRND_GRID ||
                         models->tereg == HXG_TEREG_GRID || models->ternd == HXG_TERND_GRID;
  if (uses_grid && (!grid || !d_records)) return HXG_ERR_INVALID;
  if (uses_grid && (grid->nx < 2 || grid->ny < 2 || grid->nz < 2 ||
                    !(grid->x_max > grid->x_min) || !(grid->y_max > grid->y_min) ||
                    !(grid->z_max > grid->z_min)))
    return HXG_ERR_INVALID;
  if ((obs->do_dm && !d_dm) || (obs->do_fd && !d_fd) ||
      (obs->do_sync && (!d_is || !d_qs || !d_us)))
    return HXG_ERR_INVALID;
  for (uint32_t s = 0; s < obs->total_shell; ++s)
    if (obs->nside_shell[s] > HXG_NOALLOC_MAX_NSIDE) return HXG_ERR_TOO_LARGE;
  // an error left by the caller's earlier work would surface in this
  // call's launch checks after part of the work is queued: refuse first
  if (cudaPeekAtLastError() != cudaSuccess) return HXG_ERR_CUDA;
  double *scratch = nullptr;
  int st = scratch_for_current_context(&scratch);
  if (st != HXG_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *tmp[5];
  for (int k = 0; k < 5; ++k) tmp[k] = scratch + (size_t)k * kMaxShellPix;
  // outputs start at zero (Grid_obs::build_grid); every shell map pixel is
  // rewritten by each shell launch, so the scratch needs no clearing
  const auto bytes = [](uint32_t ns) { return 12ull * ns * ns * sizeof(double); };
  if (obs->do_dm && cudaMemsetAsync(d_dm, 0, bytes(obs->nside_dm), s) != cudaSuccess)
    return HXG_ERR_CUDA;
  if (obs->do_fd && cudaMemsetAsync(d_fd, 0, bytes(obs->nside_fd), s) != cudaSuccess)
    return HXG_ERR_CUDA;
  if (obs->do_sync) {
    const size_t b = bytes(obs->nside_sync);
    if (cudaMemsetAsync(d_is, 0, b, s) != cudaSuccess ||
        cudaMemsetAsync(d_qs, 0, b, s) != cudaSuccess ||
        cudaMemsetAsync(d_us, 0, b, s) != cudaSuccess)
      return HXG_ERR_CUDA;
  }
  for (uint32_t sh = 0; sh < obs->total_shell; ++sh) {
    ShellLaunch P;
    uint64_t step = 0;
    st = noalloc_shell_launch(obs, models, grid, uses_grid ? d_records : nullptr, sh, &P,
                              &step);
    if (st != HXG_OK) return st;
    P.fdmap = obs->do_fd ? d_fd : nullptr;
    P.nside_fdmap = obs->do_fd ? (int)obs->nside_fd : 0;
    P.mask = nullptr;
    for (int k = 0; k < 5; ++k) P.out[k] = tmp[k];
    const uint64_t npix = 12ull * obs->nside_shell[sh] * obs->nside_shell[sh];
    // whole warps of 32 pixels, one lane per pixel
    P.chunks = 1;
    P.log2_chunks = 0;
    const unsigned threads = HXG_FP64_THREADS;
    const unsigned blocks = (unsigned)((npix + threads - 1) / threads);
    if (launch_shell(s, false, P, blocks, threads) != cudaSuccess) return HXG_ERR_CUDA;
    const int ns = (int)obs->nside_shell[sh];
    if (obs->do_dm) {
      double *d[1] = {d_dm};
      const double *sr[1] = {tmp[0]};
      if (launch_accumulate(s, (int)obs->nside_dm, ns, 1, d, sr) != cudaSuccess)
        return HXG_ERR_CUDA;
    }
    if (obs->do_sync) {
      double *d[3] = {d_is, d_qs, d_us};
      const double *sr[3] = {tmp[2], tmp[3], tmp[4]};
      if (launch_accumulate(s, (int)obs->nside_sync, ns, 3, d, sr) != cudaSuccess)
        return HXG_ERR_CUDA;
    }
    if (obs->do_fd) {
      double *d[1] = {d_fd};
      const double *sr[1] = {tmp[1]};
      if (launch_accumulate(s, (int)obs->nside_fd, ns, 1, d, sr) != cudaSuccess)
        return HXG_ERR_CUDA;
    }
  }
  return HXG_OK;
}
