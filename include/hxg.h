/*
 * hxg.h -- C ABI of the B200 line-of-sight integrator (hammurabiX hot path).
 *
 * One call of hxg_write_grid() is one call of the reference's
 *   void Integrator::write_grid(const Breg*, const Brnd*, const TEreg*,
 *        const TErnd*, const CREfield*, const Grid_breg*, const Grid_brnd*,
 *        const Grid_tereg*, const Grid_ternd*, const Grid_cre*, Grid_obs*,
 *        const Param*) const;                  (include/integrator.h:25-28)
 * i.e. one frequency pass over all shells, producing the DM / FD / sync I,Q,U
 * HEALPix RING maps that the reference accumulates into Grid_obs
 * (source/integrator/integrator.cc:23-134).  The virtual field objects and
 * the Param block of the reference become the plain structs below: a model
 * enum per field slot plus the model's parameters, in the CGS units the
 * reference's Param holds after parsing (source/param/param.cc).
 *
 * Conventions
 *  - every entry point returns an int status (HXG_OK == 0); hxg_last_error()
 *    gives the message of the last failure on a handle.  There is no CPU
 *    fallback: without a usable CUDA device every compute call fails with
 *    HXG_ERR_NO_DEVICE.
 *  - all floating-point inputs and outputs are IEEE double in CGS units
 *    (positions/lengths in cm, fields in Gauss, densities in cm^-3,
 *    frequencies in Hz), exactly as the reference's Param and Grid_* hold
 *    them.  Maps are HEALPix RING order, 12*nside^2 doubles.
 *  - a handle owns one CUDA stream (or the stream given to hxg_set_stream)
 *    and is not re-entrant; use one handle per host thread.
 */
#ifndef HXG_H
#define HXG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HXG_ABI_VERSION 1
#define HXG_MAX_SHELLS 16

/* ---- status codes -------------------------------------------------------
 * The reference throws std::runtime_error for unsupported models
 * (source/pipeline/pipeline.cc:47,78,101,123,133,155) and asserts otherwise;
 * the ABI returns these codes instead.                                      */
enum {
  HXG_OK = 0,
  HXG_ERR_INVALID = 1,     /* bad argument, size or descriptor              */
  HXG_ERR_UNSUPPORTED = 2, /* model / precision / combination unsupported   */
  HXG_ERR_CUDA = 3,        /* a CUDA runtime call failed                    */
  HXG_ERR_OOM = 4,         /* device allocation failed                      */
  HXG_ERR_TIMEOUT = 5,     /* a bounded device wait ran out                 */
  HXG_ERR_STATE = 6,       /* call order: e.g. grid not uploaded            */
  HXG_ERR_NO_DEVICE = 7,   /* no CUDA device / library built without one    */
  HXG_ERR_TOO_LARGE = 8    /* request exceeds the fixed scratch of
                              hxg_write_grid_noalloc                         */
};

/* ---- precision forms ---------------------------------------------------- */
enum {
  HXG_FP64 = 0,  /* plain FP64 everywhere (parity form)                     */
  HXG_FP32C = 1  /* FP32 field sampling + Kahan-compensated FP32 sums; FP64
                    for ray setup, grid coordinates, Faraday depth and its
                    phase, and the cross-shell map sums                     */
};

/* ---- field slots (Grid_breg/brnd/tereg/ternd/cre, include/grid.h:49-168) */
enum {
  HXG_FIELD_BREG = 0,
  HXG_FIELD_BRND = 1,
  HXG_FIELD_TEREG = 2,
  HXG_FIELD_TERND = 3,
  HXG_FIELD_CRE = 4
};

/* ---- model enums (replace the virtual dispatch of Breg::read_field
 *      source/field/b/breg.cc:11-26, Brnd::read_field brnd.cc:12-23,
 *      TEreg::read_field tereg.cc:11-25, TErnd::read_field ternd.cc:12-19,
 *      and the CREfield subclasses include/crefield.h)                     */
enum {
  HXG_BREG_NONE = 0,   /* Breg base class: zero field                        */
  HXG_BREG_GRID = 1,   /* read_grid, trilinear (breg.cc:28-97)               */
  HXG_BREG_LSA = 2,    /* Breg_lsa   (source/field/b/breg_lsa.cc:9-26)       */
  HXG_BREG_UNIF = 3,   /* Breg_unif  (breg_unif.cc:7-12)                     */
  HXG_BREG_CART = 4,   /* Breg_cart  (breg_cart.cc:7-11)                     */
  HXG_BREG_HELIX = 5,  /* Breg_helix (breg_helix.cc:13-30)                   */
  HXG_BREG_JAFFE = 6,  /* Breg_jaffe (breg_jaffe.cc)                         */
  HXG_BREG_JF12 = 7,   /* Breg_jf12  (breg_jf12.cc)                          */
  HXG_BREG_SPIRAL = 8  /* exponential-disk logarithmic spiral; not a
                          reference model, defined by hxg_breg_spiral_t      */
};
enum { HXG_BRND_NONE = 0, HXG_BRND_GRID = 1 };
enum {
  HXG_TEREG_NONE = 0,
  HXG_TEREG_GRID = 1,
  HXG_TEREG_UNIF = 2,   /* TEreg_unif (source/field/te/tereg_unif.cc:6-12)  */
  HXG_TEREG_YMW16 = 3,  /* TEreg_ymw16 (tereg_ymw16.cc)                     */
  HXG_TEREG_EXPDISK = 4 /* exponential disk; not a reference model          */
};
enum { HXG_TERND_NONE = 0, HXG_TERND_GRID = 1 };
enum {
  HXG_CRE_NONE = 0,
  HXG_CRE_ANA = 1,  /* CRE_ana  (source/field/cre/cre_ana.cc:11-63)        */
  HXG_CRE_UNIF = 2, /* CRE_unif (cre_unif.cc:11-59)                        */
  HXG_CRE_GRID = 3  /* CRE_num: spectral integral over a 4-D grid
                       (integrator.cc:288-330, 357-400)                    */
};

/* ---- model parameters: field-for-field copies of Param (include/param.h) */
typedef struct { double b0, psi0, psi1, chi0; } hxg_breg_lsa_t;   /* param.h:121-126 */
typedef struct { double bp, bv, l0; } hxg_breg_unif_t;            /* param.h:128-131 */
typedef struct { double bx, by, bz; } hxg_breg_cart_t;            /* param.h:149-152 */
typedef struct { double bx, by, bz, r_min, r_max; } hxg_breg_helix_t; /* param.h:153-156 */
typedef struct {                                                   /* param.h:133-148 */
  int32_t quadruple, bss, ring, bar;
  uint32_t arm_num, _pad;
  double disk_amp, disk_z0, halo_amp, halo_z0;
  double r_inner, r_scale, r_peak;
  double ring_amp, bar_amp, ring_r, bar_a, bar_b, bar_phi0;
  double arm_amp[8], arm_phi0[8];
  double arm_pitch, arm_r0, arm_z0;
  double comp_r, comp_c, comp_d, comp_p;
} hxg_breg_jaffe_t;
typedef struct {                                                   /* param.h:157-162 */
  double b_arm1, b_arm2, b_arm3, b_arm4, b_arm5, b_arm6, b_arm7;
  double b_ring, h_disk, w_disk;
  double Bn, Bs, rn, rs, wh, z0;
  double B0_X, Xtheta, rpc_X, r0_X;
} hxg_breg_jf12_t;
/* Exponential-disk logarithmic spiral (not in the reference):
 *   r = sqrt(x^2+y^2); B = 0 if r > 20 kpc or r < 3 kpc, else
 *   B = b0 * exp(-(r - r_sun)/r_scale) * exp(-|z|/h_scale)
 *       * ( sin(pitch)cos(p) - cos(pitch)sin(p),
 *           sin(pitch)sin(p) + cos(pitch)cos(p), 0 ),  cos(p)=x/r, sin(p)=y/r
 * with r_sun the observer's cylindrical radius: the Breg_lsa form with
 * psi0 = pitch, psi1 = chi0 = 0, times an exponential-disk amplitude.      */
typedef struct { double b0, pitch, r_scale, h_scale; } hxg_breg_spiral_t;
typedef struct { double n0, r0; } hxg_tereg_unif_t;               /* param.h:208-211 */
/* Exponential disk (not in the reference): n = n0 exp(-r/r_scale) exp(-|z|/h_scale) */
typedef struct { double n0, r_scale, h_scale; } hxg_tereg_expdisk_t;
typedef struct {                                                   /* param.h:193-206 */
  double r_warp, r0, t0_gamma_w;
  double t1_ad, t1_bd, t1_n1, t1_h1;
  double t2_a2, t2_b2, t2_n2, t2_k2;
  double t3_b2s, t3_ka, t3_narm[5], t3_warm[5], t3_aa, t3_ncn, t3_wcn,
      t3_thetacn, t3_nsg, t3_wsg, t3_thetasg, t3_rmin[5], t3_phimin[5],
      t3_tpitch[5], t3_cpitch[5];
  double t4_ngc, t4_agc, t4_hgc;
  double t5_kgn, t5_ngn, t5_wgn, t5_agn;
  double t6_j_lb, t6_nlb1, t6_detlb1, t6_wlb1, t6_hlb1, t6_thetalb1, t6_nlb2,
      t6_detlb2, t6_wlb2, t6_hlb2, t6_thetalb2;
  double t7_nli, t7_rli, t7_wli, t7_detthetali, t7_thetali;
} hxg_tereg_ymw16_t;
/* Random-field generator parameters, as Param holds them after parsing
 * (source/param/param.cc:366-374, 693-697): rms in G for B (the n_e rms in
 * cm^-3), k0/k1 in 1/kpc, r0/z0 in cm.                                     */
typedef struct { double rms, k0, k1, a0, a1, rho, r0, z0; } hxg_brnd_es_t; /* param.h:167-173 */
typedef struct { double rms, k0, a0, r0, z0; } hxg_ternd_dft_t;            /* param.h:216-221 */
typedef struct { double alpha, beta, theta, r0, z0, E0, j0; } hxg_cre_ana_t; /* param.h:225-229 */
typedef struct { double alpha, r0, E0, j0; } hxg_cre_unif_t;                 /* param.h:231-235 */

typedef struct {
  int32_t breg, brnd, tereg, ternd, cre, _pad;
  hxg_breg_lsa_t lsa;
  hxg_breg_unif_t unif;
  hxg_breg_cart_t cart;
  hxg_breg_helix_t helix;
  hxg_breg_jaffe_t jaffe;
  hxg_breg_jf12_t jf12;
  hxg_breg_spiral_t spiral;
  hxg_tereg_unif_t te_unif;
  hxg_tereg_ymw16_t ymw16;
  hxg_tereg_expdisk_t te_exp;
  hxg_cre_ana_t cre_ana;
  hxg_cre_unif_t cre_unif;
} hxg_models_t;

/* ---- grid geometry: Param::grid_{breg,brnd,tereg,ternd,cre}
 *      (include/param.h:25-85).  Vertex grid, x-major, z fastest
 *      (toolkit::index3d, include/toolkit.h:29-34); the CRE grid has the
 *      energy index fastest, ((i*ny+j)*nz+k)*nE+e (source/field/cre/cre.cc:202-227). */
typedef struct {
  uint32_t nx, ny, nz, nE;
  double x_min, x_max, y_min, y_max, z_min, z_max;
  double E_min, E_max, E_fact; /* CRE only */
} hxg_grid_desc_t;

/* ---- one frequency pass: Param::grid_obs (include/param.h:87-117) ----- */
typedef struct {
  double observer[3];                          /* cm                        */
  double gc_r_min, gc_r_max, gc_z_min, gc_z_max; /* cm; spherical |pos| and z */
  double oc_r_res;                             /* cm                        */
  uint32_t total_shell;
  uint32_t nside_shell[HXG_MAX_SHELLS];
  double radii_shell[HXG_MAX_SHELLS + 1];      /* cm, total_shell+1 entries */
  int32_t do_dm, do_fd, do_sync, do_mask;
  uint32_t nside_dm, nside_fd, nside_sync, _pad;
  double sync_freq;                            /* Hz (sim_sync_freq.back()) */
} hxg_obs_t;

typedef struct hxg_handle hxg_handle;

/* ---- library --------------------------------------------------------- */
/* ABI version of the loaded library (HXG_ABI_VERSION at build time).      */
int hxg_abi_version(void);
/* Number of CUDA devices the library can see (0 without a GPU).           */
int hxg_device_count(void);

/* ---- handle lifecycle ------------------------------------------------
 * Replaces the construction of Integrator + the upload of the Grid_*
 * arrays that the reference reads in place (source/pipeline/pipeline.cc:23-30,
 * 165-190).  precision is HXG_FP64 or HXG_FP32C.                         */
int hxg_create(int device, int precision, hxg_handle **out);
int hxg_destroy(hxg_handle *h);
const char *hxg_last_error(const hxg_handle *h);
/* Launch on this CUDA stream (cudaStream_t passed as void*; NULL = the
 * handle's own stream).  Work the handle queued on its previous stream is
 * ordered before its later work on the new one (an event wait); the
 * previous stream must still exist when this is called.                   */
int hxg_set_stream(hxg_handle *h, void *stream);

/* ---- field models: replaces Pipeline::assemble_breg/tereg/cre model
 *      selection (source/pipeline/pipeline.cc:33-84, 145-162).            */
int hxg_set_models(hxg_handle *h, const hxg_models_t *m);

/* ---- grids: the Grid_* SoA arrays (include/grid.h:63,94,117,144,167).
 * field = HXG_FIELD_*; c0,c1,c2 = bx,by,bz for B slots, c0 = te for n_e
 * slots, c0 = cre_flux for the CRE slot (c1,c2 ignored).  Host FP64; the
 * library keeps its own device copy (FP64 and/or FP32 per precision).
 * 2 to 2^19 vertices per axis and at most 2^32 - 1 in all
 * (HXG_ERR_INVALID otherwise).                                            */
int hxg_upload_grid(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                    const double *c0, const double *c1, const double *c2);
/* Same, from host FP32 arrays (no counterpart in the reference, whose grids
 * are FP64): the values are widened to FP64 on the device (exactly), so the
 * slot and every map equal those of hxg_upload_grid with the same values as
 * FP64, for half the host-to-device bytes.  The copies and the widening
 * run after the work already queued on the handle's stream, on a stream of
 * the device's greatest priority (so an integration running on another
 * handle's stream does not hold up the widening), and the handle's stream
 * waits for them.  Synchronous: returns when the slot holds the values.   */
int hxg_upload_grid_f32(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                        const float *c0, const float *c1, const float *c2);
/* Load a grid straight from the reference's binary grid file
 * (Grid_*::import_grid, source/grid/grid_breg.cc:48-66 and its tereg /
 * brnd / ternd / cre twins): raw native-endian FP64, the B slots with
 * (bx, by, bz) interleaved per voxel, x-major with z fastest; the CRE slot
 * nx*ny*nz*nE values with the energy fastest.  The file is read in large
 * chunks into pinned host buffers, copied while the next chunk is read, and
 * split into components on the device.  A file whose size does not match
 * the descriptor is rejected (HXG_ERR_INVALID).  Synchronous.              */
int hxg_upload_grid_file(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                         const char *path);
/* Same, from device-resident FP64 SoA arrays (no host copy).              */
int hxg_upload_grid_device(hxg_handle *h, int field, const hxg_grid_desc_t *g,
                           const double *d_c0, const double *d_c1,
                           const double *d_c2);
/* Copy a slot's FP64 SoA arrays (c0,c1,c2 as in hxg_upload_grid; c1,c2
 * ignored for scalar slots) back to host memory: the Grid_* member arrays
 * the reference holds (include/grid.h:63,94,117,144,167).  Synchronous.  */
int hxg_download_grid(hxg_handle *h, int field, double *c0, double *c1, double *c2);
/* Write a slot in the reference's binary grid format: Grid_*::export_grid
 * (source/grid/grid_brnd.cc:57-73 and its breg / tereg / ternd / cre twins;
 * the B slots with (bx, by, bz) interleaved per voxel).  Interleaved on the
 * device, written from pinned double buffers.  Synchronous.               */
int hxg_export_grid_file(hxg_handle *h, int field, const char *path);

/* ---- random-field generators: fill a grid slot on the device, as the
 * reference's Pipeline::assemble_brnd / assemble_ternd do with
 * build_permission (source/pipeline/pipeline.cc:87-140).  The slot is then
 * read like an uploaded grid.  FFTs are cuFFT double-complex transforms;
 * the Gaussian deviates of k-space cell c (x-major index, z fastest) are
 * Philox4x32-10 keyed by seed with counter {c, c >> 32, b, 0x52464721}
 * (b = 0, 1), through Box-Muller, so a field depends on the seed alone.
 * The k-space workspace (16 bytes per cell, 32 for Brnd_es) and the FFT
 * plan stay on the handle for the next call of the same grid shape;
 * hxg_destroy releases them.
 * seed 0 draws a seed from the clock, as toolkit::random_seed(0) does
 * (include/toolkit.h:122-140).  observer = Param::observer (cm), used by
 * the spatial profile.  Synchronous.
 *
 * Brnd_es::write_grid (source/field/b/brnd_es.cc:76-308) into the BRND
 * slot: the anisotropy direction is the regular field of the handle's
 * models (hxg_set_models first): HXG_BREG_GRID reads the uploaded BREG
 * slot trilinearly (breg.cc:28-97), analytic models are evaluated.       */
int hxg_generate_brnd_es(hxg_handle *h, const hxg_grid_desc_t *g, const hxg_brnd_es_t *p,
                         const double observer[3], uint64_t seed);
/* TErnd_dft::write_grid (source/field/te/ternd_dft.cc:35-128) into the
 * TERND slot.                                                               */
int hxg_generate_ternd_dft(hxg_handle *h, const hxg_grid_desc_t *g,
                           const hxg_ternd_dft_t *p, const double observer[3],
                           uint64_t seed);

/* ---- mask: Grid_obs::mask_map (source/grid/grid_obs.cc:44-50) and its
 * per-shell Hampisk::duplicate (include/hamsk.h:55-103).  A pixel is
 * integrated iff its duplicated mask value == 1.0 (integrator.cc:69-70).
 * mask == NULL clears it.                                                 */
int hxg_set_mask(hxg_handle *h, uint32_t nside, const double *mask);

/* ---- the integrator: Integrator::write_grid (integrator.cc:23-134) -----
 * Outputs are the Grid_obs maps after the shell loop, before
 * Grid_obs::export_grid's unit rescale: dm at nside_dm, fd at nside_fd,
 * is/qs/us at nside_sync.  Pointers for observables not requested by obs
 * may be NULL.  Host buffers; the call synchronises its stream.  A shell
 * may have up to 2^30 radial steps (HXG_ERR_INVALID beyond).              */
int hxg_write_grid(hxg_handle *h, const hxg_obs_t *obs, double *dm,
                   double *fd, double *is, double *qs, double *us);
/* Same with device output buffers; asynchronous on the handle's stream.   */
int hxg_write_grid_device(hxg_handle *h, const hxg_obs_t *obs, double *d_dm,
                          double *d_fd, double *d_is, double *d_qs,
                          double *d_us);
/* Wait for the handle's stream; returns the first asynchronous error.     */
int hxg_sync(hxg_handle *h);

/* ---- several frequency passes at once -------------------------------------
 * Pipeline::assemble_obs runs write_grid once per <sync> frequency
 * (source/pipeline/pipeline.cc:165-190), each pass sampling the same rays
 * at the same positions.  hxg_write_grid_multi takes the npass passes in
 * that order (obs[k], outputs d_outs[5k .. 5k+4] = dm, fd, is, qs, us of
 * pass k, as for hxg_write_grid_device) and, in the FP32C form, runs up to
 * three consecutive passes that share observer, shells, radial step, limits
 * and mask switch, all with synchrotron output and no CRE grid, in one
 * traversal per shell: positions, field samples, emissivity weights, DM and
 * FD once, then each pass's Faraday phase (with the inner-shell FD only for
 * passes that request FD, as write_grid does) and I/Q/U sums.  Every map
 * equals the one hxg_write_grid_device gives for that pass alone, to the
 * FP32C tolerance.  Other passes run one by one.  Asynchronous on the
 * handle's stream.  No counterpart in the reference.                       */
int hxg_write_grid_multi(hxg_handle *h, int npass, const hxg_obs_t *obs,
                         double *const *d_outs);
/* Same with host output buffers (outs[5k..5k+4] of pass k, NULL where the
 * pass writes no such map); synchronous.                                 */
int hxg_write_grid_multi_host(hxg_handle *h, int npass, const hxg_obs_t *obs,
                              double *const *outs);

/* ---- one shell at a time, over a shard of its pixels ---------------------
 * The two halves of one iteration of write_grid's shell loop
 * (integrator.cc:56-133), for callers that split a pass across GPUs: the
 * pixels of a shell are independent, and the only exchange is the
 * accumulated FD map, which the next shell reads for its inner-shell Faraday
 * depth (integrator.cc:78-86).
 *
 * hxg_shell_integrate_device: radial integration of shell `shell` for the
 * pixels of shard `shard` of `nshards` (NESTED blocks b of 2^k pixels with
 * b mod nshards == shard, 32 <= 2^k <= 2048 and at least 8 blocks per shard
 * where the shell allows: compact sky patches, interleaved so that every
 * shard gets the same mix of ray lengths) into the caller's shell maps at
 * nside_shell[shell] (RING; d_tmp_fd is written whenever FD or sync is on).
 * With nshards > 1 the maps are zero outside the shard, so the shard maps of
 * all shards add up to the shell's maps.  d_fd = the accumulated FD output
 * of the inner shells, complete over all pixels (read when obs->do_fd).
 * hxg_shell_merge_device: Hampix::accumulate of the shell maps into the
 * pass outputs (integrator.cc:121-132); the caller zeroes the outputs before
 * shell 0.  A pass split this way over shards: for each shell, integrate,
 * sum the shell FD maps over the shards, merge; at the end sum the DM, I, Q,
 * U outputs over the shards.  Both calls are asynchronous on the handle's
 * stream.  No counterpart in the reference (its shell loop is internal).  */
int hxg_shell_integrate_device(hxg_handle *h, const hxg_obs_t *obs, uint32_t shell,
                               uint32_t shard, uint32_t nshards, const double *d_fd,
                               double *d_tmp_dm, double *d_tmp_fd, double *d_tmp_is,
                               double *d_tmp_qs, double *d_tmp_us);
/* The same for npass = 2 or 3 passes that hxg_write_grid_multi would fuse
 * (else HXG_ERR_UNSUPPORTED): one traversal of the shard into the shared
 * shell DM / FD maps and the per-pass I, Q, U shell maps d_tmp_iqu[3k ..
 * 3k+2]; each pass then merges with hxg_shell_merge_device (the DM / FD
 * shell maps are the same for every pass that requests them).            */
int hxg_shell_integrate_multi_device(hxg_handle *h, int npass, const hxg_obs_t *obs,
                                     uint32_t shell, uint32_t shard, uint32_t nshards,
                                     const double *d_fd, double *d_tmp_dm, double *d_tmp_fd,
                                     double *const *d_tmp_iqu);
int hxg_shell_merge_device(hxg_handle *h, const hxg_obs_t *obs, uint32_t shell,
                           const double *d_tmp_dm, const double *d_tmp_fd,
                           const double *d_tmp_is, const double *d_tmp_qs,
                           const double *d_tmp_us, double *d_dm, double *d_fd,
                           double *d_is, double *d_qs, double *d_us);

/* ---- adjoint (gradients of a scalar loss of the maps) -------------------
 * Reverse mode of hxg_write_grid_device, in the handle's form.  With
 * checkpointing on, every forward call stores per shell the chunk Faraday
 * depths and Q, U partial sums and the inner-shell Faraday depth of each
 * pixel; the adjoint then runs one backward sweep per shell, outer shells
 * first.  The FP64 form covers every model the forward does except the
 * CRE grid; the FP32C form (FP32 fields and emissivity, FP64 Faraday path,
 * agreeing with the FP64 gradient to about 1e-5) covers the grid
 * workloads' models -- spiral or no regular B, exponential disk or no
 * regular n_e, CRE_ana with a constant index, gc_r_min = 0 -- and returns
 * HXG_ERR_UNSUPPORTED for others.
 *
 * Inputs: dL/d(output maps) on the device (same sizes as the forward's
 * outputs; NULL = zero).  Outputs (device, overwritten, NULL = skip):
 *   d_grad_params[HXG_NUM_PARAMS]: dL/d(parameter) in the order below, for
 *     the spiral B model, the exponential n_e disk and the CRE j0 (zero for
 *     the parameters of models that are not active);
 *   d_grad_bx/by/bz: dL/d(B grid value) per voxel of the gridded B slot(s);
 *   d_grad_ne: dL/d(n_e grid value) per voxel of the gridded n_e slot(s).
 * One grid geometry at most.                                              */
enum {
  HXG_PARAM_SPIRAL_B0 = 0,
  HXG_PARAM_SPIRAL_PITCH = 1,
  HXG_PARAM_SPIRAL_R = 2,
  HXG_PARAM_SPIRAL_H = 3,
  HXG_PARAM_EXPDISK_N0 = 4,
  HXG_PARAM_EXPDISK_R = 5,
  HXG_PARAM_EXPDISK_H = 6,
  HXG_PARAM_CRE_J0 = 7,
  HXG_NUM_PARAMS = 8
};
int hxg_set_checkpointing(hxg_handle *h, int enable);
int hxg_adjoint_device(hxg_handle *h, const hxg_obs_t *obs,
                       const double *g_dm, const double *g_fd,
                       const double *g_is, const double *g_qs,
                       const double *g_us, double *d_grad_params,
                       double *d_grad_bx, double *d_grad_by,
                       double *d_grad_bz, double *d_grad_ne);

/* ---- sharded adjoint (the multi-GPU form of the above) -------------------
 * No counterpart in the reference.  One rank's part of the reverse pass
 * of a pass whose forward ran shell by shell on shard `shard` of `nshards`
 * (hxg_shell_integrate_device with checkpointing on, every shell, the
 * same obs and models).  The ranks exchange what the unsharded adjoint
 * keeps in one map: dL/d(accumulated FD map), which every pixel of the
 * inner shells reads.
 *  - hxg_adjoint_shard_begin: checks the checkpoints and zeroes the
 *    gradient accumulators.
 *  - hxg_adjoint_shard_shell, shells from the outermost to the innermost:
 *    g_dm / g_is / g_qs / g_us as in hxg_adjoint_device; g_fdmap = the
 *    complete dL/d(FD output) including the inner-FD terms of all outer
 *    shells (the same on every rank; start from dL/d(FD output));
 *    d_gfd_inc (npix(nside_fd) doubles) receives this shard's inner-FD
 *    terms of this shell.  Before the next shell the caller sums d_gfd_inc
 *    over the ranks and adds it to g_fdmap.  FD passes need both maps.
 *  - hxg_adjoint_shard_finish: this shard's gradients in the outputs of
 *    hxg_adjoint_device; their sum over the ranks is the full gradient.
 * Launches on the handle's stream; finish synchronizes it.                */
int hxg_adjoint_shard_begin(hxg_handle *h, const hxg_obs_t *obs, uint32_t shard,
                            uint32_t nshards);
int hxg_adjoint_shard_shell(hxg_handle *h, const hxg_obs_t *obs, uint32_t shell,
                            const double *g_dm, const double *g_fdmap, const double *g_is,
                            const double *g_qs, const double *g_us, double *d_gfd_inc);
int hxg_adjoint_shard_finish(hxg_handle *h, double *d_grad_params, double *d_grad_bx,
                             double *d_grad_by, double *d_grad_bz, double *d_grad_ne);

/* ---- batched forward ---------------------------------------------------
 * Many independent passes -- parameter sets x frequencies, each one
 * Integrator::write_grid call (source/integrator/integrator.cc:23-134)
 * with its own models and hxg_obs_t -- planned once and run as one CUDA
 * graph.  The reference has no batch entry point; a caller loops over
 * Pipeline runs (source/pipeline/pipeline.cc:165-190).
 *
 *  - every entry shares the handle's grids and precision, and its models
 *    must read the same fields from grids as the handle's models (the
 *    analytic parameters may differ); masks are not supported;
 *  - outputs are the caller's device maps (RING), distinct per entry;
 *  - the plan holds per-entry shell temporaries and launch blocks and a
 *    graph with, per shell level, one persistent shell kernel over all
 *    entries (warps take pixel tiles from a work counter) and one kernel
 *    that merges the shell maps into the outputs; an entry's outer shells
 *    read the Faraday depth its inner shells accumulated, as in
 *    write_grid;
 *  - in the FP32C form, up to three consecutive entries with the same
 *    models and geometry and synchrotron output (one parameter set at
 *    several frequencies, as hxg_write_grid_multi takes them; no CRE grid)
 *    share one traversal per shell;
 *  - tune != 0: the launch shapes (lanes per pixel x tiles per fetch) are
 *    timed once in hxg_batch_create and the fastest is kept;
 *  - hxg_batch_run launches the graph on the handle's stream and does not
 *    synchronise; the entries' host data are not read again;
 *  - grids uploaded to the handle after hxg_batch_create with the same
 *    geometries are used by the next run; if the handle's grids change
 *    geometry or fields, hxg_batch_run returns HXG_ERR_STATE.            */
typedef struct {
  hxg_models_t models;
  hxg_obs_t obs;
  double *d_dm, *d_fd, *d_is, *d_qs, *d_us;
} hxg_batch_entry_t;
typedef struct hxg_batch hxg_batch;
int hxg_batch_create(hxg_handle *h, int n, const hxg_batch_entry_t *entries,
                     int tune, hxg_batch **out);
int hxg_batch_run(hxg_batch *b);
/* Launch shape in use (lanes per pixel, tiles per fetch), the number of
 * shapes timed and the best graph time (ms; 0 without tuning), and the
 * LOS samples one run covers.                                             */
int hxg_batch_info(const hxg_batch *b, int *lanes_per_pixel, int *grain,
                   int *tried, double *best_ms, int64_t *samples);
int hxg_batch_destroy(hxg_batch *b);

/* ---- timing of the integration kernels ------------------------------
 * enable != 0: every shell-integration launch is bracketed by CUDA events
 * on the launching stream.  hxg_get_timing returns the summed device time
 * (ms), the number of launches and the number of LOS samples they covered
 * since the last reset.                                                   */
int hxg_set_timing(hxg_handle *h, int enable);
int hxg_get_timing(hxg_handle *h, double *kernel_ms, int64_t *launches,
                   int64_t *samples);
/* Total number of kernels this handle has launched (all kinds).          */
int hxg_get_launch_count(hxg_handle *h, int64_t *count);

/* ---- interpolation tables of the shell merges -------------------------
 * No counterpart in the reference (Hampix::accumulate, hamdis.h:698-721,
 * finds the interpolation weights of every output pixel on every call).  A
 * shell map merged into an output of another Nside is interpolated at each
 * output pixel; the handle keeps the 4 source pixels and weights of every
 * output pixel per pair of Nsides (48 bytes per output pixel: 604 MB for
 * Nside 1024), made on first use and held until hxg_destroy.  bytes bounds
 * their total (default 8 GiB); pairs beyond it, or all of them when bytes
 * is 0, find the weights in place.  The maps are the same either way.
 * Lowering the bound frees no table already made.                        */
int hxg_set_interp_cache(hxg_handle *h, uint64_t bytes);

/* ---- allocation-free integration ---------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate
 * device memory -- plugins whose host application owns every device
 * allocation through its own pool, pipelines whose memory is fixed at
 * start-up and must not touch the allocator afterwards -- this entry
 * point runs the FP64 integrator without any cudaMalloc/cudaFree.  Inputs
 * and outputs are the caller's device buffers; the only scratch (the
 * per-shell HEALPix maps) is a fixed static device array of
 * 5 x 12 x HXG_NOALLOC_MAX_NSIDE^2 doubles (7.5 MiB) that every GPU loading
 * the library holds until exit.
 *
 *  - grid / d_records: one packed grid of FP64 voxel records
 *    {bx, by, bz, ne} (32 B per voxel, x-major, z fastest), holding the sum
 *    of all gridded B slots and of all gridded n_e slots the models read;
 *    NULL when the models read no grid.
 *  - shells larger than HXG_NOALLOC_MAX_NSIDE return HXG_ERR_TOO_LARGE;
 *    masks (do_mask) return HXG_ERR_UNSUPPORTED.
 *  - work is queued on `stream` (cudaStream_t; NULL = legacy default) of
 *    the current device; the call does not synchronise.
 *  - the first call in a CUDA context (per device, for runtime-API
 *    callers: its primary context) looks the scratch address up there
 *    (cudaGetSymbolAddress); make that first call before any stream
 *    capture.  A device reset (cudaDeviceReset) makes a new context, and
 *    the next call looks the address up again; a failed lookup is retried
 *    on the next call.
 *  - an error already pending in the CUDA runtime (cudaPeekAtLastError)
 *    makes the call return HXG_ERR_CUDA before it queues any work; when
 *    the call returns HXG_ERR_CUDA the outputs are undefined.
 *  - all calls share the scratch and it keeps the last call's contents;
 *    calls whose GPU work overlaps (other streams, other threads) race on
 *    it, so serialise them.                                                */
#define HXG_NOALLOC_MAX_NSIDE 128
int hxg_write_grid_noalloc(const hxg_obs_t *obs, const hxg_models_t *models,
                           const hxg_grid_desc_t *grid,
                           const double *d_records, double *d_dm,
                           double *d_fd, double *d_is, double *d_qs,
                           double *d_us, void *stream);

/* ---- host helpers ------------------------------------------------------*/
/* The synchrotron functions the CRE-grid emissivity integrates
 * (gsl_sf_synchrotron_1 / _2 at integrator.cc:320, 396): which = 1:
 * F(x) = x Int_x^inf K_{5/3}(t) dt, which = 2: G(x) = x K_{2/3}(x), from the
 * same tables and interpolation the device uses; 0 for x <= 0.            */
int hxg_synchrotron(int which, uint64_t n, const double *x, double *out);
/* Integrator::assemble_shell_ref (integrator.cc:231-254): step count,
 * radial step and start distance of shell `shell`.                        */
int hxg_shell_ref(const hxg_obs_t *obs, uint32_t shell, double *d_start,
                  double *delta_d, uint64_t *step);
/* Hampisk::duplicate (include/hamsk.h:55-103): mask at pivot nside ->
 * mask at nside (OR-downgrade / replicate-upgrade).                       */
int hxg_mask_duplicate(uint32_t pivot_nside, const double *pivot_mask,
                       uint32_t nside, double *out);

/* ---- device known-answer helpers (run the kernels' own device code) ---*/
/* Hampix fillpoint = HEALPix RING pix2ang (include/hamdis.h:302-356).     */
int hxg_pix2ang(uint32_t nside, uint64_t npix, double *theta, double *phi);
/* Hampix::interpolate (include/hamdis.h:609-696) of a RING map.          */
int hxg_interpolate(uint32_t nside, const double *map, uint64_t n,
                    const double *theta, const double *phi, double *out);
/* Hampix::accumulate (include/hamdis.h:698-721): dst += src.              */
int hxg_accumulate(uint32_t nside_dst, double *dst, uint32_t nside_src,
                   const double *src);
/* los_versor, los_parproj, los_perproj (integrator.h:35-49,
 * integrator.cc:268-272) and cos/sin(2*sync_ipa) (integrator.cc:257-265)
 * for n directions/fields; b is 3n doubles, versor 3n doubles.            */
int hxg_los_geometry(uint64_t n, const double *theta, const double *phi,
                     const double *b, double *versor, double *b_par,
                     double *b_per, double *cos2ipa, double *sin2ipa);
/* Trilinear read of an uploaded grid slot at n positions (3n doubles, cm):
 * Breg/Brnd::read_grid (breg.cc:28-97, brnd.cc:25-88), TEreg/TErnd::read_grid
 * (tereg.cc:27-74, ternd.cc:21-71).  out gets 3n (B) or n (n_e) doubles.  */
int hxg_read_grid(hxg_handle *h, int field, uint64_t n, const double *pos,
                  double *out);

#ifdef __cplusplus
}
#endif
#endif /* HXG_H */
