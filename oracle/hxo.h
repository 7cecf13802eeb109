/*
 * hxo.h -- CPU oracle for the line-of-sight integrator.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of
 * hammurabiX's Integrator::write_grid path, used by tests/ (as the checker)
 * and by bench.py's CPU-baseline leg.  Nothing in the hammurabix_b200
 * product links, loads or calls it.
 */
#ifndef HXO_H
#define HXO_H

#include <stdint.h>

#include "../include/hxg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One grid slot: geometry + host SoA arrays (NULL when absent). */
typedef struct {
  hxg_grid_desc_t desc;
  const double *c[3];
} hxo_grid_t;

typedef struct {
  hxo_grid_t slot[5]; /* indexed by HXG_FIELD_* */
} hxo_grids_t;

int hxo_write_grid(const hxg_obs_t *obs, const hxg_models_t *m,
                   const hxo_grids_t *grids, uint32_t mask_nside,
                   const double *mask, double *dm, double *fd, double *is,
                   double *qs, double *us);

int hxo_shell_ref(const hxg_obs_t *obs, uint32_t shell, double *d_start,
                  double *delta_d, uint64_t *step);
void hxo_pix2ang(uint32_t nside, uint64_t npix, double *theta, double *phi);
void hxo_interpolate(uint32_t nside, const double *map, uint64_t n,
                     const double *theta, const double *phi, double *out);
void hxo_accumulate(uint32_t nside_dst, double *dst, uint32_t nside_src,
                    const double *src);
int hxo_mask_duplicate(uint32_t pivot_nside, const double *pivot_mask,
                       uint32_t nside, double *out);
void hxo_los_geometry(uint64_t n, const double *theta, const double *phi,
                      const double *b, double *versor, double *b_par,
                      double *b_per, double *ipa);
int hxo_read_grid(const hxo_grid_t *g, int ncomp, uint64_t n,
                  const double *pos, double *out);
double hxo_temp_convert(double temp_br, double freq);
/* analytic synchrotron emissivities J_tot, J_pol at pos for |B_perp| */
void hxo_sync_emissivity(const hxg_models_t *m, const double obs[3],
                         double freq, const double pos[3], double b_per,
                         double *jt, double *jp);
/* regular-field / electron-density model evaluation (write_field) */
void hxo_breg_field(const hxg_models_t *m, const double obs[3],
                    const double pos[3], double out[3]);
double hxo_tereg_field(const hxg_models_t *m, const double obs[3],
                       const double pos[3]);

#ifdef __cplusplus
}
#endif
#endif
