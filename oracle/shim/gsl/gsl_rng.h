/* Stand-in for GSL's gsl_rng.h.  Only the random-field generators use it.
 * GSL's taus stream is not reproduced: by default the generator is
 * splitmix64; with hxo_shim_cell_stream(k) > 0 the Gaussian deviates are the
 * cell-indexed Philox4x32-10 / Box-Muller deviates of the device generators
 * (see shim.cc), so that a single-threaded reference generator run consumes
 * exactly the deviates the device uses for each k-space cell. */
#ifndef HXO_SHIM_GSL_RNG_H
#define HXO_SHIM_GSL_RNG_H
typedef struct {
  unsigned long long state;
  unsigned long long seed, draws;
  int cells; /* deviates per k-space cell in cell-stream mode, 0 = off */
} gsl_rng;
typedef struct { int id; } gsl_rng_type;
extern const gsl_rng_type *gsl_rng_taus;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
void gsl_rng_free(gsl_rng *r);
double gsl_rng_uniform(const gsl_rng *r);
/* k deviates per k-space cell (4 for Brnd_es, 2 for TErnd_dft) for every
 * generator seeded from now on; 0 = off, then the environment variable
 * HXO_SHIM_CELL_STREAM decides: "k" for all, or "k0,k1,..." for the 1st,
 * 2nd, ... gsl_rng_set call of the process (the last value repeats). */
extern "C" void hxo_shim_cell_stream(int k);
#endif
