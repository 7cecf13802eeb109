/* Stand-in for GSL's gsl_rng.h.  Only the random-field generators use it;
 * they are outside the integration path and the oracle never runs them.
 * The generator here is splitmix64, not GSL's taus stream. */
#ifndef HXO_SHIM_GSL_RNG_H
#define HXO_SHIM_GSL_RNG_H
typedef struct { unsigned long long state; } gsl_rng;
typedef struct { int id; } gsl_rng_type;
extern const gsl_rng_type *gsl_rng_taus;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
void gsl_rng_free(gsl_rng *r);
double gsl_rng_uniform(const gsl_rng *r);
#endif
