/* Declarations of the GSL random-number entry points the hammurabiX
 * objects linked into the drop-in call (Brnd_jf12, Brnd_mhd), for builds
 * where GSL is not installed; GSL's public API with C linkage.  The
 * generator type is opaque here.  extern_stubs.cc makes gsl_rng_alloc
 * throw: the generators that draw from GSL are not replaced on the B200
 * build.  With GSL installed, build against its headers and library. */
#ifndef HXG_DROPIN_GSL_RNG_H
#define HXG_DROPIN_GSL_RNG_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct hxg_dropin_gsl_rng_s gsl_rng;
typedef struct hxg_dropin_gsl_rng_type_s gsl_rng_type;
extern const gsl_rng_type *gsl_rng_taus;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long int seed);
void gsl_rng_free(gsl_rng *r);
double gsl_rng_uniform(const gsl_rng *r);
#ifdef __cplusplus
}
#endif
#endif
