/* GSL's gsl_ran_ugaussian, for builds without GSL (see gsl_rng.h). */
#ifndef HXG_DROPIN_GSL_RANDIST_H
#define HXG_DROPIN_GSL_RANDIST_H
#include <gsl/gsl_rng.h>
#ifdef __cplusplus
extern "C" {
#endif
double gsl_ran_ugaussian(const gsl_rng *r);
#ifdef __cplusplus
}
#endif
#endif
