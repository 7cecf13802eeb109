/* Stand-in for GSL's gsl_randist.h (see gsl_rng.h). */
#ifndef HXO_SHIM_GSL_RANDIST_H
#define HXO_SHIM_GSL_RANDIST_H
#include <gsl/gsl_rng.h>
double gsl_ran_ugaussian(const gsl_rng *r);
#endif
