/* Stand-in for GSL's gsl_sf_gamma.h (GSL is not installed here).
 * gsl_sf_gamma(x) is the Gamma function; std::tgamma computes the same
 * function to within a few ulp, far inside the oracle's 1e-10 tolerance. */
#ifndef HXO_SHIM_GSL_SF_GAMMA_H
#define HXO_SHIM_GSL_SF_GAMMA_H
#include <cmath>
inline double gsl_sf_gamma(const double x) { return std::tgamma(x); }
#endif
