/* Stand-in for GSL's gsl_sf_synchrotron.h.  Written from the published
 * definitions F(x) = x * Int_x^inf K_{5/3}(t) dt and G(x) = x * K_{2/3}(x)
 * (Rybicki & Lightman eq. 6.31c); implementation in shim.cc. */
#ifndef HXO_SHIM_GSL_SF_SYNCHROTRON_H
#define HXO_SHIM_GSL_SF_SYNCHROTRON_H
double gsl_sf_synchrotron_1(const double x);
double gsl_sf_synchrotron_2(const double x);
#endif
