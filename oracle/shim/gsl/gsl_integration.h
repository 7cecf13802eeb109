/* Stand-in for GSL's gsl_integration.h: included by the random-field
 * generators, which call none of its functions. */
#ifndef HXO_SHIM_GSL_INTEGRATION_H
#define HXO_SHIM_GSL_INTEGRATION_H
#endif
