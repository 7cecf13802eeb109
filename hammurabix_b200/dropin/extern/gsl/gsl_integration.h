/* Included by Brnd_jf12, which calls none of its functions. */
#ifndef HXG_DROPIN_GSL_INTEGRATION_H
#define HXG_DROPIN_GSL_INTEGRATION_H
#endif
