/* oracle shim (test infrastructure): see hx_gsl_impl.h */
#include "hx_gsl_impl.h"
