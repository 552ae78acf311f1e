/* Test infrastructure: forwards to the oracle harness's GSL interface subset. */
#include "gsl_shim_all.h"
