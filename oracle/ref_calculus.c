/*
 * Checker shim: the reference's calculus macros (src/toolbox/utilities/
 * lsm_calculus_toolbox.h:41-60, LSM_HEAVISIDE and LSM_DELTA_FUNCTION) as
 * callable functions, compiled from the reference header by `make -C oracle
 * ref` into oracle/_ref/libcalculus.so.  Test infrastructure only.
 */
#define _GNU_SOURCE
#include <math.h>

#include "lsm_calculus_toolbox.h"

double ref_heaviside(double x, double eps) { return LSM_HEAVISIDE(x, eps); }
double ref_delta_function(double x, double eps) { return LSM_DELTA_FUNCTION(x, eps); }
