/*
 * The configure results of the reference's double-precision build
 * (configure.ac:255-281 fills config/LSMLIB_config.h.in with these), so that
 * its fast-marching sources compile on their own for the checkers in
 * oracle/_ref.
 */
#ifndef included_LSMLIB_config_h
#define included_LSMLIB_config_h

#include <float.h>

#define LSMLIB_DOUBLE_PRECISION 1
#define LSMLIB_REAL double
#define LSMLIB_ZERO_TOL 1.e-11
#define LSMLIB_REAL_MAX DBL_MAX
#define LSMLIB_REAL_MIN DBL_MIN
#define LSMLIB_REAL_EPSILON DBL_EPSILON

#endif
