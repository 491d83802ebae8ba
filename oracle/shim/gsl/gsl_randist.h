/* GSL stand-in (see gsl_rng.h): the Gaussian deviates the field generators
 * draw (ngrf_2d_funcs.c:376 and on), here draw n of the Philox normal stream. */
#ifndef BEAM_GSL_RANDIST_SHIM_H
#define BEAM_GSL_RANDIST_SHIM_H
#include <gsl/gsl_rng.h>
double gsl_ran_gaussian_ziggurat(gsl_rng *r, double sigma);
double gsl_ran_gaussian(gsl_rng *r, double sigma);
#endif
