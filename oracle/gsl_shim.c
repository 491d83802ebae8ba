/* GSL stand-in for compiling the reference field generator into oracle/_ref/
 * (see oracle/shim/gsl/gsl_rng.h). Test infrastructure only.
 *
 * gsl_rng_set(r, s) starts the stream with seed s at draw 0, and each
 * gsl_ran_gaussian_ziggurat(r, sigma) returns sigma * orc_normal(s, n) for the
 * next draw n. The generator's mode order is untouched, so draw n lands on the
 * same mode as in the reference; only the deviates differ from GSL's
 * MT19937 + ziggurat stream. */
#include <stdint.h>
#include <stdlib.h>

#include "philox_normal.h"
#include "shim/gsl/gsl_randist.h"

struct beam_shim_rng_type {
  int unused;
};
struct beam_shim_rng {
  uint64_t seed, n;
};

static const struct beam_shim_rng_type mt19937_stand_in = {0};
const gsl_rng_type *gsl_rng_mt19937 = &mt19937_stand_in;
const gsl_rng_type *gsl_rng_cmrg = &mt19937_stand_in;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
  (void)T;
  return (gsl_rng *)calloc(1, sizeof(gsl_rng));
}

void gsl_rng_set(gsl_rng *r, unsigned long int s) {
  r->seed = s;
  r->n = 0;
}

void gsl_rng_free(gsl_rng *r) { free(r); }

double gsl_ran_gaussian_ziggurat(gsl_rng *r, double sigma) { return sigma * orc_normal(r->seed, r->n++); }

double gsl_ran_gaussian(gsl_rng *r, double sigma) { return gsl_ran_gaussian_ziggurat(r, sigma); }
