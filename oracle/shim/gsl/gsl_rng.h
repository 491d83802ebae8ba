/* GSL stand-in used only to compile reference programs into oracle/_ref/.
 * The estimator (barbie.c, funcs.c, calpow_mom.c) includes this header but
 * links no GSL symbol. The field generator (ngrf_2d_funcs.c:356-360,509) uses
 * the functions below; oracle/gsl_shim.c implements them over the
 * counter-based normal stream of oracle/philox_normal.h (GSL itself is not
 * available). gsl_rng_cmrg is only named by the 2D generator
 * (ngrf_2d_funcs.c:605), which the 3D program never calls. */
#ifndef BEAM_GSL_RNG_SHIM_H
#define BEAM_GSL_RNG_SHIM_H
typedef struct beam_shim_rng_type gsl_rng_type;
typedef struct beam_shim_rng gsl_rng;
extern const gsl_rng_type *gsl_rng_mt19937;
extern const gsl_rng_type *gsl_rng_cmrg;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(gsl_rng *r, unsigned long int s);
void gsl_rng_free(gsl_rng *r);
#endif
