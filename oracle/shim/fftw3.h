/* FFTW-API shim header used only to compile the reference programs
 * (barbie.c + funcs.c, calpow_mom.c, generate_field.c + ngrf_2d_funcs.c of
 * sukhdeepsinghgill/BARBIE) into oracle/_ref/ for parity checks. FFTW itself is
 * not installed here. The estimator uses five of its symbols
 * (fftw_plan_dft_2d, fftw_execute, fftw_destroy_plan, fftw_init_threads,
 * fftw_plan_with_nthreads) and the field generator two more
 * (fftw_plan_dft_r2c_3d, fftw_plan_dft_c2r_3d); oracle/fftw_shim.c provides
 * them on top of the oracle's own DFT (oracle/fft.c).
 *
 * It also defines beam_ref_env_long(), which the build recipe substitutes for
 * the reference's hard-coded plane/ring counts (barbie.c:71-72) so that one
 * binary serves every configuration. */
#ifndef BEAM_FFTW_SHIM_H
#define BEAM_FFTW_SHIM_H
#include <stdlib.h>

typedef double fftw_complex[2];
typedef struct beam_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);

static inline long beam_ref_env_long(const char *name, long fallback) {
  const char *v = getenv(name);
  return (v && *v) ? strtol(v, NULL, 10) : fallback;
}
#endif
