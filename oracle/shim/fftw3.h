/* FFTW-API shim header used only to compile the reference estimator
 * (barbie.c + funcs.c of sukhdeepsinghgill/BARBIE) into oracle/_ref/ for
 * parity checks. FFTW itself is not installed here; the reference uses five of
 * its symbols (fftw_plan_dft_2d, fftw_execute, fftw_destroy_plan,
 * fftw_init_threads, fftw_plan_with_nthreads), which oracle/fftw_shim.c
 * provides on top of the oracle's own DFT (oracle/fft.c).
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
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);

static inline long beam_ref_env_long(const char *name, long fallback) {
  const char *v = getenv(name);
  return (v && *v) ? strtol(v, NULL, 10) : fallback;
}
#endif
