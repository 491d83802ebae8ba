/* FFTW-API shim over the oracle DFT (oracle/fft.c); see oracle/shim/fftw3.h.
 * Only complex 2D plans are supported, which is all the reference estimator
 * creates (funcs.c:349,546). Test infrastructure only. */
#include <stdlib.h>
#include <string.h>

#include "fft.h"
#include "shim/fftw3.h"

/* thread count requested through fftw_plan_with_nthreads (barbie.c:152 asks for 4) */
static int shim_threads = 1;

struct beam_shim_plan {
  int n0, n1, sign;
  fftw_complex *in, *out;
};

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
  return p;
}

void fftw_execute(const fftw_plan p) {
  if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)p->n0 * (size_t)p->n1);
  orc_fft2d_threads(p->n0, p->n1, p->sign, &p->out[0][0], shim_threads);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { shim_threads = nthreads > 0 ? nthreads : 1; }
