/* FFTW-API shim over the oracle DFT (oracle/fft.c); see oracle/shim/fftw3.h.
 * Complex 2D plans (the estimator, funcs.c:349,546) and real 3D r2c / c2r
 * plans (the field generator, generate_field.c:78-79). Test infrastructure
 * only. */
#include <stdlib.h>
#include <string.h>

#include "fft.h"
#include "shim/fftw3.h"

/* thread count requested through fftw_plan_with_nthreads (barbie.c:152 asks for 4) */
static int shim_threads = 1;

enum { SHIM_DFT_2D, SHIM_R2C_3D, SHIM_C2R_3D };

struct beam_shim_plan {
  int kind, n0, n1, n2, sign;
  void *in, *out;
};

static fftw_plan shim_plan(int kind, int n0, int n1, int n2, int sign, void *in, void *out) {
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  p->kind = kind, p->n0 = n0, p->n1 = n1, p->n2 = n2, p->sign = sign, p->in = in, p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  return shim_plan(SHIM_DFT_2D, n0, n1, 1, sign, in, out);
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
  (void)flags;
  return shim_plan(SHIM_R2C_3D, n0, n1, n2, -1, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags) {
  (void)flags;
  return shim_plan(SHIM_C2R_3D, n0, n1, n2, +1, in, out);
}

/* The real 3D transforms work in place on the padded layout double[n0][n1][n2+2]
 * (2*(n2/2+1) doubles per row); out-of-place plans (unpadded real arrays) go
 * through a padded copy. */
void fftw_execute(const fftw_plan p) {
  if (p->kind == SHIM_DFT_2D) {
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)p->n0 * (size_t)p->n1);
    orc_fft2d_threads(p->n0, p->n1, p->sign, (double *)p->out, shim_threads);
    return;
  }
  const size_t rows = (size_t)p->n0 * p->n1, n2 = (size_t)p->n2, pitch = 2 * (n2 / 2 + 1);
  if (p->kind == SHIM_R2C_3D) {
    double *buf = (double *)p->out;
    if (p->in != p->out)
      for (size_t r = 0; r < rows; ++r) memcpy(buf + r * pitch, (const double *)p->in + r * n2, sizeof(double) * n2);
    orc_r2c_3d(p->n0, p->n1, p->n2, buf);
    return;
  }
  if (p->in == p->out) {
    orc_c2r_3d(p->n0, p->n1, p->n2, (double *)p->out);
    return;
  }
  double *buf = (double *)malloc(sizeof(double) * rows * pitch);
  memcpy(buf, p->in, sizeof(double) * rows * pitch);
  orc_c2r_3d(p->n0, p->n1, p->n2, buf);
  for (size_t r = 0; r < rows; ++r) memcpy((double *)p->out + r * n2, buf + r * pitch, sizeof(double) * n2);
  free(buf);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { shim_threads = nthreads > 0 ? nthreads : 1; }
