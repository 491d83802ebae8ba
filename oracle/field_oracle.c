/* Oracle: CPU restatement of the reference's field generator
 * (generate_field.c + ngrf_2d_funcs.c of sukhdeepsinghgill/BARBIE) and of its
 * real-space-to-r2c step. TEST INFRASTRUCTURE ONLY (see beam_oracle.h).
 *
 * Parity is pinned against the reference generator compiled from its own
 * sources (oracle/Makefile, _ref/field_ref) with the FFTW and GSL stand-ins;
 * the normal deviates of both come from oracle/philox_normal.h. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "beam_oracle.h"
#include "fft.h"
#include "philox_normal.h"

/* Pk, ngrf_2d_funcs.c:143-155, with p(k) = 1.0 * k^-2 (ngrf_2d_funcs.c:132-140) */
static double field_pk(double C, long i, long j, long k) {
  const double kx = C * i, ky = C * j, kz = C * k;
  const double kk = sqrt(kx * kx + ky * ky + kz * kz);
  return 1.0 * pow(kk, -2.0);
}

typedef struct {
  uint64_t seed, n;
} orc_stream;

static double draw(orc_stream *s) { return orc_normal(s->seed, s->n++); }

/* Fill_Modes, ngrf_2d_funcs.c:341-510: points, lines, planes and cubes of the
 * half-complex array A[N][N][N/2+1], in the reference's draw order. */
void orc_field_fill_modes(long N, uint64_t seed, double LL, double *Ad) {
  double(*A)[2] = (double(*)[2])Ad;
  const long h = N / 2, NH = N / 2 + 1;
  const double vol = pow(N * LL, 3), volfac = vol / 2., C = 2. * M_PI / (N * LL);
  orc_stream st = {seed, 0};
#define AT(i, j, k) (((long)(i) * N + (long)(j)) * NH + (long)(k))
  /* points, ngrf_2d_funcs.c:364-383 */
  for (long i = 0; i < 2; ++i)
    for (long j = 0; j < 2; ++j)
      for (long k = 0; k < 2; ++k) {
        if (i == 0 && j == 0 && k == 0) {
          A[0][0] = 0.0, A[0][1] = 0.0;
          continue;
        }
        const long x = AT(i * h, j * h, k * h);
        const double amp = sqrt(volfac * field_pk(C, i * h, j * h, k * h));
        A[x][0] = amp * draw(&st);
        A[x][1] = 0.0;
      }
  /* lines, ngrf_2d_funcs.c:387-428 */
  for (long i = 0; i < 2; ++i)
    for (long j = 0; j < 2; ++j) {
      for (long k = 1; k < h; ++k) {
        const double amp = sqrt(volfac * field_pk(C, k, i * h, j * h));
        const long x1 = AT(k, i * h, j * h), x2 = AT(N - k, i * h, j * h);
        A[x1][0] = amp * draw(&st);
        A[x1][1] = amp * draw(&st);
        A[x2][0] = A[x1][0], A[x2][1] = -A[x1][1];
      }
      for (long k = 1; k < h; ++k) {
        const double amp = sqrt(volfac * field_pk(C, i * h, k, j * h));
        const long x1 = AT(i * h, k, j * h), x2 = AT(i * h, N - k, j * h);
        A[x1][0] = amp * draw(&st);
        A[x1][1] = amp * draw(&st);
        A[x2][0] = A[x1][0], A[x2][1] = -A[x1][1];
      }
      for (long k = 1; k < h; ++k) {
        const double amp = sqrt(volfac * field_pk(C, i * h, j * h, k));
        const long x1 = AT(i * h, j * h, k);
        A[x1][0] = amp * draw(&st);
        A[x1][1] = amp * draw(&st);
      }
    }
  /* planes, ngrf_2d_funcs.c:432-481 */
  for (long i = 0; i < 2; ++i)
    for (long m = 0; m < 2; ++m) {
      for (long j = 1; j < h; ++j)
        for (long k = 1; k < h; ++k) {
          const double amp = sqrt(volfac * field_pk(C, i * h, j, k));
          const long x1 = AT(i * h, m ? N - j : j, k);
          A[x1][0] = amp * draw(&st);
          A[x1][1] = amp * draw(&st);
        }
      for (long j = 1; j < h; ++j)
        for (long k = 1; k < h; ++k) {
          const double amp = sqrt(volfac * field_pk(C, j, i * h, k));
          const long x1 = AT(m ? N - j : j, i * h, k);
          A[x1][0] = amp * draw(&st);
          A[x1][1] = amp * draw(&st);
        }
      for (long j = 1; j < h; ++j)
        for (long k = 1; k < h; ++k) {
          const double amp = sqrt(volfac * field_pk(C, j, k, i * h));
          const long x1 = AT(m ? N - j : j, k, i * h), x2 = AT(m ? j : N - j, N - k, i * h);
          A[x1][0] = amp * draw(&st);
          A[x1][1] = amp * draw(&st);
          A[x2][0] = A[x1][0], A[x2][1] = -A[x1][1];
        }
    }
  /* cubes, ngrf_2d_funcs.c:483-505 */
  for (long i = 1; i < h; ++i)
    for (long j = 1; j < h; ++j)
      for (long k = 1; k < h; ++k) {
        const double amp = sqrt(volfac * field_pk(C, i, j, k));
        const long xs[4] = {AT(i, j, k), AT(N - i, j, k), AT(i, N - j, k), AT(N - i, N - j, k)};
        for (int q = 0; q < 4; ++q) {
          A[xs[q]][0] = amp * draw(&st);
          A[xs[q]][1] = amp * draw(&st);
        }
      }
#undef AT
}

/* RSD, ngrf_2d_funcs.c:734-765: Delta(k) *= 1 + beta mu^2, mu = k_z/|k| with
 * the line of sight along the last axis; the k = 0 mode is left alone. */
static void field_rsd(long N, double beta, double *padded) {
  const long NH = N / 2 + 1;
  for (long i = 0; i < N; ++i)
    for (long j = 0; j < N; ++j)
      for (long k = 0; k <= N / 2; ++k) {
        const double ia = (i > N / 2) ? (N - i) : i, ja = (j > N / 2) ? (N - j) : j;
        const double kk = sqrt(1. * (ia * ia + ja * ja + k * k));
        if (i + j + k != 0) {
          const double myu = k / kk;
          double *a = padded + 2 * ((i * N + j) * NH + k);
          a[0] *= (1. + beta * myu * myu);
          a[1] *= (1. + beta * myu * myu);
        }
      }
}

/* Get_Modes, ngrf_2d_funcs.c:534-550: x *= LL^3, then the r2c transform. */
static void field_get_modes(long N, double LL, double *padded) {
  const long pitch = N + 2;
  const double Lcube = pow(LL, 3.);
  for (long ij = 0; ij < N * N; ++ij)
    for (long k = 0; k < N; ++k) padded[ij * pitch + k] = padded[ij * pitch + k] * Lcube;
  orc_r2c_3d(N, N, N, padded);
}

int orc_field_generate(long N, uint64_t seed, double LL, double ff, double beta, double *padded, double *sigma) {
  if (N < 4 || N % 2 || !padded || !(LL > 0)) return -1;
  const long NH = N / 2 + 1, pitch = N + 2;
  const double vol = pow(N * LL, 3);
  orc_field_fill_modes(N, seed, LL, padded);
  /* Make_Image, ngrf_2d_funcs.c:512-531 */
  for (long x = 0; x < 2 * N * N * NH; ++x) padded[x] = padded[x] / (vol);
  orc_c2r_3d(N, N, N, padded);
  /* Non_Gauss, ngrf_2d_funcs.c:553-584 */
  double var = 0.;
  for (long ij = 0; ij < N * N; ++ij)
    for (long k = 0; k < N; ++k) var += pow(padded[ij * pitch + k], 2.);
  var /= (1. * N * N * N);
  for (long ij = 0; ij < N * N; ++ij)
    for (long k = 0; k < N; ++k) padded[ij * pitch + k] += ff * (pow(padded[ij * pitch + k], 2.) - var);
  if (sigma) *sigma = pow(var, 0.5);
  field_get_modes(N, LL, padded);
  field_rsd(N, beta, padded);
  return 0;
}

int orc_field_ingest(long N, double LL, double beta, const double *cube, double *padded) {
  if (N < 4 || N % 2 || !cube || !padded || !(LL > 0)) return -1;
  const long pitch = N + 2;
  for (long ij = 0; ij < N * N; ++ij) {
    memcpy(padded + ij * pitch, cube + ij * N, sizeof(double) * N);
    padded[ij * pitch + N] = padded[ij * pitch + N + 1] = 0.0;
  }
  field_get_modes(N, LL, padded);
  field_rsd(N, beta, padded);
  return 0;
}
