/* CPU FP64 DFTs for the oracle; the definition followed is stated in fft.h.
 * Test infrastructure only: nothing on the GPU product path calls this file. */
#include "fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  long n;      /* transform length */
  double *tw;  /* tw[2j], tw[2j+1] = cos, sin of sign*2*pi*j/n, j in [0,n) */
} orc_table;

static void table_init(orc_table *t, long n, int sign) {
  t->n = n;
  t->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (long j = 0; j < n; ++j) {
    /* reduce j/n into [0,1) exactly in integers before scaling to an angle */
    double a = (double)sign * 2.0 * M_PI * (double)j / (double)n;
    t->tw[2 * j] = cos(a);
    t->tw[2 * j + 1] = sin(a);
  }
}

static void table_free(orc_table *t) { free(t->tw); t->tw = NULL; }

static long pick_radix(long n) {
  if (n % 4 == 0) return 4;
  if (n % 2 == 0) return 2;
  if (n % 3 == 0) return 3;
  for (long p = 5; p * p <= n; p += 2)
    if (n % p == 0) return p;
  return n; /* prime: direct DFT */
}

/* Decimation in time: out[0..n) = DFT_n of in[0], in[is], in[2*is], ...
 * w_n^j is t->tw[j * (t->n / n)] because n divides the table length. */
static void dit(const double *in, long is, double *out, long n, const orc_table *t) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  long R = pick_radix(n);
  long m = n / R;
  for (long q = 0; q < R; ++q) dit(in + 2 * q * is, is * R, out + 2 * q * m, m, t);
  long step = t->n / n;
  double tq_stack[2 * 16];
  double *tq = R <= 16 ? tq_stack : (double *)malloc(sizeof(double) * 2 * (size_t)R);
  for (long k = 0; k < m; ++k) {
    for (long q = 0; q < R; ++q) {
      const double *y = out + 2 * (q * m + k);
      long j = ((q * k) % n) * step;
      double c = t->tw[2 * j], s = t->tw[2 * j + 1];
      tq[2 * q] = y[0] * c - y[1] * s;
      tq[2 * q + 1] = y[0] * s + y[1] * c;
    }
    for (long s = 0; s < R; ++s) {
      double re = 0.0, im = 0.0;
      for (long q = 0; q < R; ++q) {
        long j = (((q * s) % R) * m) * step; /* w_R^{qs} = w_n^{(qs mod R) m} */
        double c = t->tw[2 * j], sn = t->tw[2 * j + 1];
        re += tq[2 * q] * c - tq[2 * q + 1] * sn;
        im += tq[2 * q] * sn + tq[2 * q + 1] * c;
      }
      out[2 * (k + s * m)] = re;
      out[2 * (k + s * m) + 1] = im;
    }
  }
  if (tq != tq_stack) free(tq);
}

static void fft_strided(long n, long stride, double *data, const orc_table *t, double *tmp_in, double *tmp_out) {
  for (long k = 0; k < n; ++k) {
    tmp_in[2 * k] = data[2 * k * stride];
    tmp_in[2 * k + 1] = data[2 * k * stride + 1];
  }
  dit(tmp_in, 1, tmp_out, n, t);
  for (long k = 0; k < n; ++k) {
    data[2 * k * stride] = tmp_out[2 * k];
    data[2 * k * stride + 1] = tmp_out[2 * k + 1];
  }
}

void orc_fft1d(long n, int sign, double *data) {
  if (n <= 1) return;
  orc_table t;
  table_init(&t, n, sign);
  double *a = (double *)malloc(sizeof(double) * 4 * (size_t)n);
  fft_strided(n, 1, data, &t, a, a + 2 * n);
  free(a);
  table_free(&t);
}

void orc_fft2d(long n0, long n1, int sign, double *data) {
  orc_table t0, t1;
  table_init(&t0, n0, sign);
  table_init(&t1, n1, sign);
  long nm = n0 > n1 ? n0 : n1;
  double *a = (double *)malloc(sizeof(double) * 4 * (size_t)nm);
  for (long i = 0; i < n0; ++i) fft_strided(n1, 1, data + 2 * i * n1, &t1, a, a + 2 * nm);
  for (long j = 0; j < n1; ++j) fft_strided(n0, n1, data + 2 * j, &t0, a, a + 2 * nm);
  free(a);
  table_free(&t0);
  table_free(&t1);
}

void orc_fft3d(long n0, long n1, long n2, int sign, double *data) {
  orc_table t0, t1, t2;
  table_init(&t0, n0, sign);
  table_init(&t1, n1, sign);
  table_init(&t2, n2, sign);
  long nm = n0 > n1 ? n0 : n1;
  if (n2 > nm) nm = n2;
  double *a = (double *)malloc(sizeof(double) * 4 * (size_t)nm);
  for (long i = 0; i < n0 * n1; ++i) fft_strided(n2, 1, data + 2 * i * n2, &t2, a, a + 2 * nm);
  for (long i = 0; i < n0; ++i)
    for (long k = 0; k < n2; ++k) fft_strided(n1, n2, data + 2 * (i * n1 * n2 + k), &t1, a, a + 2 * nm);
  for (long jk = 0; jk < n1 * n2; ++jk) fft_strided(n0, n1 * n2, data + 2 * jk, &t0, a, a + 2 * nm);
  free(a);
  table_free(&t0);
  table_free(&t1);
  table_free(&t2);
}

void orc_fft2d_threads(long n0, long n1, int sign, double *data, int nthreads) {
  if (nthreads <= 1) {
    orc_fft2d(n0, n1, sign, data);
    return;
  }
  orc_table t0, t1;
  table_init(&t0, n0, sign);
  table_init(&t1, n1, sign);
  long nm = n0 > n1 ? n0 : n1;
#pragma omp parallel num_threads(nthreads)
  {
    double *a = (double *)malloc(sizeof(double) * 4 * (size_t)nm);
#pragma omp for schedule(static)
    for (long i = 0; i < n0; ++i) fft_strided(n1, 1, data + 2 * i * n1, &t1, a, a + 2 * nm);
#pragma omp for schedule(static)
    for (long j = 0; j < n1; ++j) fft_strided(n0, n1, data + 2 * j, &t0, a, a + 2 * nm);
    free(a);
  }
  table_free(&t0);
  table_free(&t1);
}

void orc_r2c_3d(long n0, long n1, long n2, double *padded) {
  const long nh = n2 / 2 + 1, pitch = 2 * nh;
  double *z = (double *)calloc(2 * (size_t)n0 * n1 * n2, sizeof(double));
  for (long ij = 0; ij < n0 * n1; ++ij)
    for (long k = 0; k < n2; ++k) z[2 * (ij * n2 + k)] = padded[ij * pitch + k];
  orc_fft3d(n0, n1, n2, -1, z);
  for (long ij = 0; ij < n0 * n1; ++ij)
    for (long k = 0; k < nh; ++k) {
      padded[ij * pitch + 2 * k] = z[2 * (ij * n2 + k)];
      padded[ij * pitch + 2 * k + 1] = z[2 * (ij * n2 + k) + 1];
    }
  free(z);
}

void orc_c2r_3d(long n0, long n1, long n2, double *padded) {
  const long nh = n2 / 2 + 1, pitch = 2 * nh;
  double *z = (double *)malloc(sizeof(double) * 2 * (size_t)n0 * n1 * n2);
  for (long i = 0; i < n0; ++i)
    for (long j = 0; j < n1; ++j)
      for (long k = 0; k < n2; ++k) {
        double *dst = z + 2 * ((i * n1 + j) * n2 + k);
        if (k < nh) {
          dst[0] = padded[(i * n1 + j) * pitch + 2 * k];
          dst[1] = padded[(i * n1 + j) * pitch + 2 * k + 1];
        } else {
          const long ic = (n0 - i) % n0, jc = (n1 - j) % n1, kc = n2 - k;
          dst[0] = padded[(ic * n1 + jc) * pitch + 2 * kc];
          dst[1] = -padded[(ic * n1 + jc) * pitch + 2 * kc + 1];
        }
      }
  orc_fft3d(n0, n1, n2, +1, z);
  for (long ij = 0; ij < n0 * n1; ++ij)
    for (long k = 0; k < n2; ++k) padded[ij * pitch + k] = z[2 * (ij * n2 + k)];
  free(z);
}
