/* Oracle: CPU restatement of the BEAM estimator hot path. TEST INFRASTRUCTURE ONLY:
 * used by tests/, the smoke check and the benchmark's CPU-baseline leg as the
 * checker; never linked into the GPU library. Each function cites the lines of
 * the reference (barbie.c, funcs.c of sukhdeepsinghgill/BARBIE) it follows. */
#include "beam_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fft.h"

/* barbie.c:110-130. Blocks of ten rings; block b has width b+1 grid units.
 * Every lower edge but the first is pulled in by 0.1, the upper edge of ring
 * i-1 is the lower edge of ring i, the last upper edge is Nmax, and the ring
 * "average" used by the closure tests is the midpoint. */
int orc_ring_edges(long Nr, long Nmax, double *low, double *high, double *avg) {
  if (Nr <= 0 || Nr % 10 != 0) return -1;
  long edge = 0;
  for (long r = 0; r < Nr; ++r) {
    low[r] = (double)edge;
    edge += r / 10 + 1;
  }
  for (long r = 1; r < Nr; ++r) {
    low[r] -= 0.1;
    high[r - 1] = low[r];
  }
  high[Nr - 1] = (double)Nmax;
  for (long r = 0; r < Nr; ++r) avg[r] = (high[r] + low[r]) / 2.;
  return 0;
}

/* Signed frequency of FFT index i on an NN grid, as at barbie.c:141-142. */
static long signed_freq(long i, long NN) { return i > NN / 2 ? i - NN : i; }

/* barbie.c:135-148 */
void orc_ring_masks(long NN, long Nr, const double *low, const double *high, double *RR) {
  for (long r = 0; r < Nr; ++r)
    for (long i = 0; i < NN; ++i)
      for (long j = 0; j < NN; ++j) {
        long ia = signed_freq(i, NN), ja = signed_freq(j, NN);
        double kk = sqrt(1. * (double)(ia * ia + ja * ja));
        RR[(r * NN + i) * NN + j] = (kk >= low[r] && kk < high[r]) ? 1. : 0.;
      }
}

/* Closure test of funcs.c:389-395 on ring midpoints: t = a2/a1 in [0.5,1] and
 * mu = (t + 1/t - (a3/a1)(a3/a2))/2 in [0.5/t, 1]. */
static int ring_triplet_closes(const double *avg, long r1, long r2, long r3, int *t_ok) {
  double tt = avg[r2] / avg[r1];
  *t_ok = (tt >= 0.5 && tt <= 1.);
  if (!*t_ok) return 0;
  double mu = 0.5 * (tt + 1. / tt - (avg[r3] / avg[r1]) * (avg[r3] / avg[r2]));
  return mu >= 0.5 / tt && mu <= 1.;
}

/* funcs.c:328-424 (calCR). The ring masks are transformed with an unnormalised
 * backward 2D DFT and only the real part is kept (funcs.c:367-382); Num is the
 * pixel sum of the three real transforms in row-major order (funcs.c:396-399). */
long orc_closed_rings(long NN, long Nr, const double *low, const double *high,
                      const double *avg, double *out4, long cap) {
  size_t n2 = (size_t)NN * (size_t)NN;
  double *RR = (double *)malloc(sizeof(double) * n2 * (size_t)Nr);
  double *II = (double *)malloc(sizeof(double) * n2 * (size_t)Nr);
  double *A = (double *)malloc(sizeof(double) * 2 * n2);
  if (!RR || !II || !A) {
    free(RR); free(II); free(A);
    return -1;
  }
  orc_ring_masks(NN, Nr, low, high, RR);
  for (long r = 0; r < Nr; ++r) {
    for (size_t x = 0; x < n2; ++x) {
      A[2 * x] = RR[r * n2 + x];
      A[2 * x + 1] = 0.;
    }
    orc_fft2d(NN, NN, +1, A);
    for (size_t x = 0; x < n2; ++x) II[r * n2 + x] = A[2 * x];
  }
  long count = 0;
  for (long r1 = 0; r1 < Nr; ++r1)
    for (long r2 = 0; r2 <= r1; ++r2) {
      int t_ok;
      ring_triplet_closes(avg, r1, r2, 0, &t_ok);
      if (!t_ok) continue;
      for (long r3 = 0; r3 <= r2; ++r3) {
        if (!ring_triplet_closes(avg, r1, r2, r3, &t_ok)) continue;
        double num = 0.;
        const double *i1 = II + r1 * n2, *i2 = II + r2 * n2, *i3 = II + r3 * n2;
        for (size_t x = 0; x < n2; ++x) num += i1[x] * i2[x] * i3[x];
        if (out4 && count < cap) {
          out4[4 * count + 0] = (double)r1;
          out4[4 * count + 1] = (double)r2;
          out4[4 * count + 2] = (double)r3;
          out4[4 * count + 3] = num;
        }
        ++count;
      }
    }
  free(RR); free(II); free(A);
  return count;
}

int64_t orc_triangle_count_direct(long NN, const double *RR, long r1, long r2, long r3) {
  size_t n2 = (size_t)NN * (size_t)NN;
  const double *m1 = RR + r1 * n2, *m2 = RR + r2 * n2, *m3 = RR + r3 * n2;
  int64_t count = 0;
  for (long i1 = 0; i1 < NN; ++i1)
    for (long j1 = 0; j1 < NN; ++j1) {
      if (m1[i1 * NN + j1] == 0.) continue;
      for (long i2 = 0; i2 < NN; ++i2)
        for (long j2 = 0; j2 < NN; ++j2) {
          if (m2[i2 * NN + j2] == 0.) continue;
          long i3 = (2 * NN - i1 - i2) % NN, j3 = (2 * NN - j1 - j2) % NN;
          if (m3[i3 * NN + j3] != 0.) ++count;
        }
    }
  return count;
}

/* funcs.c:88-109 with sign=+1 (the only sign barbie passes, funcs.c:553).
 * Element (i,j) of plane p is complex index i*NN*(NN/2+1) + j*(NN/2+1) + p of
 * the r2c buffer (funcs.c:97). */
void orc_plane_ring(long NN, long p, long r, const double *r2c, const double *RR, double *out) {
  long nh = NN / 2 + 1;
  size_t n2 = (size_t)NN * (size_t)NN;
  const double *mask = RR + (size_t)r * n2;
  for (long i = 0; i < NN; ++i)
    for (long j = 0; j < NN; ++j) {
      size_t src = (size_t)i * NN * nh + (size_t)j * nh + (size_t)p;
      size_t dst = (size_t)i * NN + j;
      out[2 * dst] = r2c[2 * src] * mask[dst];
      out[2 * dst + 1] = r2c[2 * src + 1] * mask[dst];
    }
  if (p == 0) { /* k = 0 mode excluded, funcs.c:102-106 */
    out[0] = 0.;
    out[1] = 0.;
  }
  orc_fft2d(NN, NN, +1, out);
}

/* funcs.c:708-745. Legendre-based orientation weights bs[] for the 16 (l,m)
 * multipoles (l=0; l=2,m=0..2; l=4,m=0..4; l=6,m=0..6) and the matching
 * normalisation polynomials norm[], as functions of the triangle orientation
 * (px, pz). Written with z = pz^2, x = px^2, w = pz^2 - 1. */
void orc_cal_coeff(double px, double pz, double *bs, double *norm) {
  const double z = pz * pz, x = px * px, w = z - 1.;
  const double c2 = 2. * x + z - 1.;             /* -1 + 2px^2 + pz^2 */
  const double c4 = 8. * x * x + 8. * x * w + w * w;
  bs[0] = 1.;
  bs[1] = 2. * (3. * z - 1.);
  bs[2] = -sqrt(2. / 3.) * px * pz;
  bs[3] = 2. * sqrt(2. / 3.) * c2;
  bs[4] = 8. * (3. - 30. * z + 35. * z * z);
  bs[5] = -4. * px * pz * (7. * z - 3.) / sqrt(5.);
  bs[6] = 4. * sqrt(0.4) * c2 * (7. * z - 1.);
  bs[7] = -4. * px * pz * (4. * x + 3. * z - 3.) / sqrt(35.);
  bs[8] = 8. * sqrt(2. / 35.) * c4;
  bs[9] = 16. * (-5. + 105. * z - 315. * z * z + 231. * z * z * z);
  bs[10] = -8. * sqrt(2. / 21.) * px * pz * (5. - 30. * z + 33. * z * z);
  bs[11] = 32. * c2 * (1. - 18. * z + 33. * z * z) / sqrt(105.);
  bs[12] = -16. * px * pz * (4. * x + 3. * z - 3.) * (11. * z - 3.) / sqrt(105.);
  bs[13] = 16. * sqrt(2. / 7.) * (11. * z - 1.) * c4 / 3.;
  bs[14] = -16. * pz * px * (16. * x * x + 20. * x * w + 5. * w * w) / (3. * sqrt(77.));
  bs[15] = 32. * (32. * x * x * x + 48. * x * x * w + 18. * x * w * w + w * w * w) / sqrt(231.);

  const double u = 1. - z; /* 1 - pz^2 */
  const double l2 = 3. * z - 1.;
  const double l4 = 3. - 30. * z + 35. * z * z;
  const double a5 = pz * (7. * z - 3.);
  const double a6 = 7. * z - 1.;
  const double l6 = -5. + 105. * z - 315. * z * z + 231. * z * z * z;
  const double a10 = pz * (5. - 30. * z + 33. * z * z);
  const double a11 = 1. - 18. * z + 33. * z * z;
  const double a12 = pz * (11. * z - 3.);
  const double a13 = 11. * z - 1.;
  norm[0] = 1.;
  norm[1] = l2 * l2;
  norm[2] = z * u;
  norm[3] = u * u;
  norm[4] = l4 * l4;
  norm[5] = u * a5 * a5;
  norm[6] = u * u * a6 * a6;
  norm[7] = z * u * u * u;
  norm[8] = u * u * u * u;
  norm[9] = l6 * l6;
  norm[10] = u * a10 * a10;
  norm[11] = u * u * a11 * a11;
  norm[12] = u * u * u * a12 * a12;
  norm[13] = u * u * u * u * a13 * a13;
  norm[14] = z * u * u * u * u * u;
  norm[15] = u * u * u * u * u * u;
}

/* Stable descending sort of the three legs by |K| (ties keep leg order), as the
 * bubble sort of funcs.c:113-126 with its strict comparison. */
static void sort_legs(double K[3][2]) {
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2 - i; ++j)
      if (K[j][0] < K[j + 1][0]) {
        double a = K[j][0], b = K[j][1];
        K[j][0] = K[j + 1][0];
        K[j][1] = K[j + 1][1];
        K[j + 1][0] = a;
        K[j + 1][1] = b;
      }
}

/* p2 range for a ring triplet by ring-equality symmetry, barbie.c:257-268. */
static void p2_range(long p1, long Nmax, long r1, long r2, long r3, long *lo, long *hi) {
  if (r1 == r2 && r2 == r3) {
    *lo = 0; *hi = p1;
  } else if (r1 == r2) {
    *lo = -p1; *hi = p1;
  } else if (r2 == r3) {
    *lo = (int)(-p1 / 2); *hi = Nmax;
  } else {
    *lo = (p1 == 0) ? 0 : -Nmax + 1; *hi = Nmax;
  }
}

/* Bin index on [0.5,1] with n bins, value 1 going to the last bin (barbie.c:344-345). */
static int shape_bin(double v, int n) {
  return (v == 1) ? (n - 1) : (int)floor((v - .5) / (.5 / (1. * n)));
}

/* barbie.c:247-298 and 343-345. */
long orc_enumerate(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, int n_mtbin,
                   const double *avg, const double *rings4, long rcount,
                   orc_triple *out, long cap, long *iterations) {
  (void)NN; (void)Nr;
  long n = 0, iters = 0;
  for (long p1 = 0; p1 < Nmax; ++p1)
    for (long rp = 0; rp < rcount; ++rp) {
      long r1 = (long)rings4[4 * rp], r2 = (long)rings4[4 * rp + 1], r3 = (long)rings4[4 * rp + 2];
      long lo, hi;
      p2_range(p1, Nmax, r1, r2, r3, &lo, &hi);
      for (long p2 = lo; p2 <= hi; ++p2) {
        ++iters;
        long p3 = -p1 - p2;
        if (labs(p3) >= Nmax) continue;
        double K[3][2] = {{sqrt(avg[r1] * avg[r1] + (double)(p1 * p1)), (double)p1},
                          {sqrt(avg[r2] * avg[r2] + (double)(p2 * p2)), (double)p2},
                          {sqrt(avg[r3] * avg[r3] + (double)(p3 * p3)), (double)p3}};
        sort_legs(K);
        if (!(K[0][0] > LL_k1 && K[0][0] < UL_k1)) continue;
        if (out && n < cap) {
          orc_triple *t = out + n;
          double K1 = K[0][0];
          double T = K[1][0] / K[0][0];
          double MU = 0.5 * (T + 1. / T - (K[2][0] / K[0][0]) * (K[2][0] / K[1][0]));
          double pz = K[0][1] / K[0][0];
          double px = ((K[1][1] / K[1][0]) + MU * pz) / (sqrt(1. - (MU * MU)));
          t->p1 = (int32_t)p1; t->r1 = (int32_t)r1;
          t->p2 = (int32_t)p2; t->r2 = (int32_t)r2;
          t->p3 = (int32_t)p3; t->r3 = (int32_t)r3;
          t->rp = (int32_t)rp;
          t->K1 = K1; t->T = T; t->MU = MU; t->px = px; t->pz = pz;
          t->num = rings4[4 * rp + 3];
          for (int i = 0; i < 3; ++i) {
            t->leg_k[i] = K[i][0];
            t->leg_p[i] = K[i][1];
          }
          t->k1_bin = (int32_t)floor((K1 - (LL_k1)) / (1. * BW_k1));
          t->t_bin = shape_bin(T, n_mtbin);
          t->mu_bin = shape_bin(MU, n_mtbin);
        }
        ++n;
      }
    }
  if (iterations) *iterations = iters;
  return n;
}

/* barbie.c:329-337: sum over pixels of Re(F1 * F2^(s2) * F3^(s3)), where ^(-1)
 * is complex conjugation (the caches hold planes p >= 0 only). */
double orc_triple_product(long NN, const double *F1, const double *F2, const double *F3, int sign2, int sign3) {
  size_t n2 = (size_t)NN * (size_t)NN;
  double s2 = (double)sign2, s3 = (double)sign3, acc = 0.;
  for (size_t x = 0; x < n2; ++x) {
    double ar = F1[2 * x], ai = F1[2 * x + 1];
    double br = F2[2 * x], bi = s2 * F2[2 * x + 1];
    double cr = F3[2 * x], ci = s3 * F3[2 * x + 1];
    acc += ar * br * cr - ar * bi * ci - ai * br * ci - ai * bi * cr;
  }
  return acc;
}

/* The same pixel sum with the products and the running sum in long double
 * (64-bit significand on x86-64). Test infrastructure for the largest
 * fixtures: at NN=384 the double running sum over 147,456 pixels carries
 * rounding of up to ~4e-12 of a triangle's scale, which bins that cancel by
 * ~3e5 turn into ~1e-10; the wider sum keeps the oracle's own error well
 * below the parity bar. */
static double triple_product_wide(long NN, const double *F1, const double *F2, const double *F3, int sign2,
                                  int sign3) {
  size_t n2 = (size_t)NN * (size_t)NN;
  long double s2 = (long double)sign2, s3 = (long double)sign3, acc = 0.L;
  for (size_t x = 0; x < n2; ++x) {
    long double ar = F1[2 * x], ai = F1[2 * x + 1];
    long double br = F2[2 * x], bi = s2 * F2[2 * x + 1];
    long double cr = F3[2 * x], ci = s3 * F3[2 * x + 1];
    acc += ar * br * cr - ar * bi * ci - ai * br * ci - ai * bi * cr;
  }
  return (double)acc;
}

/* funcs.c:73-81 */
static double input_ps(double kk) {
  double Av = 1.0, betav = -2.0;
  return Av * pow(kk, betav);
}

double orc_biana(long NN, double LL, const double leg_k[3], const double leg_p[3]) {
  const double ff = 0.1, beta = 1.;           /* barbie.c:79-80 */
  const double Cunits = 2. * M_PI / (NN * LL);  /* barbie.c:77 */
  double mu_1 = leg_p[0] / leg_k[0], mu_2 = leg_p[1] / leg_k[1], mu_3 = leg_p[2] / leg_k[2];
  double Biana = 2. * ff * (input_ps(Cunits * leg_k[0]) * input_ps(Cunits * leg_k[1]) +
                            input_ps(Cunits * leg_k[1]) * input_ps(Cunits * leg_k[2]) +
                            input_ps(Cunits * leg_k[2]) * input_ps(Cunits * leg_k[0]));
  return Biana * (1 + beta * mu_1 * mu_1) * (1 + beta * mu_2 * mu_2) * (1 + beta * mu_3 * mu_3);
}

void orc_biana_all(long NN, double LL, const orc_triple *tri, long n, double *out) {
  for (long t = 0; t < n; ++t) out[t] = orc_biana(NN, LL, tri[t].leg_k, tri[t].leg_p);
}

int orc_estimate(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, int n_mtbin,
                 double LL, const double *r2c, double *bin_bs, double *bin_norm, double *bin_out,
                 int64_t *counts, double *tri_B, long tri_cap, int nthreads, double *bin_ana) {
  return orc_estimate_ex(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin, LL, r2c, bin_bs, bin_norm, bin_out, counts,
                         tri_B, tri_cap, nthreads, bin_ana, 0);
}

int orc_estimate_ex(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, int n_mtbin,
                    double LL, const double *r2c, double *bin_bs, double *bin_norm, double *bin_out,
                    int64_t *counts, double *tri_B, long tri_cap, int nthreads, double *bin_ana, int wide) {
  if (NN <= 0 || NN % 2 || Nmax <= 0 || Nmax > NN / 2 + 1 || BW_k1 <= 0 || UL_k1 <= LL_k1) return -1;
  double *low = (double *)calloc((size_t)Nr, sizeof(double));
  double *high = (double *)calloc((size_t)Nr, sizeof(double));
  double *avg = (double *)calloc((size_t)Nr, sizeof(double));
  if (orc_ring_edges(Nr, Nmax, low, high, avg)) {
    free(low); free(high); free(avg);
    return -1;
  }
  size_t n2 = (size_t)NN * (size_t)NN;
  long cap = Nr * Nr * Nr;
  double *rings4 = (double *)malloc(sizeof(double) * 4 * (size_t)cap);
  long rcount = orc_closed_rings(NN, Nr, low, high, avg, rings4, cap);
  double *RR = (double *)malloc(sizeof(double) * n2 * (size_t)Nr);
  double *cache = (double *)malloc(sizeof(double) * 2 * n2 * (size_t)(Nmax * Nr));
  if (rcount < 0 || !RR || !cache) {
    free(low); free(high); free(avg); free(rings4); free(RR); free(cache);
    return -1;
  }
  orc_ring_masks(NN, Nr, low, high, RR);
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
  for (long pr = 0; pr < Nmax * Nr; ++pr)
    orc_plane_ring(NN, pr / Nr, pr % Nr, r2c, RR, cache + 2 * n2 * (size_t)pr);

  long ntri = orc_enumerate(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin, avg, rings4, rcount, NULL, 0, NULL);
  orc_triple *tri = (orc_triple *)malloc(sizeof(orc_triple) * (size_t)(ntri > 0 ? ntri : 1));
  double *B = (double *)malloc(sizeof(double) * (size_t)(ntri > 0 ? ntri : 1));
  orc_enumerate(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, n_mtbin, avg, rings4, rcount, tri, ntri, NULL);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
  for (long t = 0; t < ntri; ++t) {
    const orc_triple *q = tri + t;
    const double *F1 = cache + 2 * n2 * (size_t)(q->p1 * Nr + q->r1);
    const double *F2 = cache + 2 * n2 * (size_t)(labs(q->p2) * Nr + q->r2);
    const double *F3 = cache + 2 * n2 * (size_t)(labs(q->p3) * Nr + q->r3);
    B[t] = wide ? triple_product_wide(NN, F1, F2, F3, q->p2 < 0 ? -1 : 1, q->p3 < 0 ? -1 : 1)
                : orc_triple_product(NN, F1, F2, F3, q->p2 < 0 ? -1 : 1, q->p3 < 0 ? -1 : 1);
  }

  int n_k1bin = (int)((UL_k1 - LL_k1) / (1. * BW_k1));
  size_t nbins = (size_t)n_k1bin * n_mtbin * n_mtbin;
  memset(bin_bs, 0, sizeof(double) * nbins * ORC_NPOLES);
  memset(bin_norm, 0, sizeof(double) * nbins * ORC_NPOLES);
  if (bin_ana) memset(bin_ana, 0, sizeof(double) * nbins * ORC_NPOLES);
  if (counts) memset(counts, 0, sizeof(int64_t) * nbins);
  int rc = 0;
  for (long t = 0; t < ntri; ++t) { /* barbie.c:343-363, in loop order */
    const orc_triple *q = tri + t;
    if (q->k1_bin < 0 || q->k1_bin >= n_k1bin || q->t_bin < 0 || q->t_bin >= n_mtbin ||
        q->mu_bin < 0 || q->mu_bin >= n_mtbin) {
      rc = -1; /* the reference indexes out of bounds here */
      continue;
    }
    double bs[ORC_NPOLES], nm[ORC_NPOLES];
    orc_cal_coeff(q->px, q->pz, bs, nm);
    double num = q->num;
    double ana = orc_biana(NN, LL, q->leg_k, q->leg_p);
    if (B[t] == 0.) { /* barbie.c:355-357 */
      ana = 0.;
      num = 0.;
    }
    size_t b = ((size_t)q->k1_bin * n_mtbin + q->t_bin) * n_mtbin + q->mu_bin;
    for (int ii = 0; ii < ORC_NPOLES; ++ii) {
      bin_bs[b * ORC_NPOLES + ii] += B[t] * bs[ii];
      if (bin_ana) bin_ana[b * ORC_NPOLES + ii] += ana * num * bs[ii];
      bin_norm[b * ORC_NPOLES + ii] += num * nm[ii];
    }
    if (counts && B[t] != 0.) counts[b] += (int64_t)llround(q->num / (double)n2);
  }
  double vol = pow((double)NN * LL, 3);
  for (size_t i = 0; i < nbins * ORC_NPOLES; ++i) bin_out[i] = bin_bs[i] / (vol * bin_norm[i]);
  if (tri_B)
    for (long t = 0; t < ntri && t < tri_cap; ++t) tri_B[t] = B[t];
  free(low); free(high); free(avg); free(rings4); free(RR); free(cache); free(tri); free(B);
  return rc;
}

static double wall_seconds(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

int orc_time_sample(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, const double *r2c,
                    const long *sample, long nsample, int nthreads, double *t_fft, long *n_fft, double *t_sum,
                    double *checksum) {
  double *low = (double *)calloc((size_t)Nr, sizeof(double));
  double *high = (double *)calloc((size_t)Nr, sizeof(double));
  double *avg = (double *)calloc((size_t)Nr, sizeof(double));
  if (orc_ring_edges(Nr, Nmax, low, high, avg)) {
    free(low); free(high); free(avg);
    return -1;
  }
  size_t n2 = (size_t)NN * (size_t)NN;
  long cap = Nr * Nr * Nr;
  double *rings4 = (double *)malloc(sizeof(double) * 4 * (size_t)cap);
  long rcount = orc_closed_rings(NN, Nr, low, high, avg, rings4, cap);
  long ntri = orc_enumerate(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, 5, avg, rings4, rcount, NULL, 0, NULL);
  orc_triple *tri = (orc_triple *)malloc(sizeof(orc_triple) * (size_t)(ntri > 0 ? ntri : 1));
  orc_enumerate(NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, 5, avg, rings4, rcount, tri, ntri, NULL);
  double *RR = (double *)malloc(sizeof(double) * n2 * (size_t)Nr);
  orc_ring_masks(NN, Nr, low, high, RR);
  /* distinct (|p|, ring) arrays the sample needs */
  long *slot = (long *)malloc(sizeof(long) * (size_t)(Nmax * Nr));
  for (long k = 0; k < Nmax * Nr; ++k) slot[k] = -1;
  long nslot = 0;
  long *slot_pr = (long *)malloc(sizeof(long) * (size_t)(Nmax * Nr));
  for (long s = 0; s < nsample; ++s) {
    if (sample[s] < 0 || sample[s] >= ntri) continue;
    const orc_triple *q = tri + sample[s];
    long key[3] = {q->p1 * Nr + q->r1, labs(q->p2) * Nr + q->r2, labs(q->p3) * Nr + q->r3};
    for (int k = 0; k < 3; ++k)
      if (slot[key[k]] < 0) {
        slot[key[k]] = nslot;
        slot_pr[nslot++] = key[k];
      }
  }
  double *F = (double *)malloc(sizeof(double) * 2 * n2 * (size_t)(nslot > 0 ? nslot : 1));
  int nt = nthreads > 0 ? nthreads : 1;
  double t0 = wall_seconds();
#pragma omp parallel for schedule(dynamic) num_threads(nt)
  for (long k = 0; k < nslot; ++k) orc_plane_ring(NN, slot_pr[k] / Nr, slot_pr[k] % Nr, r2c, RR, F + 2 * n2 * (size_t)k);
  double t1 = wall_seconds();
  double sum = 0.0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt) reduction(+ : sum)
  for (long s = 0; s < nsample; ++s) {
    if (sample[s] < 0 || sample[s] >= ntri) continue;
    const orc_triple *q = tri + sample[s];
    const double *F1 = F + 2 * n2 * (size_t)slot[q->p1 * Nr + q->r1];
    const double *F2 = F + 2 * n2 * (size_t)slot[labs(q->p2) * Nr + q->r2];
    const double *F3 = F + 2 * n2 * (size_t)slot[labs(q->p3) * Nr + q->r3];
    sum += orc_triple_product(NN, F1, F2, F3, q->p2 < 0 ? -1 : 1, q->p3 < 0 ? -1 : 1);
  }
  double t2 = wall_seconds();
  *t_fft = t1 - t0;
  *n_fft = nslot;
  *t_sum = t2 - t1;
  *checksum = sum;
  free(low); free(high); free(avg); free(rings4); free(tri); free(RR); free(slot); free(slot_pr); free(F);
  return 0;
}

/* funcs.c:860-1074 (calpow_mom): power spectrum multipoles of the r2c buffer in
 * Nbin logarithmic bins of |k|, with the reference's float/double types so the
 * bin of every mode and the Legendre weights round as there. The three loops
 * (half lines, half planes, half cube) visit each independent mode once. out
 * receives [6][Nbin]: kmode, P0, P2, P4, P6, mode count (normalised as
 * funcs.c:1050-1066 with cell size LL). */
static void orc_pk_add(double *acc, int Nbin, long NN, float fac1, float fac2, float fac3, float scale, long a,
                       long b, long c, const double *z) {
  float m, mu, P2, P4, P6;
  m = sqrt(fac1 * a * a + fac2 * b * b + fac3 * c * c);
  mu = (1.0 * c) / (NN * m);
  P2 = 0.5 * (3. * mu * mu - 1.);
  P4 = 0.125 * (35.0 * powf(mu, 4.0) - 30.0 * mu * mu + 3);
  P6 = 0.0625 * (231.0 * powf(mu, 6.0) - 315.0 * powf(mu, 4.0) + 105.0 * mu * mu - 5);
  long d = (int)floorf(log10(m * NN) / scale);
  if (d < 0 || d >= Nbin) return;
  double pw = (z[0] * z[0]) + (z[1] * z[1]);
  double *q = acc + 9 * d;
  q[0] += pw;
  q[1] += (double)(pw * P2);
  q[2] += (double)(pw * P4);
  q[3] += (double)(pw * P6);
  q[4] += (double)m;
  q[5] += 1.0;
  q[6] += (double)(P2 * P2);
  q[7] += (double)(P4 * P4);
  q[8] += (double)(P6 * P6);
}

int orc_power_multipoles(long NN, double LL, int Nbin, const double *r2c, double *out) {
  if (NN <= 0 || NN % 2 || Nbin <= 0 || !r2c || !out) return -1;
  const long N1 = NN, N2 = NN, N3 = NN, NH = N3 / 2 + 1;
  double *acc = (double *)calloc((size_t)Nbin * 9, sizeof(double));
  if (!acc) return -1;
  float fac1 = 1. / (1. * N1 * N1), fac2 = 1. / (1. * N2 * N2), fac3 = 1. / (1. * N3 * N3);
  float scale = log10(0.5 * N1) / Nbin;
  const double *z = r2c;
  for (long i = 1; i <= N1 / 2; i++) /* half lines */
    for (long j = 0; j <= N2 / 2; j = j + N2 / 2)
      for (long k = 0; k <= N3 / 2; k = k + N3 / 2)
        orc_pk_add(acc, Nbin, NN, fac1, fac2, fac3, scale, i, j, k, z + 2 * ((i * N2 + j) * NH + k));
  for (long i = 0; i < N1; i++) { /* half planes */
    long a = (i > N1 / 2) ? N1 - i : i;
    for (long j = 1; j < N2 / 2; j++)
      for (long k = 0; k <= N3 / 2; k = k + N3 / 2)
        orc_pk_add(acc, Nbin, NN, fac1, fac2, fac3, scale, a, j, k, z + 2 * ((i * N2 + j) * NH + k));
  }
  for (long i = 0; i < N1; i++) { /* half cube */
    long a = (i > N1 / 2) ? N1 - i : i;
    for (long j = 0; j < N2; j++) {
      long b = (j > N2 / 2) ? N2 - j : j;
      for (long k = 1; k < N3 / 2; k++)
        orc_pk_add(acc, Nbin, NN, fac1, fac2, fac3, scale, a, b, k, z + 2 * ((i * N2 + j) * NH + k));
    }
  }
  double norml = 1. / (1. * N1 * N2 * N3), pi = M_PI;
  for (int d = 0; d < Nbin; d++) {
    const double *q = acc + 9 * d;
    double kmode = q[4], P0 = q[0], P2 = q[1], P4 = q[2], P6 = q[3];
    if (q[5] > 0.0) {
      P0 = norml * P0 / (1.0 * q[5] * pow(LL, 3.));
      kmode = 2. * pi * kmode / (q[5] * LL);
    }
    if (q[6] > 0.0) P2 = norml * P2 / (1.0 * q[6] * pow(LL, 3.));
    if (q[7] > 0.0) P4 = norml * P4 / (1.0 * q[7] * pow(LL, 3.));
    if (q[8] > 0.0) P6 = norml * P6 / (1.0 * q[8] * pow(LL, 3.));
    out[d] = kmode;
    out[Nbin + d] = P0;
    out[2 * Nbin + d] = P2;
    out[3 * Nbin + d] = P4;
    out[4 * Nbin + d] = P6;
    out[5 * Nbin + d] = q[5];
  }
  free(acc);
  return 0;
}
