/* Host-side estimator geometry for libbeam_gpu (see geometry.h).
 *
 * The floating-point expressions that decide ring membership, triplet closure,
 * the k1 window and the bins are kept in the same operation order as the
 * reference so that they round identically; this file must be compiled without
 * FMA contraction (-ffp-contract=off) and without fast-math. */
#include "geometry.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* barbie.c:110-130: blocks of ten rings, block b of width b+1; inner edges
 * lowered by 0.1; ring i-1 ends where ring i starts; outer edge Nmax; the ring
 * value used by the closure tests is the midpoint of its edges. */
int beam_ring_edges(long Nr, long Nmax, double *low, double *high, double *avg) {
  if (Nr < 10 || Nr % 10 != 0) return BEAM_EINVAL;
  long start = 0;
  for (long r = 0; r < Nr; ++r) {
    low[r] = (double)start;
    start += 1 + r / 10;
  }
  for (long r = 1; r < Nr; ++r) {
    low[r] -= .1;
    high[r - 1] = low[r];
  }
  high[Nr - 1] = 1. * (double)Nmax;
  for (long r = 0; r < Nr; ++r) avg[r] = (high[r] + low[r]) / 2.;
  return BEAM_OK;
}

void beam_geom_free(beam_geom *g) {
  free(g->low); free(g->high); free(g->avg); free(g->ringmap); free(g->rp);
  free(g->t_rp); free(g->t_p1); free(g->t_p2); free(g->t_bin); free(g->t_px); free(g->t_pz); free(g->t_ana);
  memset(g, 0, sizeof(*g));
}

/* Ring membership of every pixel (barbie.c:135-148). Rings are half-open
 * intervals [low, high) of |k_perp| that share their edges, so a pixel is in at
 * most one ring; membership is tested per ring exactly as the reference does. */
static int build_ringmap(beam_geom *g) {
  long NN = g->NN;
  g->ringmap = (int16_t *)malloc(sizeof(int16_t) * (size_t)(NN * NN));
  if (!g->ringmap) return BEAM_ENOMEM;
  for (long i = 0; i < NN; ++i)
    for (long j = 0; j < NN; ++j) {
      int ia = (int)((i > NN / 2) ? (i - NN) : i);
      int ja = (int)((j > NN / 2) ? (j - NN) : j);
      double kk = sqrt(1. * (ia * ia + ja * ja));
      int ring = -1;
      for (long r = 0; r < g->Nr; ++r)
        if (kk >= g->low[r] && kk < g->high[r]) {
          if (ring >= 0) return BEAM_EINVAL; /* overlapping rings: not this edge rule */
          ring = (int)r;
        }
      g->ringmap[i * NN + j] = (int16_t)ring;
    }
  return BEAM_OK;
}

/* funcs.c:389-395: sorted triplets r1 >= r2 >= r3 whose midpoints close:
 * t = a2/a1 in [0.5, 1] and mu = (t + 1/t - (a3/a1)(a3/a2))/2 in [0.5/t, 1]. */
static int build_triplets(beam_geom *g) {
  const double *a = g->avg;
  long Nr = g->Nr, n = 0, cap = 64;
  g->rp = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)cap);
  if (!g->rp) return BEAM_ENOMEM;
  for (long r1 = 0; r1 < Nr; ++r1)
    for (long r2 = 0; r2 <= r1; ++r2) {
      double tt = a[r2] / a[r1];
      if (!(tt >= 0.5 && tt <= 1.)) continue;
      for (long r3 = 0; r3 <= r2; ++r3) {
        double mu = 0.5 * (tt + 1. / tt - (a[r3] / a[r1]) * (a[r3] / a[r2]));
        if (!(mu >= 0.5 / tt && mu <= 1.)) continue;
        if (n == cap) {
          cap *= 2;
          int32_t *p = (int32_t *)realloc(g->rp, sizeof(int32_t) * 3 * (size_t)cap);
          if (!p) return BEAM_ENOMEM;
          g->rp = p;
        }
        g->rp[3 * n] = (int32_t)r1;
        g->rp[3 * n + 1] = (int32_t)r2;
        g->rp[3 * n + 2] = (int32_t)r3;
        ++n;
      }
    }
  g->nrp = n;
  return BEAM_OK;
}

/* One (p1, rp, p2) visit of the loop barbie.c:280-298 and its bins (:343-345).
 * Returns 1 if the triangle passes |p3| < Nmax and LL_k1 < K1 < UL_k1. */
typedef struct {
  double px, pz;
  double ana;
  int bin;
  int bad_bin;
} tri_eval;

/* funcs.c:73-81: the input power spectrum P(k) = Av k^betav. */
static double input_ps(double kk) {
  double Av = 1.0, betav = -2.0;
  return Av * pow(kk, betav);
}

static int eval_triangle(const beam_geom *g, int r1, int r2, int r3, int p1, int p2, tri_eval *e) {
  int p3 = -p1 - p2;
  int s3 = p3 < 0 ? -1 : 1;
  if (!(s3 * p3 < g->Nmax)) return 0;
  const double *a = g->avg;
  /* legs as (|K|, p); |K| = sqrt(k_perp_avg^2 + p^2) */
  double k[3] = {sqrt(a[r1] * a[r1] + p1 * p1), sqrt(a[r2] * a[r2] + p2 * p2), sqrt(a[r3] * a[r3] + p3 * p3)};
  double p[3] = {(double)p1, (double)p2, (double)p3};
  /* stable descending order by |K| (ties keep leg order), as funcs.c:113-126 */
  for (int pass = 0; pass < 2; ++pass)
    for (int j = 0; j < 2 - pass; ++j)
      if (k[j] < k[j + 1]) {
        double t = k[j]; k[j] = k[j + 1]; k[j + 1] = t;
        t = p[j]; p[j] = p[j + 1]; p[j + 1] = t;
      }
  if (!(k[0] > g->LL_k1 && k[0] < g->UL_k1)) return 0;
  double K1 = k[0];
  double T = k[1] / k[0];
  double MU = 0.5 * (T + 1. / T - (k[2] / k[0]) * (k[2] / k[1]));
  e->pz = p[0] / k[0];
  e->px = ((p[1] / k[1]) + MU * e->pz) / (sqrt(1. - (MU * MU)));
  /* barbie.c:300-305 with ff = 0.1, beta = 1 (barbie.c:79-80), Cunits of :77 */
  {
    const double ff = 0.1, beta = 1., Cunits = 2. * M_PI / (g->NN * g->LL);
    double mu_1 = p[0] / k[0], mu_2 = p[1] / k[1], mu_3 = p[2] / k[2];
    /* each leg's P(k) once: the same values the reference computes twice */
    double P0 = input_ps(Cunits * k[0]), P1 = input_ps(Cunits * k[1]), P2 = input_ps(Cunits * k[2]);
    double ana = 2. * ff * (P0 * P1 + P1 * P2 + P2 * P0);
    e->ana = ana * (1 + beta * mu_1 * mu_1) * (1 + beta * mu_2 * mu_2) * (1 + beta * mu_3 * mu_3);
  }
  int n = g->n_mtbin;
  double kb = floor((K1 - (g->LL_k1)) / (1. * g->BW_k1));
  double tb = (T == 1) ? (n - 1) : floor((T - .5) / (.5 / (1. * n)));
  double mb = (MU == 1) ? (n - 1) : floor((MU - .5) / (.5 / (1. * n)));
  e->bad_bin = !(kb >= 0 && kb < g->n_k1bin && tb >= 0 && tb < n && mb >= 0 && mb < n);
  e->bin = e->bad_bin ? -1 : (int)(((long)kb * n + (long)tb) * n + (long)mb);
  return 1;
}

/* p2 range of barbie.c:257-268 by ring equality. */
static void p2_limits(int p1, long Nmax, int r1, int r2, int r3, int *lo, int *hi) {
  if (r1 == r2 && r2 == r3) {
    *lo = 0; *hi = p1;
  } else if (r1 == r2) {
    *lo = -p1; *hi = p1;
  } else if (r2 == r3) {
    *lo = (int)(-p1 / 2); *hi = (int)Nmax;
  } else {
    *lo = (p1 == 0) ? 0 : (int)(-Nmax + 1); *hi = (int)Nmax;
  }
}

/* Acceptance alone (barbie.c:285,292): |p3| < Nmax and LL_k1 < K1 < UL_k1,
 * K1 the largest of the three legs' |K| -- the same sqrt expressions as
 * eval_triangle, so the same triangles pass. */
static int accepted(const beam_geom *g, int r1, int r2, int r3, int p1, int p2) {
  int p3 = -p1 - p2;
  if (!((p3 < 0 ? -p3 : p3) < g->Nmax)) return 0;
  const double *a = g->avg;
  double k1 = sqrt(a[r1] * a[r1] + p1 * p1), k2 = sqrt(a[r2] * a[r2] + p2 * p2), k3 = sqrt(a[r3] * a[r3] + p3 * p3);
  double K1 = k1 > k2 ? k1 : k2;
  K1 = K1 > k3 ? K1 : k3;
  return K1 > g->LL_k1 && K1 < g->UL_k1;
}

/* The loop is split over p1 (the reference's outer loop) between threads; each
 * p1 first counts, then fills its own slice, so triangles keep loop order.
 * A leg's |K| = sqrt(avg^2 + p^2) is at least |p|, so no triangle with a plane
 * |p| >= UL_k1 passes the k1 window: those iterations are counted, not
 * visited. */
typedef struct {
  beam_geom *g;
  long *count;       /* [Nmax] accepted per p1 */
  long *offset;      /* [Nmax] first triangle of p1 */
  long *iters;       /* [Nmax] visits per p1 */
  int *bad;          /* [Nmax] out-of-range bins met */
  int fill;
  long next;         /* next p1 to take */
  pthread_mutex_t lock;
} enum_job;

static void enumerate_p1(enum_job *job, int p1) {
  beam_geom *g = job->g;
  long n = 0, it = 0, at = job->fill ? job->offset[p1] : 0;
  const int U = g->UL_k1;
  for (long rp = 0; rp < g->nrp; ++rp) {
    int r1 = g->rp[3 * rp], r2 = g->rp[3 * rp + 1], r3 = g->rp[3 * rp + 2];
    int lo, hi;
    p2_limits(p1, g->Nmax, r1, r2, r3, &lo, &hi);
    if (hi >= lo) it += hi - lo + 1;
    if (p1 >= U) continue;
    /* |p2| < U and |p1 + p2| < U */
    int clo = lo > -U + 1 ? lo : -U + 1, chi = hi < U - 1 ? hi : U - 1;
    if (clo < -U + 1 - p1) clo = -U + 1 - p1;
    if (chi > U - 1 - p1) chi = U - 1 - p1;
    for (int p2 = clo; p2 <= chi; ++p2) {
      if (!job->fill) {
        n += accepted(g, r1, r2, r3, p1, p2);
        continue;
      }
      tri_eval e;
      if (!eval_triangle(g, r1, r2, r3, p1, p2, &e)) continue;
      if (e.bad_bin) job->bad[p1] = 1;
      if (at >= job->offset[p1] + job->count[p1]) { /* the count pass disagreed: never write past p1's slice */
        job->bad[p1] |= 2;
        continue;
      }
      {
        g->t_rp[at] = (int32_t)rp;
        g->t_p1[at] = p1;
        g->t_p2[at] = p2;
        g->t_bin[at] = e.bin;
        g->t_px[at] = e.px;
        g->t_pz[at] = e.pz;
        g->t_ana[at] = e.ana;
        ++at;
      }
      ++n;
    }
  }
  if (!job->fill) {
    job->count[p1] = n;
    job->iters[p1] = it;
  }
}

static void *enum_worker(void *arg) {
  enum_job *job = (enum_job *)arg;
  for (;;) {
    pthread_mutex_lock(&job->lock);
    long p1 = job->next++;
    pthread_mutex_unlock(&job->lock);
    if (p1 >= job->g->Nmax) break;
    enumerate_p1(job, (int)p1);
  }
  return NULL;
}

static void run_pass(enum_job *job, int nthreads) {
  job->next = 0;
  pthread_t th[64];
  int started = 0;
  for (int t = 0; t < nthreads && t < 64; ++t)
    if (pthread_create(&th[t], NULL, enum_worker, job) == 0) ++started;
  if (started == 0) enum_worker(job);
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
}

static int build_triangles(beam_geom *g) {
  long Nmax = g->Nmax;
  enum_job job;
  memset(&job, 0, sizeof(job));
  job.g = g;
  job.count = (long *)calloc((size_t)Nmax, sizeof(long));
  job.offset = (long *)calloc((size_t)Nmax, sizeof(long));
  job.iters = (long *)calloc((size_t)Nmax, sizeof(long));
  job.bad = (int *)calloc((size_t)Nmax, sizeof(int));
  if (!job.count || !job.offset || !job.iters || !job.bad) {
    free(job.count); free(job.offset); free(job.iters); free(job.bad);
    return BEAM_ENOMEM;
  }
  pthread_mutex_init(&job.lock, NULL);
  long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
  int nthreads = (int)(ncpu > 32 ? 32 : (ncpu < 1 ? 1 : ncpu));
  if (nthreads > Nmax) nthreads = (int)Nmax;

  run_pass(&job, nthreads);
  long total = 0, iters = 0;
  int bad = 0;
  for (long p = 0; p < Nmax; ++p) {
    job.offset[p] = total;
    total += job.count[p];
    iters += job.iters[p];
  }
  int rc = BEAM_OK;
  size_t n = (size_t)(total > 0 ? total : 1);
  g->t_rp = (int32_t *)malloc(sizeof(int32_t) * n);
  g->t_p1 = (int32_t *)malloc(sizeof(int32_t) * n);
  g->t_p2 = (int32_t *)malloc(sizeof(int32_t) * n);
  g->t_bin = (int32_t *)malloc(sizeof(int32_t) * n);
  g->t_px = (double *)malloc(sizeof(double) * n);
  g->t_pz = (double *)malloc(sizeof(double) * n);
  g->t_ana = (double *)malloc(sizeof(double) * n);
  if (!g->t_rp || !g->t_p1 || !g->t_p2 || !g->t_bin || !g->t_px || !g->t_pz || !g->t_ana) {
    rc = BEAM_ENOMEM;
  } else {
    job.fill = 1;
    run_pass(&job, nthreads);
    g->ntri = total;
    g->iterations = iters;
    for (long p = 0; p < Nmax; ++p) bad |= job.bad[p];
    if (bad & 2) rc = BEAM_EINVAL; /* count and fill passes disagree (not expected) */
    else if (bad) rc = BEAM_EBOUNDS;
  }
  pthread_mutex_destroy(&job.lock);
  free(job.count); free(job.offset); free(job.iters); free(job.bad);
  return rc;
}

int beam_geom_build(beam_geom *g, const beam_cfg *cfg) {
  memset(g, 0, sizeof(*g));
  if (!cfg || cfg->NN < 4 || cfg->NN % 2 || cfg->NN > 4096 || cfg->Nmax < 1 || cfg->Nmax > cfg->NN / 2 ||
      cfg->Nr < 10 || cfg->Nr % 10 || cfg->Nr > 1000 || cfg->BW_k1 <= 0 || cfg->UL_k1 <= cfg->LL_k1 ||
      (cfg->UL_k1 - cfg->LL_k1) % cfg->BW_k1 != 0 || cfg->n_mtbin < 1 || cfg->n_mtbin > 64 || !(cfg->LL > 0))
    return BEAM_EINVAL;
  g->NN = cfg->NN;
  g->Nmax = cfg->Nmax;
  g->Nr = cfg->Nr;
  g->UL_k1 = cfg->UL_k1;
  g->LL_k1 = cfg->LL_k1;
  g->BW_k1 = cfg->BW_k1;
  g->n_mtbin = cfg->n_mtbin;
  g->n_k1bin = (int)((cfg->UL_k1 - cfg->LL_k1) / (1. * cfg->BW_k1));
  g->LL = cfg->LL;
  g->vol = pow((double)g->NN * g->LL, 3);
  g->low = (double *)calloc((size_t)g->Nr, sizeof(double));
  g->high = (double *)calloc((size_t)g->Nr, sizeof(double));
  g->avg = (double *)calloc((size_t)g->Nr, sizeof(double));
  if (!g->low || !g->high || !g->avg) {
    beam_geom_free(g);
    return BEAM_ENOMEM;
  }
  int rc = beam_ring_edges(g->Nr, g->Nmax, g->low, g->high, g->avg);
  if (rc == BEAM_OK) rc = build_ringmap(g);
  if (rc == BEAM_OK) rc = build_triplets(g);
  if (rc == BEAM_OK) rc = build_triangles(g);
  if (rc != BEAM_OK && rc != BEAM_EBOUNDS) beam_geom_free(g);
  return rc;
}
