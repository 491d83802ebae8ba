/* Oracle: a plain-C CPU restatement of the BEAM bispectrum estimator hot path
 * (reference: barbie.c + funcs.c of sukhdeepsinghgill/BARBIE).
 *
 * TEST INFRASTRUCTURE ONLY. The pytest suite, the smoke entry point and the
 * benchmark's CPU-baseline leg compare against it or time it; the GPU product
 * library (libbeam_gpu.so) never links or calls it.
 *
 * Parity of this restatement is pinned against the reference program itself,
 * compiled from its own sources with an FFTW-API shim (oracle/Makefile), on the
 * golden cases committed under tests/golden/.
 *
 * Array conventions follow the reference:
 *   r2c   : double[NN][NN][NN+2]   FFTW in-place r2c buffer (barbie.c:176-185)
 *   plane : double[NN][NN][2]      one (plane, ring) transform (funcs.c:88-109)
 *   bins  : double[n_k1bin][n_mtbin][n_mtbin][16]  (barbie.c:87)
 */
#ifndef BEAM_ORACLE_H
#define BEAM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NPOLES 16

/* Ring edges, barbie.c:110-130. Nr must be a multiple of 10. Returns 0 or -1. */
int orc_ring_edges(long Nr, long Nmax, double *low, double *high, double *avg);

/* Ring masks RR[Nr][NN][NN], barbie.c:135-148. */
void orc_ring_masks(long NN, long Nr, const double *low, const double *high, double *RR);

/* calCR, funcs.c:328-424: closed sorted ring triplets and their FFT-based
 * triangle sums Num = sum_x I1*I2*I3. Writes up to cap records of
 * {r1,r2,r3,Num} into out4; returns the number of triplets found. */
long orc_closed_rings(long NN, long Nr, const double *low, const double *high,
                      const double *avg, double *out4, long cap);

/* Exact integer in-plane triangle count of one ring triplet by direct lattice
 * enumeration: #{(k1,k2,k3) in R1 x R2 x R3 : k1+k2+k3 = 0 mod NN}.
 * This is what funcs.c:396-399 computes as Num/NN^2 up to FFT round-off. */
int64_t orc_triangle_count_direct(long NN, const double *RR, long r1, long r2, long r3);

/* Df, funcs.c:88-109 (sign=+1 only): gather plane p of the r2c buffer, mask
 * with ring r, zero k_perp=0 on plane 0, unnormalised 2D backward DFT. */
void orc_plane_ring(long NN, long p, long r, const double *r2c, const double *RR, double *out);

/* cal_coeff, funcs.c:708-745: the 16 orientation weights and norms. */
void orc_cal_coeff(double px, double pz, double *bs, double *norm);

/* One accepted triangle of the loop barbie.c:247-298. */
typedef struct {
  int32_t p1, r1, p2, r2, p3, r3; /* planes (signed) and rings of the three legs */
  int32_t rp;                     /* index of the ring triplet */
  int32_t k1_bin, t_bin, mu_bin;  /* bins, barbie.c:343-345 */
  double K1, T, MU, px, pz;       /* shape parameters, barbie.c:293-297 */
  double num;                     /* rdata[rp][3], barbie.c:298 */
  double leg_k[3], leg_p[3];      /* sorted legs K[i][0], K[i][1] (barbie.c:285-287) */
} orc_triple;

/* Enumerate the accepted triangles in the reference's loop order
 * (p1 outer, rp middle, p2 inner; barbie.c:247-292). If out is non-NULL up
 * to cap records are written. Returns the total number of accepted triangles,
 * and the number of (p1,rp,p2) iterations through *iterations if non-NULL. */
long orc_enumerate(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, int n_mtbin,
                   const double *avg, const double *rings4, long rcount,
                   orc_triple *out, long cap, long *iterations);

/* The complete estimator (barbie.c:110-397 with funcs.c helpers) on an r2c
 * buffer held in memory, the plane-ring cache held in RAM instead of on disk.
 * Outputs (caller-allocated, n_k1bin*n_mtbin*n_mtbin*16 doubles each):
 *   bin_bs    accumulated sum B*bs            (bin_BS_real before line 390)
 *   bin_norm  accumulated sum Num*norm        (bin_normalization)
 *   bin_out   bin_bs/(vol*bin_norm)           (barbie.c:390)
 * counts (optional, n_k1bin*n_mtbin*n_mtbin int64): sum over accepted
 * triangles with B != 0 of the exact integer triangle count round(Num/NN^2).
 * B per accepted triangle in enumeration order is written to tri_B if non-NULL.
 * bin_ana (optional, same shape as bin_bs): sum of Biana*Num*bs, the analytic
 * bispectrum accumulator of barbie.c:300-305,356-361 started from zero (the
 * reference prints bin_ana/bin_norm as column 5, barbie.c:391-393).
 * nthreads > 1 splits the pixel sums over OpenMP threads.
 * Returns 0, or -1 on invalid arguments / allocation failure. */
int orc_estimate(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, int n_mtbin,
                 double LL, const double *r2c, double *bin_bs, double *bin_norm, double *bin_out,
                 int64_t *counts, double *tri_B, long tri_cap, int nthreads, double *bin_ana);

/* orc_estimate with the per-triangle pixel sums accumulated in long double
 * when wide != 0 (same pixel order; the bins then carry far less of the
 * oracle's own rounding, for fixtures at NN >= 384). */
int orc_estimate_ex(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, int n_mtbin,
                    double LL, const double *r2c, double *bin_bs, double *bin_norm, double *bin_out,
                    int64_t *counts, double *tri_B, long tri_cap, int nthreads, double *bin_ana, int wide);

/* barbie.c:300-305: analytic redshift-space bispectrum of a triangle from its
 * sorted legs (|K_i|, p_i) in grid units, cell size LL: P(k) = k^-2
 * (input_ps, funcs.c:73-81), ff = 0.1, beta = 1 (barbie.c:79-80). */
double orc_biana(long NN, double LL, const double leg_k[3], const double leg_p[3]);
/* orc_biana of each of n enumerated triangles. */
void orc_biana_all(long NN, double LL, const orc_triple *tri, long n, double *out);

/* CPU-baseline timing on a bounded sample of one bispectrum's work: the
 * plane-ring transforms (Df) the sampled accepted triangles need and their
 * pixel sums (barbie.c:329-337), each stage spread over nthreads OpenMP
 * threads. sample[] holds triangle indices in loop order. Outputs: wall
 * seconds of the transforms (*t_fft over *n_fft arrays) and of the sums
 * (*t_sum), and the sum of the sampled B values (*checksum). */
int orc_time_sample(long NN, long Nmax, long Nr, int UL_k1, int LL_k1, int BW_k1, const double *r2c,
                    const long *sample, long nsample, int nthreads, double *t_fft, long *n_fft, double *t_sum,
                    double *checksum);

/* The pixel sum of barbie.c:329-337 for one triangle, given three plane-ring
 * arrays (stored for planes |p| >= 0) and the conjugation signs. */
double orc_triple_product(long NN, const double *F1, const double *F2, const double *F3, int sign2, int sign3);

/* funcs.c:860-1074 (calpow_mom): power spectrum multipoles P0, P2, P4, P6 of the
 * r2c buffer in Nbin logarithmic |k| bins, cell size LL. out: [6][Nbin] =
 * kmode, P0, P2, P4, P6, mode count (the columns of calpow_mom.c:115). */
int orc_power_multipoles(long NN, double LL, int Nbin, const double *r2c, double *out);

/* Field generator (field_oracle.c). Normal deviates: orc_normal of
 * philox_normal.h, draw n of the stream with the given seed.
 *
 * Fill_Modes (ngrf_2d_funcs.c:341-510): the Gaussian modes of the half-complex
 * array A[N][N][N/2+1] (interleaved re,im), amplitude sqrt(vol/2 * k^-2). */
void orc_field_fill_modes(long N, uint64_t seed, double LL, double *A);
/* generate_field.c:81-86: Fill_Modes, Make_Image, Non_Gauss (x += ff (x^2 - var)),
 * Get_Modes, RSD(beta), into the r2c buffer double[N][N][N+2]; sigma = sqrt(var)
 * of the Gaussian image. Returns 0, or -1 on invalid arguments. */
int orc_field_generate(long N, uint64_t seed, double LL, double ff, double beta, double *r2c, double *sigma);
/* A real-space cube double[N][N][N] to the r2c buffer: Get_Modes (x LL^3, r2c
 * transform, ngrf_2d_funcs.c:534-550) and RSD(beta) (ngrf_2d_funcs.c:734-765). */
int orc_field_ingest(long N, double LL, double beta, const double *cube, double *r2c);

#ifdef __cplusplus
}
#endif
#endif
