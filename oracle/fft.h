/* CPU FP64 discrete Fourier transforms for the oracle (test infrastructure only).
 *
 * The reference links FFTW3 (Makefile:3) and uses exactly one transform on the
 * estimator path: an unnormalised 2D complex backward DFT, planned with
 * fftw_plan_dft_2d(NN, NN, ..., FFTW_BACKWARD, FFTW_ESTIMATE) (funcs.c:349,546).
 * FFTW is not vendored and not installed here, so this file restates the
 * mathematical definition FFTW documents for that call:
 *
 *     out[j0][j1] = sum_{k0,k1} in[k0][k1] * exp(sign * 2*pi*i * (j0*k0/n0 + j1*k1/n1))
 *
 * with sign = +1 for backward, and no scaling. Sizes 2^a * 3^b use a mixed
 * radix 2/3/4 decimation-in-time recursion; any other factor falls back to a
 * direct DFT of that factor. Twiddles are taken from one table of
 * exp(sign*2*pi*i*j/n) evaluated with libm cos/sin per entry.
 */
#ifndef BEAM_ORACLE_FFT_H
#define BEAM_ORACLE_FFT_H

#ifdef __cplusplus
extern "C" {
#endif

/* In-place 1D DFT of n complex values (interleaved re,im) with given sign (+1 backward, -1 forward). */
void orc_fft1d(long n, int sign, double *data);

/* In-place 2D DFT of an n0 x n1 row-major complex array (interleaved re,im). */
void orc_fft2d(long n0, long n1, int sign, double *data);

/* orc_fft2d with the row and column passes spread over nthreads OpenMP threads. */
void orc_fft2d_threads(long n0, long n1, int sign, double *data, int nthreads);

/* In-place 3D DFT of an n0 x n1 x n2 row-major complex array (interleaved re,im). */
void orc_fft3d(long n0, long n1, long n2, int sign, double *data);

/* The two real 3D transforms the reference's field generator plans in place on
 * a double[n0][n1][n2+2] buffer (fftw_plan_dft_r2c_3d / fftw_plan_dft_c2r_3d,
 * generate_field.c:78-79), by their FFTW definitions:
 *   r2c: the unnormalised forward DFT (sign -1) of the n0*n1*n2 real values
 *        x[i][j][k] (k < n2 of each padded row), keeping the n2/2+1 complex
 *        values k2 <= n2/2 of each row;
 *   c2r: the unnormalised backward DFT (sign +1) of the Hermitian extension
 *        X[i][j][n2-k] = conj X[-i][-j][k] of the half spectrum; the real parts
 *        are written to k < n2 of each row (the imaginary parts of an exactly
 *        Hermitian input cancel).
 * Both go through one complex n0*n1*n2 array. */
void orc_r2c_3d(long n0, long n1, long n2, double *padded);
void orc_c2r_3d(long n0, long n1, long n2, double *padded);

#ifdef __cplusplus
}
#endif
#endif
