/* Counter-based normal deviates for the field generator's oracle and for the
 * GSL stand-in that the reference generator is compiled against
 * (oracle/gsl_shim.c). Test infrastructure only.
 *
 * The reference draws its Gaussian modes from GSL (gsl_rng_mt19937 seeded with
 * gsl_rng_set, gsl_ran_gaussian_ziggurat; ngrf_2d_funcs.c:356-360). GSL is not
 * vendored with the reference and not installed here, so its stream cannot be
 * reproduced. Draw n of a stream with seed s is instead
 *
 *   (x0, x1, x2, x3) = Philox4x32-10(counter = (n mod 2^32, n / 2^32, 0, 0),
 *                                    key = (s mod 2^32, s / 2^32))
 *   u1 = ((x1:x0 >> 11) + 1) * 2^-53     in (0, 1]
 *   u2 =  (x3:x2 >> 11)      * 2^-53     in [0, 1)
 *   g  = sqrt(-2 ln u1) * cos(2 pi u2)   (Box-Muller)
 *
 * Philox4x32-10 is the counter-based generator of Salmon, Moraes, Dror and
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of
 * two 32x32->64 multiplies (0xD2511F53, 0xCD9E8D57), the key bumped by the
 * Weyl constants (0x9E3779B9, 0xBB67AE85) between rounds. A counter-based
 * stream lets the GPU compute every draw where it is used; the GPU library has
 * its own implementation of the same definition. */
#ifndef BEAM_PHILOX_NORMAL_H
#define BEAM_PHILOX_NORMAL_H

#include <math.h>
#include <stdint.h>

static inline void orc_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1, n3 = (uint32_t)p0;
    c[0] = n0, c[1] = n1, c[2] = n2, c[3] = n3;
    if (r < 9) k0 += 0x9E3779B9u, k1 += 0xBB67AE85u;
  }
}

static inline double orc_normal(uint64_t seed, uint64_t n) {
  uint32_t c[4] = {(uint32_t)n, (uint32_t)(n >> 32), 0u, 0u};
  orc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t a = (((uint64_t)c[1] << 32) | c[0]) >> 11, b = (((uint64_t)c[3] << 32) | c[2]) >> 11;
  const double u1 = (double)(a + 1) * 0x1.0p-53, u2 = (double)b * 0x1.0p-53;
  return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

#endif
