/* Host-side estimator geometry for libbeam_gpu: everything that depends only on
 * the configuration (not on the field). Compiled as C with IEEE double
 * semantics (no FMA contraction, no fast-math) so that ring membership, the
 * closure tests, K1/T/MU/px/pz and the bin indices are bit-identical to the
 * reference's own C expressions. */
#ifndef BEAM_GEOMETRY_H
#define BEAM_GEOMETRY_H

#include <stdint.h>

#include "beam_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct beam_geom {
  long NN, Nmax, Nr;
  int UL_k1, LL_k1, BW_k1, n_mtbin, n_k1bin;
  double LL, vol;
  double *low, *high, *avg; /* [Nr] ring edges and midpoints */
  int16_t *ringmap;         /* [NN*NN] ring of pixel (i,j), or -1 */

  long nrp;                 /* closed ring triplets, reference order */
  int32_t *rp;              /* [nrp][3] = r1, r2, r3 */

  long ntri;                /* accepted triangles, loop order */
  int32_t *t_rp;            /* [ntri] ring triplet index */
  int32_t *t_p1, *t_p2;     /* [ntri] planes of legs 1 and 2 (p3 = -p1-p2) */
  int32_t *t_bin;           /* [ntri] flattened (k1_bin, t_bin, mu_bin) */
  double *t_px, *t_pz;      /* [ntri] orientation parameters */
  double *t_ana;            /* [ntri] analytic bispectrum of the triangle (barbie.c:300-305) */
  long iterations;          /* (p1, rp, p2) loop iterations visited */
} beam_geom;

/* Build the geometry. Returns BEAM_OK, BEAM_EINVAL, BEAM_ENOMEM or BEAM_EBOUNDS. */
BEAM_API int beam_geom_build(beam_geom *g, const beam_cfg *cfg);
BEAM_API void beam_geom_free(beam_geom *g);

/* Ring edges of barbie.c:110-130 (exposed for tests and the host drop-in). */
BEAM_API int beam_ring_edges(long Nr, long Nmax, double *low, double *high, double *avg);

#ifdef __cplusplus
}
#endif
#endif
