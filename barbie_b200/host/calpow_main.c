/* Drop-in for the reference's power-spectrum-multipole program
 * `calpow_mom NN NRi` (calpow_mom.c of sukhdeepsinghgill/BARBIE), running on a
 * B200 through libbeam_gpu.
 *
 * Same command line, input and output as the reference:
 *   input   ResFiles_N<NN>/data_files/field_N<NN>_R<NRi>.txt  raw native doubles,
 *           r2c layout [NN][NN][NN+2] (calpow_mom.c:72-81)
 *   output  ResFiles_N<NN>/psoutN<NN>_R<NRi>.dat, rows "%e\t%e\t%e\t%e\t%e\t%e\n" =
 *           mean k, P0, P2, P4, P6, mode count for the bins with modes
 *           (calpow_mom.c:109-117)
 * with the reference's constants: cell size 0.56, 10 bins (calpow_mom.c:50,91).
 * BEAM_PRINT_DIGITS (optional) prints more significant digits; BEAM_DEVICE picks
 * the CUDA device. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "beam_gpu.h"

int main(int argc, char *argv[]) {
  if (argc != 3) {
    printf("Usage: %s NN(384) NRi(1) UL_k1(Nmax) LL_k1(Nmax-10) BW_k1(1)\n", argv[0]);
    return 1;
  }
  long NN = atol(argv[1]);
  int NRi = atoi(argv[2]);
  printf("\n Calculating PS Multipoles for Realization(NRi) = %d and Grids(NN) = %ld\n", NRi, NN);
  if (NN < 2 || NN % 2 || NN > 4096) {
    fprintf(stderr, "calpow_mom: NN must be even and at most 4096\n");
    return 1;
  }
  const double LL = .56;
  const int NB = 10;
  char path[256];
  snprintf(path, sizeof(path), "ResFiles_N%ld/data_files/field_N%ld_R%d.txt", NN, NN, NRi);
  FILE *fp = fopen(path, "rb");
  if (!fp) {
    fprintf(stderr, "calpow_mom: cannot open %s\n", path);
    return 1;
  }
  size_t n = (size_t)NN * NN * (NN + 2);
  double *field = (double *)malloc(sizeof(double) * n);
  if (!field) {
    fclose(fp);
    fprintf(stderr, "calpow_mom: out of host memory\n");
    return 1;
  }
  size_t got = fread(field, sizeof(double), n, fp);
  fclose(fp);
  if (got != n) {
    fprintf(stderr, "calpow_mom: %s holds %zu of %zu doubles\n", path, got, n);
    return 1;
  }
  const char *dev = getenv("BEAM_DEVICE");
  beam_gpu_ctx *ctx = NULL;
  int rc = beam_gpu_init(dev ? atoi(dev) : 0, &ctx);
  if (rc) {
    fprintf(stderr, "calpow_mom: %s: %s\n", beam_gpu_strerror(rc), beam_gpu_last_error_detail());
    return 1;
  }
  double out[6 * NB];
  rc = beam_gpu_power_multipoles(ctx, NN, LL, NB, field, 0, out);
  if (rc) {
    fprintf(stderr, "calpow_mom: %s: %s\n", beam_gpu_strerror(rc), beam_gpu_last_error_detail());
    return 1;
  }
  snprintf(path, sizeof(path), "ResFiles_N%ld/psoutN%ld_R%d.dat", NN, NN, NRi);
  fp = fopen(path, "w");
  if (!fp) {
    fprintf(stderr, "calpow_mom: cannot write %s\n", path);
    return 1;
  }
  const char *dg = getenv("BEAM_PRINT_DIGITS");
  int digits = dg ? atoi(dg) : 0;
  for (int i = 0; i < NB; ++i)
    if (out[5 * NB + i] > 0) {
      if (digits > 0)
        fprintf(fp, "%.*e\t%.*e\t%.*e\t%.*e\t%.*e\t%.*e\n", digits - 1, out[i], digits - 1, out[NB + i], digits - 1,
                out[2 * NB + i], digits - 1, out[3 * NB + i], digits - 1, out[4 * NB + i], digits - 1,
                out[5 * NB + i]);
      else
        fprintf(fp, "%e\t%e\t%e\t%e\t%e\t%e\n", out[i], out[NB + i], out[2 * NB + i], out[3 * NB + i],
                out[4 * NB + i], out[5 * NB + i]);
    }
  fclose(fp);
  beam_gpu_destroy(ctx);
  free(field);
  return 0;
}
