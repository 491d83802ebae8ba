/* Drop-in for the reference's field generator `field NN NRi`
 * (generate_field.c + ngrf_2d_funcs.c of sukhdeepsinghgill/BARBIE), running
 * on a B200 through libbeam_gpu (beam_gpu_field_generate).
 *
 * Same command line, messages and output as the reference:
 *   output  ResFiles_N<NN>/data_files/field_N<NN>_R<NRi>.txt, raw native
 *           doubles, r2c layout [NN][NN][NN+2] (generate_field.c:100-109) --
 *           the input of `barbie` and `calpow_mom`
 * with the reference's constants: cell size 0.56, ff = 0.5, beta = 1, seed
 * 100020 + 146 NRi (generate_field.c:45-50). The Gaussian draws are the
 * library's counter-based stream, not GSL's, so the field is a different
 * realization with the same statistics. BEAM_DEVICE picks the CUDA device. */
#include <stdio.h>
#include <stdlib.h>

#include "beam_gpu.h"

int main(int argc, char *argv[]) {
  if (argc != 3) {
    printf("Usage: %s <Number of Grids> <Realization>\n", argv[0]);
    return 1;
  }
  long NN = atol(argv[1]);
  int NRi = atoi(argv[2]);
  printf("\n Generating field Realization(NRi) = %d for Grids(NN) = %ld\n\n", NRi, NN);
  const double LL = 0.56, ff = 0.5, beta = 1.;
  const unsigned long long seed = 100020 + 146 * (unsigned long long)NRi;
  if (NN < 4 || NN > 1024) {
    fprintf(stderr, "field: NN must be 2^a 3^b, even, in [4, 1024]\n");
    return 1;
  }
  const size_t n = (size_t)NN * NN * (NN + 2);
  char path[256];
  snprintf(path, sizeof(path), "ResFiles_N%ld/data_files/field_N%ld_R%d.txt", NN, NN, NRi);
  FILE *fp = fopen(path, "wb");
  if (!fp) {
    fprintf(stderr, "field: cannot write %s\n", path);
    return 1;
  }
  const char *dev = getenv("BEAM_DEVICE");
  beam_gpu_ctx *ctx = NULL;
  int rc = beam_gpu_init(dev ? atoi(dev) : 0, &ctx);
  double *field = NULL;
  double sigma = 0.0;
  if (rc == BEAM_OK) {
    field = (double *)malloc(sizeof(double) * n);
    rc = field ? beam_gpu_field_generate(ctx, NN, seed, LL, ff, beta, field, 0, &sigma) : BEAM_ENOMEM;
  }
  if (rc != BEAM_OK) {
    fclose(fp);
    remove(path);
    fprintf(stderr, "field: %s: %s\n", beam_gpu_strerror(rc), beam_gpu_last_error_detail());
    free(field);
    beam_gpu_destroy(ctx);
    return 1;
  }
  fprintf(stdout, "sigma = %e\n", sigma);
  size_t put = fwrite(field, sizeof(double), n, fp);
  int bad = fclose(fp) != 0 || put != n;
  free(field);
  beam_gpu_destroy(ctx);
  if (bad) {
    fprintf(stderr, "field: short write to %s\n", path);
    return 1;
  }
  return 0;
}
