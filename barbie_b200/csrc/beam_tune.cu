// Autotuner of the triangle-sum work decomposition (beam_gpu_plan_autotune).
//
// The decomposition of a plan's triangle sums into CTA work items has two
// free parameters (build_work in beam_plan.cu):
//   tau0     the first cap on the in-plane triangles one CTA walks -- the
//            split-K factor of each ring triplet's triangle list (the cap
//            doubles while the partial sums would outgrow their budget);
//   balance  how many items' worth of work per SM the load balance aims at
//            (more, smaller items: better tail balance, more partial sums).
// Their best values depend on the geometry (NN, Nmax, Nr, bins) and the
// device. The tuner rebuilds the plan's tables for each candidate, fills the
// mode data with a fixed pseudo-random pattern, times the triangle phase
// (triangle sums + split reduction) with CUDA events on the plan's stream,
// and keeps the fastest. Results are the same to round-off for every
// candidate (only the order of the partial sums changes).
#include <algorithm>
#include <vector>

#include "beam_internal.h"

namespace beam {

// a fixed pseudo-random pattern in [-1, 1) for every staged mode value
__global__ void k_fill_pattern(double *__restrict__ v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long x = (i + 1) * 0x9E3779B97F4A7C15ull;
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 29;
    v[i] = (double)(x >> 11) * 0x1.0p-52 - 1.0;
  }
}
__global__ void k_fill_pattern_f(float *__restrict__ v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned x = (unsigned)(i + 1) * 0x9E3779B9u;
    x ^= x >> 15;
    x *= 0x2C1B3C6Du;
    x ^= x >> 12;
    v[i] = (float)(x >> 8) * 0x1.0p-23f - 1.0f;
  }
}

int ctx_scratch(beam_gpu_ctx *ctx, size_t bytes, void **out) {
  if (ctx->scratch_bytes < bytes) {
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    size_t got = 0;
    char *p = nullptr;
    int rc = dev_alloc(&got, &p, bytes);
    if (rc != BEAM_OK) return rc;
    ctx->scratch = p;
    ctx->scratch_bytes = bytes;
  }
  *out = ctx->scratch;
  return BEAM_OK;
}

int fill_pattern(double *v, size_t n, cudaStream_t st, int num_sms) {
  k_fill_pattern<<<4 * std::max(1, num_sms), 256, 0, st>>>(v, n);
  BEAM_CUDA(cudaGetLastError());
  return BEAM_OK;
}

// the plan's tables and main slot rebuilt for the given decomposition
static int rebuild(beam_gpu_plan *p, long long tau0, double balance) {
  slot_destroy(p->main);
  p->main = nullptr;
  for (RunSlot *&s : p->batch) {
    slot_destroy(s);
    s = nullptr;
  }
  free_plan_tables(p);
  p->device_bytes = 0;
  p->tau0 = tau0;
  p->balance = balance;
  int rc = host_guard([&] { return build_plan_tables(p); });
  if (rc == BEAM_OK) rc = host_guard([&] { return slot_create(p, 1, &p->ctx->lane, &p->main); });
  return rc;
}

// triangle phase of one realization on the pattern, best of reps (ms)
static int time_triangle_phase(beam_gpu_plan *p, int reps, float *best) {
  RunSlot *s = p->main;
  cudaStream_t st = p->ctx->stream;
  const size_t n = (size_t)p->d.n_modes * p->d.W * 2;  // real values of one realization's S
  if (p->d.elem == sizeof(float2))
    k_fill_pattern_f<<<4 * p->ctx->num_sms, 256, 0, st>>>((float *)s->S, n);
  else  // FP64 rows (the int8 path's come first, its slice tables are cut from them)
    k_fill_pattern<<<4 * p->ctx->num_sms, 256, 0, st>>>((double *)s->S, n);
  BEAM_CUDA(cudaGetLastError());
  if (p->d.i8) BEAM_TRY(build_slices(p, s, 1));
  cudaEvent_t e0, e1;
  BEAM_CUDA(cudaEventCreate(&e0));
  BEAM_CUDA(cudaEventCreate(&e1));
  *best = 1e30f;
  int rc = BEAM_OK;
  for (int r = -1; r < reps && rc == BEAM_OK; ++r) {  // r = -1: warm-up
    cudaEventRecord(e0, st);
    rc = run_triangle_sums(p, s, 1);
    cudaEventRecord(e1, st);
    if (rc == BEAM_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = BEAM_ECUDA;
    float ms = 0.f;
    if (rc == BEAM_OK && r >= 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) *best = std::min(*best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == BEAM_OK) rc = check_status(s);
  return rc;
}

}  // namespace beam

using namespace beam;

extern "C" int beam_gpu_plan_autotune(beam_gpu_plan *p, int reps, beam_tune_report *rep) {
  if (!p || p->cfg.method != BEAM_METHOD_TRIANGLE) {
    set_detail("autotune: a triangle-method plan is required");
    return BEAM_EINVAL;
  }
  if (reps <= 0) reps = 3;
  reps = std::min(reps, 20);
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  BEAM_CUDA(cudaStreamSynchronize(p->ctx->stream));
  static const long long taus[] = {256, 512, 1024, 2048};
  static const double bals[] = {4.0, 8.0, 16.0};
  struct Cand {
    long long tau0;
    double balance;
    float ms;
    int items;
  };
  std::vector<Cand> cands;
  for (long long t : taus)
    for (double b : bals) cands.push_back(Cand{t, b, 0.f, 0});
  static_assert(sizeof(taus) / sizeof(taus[0]) * sizeof(bals) / sizeof(bals[0]) <= BEAM_TUNE_MAX, "report size");
  int rc = BEAM_OK;
  for (Cand &c : cands) {
    rc = rebuild(p, c.tau0, c.balance);
    if (rc == BEAM_OK) rc = time_triangle_phase(p, reps, &c.ms);
    if (rc != BEAM_OK) break;
    c.items = p->d.n_items;
  }
  size_t best = 0;
  for (size_t k = 1; k < cands.size(); ++k)
    if (cands[k].ms < cands[best].ms) best = k;
  // the kept decomposition, with fresh (zeroed) run buffers; after a failure
  // the default one
  const int rc2 = rc == BEAM_OK ? rebuild(p, cands[best].tau0, cands[best].balance) : rebuild(p, p->cfg.precision == BEAM_PREC_FP64 ? 2 * TRI_TAU_MAX : TRI_TAU_MAX, 8.0);
  if (rc == BEAM_OK) rc = rc2;
  if (rep && rc == BEAM_OK) {
    rep->n = (int)cands.size();
    rep->best = (int)best;
    for (size_t k = 0; k < cands.size(); ++k) {
      rep->tau0[k] = cands[k].tau0;
      rep->balance[k] = cands[k].balance;
      rep->ms[k] = cands[k].ms;
      rep->items[k] = cands[k].items;
    }
  }
  return rc;
}
