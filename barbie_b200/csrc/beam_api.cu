// C-ABI entry points of libbeam_gpu (declared in include/beam_gpu.h).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>

#include "beam_internal.h"

namespace beam {
static thread_local std::string g_detail;
void set_detail(const std::string &s) { g_detail = s; }
int plane_rings(beam_gpu_plan *p, const double *r2c, int on_device, const int *planes, const int *rings, int n,
                double *out, int out_on_device);
int pixel_triangle_sums(beam_gpu_plan *p, const double *r2c, int on_device);
bool pixel_method(const beam_gpu_plan *p);
int build_pixel_path(beam_gpu_plan *p);
void free_pixel_path(beam_gpu_plan *p);
}  // namespace beam

using namespace beam;

extern "C" {

void beam_cfg_default(beam_cfg *cfg, long NN, int UL_k1, int LL_k1, int BW_k1) {
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->NN = NN;
  cfg->Nmax = 100;   // barbie.c:71
  cfg->Nr = 40;      // barbie.c:72
  cfg->UL_k1 = UL_k1;
  cfg->LL_k1 = LL_k1;
  cfg->BW_k1 = BW_k1;
  cfg->n_mtbin = 5;  // barbie.c:84
  cfg->LL = 1.0;     // barbie.c:67
  cfg->precision = BEAM_PREC_FP64;
  cfg->method = BEAM_METHOD_TRIANGLE;
}

const char *beam_gpu_strerror(int code) {
  switch (code) {
    case BEAM_OK: return "ok";
    case BEAM_EINVAL: return "invalid configuration or argument";
    case BEAM_ENOMEM: return "host allocation failed";
    case BEAM_EDEVMEM: return "device allocation failed or footprint refused";
    case BEAM_ECUDA: return "CUDA runtime error";
    case BEAM_ETIMEDOUT: return "bounded device wait timed out";
    case BEAM_EBUSY: return "busy";
    case BEAM_EBOUNDS: return "a triangle's bin index is outside the bin arrays";
    case BEAM_ENODEV: return "no usable CUDA device";
    case BEAM_ENOTFOUND: return "unknown job";
    default: return "unknown error";
  }
}

const char *beam_gpu_last_error_detail(void) { return g_detail.c_str(); }

int beam_gpu_init(int device, beam_gpu_ctx **out) {
  if (!out) return BEAM_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    set_detail("no CUDA device visible");
    return BEAM_ENODEV;
  }
  if (device < 0 || device >= n) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  BEAM_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    set_detail(std::string("libbeam_gpu is built for sm_100a; device is ") + prop.name);
    return BEAM_ENODEV;
  }
  beam_gpu_ctx *c = new (std::nothrow) beam_gpu_ctx();
  if (!c) return BEAM_ENOMEM;
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  for (int k = 0; k < TRI_WARPS && e == cudaSuccess; ++k) {
    e = cudaStreamCreateWithFlags(&c->side[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->join[k], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    set_detail(cudaGetErrorString(e));
    beam_gpu_destroy(c);
    return BEAM_ECUDA;
  }
  *out = c;
  return BEAM_OK;
}

void beam_gpu_destroy(beam_gpu_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (int k = 0; k < TRI_WARPS; ++k) {
    if (ctx->side[k]) cudaStreamDestroy(ctx->side[k]);
    if (ctx->join[k]) cudaEventDestroy(ctx->join[k]);
  }
  if (ctx->fork) cudaEventDestroy(ctx->fork);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int beam_gpu_plan_create(beam_gpu_ctx *ctx, const beam_cfg *cfg, beam_gpu_plan **out) {
  if (!ctx || !cfg || !out) return BEAM_EINVAL;
  *out = nullptr;
  if ((cfg->precision != BEAM_PREC_FP64 && cfg->precision != BEAM_PREC_MIXED) ||
      (cfg->method != BEAM_METHOD_TRIANGLE && cfg->method != BEAM_METHOD_PIXEL)) {
    set_detail("unknown precision or method");
    return BEAM_EINVAL;
  }
  BEAM_CUDA(cudaSetDevice(ctx->device));
  beam_gpu_plan *p = new (std::nothrow) beam_gpu_plan();
  if (!p) return BEAM_ENOMEM;
  p->ctx = ctx;
  p->cfg = *cfg;
  int rc = beam_geom_build(&p->geom, cfg);
  if (rc == BEAM_EBOUNDS) set_detail("a triangle's (k1, t, mu) bin falls outside the bin arrays");
  if (rc == BEAM_EINVAL) set_detail("invalid configuration (NN even, Nmax <= NN/2, Nr a multiple of 10, "
                                    "BW_k1 > 0 dividing UL_k1 - LL_k1 > 0)");
  if (rc == BEAM_OK) rc = build_plan_tables(p);
  if (rc == BEAM_OK && pixel_method(p)) rc = build_pixel_path(p);
  for (int k = 0; k < 5 && rc == BEAM_OK; ++k)
    if (cudaEventCreate(&p->ev[k]) != cudaSuccess) rc = BEAM_ECUDA;
  if (rc != BEAM_OK) {
    beam_gpu_plan_destroy(p);
    return rc;
  }
  *out = p;
  return BEAM_OK;
}

void beam_gpu_plan_destroy(beam_gpu_plan *p) {
  if (!p) return;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  for (int k = 0; k < 5; ++k)
    if (p->ev[k]) cudaEventDestroy(p->ev[k]);
  free_pixel_path(p);
  free_plan_tables(p);
  beam_geom_free(&p->geom);
  delete p;
}

int beam_gpu_plan_get_info(const beam_gpu_plan *p, beam_plan_info *info) {
  if (!p || !info) return BEAM_EINVAL;
  std::memset(info, 0, sizeof(*info));
  info->n_k1bin = p->geom.n_k1bin;
  info->n_bins = p->d.n_bins;
  info->n_closed_triplets = p->geom.nrp;
  info->n_triples = p->geom.ntri;
  info->n_used_triplets = p->d.n_used;
  long long terms = 0;
  // sum over accepted triangles of the in-plane triangle count of their triplet
  std::vector<long long> per_u(p->d.n_used, 0);
  for (size_t u = 0; u + 1 < p->tri_first.size(); ++u) per_u[u] = p->tri_first[u + 1] - p->tri_first[u];
  std::vector<int> u_of_rp(p->geom.nrp, -1);
  for (size_t u = 0; u < p->used_rp.size(); ++u) u_of_rp[p->used_rp[u]] = (int)u;
  for (long long t = 0; t < p->geom.ntri; ++t) terms += per_u[u_of_rp[p->geom.t_rp[t]]];
  info->n_fourier_terms = terms;
  info->n_modes = p->d.n_modes;
  info->n_planes = p->d.Q;
  info->device_bytes = p->device_bytes;
  info->vol = p->geom.vol;
  return BEAM_OK;
}

static int copy_results(beam_gpu_plan *p, beam_result *res) {
  DevPlan &d = p->d;
  cudaStream_t s = p->ctx->stream;
  size_t nb = (size_t)d.n_bins;
  if (nb) {
    BEAM_CUDA(cudaMemcpyAsync(p->h_bins, d.bins, sizeof(double) * 3 * nb * BEAM_NPOLES, cudaMemcpyDeviceToHost, s));
    BEAM_CUDA(cudaMemcpyAsync(p->h_count, d.bin_count, sizeof(long long) * nb, cudaMemcpyDeviceToHost, s));
  }
  BEAM_TRY(check_status(p));  // synchronizes the stream
  if (!res) return BEAM_OK;
  size_t n = nb * BEAM_NPOLES;
  if (res->bs) std::memcpy(res->bs, p->h_bins, sizeof(double) * n);
  if (res->norm) std::memcpy(res->norm, p->h_bins + n, sizeof(double) * n);
  if (res->out) std::memcpy(res->out, p->h_bins + 2 * n, sizeof(double) * n);
  if (res->count)
    for (size_t b = 0; b < nb; ++b) res->count[b] = (int64_t)p->h_count[b];
  return BEAM_OK;
}

static int compute_B(beam_gpu_plan *p, const double *r2c, int on_device) {
  p->timed = false;
  mark(p, 0);
  if (pixel_method(p)) return pixel_triangle_sums(p, r2c, on_device);
  if (on_device)
    BEAM_TRY(upload_modes_device(p, r2c));
  else
    BEAM_TRY(upload_modes_host(p, r2c));
  return run_triangle_sums(p);
}

int beam_gpu_run(beam_gpu_plan *p, const double *r2c, int r2c_on_device, beam_result *res) {
  if (!p || !r2c) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  BEAM_TRY(compute_B(p, r2c, r2c_on_device));
  BEAM_TRY(run_epilogue(p));
  mark(p, 4);
  p->timed = true;
  return copy_results(p, res);
}

int beam_gpu_run_batch(beam_gpu_plan *p, const double *const *r2c, int n, beam_result *res) {
  if (!p || (!r2c && n > 0) || n < 0) return BEAM_EINVAL;
  for (int i = 0; i < n; ++i) BEAM_TRY(beam_gpu_run(p, r2c[i], 0, res ? &res[i] : nullptr));
  return BEAM_OK;
}

int beam_gpu_triangle_sums(beam_gpu_plan *p, const double *r2c, int r2c_on_device, double *B) {
  if (!p || !r2c || !B) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  BEAM_TRY(compute_B(p, r2c, r2c_on_device));
  mark(p, 4);
  p->timed = true;
  long long n = p->geom.ntri;
  std::vector<double> tmp((size_t)std::max<long long>(1, n));
  if (n) BEAM_CUDA(cudaMemcpyAsync(tmp.data(), p->d.B, sizeof(double) * n, cudaMemcpyDeviceToHost, p->ctx->stream));
  BEAM_TRY(check_status(p));
  for (long long i = 0; i < n; ++i) B[p->loop_of_bin[i]] = tmp[i];
  return BEAM_OK;
}

int beam_gpu_closed_rings(beam_gpu_plan *p, double *rings4, long cap, long *rcount) {
  if (!p) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  std::vector<long long> counts;
  BEAM_TRY(count_closed_triangles(p, counts));
  double nn2 = (double)p->geom.NN * (double)p->geom.NN;
  for (long k = 0; k < p->geom.nrp && k < cap && rings4; ++k) {
    rings4[4 * k] = p->geom.rp[3 * k];
    rings4[4 * k + 1] = p->geom.rp[3 * k + 1];
    rings4[4 * k + 2] = p->geom.rp[3 * k + 2];
    rings4[4 * k + 3] = nn2 * (double)counts[k];
  }
  if (rcount) *rcount = p->geom.nrp;
  return BEAM_OK;
}

int beam_gpu_plane_rings(beam_gpu_plan *p, const double *r2c, int r2c_on_device, const int *planes, const int *rings,
                         int n, double *out, int out_on_device) {
  if (!p || !r2c || !planes || !rings || !out || n < 0) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  return plane_rings(p, r2c, r2c_on_device, planes, rings, n, out, out_on_device);
}

void *beam_gpu_stream(beam_gpu_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int beam_gpu_plan_last_timings(const beam_gpu_plan *p, float *ms, int n) {
  if (!p || !ms || n < 0) return BEAM_EINVAL;
  if (!p->timed) return BEAM_EINVAL;
  BEAM_CUDA(cudaEventSynchronize(p->ev[4]));
  for (int k = 0; k < n && k < 4; ++k) BEAM_CUDA(cudaEventElapsedTime(&ms[k], p->ev[k], p->ev[k + 1]));
  return BEAM_OK;
}

}  // extern "C"
