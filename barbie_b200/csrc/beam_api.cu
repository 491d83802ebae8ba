// C-ABI entry points of libbeam_gpu (declared in include/beam_gpu.h).
#include <chrono>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>

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
int triangle_init_attributes(size_t smem_optin);
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
  cfg->shard_index = 0;
  cfg->shard_count = 1;
}

int beam_shard_assign(const double *work, int n, int shard_count, int *owner) {
  if (n < 0 || shard_count < 1 || (n > 0 && (!work || !owner))) return BEAM_EINVAL;
  std::vector<int> order(n);
  for (int u = 0; u < n; ++u) order[u] = u;
  std::stable_sort(order.begin(), order.end(), [work](int a, int b) { return work[a] > work[b]; });
  std::vector<double> load(shard_count, 0.0);
  for (int u : order) {
    int best = 0;
    for (int k = 1; k < shard_count; ++k)
      if (load[k] < load[best]) best = k;
    owner[u] = best;
    load[best] += work[u];
  }
  return BEAM_OK;
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
  int rc = lane_create(&c->lane);
  if (rc == BEAM_OK) rc = triangle_init_attributes(c->smem_optin);
  if (rc != BEAM_OK) {
    beam_gpu_destroy(c);
    return rc;
  }
  c->stream = c->lane.stream;
  *out = c;
  return BEAM_OK;
}

void beam_gpu_destroy(beam_gpu_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->field_ws) cudaFree(ctx->field_ws);
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->pk_tab) cudaFree(ctx->pk_tab);
  lane_destroy(&ctx->lane);
  delete ctx;
}

int beam_gpu_plan_create(beam_gpu_ctx *ctx, const beam_cfg *cfg, beam_gpu_plan **out) {
  if (!ctx || !cfg || !out) return BEAM_EINVAL;
  *out = nullptr;
  if ((cfg->precision != BEAM_PREC_FP64 && cfg->precision != BEAM_PREC_MIXED && cfg->precision != BEAM_PREC_INT8) ||
      (cfg->method != BEAM_METHOD_TRIANGLE && cfg->method != BEAM_METHOD_PIXEL)) {
    set_detail("unknown precision or method");
    return BEAM_EINVAL;
  }
  const int shards = cfg->shard_count < 1 ? 1 : cfg->shard_count;
  if (cfg->shard_index < 0 || cfg->shard_index >= shards || (shards > 1 && cfg->method != BEAM_METHOD_TRIANGLE)) {
    set_detail("shard_index must lie in [0, shard_count); sharding needs the triangle method");
    return BEAM_EINVAL;
  }
  BEAM_CUDA(cudaSetDevice(ctx->device));
  beam_gpu_plan *p = new (std::nothrow) beam_gpu_plan();
  if (!p) return BEAM_ENOMEM;
  p->ctx = ctx;
  p->cfg = *cfg;
  p->cfg.shard_count = shards;
  // first split cap of the triangle lists: the autotuner's best at NN=384 for
  // each path (FP64 1024, mixed 512 triangles per CTA)
  p->tau0 = cfg->precision == BEAM_PREC_FP64 ? 2 * TRI_TAU_MAX : TRI_TAU_MAX;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return (float)std::chrono::duration<double, std::milli>(b - a).count();
  };
  const auto t0 = now();
  int rc = beam_geom_build(&p->geom, cfg);
  p->build_ms[0] = ms(t0, now());
  if (rc == BEAM_EBOUNDS) set_detail("a triangle's (k1, t, mu) bin falls outside the bin arrays");
  if (rc == BEAM_EINVAL) set_detail("invalid configuration (NN even, Nmax <= NN/2, Nr a multiple of 10, "
                                    "BW_k1 > 0 dividing UL_k1 - LL_k1 > 0)");
  if (rc == BEAM_OK) rc = host_guard([&] { return build_plan_tables(p); });
  const auto t1 = now();
  if (rc == BEAM_OK) rc = host_guard([&] { return slot_create(p, 1, &ctx->lane, &p->main); });
  p->build_ms[4] = ms(t1, now());
  if (rc == BEAM_OK && pixel_method(p)) rc = host_guard([&] { return build_pixel_path(p); });
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
  for (beam::RunSlot *&s : p->batch) {
    slot_destroy(s);
    s = nullptr;
  }
  slot_destroy(p->main);
  p->main = nullptr;
  free_pixel_path(p);
  free_plan_tables(p);
  beam_geom_free(&p->geom);
  delete p;
}

int beam_gpu_plan_set_triangle_launch(beam_gpu_plan *p, int mode) {
  if (!p || (mode != BEAM_LAUNCH_CLASSES && mode != BEAM_LAUNCH_PERSISTENT)) return BEAM_EINVAL;
  if (p->cfg.precision == BEAM_PREC_INT8 && mode == BEAM_LAUNCH_PERSISTENT) {
    set_detail("the int8 path has class launches only");
    return BEAM_EINVAL;
  }
  if (p->tri_launch == mode) return BEAM_OK;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  BEAM_CUDA(cudaStreamSynchronize(p->ctx->stream));
  for (RunSlot *s : {p->main, p->batch[0], p->batch[1]}) {
    if (!s || !s->graph) continue;
    if (s->done) BEAM_CUDA(cudaEventSynchronize(s->done));
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->graph_n = 0;
  }
  p->tri_launch = mode;
  return BEAM_OK;
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
  long long mine = terms;
  if (p->cfg.shard_count > 1) {
    mine = 0;
    for (long long t = 0; t < p->geom.ntri; ++t) {
      int u = u_of_rp[p->geom.t_rp[t]];
      if (p->u_owner[u] == p->cfg.shard_index) mine += per_u[u];
    }
  }
  info->n_shard_terms = mine;
  info->n_modes = p->d.n_modes;
  info->n_planes = p->d.Q;
  size_t bytes = p->device_bytes + (p->main ? p->main->bytes : 0);
  for (const RunSlot *s : p->batch) bytes += s ? s->bytes : 0;
  info->device_bytes = bytes;
  info->vol = p->geom.vol;
  info->launches_last_run = p->main ? p->main->launches : 0;
  info->run_bytes = slot_bytes(p, 1);
  info->n_run_combos = (long)p->n_run_combos;
  for (int k = 0; k < 5; ++k) info->build_ms[k] = p->build_ms[k];
  return BEAM_OK;
}

// Host gather of one realization's mode rows, split over up to 8 host threads
// when there is more than about a megabyte to move.
static void gather_one(const beam_gpu_plan *p, RunSlot *s, const double *r2c) {
  const int nm = p->d.n_modes;
  const size_t bytes = (size_t)nm * p->d.Q * 16;
  unsigned hw = std::thread::hardware_concurrency();
  int nt = (int)std::min<size_t>(std::min<unsigned>(std::max(1u, hw), 8u), bytes >> 20);
  if (nt <= 1) {
    gather_host(p, s, 0, r2c);
    return;
  }
  host_parallel(nt, [=](int k) {
    gather_host(p, s, 0, r2c, (int)((long long)nm * k / nt), (int)((long long)nm * (k + 1) / nt));
  });
}

// Device-side address of a page-locked host buffer (cudaHostAlloc'd or
// cudaHostRegister'ed), or nullptr for pageable memory.
static const double *mapped_host(const double *r2c) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, r2c) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return at.type == cudaMemoryTypeHost ? static_cast<const double *>(at.devicePointer) : nullptr;
}

// Buffers the kernels read or write as complex128 (double2) must start on a
// 16-byte boundary.
static bool aligned16(const void *q) { return ((uintptr_t)q & 15) == 0; }

// Triangle sums of one realization on the plan's own slot. A device r2c
// buffer must be 16-byte aligned; a page-locked host one that is not is
// gathered on the host instead of being read in place.
static int compute_B(beam_gpu_plan *p, const double *r2c, int on_device) {
  if (on_device && !aligned16(r2c)) {
    set_detail("the device r2c buffer must be 16-byte aligned");
    return BEAM_EINVAL;
  }
  RunSlot *s = p->main;
  s->timed = false;
  s->launches = 0;
  mark(s, 0);
  if (pixel_method(p)) return pixel_triangle_sums(p, r2c, on_device);
  if (on_device) {
    s->h_src[s->cap] = r2c;
    BEAM_TRY(upload_modes(p, s, 1, false));
  } else if (const double *mapped = aligned16(r2c) ? mapped_host(r2c) : nullptr) {
    BEAM_TRY(gather_mapped(p, s, mapped));
    BEAM_TRY(upload_modes(p, s, 1, true, true));
  } else {
    gather_one(p, s, r2c);
    BEAM_TRY(upload_modes(p, s, 1, true));
  }
  return run_triangle_sums(p, s, 1);
}

int beam_gpu_run(beam_gpu_plan *p, const double *r2c, int r2c_on_device, beam_result *res) {
  if (!p || !r2c) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  RunSlot *s = p->main;
  BEAM_TRY(compute_B(p, r2c, r2c_on_device));
  BEAM_TRY(run_epilogue(p, s, 1));
  mark(s, 4);
  BEAM_TRY(fetch_results(p, s, 1));
  BEAM_TRY(check_status(s));
  s->timed = true;
  return copy_result(p, s, 0, res);
}

// Copy the mode rows of realizations r2c[0..n) into slot rows [0, n), split
// over a few host threads.
static void gather_batch(const beam_gpu_plan *p, RunSlot *s, const double *const *r2c, int n) {
  unsigned hw = std::thread::hardware_concurrency();
  int nt = (int)std::min<unsigned>(std::max(1u, hw), 8u);
  nt = std::min(nt, n);
  if (nt <= 1) {
    for (int r = 0; r < n; ++r) gather_host(p, s, r, r2c[r]);
    return;
  }
  host_parallel(nt, [=](int k) {
    for (int r = k; r < n; r += nt) gather_host(p, s, r, r2c[r]);
  });
}

int beam_gpu_run_batch_ex(beam_gpu_plan *p, const double *const *r2c, int n, beam_result *res, int batch) {
  if (!p || (!r2c && n > 0) || n < 0 || batch < 0) return BEAM_EINVAL;
  for (int i = 0; i < n; ++i)
    if (!r2c[i]) return BEAM_EINVAL;
  if (n == 0) return BEAM_OK;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  if (pixel_method(p)) {
    for (int i = 0; i < n; ++i) BEAM_TRY(beam_gpu_run(p, r2c[i], 0, res ? &res[i] : nullptr));
    return BEAM_OK;
  }
  int b = batch;
  if (b == 0) {
    size_t fr = 0, tot = 0;
    BEAM_CUDA(cudaMemGetInfo(&fr, &tot));
    size_t per = std::max<size_t>(1, slot_bytes(p, 1));
    b = (int)std::min<size_t>(64, std::max<size_t>(1, fr / 4 / per));  // two slots in half the free memory
  }
  b = std::min(std::min(b, n), 65535);
  const int nslots = n > b ? 2 : 1;
  for (int k = 0; k < nslots; ++k)
    if (!p->batch[k] || p->batch[k]->cap < b) {
      slot_destroy(p->batch[k]);
      p->batch[k] = nullptr;
      BEAM_TRY(slot_create(p, b, nullptr, &p->batch[k]));
    }
  int first[2] = {-1, -1}, count[2] = {0, 0};
  int rc = BEAM_OK;
  auto retire = [&](int k) {
    if (first[k] < 0) return BEAM_OK;
    int r = check_status(p->batch[k]);
    for (int j = 0; j < count[k] && r == BEAM_OK && res; ++j) copy_result(p, p->batch[k], j, &res[first[k] + j]);
    first[k] = -1;
    return r;
  };
  for (int i = 0, r0 = 0; r0 < n && rc == BEAM_OK; ++i, r0 += b) {
    const int k = i % nslots, nb = std::min(b, n - r0);
    rc = retire(k);  // the slot's previous batch has finished: its staging rows may be rewritten
    if (rc != BEAM_OK) break;
    gather_batch(p, p->batch[k], r2c + r0, nb);
    rc = slot_run_graph(p, p->batch[k], nb);
    if (rc == BEAM_OK) {
      first[k] = r0;
      count[k] = nb;
    }
  }
  for (int k = 0; k < nslots; ++k) {
    int r = retire(k);
    if (rc == BEAM_OK) rc = r;
  }
  return rc;
}

int beam_gpu_run_batch(beam_gpu_plan *p, const double *const *r2c, int n, beam_result *res) {
  return beam_gpu_run_batch_ex(p, r2c, n, res, 0);
}

int beam_gpu_triangle_sums(beam_gpu_plan *p, const double *r2c, int r2c_on_device, double *B) {
  if (!p || !r2c || !B) return BEAM_EINVAL;
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  RunSlot *s = p->main;
  BEAM_TRY(compute_B(p, r2c, r2c_on_device));
  mark(s, 4);
  long long n = p->geom.ntri;
  std::vector<double> tmp((size_t)std::max<long long>(1, n));
  cudaStream_t st = s->lane->stream;
  if (n) BEAM_CUDA(cudaMemcpyAsync(tmp.data(), s->B, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  BEAM_CUDA(cudaMemcpyAsync(s->h_status, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  BEAM_CUDA(cudaEventRecord(s->done, st));
  BEAM_TRY(check_status(s));
  s->timed = true;
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
  if ((r2c_on_device && !aligned16(r2c)) || (out_on_device && !aligned16(out))) {
    set_detail("device buffers must be 16-byte aligned");
    return BEAM_EINVAL;
  }
  BEAM_CUDA(cudaSetDevice(p->ctx->device));
  return plane_rings(p, r2c, r2c_on_device, planes, rings, n, out, out_on_device);
}

void *beam_gpu_stream(beam_gpu_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int beam_gpu_plan_last_timings(const beam_gpu_plan *p, float *ms, int n) {
  if (!p || !ms || n < 0) return BEAM_EINVAL;
  const RunSlot *s = p->main;
  if (!s || !s->timed) return BEAM_EINVAL;
  BEAM_CUDA(cudaEventSynchronize(s->ev[4]));
  for (int k = 0; k < n && k < 4; ++k) BEAM_CUDA(cudaEventElapsedTime(&ms[k], s->ev[k], s->ev[k + 1]));
  return BEAM_OK;
}

}  // extern "C"
