// Job server of libbeam_gpu (beam_gpu_server_*, declared in include/beam_gpu.h).
//
// One dispatcher thread per server owns every plan and run slot of the
// server; callers only touch the job table under the server's mutex.
//   * plans: cached per configuration (beam_cfg minus the shard fields), least
//     recently used first out when memory or the cache limit calls for it;
//   * slots: one realization's run buffers with streams of their own
//     (RunSlot with its own Lane), pooled per plan;
//   * admission: queued jobs in arrival order while fewer than max_active
//     run and the job's footprint -- its plan if not cached plus a slot -- fits
//     the budget after idle slots and idle plans are released; a job that does
//     not fit lets later jobs pass for up to kHoldMs, after which admission
//     waits for it;
//   * a job runs as the slot's captured graph (H2D of the gathered mode rows,
//     kernels, D2H of the bins), so jobs on different slots overlap on the GPU;
//     the dispatcher polls each slot's `done` event to retire it;
//   * priority by size: a plan's slots get streams whose CUDA priority falls
//     with the plan's work (one level per decade of closed-triangle terms
//     above 1e8), so as the CTAs of a large job retire, those of a small job
//     that arrived meanwhile are scheduled first and it does not wait for the
//     large one to drain.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "beam_internal.h"

using namespace beam;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

constexpr double kHoldMs = 200.0;  // how long a job that does not fit may be passed by later ones

struct CfgKey {
  long NN, Nmax, Nr;
  int UL, LL, BW, n_mtbin, precision;
  double cell;
  bool operator<(const CfgKey &o) const {
    return std::tie(NN, Nmax, Nr, UL, LL, BW, n_mtbin, precision, cell) <
           std::tie(o.NN, o.Nmax, o.Nr, o.UL, o.LL, o.BW, o.n_mtbin, o.precision, o.cell);
  }
};

CfgKey key_of(const beam_cfg &c) {
  return CfgKey{c.NN, c.Nmax, c.Nr, c.UL_k1, c.LL_k1, c.BW_k1, c.n_mtbin, c.precision, c.LL};
}

struct PlanEntry {
  CfgKey key;
  beam_gpu_plan *plan = nullptr;
  int priority = 0;         // CUDA stream priority of the plan's job slots
  std::vector<RunSlot *> free_slots;
  int active = 0;           // running jobs on this plan
  size_t bytes = 0;         // tables + the plan's own slot
  unsigned long long last_use = 0;
};

struct Job {
  int64_t id = 0;
  beam_cfg cfg{};
  const double *r2c = nullptr;
  int state = BEAM_JOB_QUEUED, error = BEAM_OK;
  std::string detail;
  Clock::time_point t_submit, t_start, t_done;
  bool blocked = false;     // did not fit at its last admission attempt
  Clock::time_point t_blocked;
  PlanEntry *entry = nullptr;
  RunSlot *slot = nullptr;
  int n_k1bin = 0, n_mtbin = 0;
  long n_bins = 0;
  std::vector<double> bins;  // [BIN_SECTIONS][n_bins][16]
  std::vector<int64_t> count;
};

}  // namespace

struct beam_gpu_server {
  beam_gpu_ctx *ctx = nullptr;
  beam_server_cfg cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job *> queue;                    // arrival order (mu)
  std::unordered_map<int64_t, Job *> jobs;    // every job not yet taken (mu)
  int64_t next_id = 1;
  bool stop = false;
  size_t used = 0, peak = 0;                  // written by the dispatcher under mu
  std::thread th;
  // dispatcher only
  std::map<CfgKey, PlanEntry *> plans;
  std::vector<Job *> active;
  unsigned long long tick = 0;
};

namespace {

void account(beam_gpu_server *s, long long delta) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->used = (size_t)((long long)s->used + delta);
  s->peak = std::max(s->peak, s->used);
}

void finish(beam_gpu_server *s, Job *j, int state, int error, const std::string &detail) {
  std::lock_guard<std::mutex> lk(s->mu);
  j->state = state;
  j->error = error;
  j->detail = detail;
  j->t_done = Clock::now();
  s->cv_done.notify_all();
}

void drop_slot(beam_gpu_server *s, RunSlot *slot) {
  long long b = (long long)slot->bytes;
  slot_destroy(slot);
  account(s, -b);
}

void drop_plan(beam_gpu_server *s, PlanEntry *e) {
  for (RunSlot *slot : e->free_slots) drop_slot(s, slot);
  e->free_slots.clear();
  beam_gpu_plan_destroy(e->plan);
  account(s, -(long long)e->bytes);
  s->plans.erase(e->key);
  delete e;
}

// Release idle memory, least recently used first -- pooled slots, then whole
// idle plans (never `keep`) -- until `need` more bytes fit the budget.
bool make_room(beam_gpu_server *s, size_t need, const PlanEntry *keep) {
  auto fits = [&]() {
    std::lock_guard<std::mutex> lk(s->mu);
    return s->used + need <= s->cfg.mem_budget;
  };
  std::vector<PlanEntry *> order;
  for (auto &kv : s->plans) order.push_back(kv.second);
  std::sort(order.begin(), order.end(), [](const PlanEntry *a, const PlanEntry *b) { return a->last_use < b->last_use; });
  for (PlanEntry *e : order) {
    if (fits()) return true;
    while (!e->free_slots.empty() && !fits()) {
      drop_slot(s, e->free_slots.back());
      e->free_slots.pop_back();
    }
  }
  for (PlanEntry *e : order) {
    if (fits()) return true;
    if (e != keep && e->active == 0) drop_plan(s, e);
  }
  return fits();
}

// Try to start job j. BEAM_OK: running; BEAM_EBUSY: must wait for memory or
// a slot; anything else: the job failed (already finished with that error).
int try_admit(beam_gpu_server *s, Job *j) {
  CfgKey key = key_of(j->cfg);
  PlanEntry *e = nullptr;
  auto it = s->plans.find(key);
  if (it != s->plans.end()) e = it->second;
  if (!e) {
    if ((int)s->plans.size() >= s->cfg.max_plans) {
      // the least recently used idle plan leaves the cache
      PlanEntry *lru = nullptr;
      for (auto &kv : s->plans)
        if (kv.second->active == 0 && (!lru || kv.second->last_use < lru->last_use)) lru = kv.second;
      if (lru) drop_plan(s, lru);
      else if (!s->active.empty()) return BEAM_EBUSY;
    }
    beam_gpu_plan *p = nullptr;
    int rc = beam_gpu_plan_create(s->ctx, &j->cfg, &p);
    if (rc == BEAM_EDEVMEM) {
      make_room(s, (size_t)-1 / 2, nullptr);  // release everything idle, then try once more
      rc = beam_gpu_plan_create(s->ctx, &j->cfg, &p);
      if (rc == BEAM_EDEVMEM && !s->active.empty()) return BEAM_EBUSY;
    }
    if (rc != BEAM_OK) {
      finish(s, j, BEAM_JOB_FAILED, rc, beam_gpu_last_error_detail());
      return rc;
    }
    beam_plan_info info;
    beam_gpu_plan_get_info(p, &info);
    e = new PlanEntry();
    e->key = key;
    e->plan = p;
    e->bytes = info.device_bytes;
    {
      int least = 0, greatest = 0;  // e.g. 0 and -5: smaller numbers are served first
      if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) least = greatest = 0;
      int level = 0;
      for (double t = (double)info.n_fourier_terms; t >= 1e9 && level < least - greatest; t /= 10.0) ++level;
      e->priority = greatest + level;
    }
    s->plans[key] = e;
    account(s, (long long)e->bytes);
    // a plan's size is known only once built: if it pushed the total over the
    // budget, release idle memory, else (while others run) wait with the plan cached
    if (!make_room(s, 0, e) && !s->active.empty()) return BEAM_EBUSY;
  }
  e->last_use = ++s->tick;
  beam_gpu_plan *p = e->plan;
  RunSlot *slot = nullptr;
  if (!e->free_slots.empty()) {
    slot = e->free_slots.back();
    e->free_slots.pop_back();
  } else {
    size_t need = slot_bytes(p, 1);
    if (!make_room(s, need, e)) {
      if (!s->active.empty()) return BEAM_EBUSY;
      finish(s, j, BEAM_JOB_FAILED, BEAM_EDEVMEM, "job footprint exceeds the server's memory budget");
      return BEAM_EDEVMEM;
    }
    int rc = slot_create(p, 1, nullptr, &slot, e->priority);
    if (rc == BEAM_EDEVMEM && !s->active.empty()) return BEAM_EBUSY;
    if (rc != BEAM_OK) {
      finish(s, j, BEAM_JOB_FAILED, rc, beam_gpu_last_error_detail());
      return rc;
    }
    account(s, (long long)slot->bytes);
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    j->t_start = Clock::now();
    j->state = BEAM_JOB_RUNNING;
    j->n_k1bin = p->geom.n_k1bin;
    j->n_mtbin = p->geom.n_mtbin;
    j->n_bins = p->d.n_bins;
  }
  gather_host(p, slot, 0, j->r2c);
  int rc = slot_run_graph(p, slot, 1);
  if (rc != BEAM_OK) {
    e->free_slots.push_back(slot);
    finish(s, j, BEAM_JOB_FAILED, rc, beam_gpu_last_error_detail());
    return rc;
  }
  j->entry = e;
  j->slot = slot;
  e->active++;
  s->active.push_back(j);
  return BEAM_OK;
}

// Retire the running jobs whose device work has finished.
bool retire(beam_gpu_server *s) {
  bool any = false;
  for (size_t k = 0; k < s->active.size();) {
    Job *j = s->active[k];
    cudaError_t q = cudaEventQuery(j->slot->done);
    if (q == cudaErrorNotReady) {
      ++k;
      continue;
    }
    int rc = check_status(j->slot);
    if (rc == BEAM_OK) {
      size_t nb = (size_t)j->n_bins;
      j->bins.assign(j->slot->h_bins, j->slot->h_bins + BIN_SECTIONS * nb * BEAM_NPOLES);
      j->count.assign(j->slot->h_count, j->slot->h_count + nb);
      finish(s, j, BEAM_JOB_DONE, BEAM_OK, "");
    } else {
      finish(s, j, BEAM_JOB_FAILED, rc, beam_gpu_last_error_detail());
    }
    j->entry->active--;
    j->entry->free_slots.push_back(j->slot);
    j->slot = nullptr;
    s->active.erase(s->active.begin() + (long)k);
    any = true;
  }
  return any;
}

void dispatcher(beam_gpu_server *s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    retire(s);
    std::vector<Job *> queued;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stop && s->queue.empty() && s->active.empty()) break;
      queued.assign(s->queue.begin(), s->queue.end());
    }
    bool hold = false;  // a job that does not fit has waited long enough: no passing
    for (Job *j : queued) {
      if ((int)s->active.size() >= s->cfg.max_active || hold) break;
      int rc = try_admit(s, j);
      if (rc == BEAM_EBUSY) {
        if (!j->blocked) {
          j->blocked = true;
          j->t_blocked = Clock::now();
        }
        hold = ms_between(j->t_blocked, Clock::now()) > kHoldMs;
        continue;
      }
      std::lock_guard<std::mutex> lk(s->mu);
      s->queue.erase(std::find(s->queue.begin(), s->queue.end(), j));
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (!s->active.empty())
      s->cv_work.wait_for(lk, std::chrono::microseconds(50));  // poll the running jobs' events
    else if (s->queue.empty() && !s->stop)
      s->cv_work.wait(lk);
  }
  // shut down: everything is idle
  while (!s->plans.empty()) drop_plan(s, s->plans.begin()->second);
}

}  // namespace

extern "C" {

void beam_server_cfg_default(beam_server_cfg *cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->max_active = 4;
  cfg->max_plans = 16;
}

int beam_gpu_server_create(beam_gpu_ctx *ctx, const beam_server_cfg *cfg, beam_gpu_server **out) {
  if (!ctx || !out) return BEAM_EINVAL;
  *out = nullptr;
  beam_server_cfg c;
  beam_server_cfg_default(&c);
  if (cfg) {
    if (cfg->max_active < 0 || cfg->max_plans < 0) return BEAM_EINVAL;
    if (cfg->mem_budget) c.mem_budget = cfg->mem_budget;
    if (cfg->max_active) c.max_active = cfg->max_active;
    if (cfg->max_plans) c.max_plans = cfg->max_plans;
  }
  BEAM_CUDA(cudaSetDevice(ctx->device));
  if (c.mem_budget == 0) {
    size_t fr = 0, tot = 0;
    BEAM_CUDA(cudaMemGetInfo(&fr, &tot));
    c.mem_budget = fr / 10 * 8;
  }
  beam_gpu_server *s = new (std::nothrow) beam_gpu_server();
  if (!s) return BEAM_ENOMEM;
  s->ctx = ctx;
  s->cfg = c;
  try {
    s->th = std::thread(dispatcher, s);
  } catch (...) {
    delete s;
    return BEAM_ENOMEM;
  }
  *out = s;
  return BEAM_OK;
}

void beam_gpu_server_destroy(beam_gpu_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  for (auto &kv : s->jobs) delete kv.second;
  delete s;
}

int beam_gpu_server_submit(beam_gpu_server *s, const beam_cfg *cfg, const double *r2c, int64_t *job) {
  if (!s || !cfg || !r2c || !job) return BEAM_EINVAL;
  if (cfg->method != BEAM_METHOD_TRIANGLE || cfg->shard_count > 1) {
    set_detail("server jobs need the triangle method and no sharding");
    return BEAM_EINVAL;
  }
  Job *j = new (std::nothrow) Job();
  if (!j) return BEAM_ENOMEM;
  j->cfg = *cfg;
  j->cfg.shard_index = 0;
  j->cfg.shard_count = 1;
  j->r2c = r2c;
  j->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete j;
    return BEAM_EINVAL;
  }
  j->id = s->next_id++;
  s->jobs[j->id] = j;
  s->queue.push_back(j);
  *job = j->id;
  s->cv_work.notify_all();
  return BEAM_OK;
}

static void fill_info(const Job *j, beam_job_info *info) {
  if (!info) return;
  std::memset(info, 0, sizeof(*info));
  info->state = j->state;
  info->error = j->error;
  info->n_k1bin = j->n_k1bin;
  info->n_mtbin = j->n_mtbin;
  info->n_bins = j->n_bins;
  bool started = j->state != BEAM_JOB_QUEUED;
  bool ended = j->state == BEAM_JOB_DONE || j->state == BEAM_JOB_FAILED;
  Clock::time_point now = Clock::now();
  info->queue_ms = ms_between(j->t_submit, started ? j->t_start : (ended ? j->t_done : now));
  info->run_ms = started ? ms_between(j->t_start, ended ? j->t_done : now) : 0.0;
  info->total_ms = ms_between(j->t_submit, ended ? j->t_done : now);
}

int beam_gpu_server_wait(beam_gpu_server *s, int64_t job, int timeout_ms, beam_job_info *info) {
  if (!s) return BEAM_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) return BEAM_ENOTFOUND;
  Job *j = it->second;
  auto ended = [j]() { return j->state == BEAM_JOB_DONE || j->state == BEAM_JOB_FAILED; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ended);
  else if (timeout_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ended);
  fill_info(j, info);
  return ended() ? BEAM_OK : BEAM_EBUSY;
}

int beam_gpu_server_take(beam_gpu_server *s, int64_t job, beam_result *res) {
  if (!s) return BEAM_EINVAL;
  Job *j = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return BEAM_ENOTFOUND;
    j = it->second;
    if (j->state != BEAM_JOB_DONE && j->state != BEAM_JOB_FAILED) return BEAM_EBUSY;
    s->jobs.erase(it);
  }
  int rc = j->state == BEAM_JOB_DONE ? BEAM_OK : j->error;
  if (rc != BEAM_OK) {
    set_detail(j->detail);
  } else if (res) {
    size_t n = (size_t)j->n_bins * BEAM_NPOLES;
    if (res->bs) std::memcpy(res->bs, j->bins.data(), sizeof(double) * n);
    if (res->norm) std::memcpy(res->norm, j->bins.data() + n, sizeof(double) * n);
    if (res->out) std::memcpy(res->out, j->bins.data() + 2 * n, sizeof(double) * n);
    if (res->ana_sum) std::memcpy(res->ana_sum, j->bins.data() + 3 * n, sizeof(double) * n);
    if (res->ana)
      for (size_t i = 0; i < n; ++i) res->ana[i] = j->bins[3 * n + i] / j->bins[n + i];  // barbie.c:391
    if (res->count) std::memcpy(res->count, j->count.data(), sizeof(int64_t) * (size_t)j->n_bins);
  }
  delete j;
  return rc;
}

int beam_gpu_server_memory(const beam_gpu_server *s, size_t *now, size_t *peak) {
  if (!s) return BEAM_EINVAL;
  std::lock_guard<std::mutex> lk(const_cast<beam_gpu_server *>(s)->mu);
  if (now) *now = s->used;
  if (peak) *peak = s->peak;
  return BEAM_OK;
}

}  // extern "C"
