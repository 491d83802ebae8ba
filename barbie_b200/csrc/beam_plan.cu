// Plan construction for libbeam_gpu: ring-mode tables, the in-plane triangle
// lists of the ring triplets in use (built on the GPU), the accepted triangles
// grouped by ring triplet, the work items of the triangle-sum kernel and the
// bin-ordered epilogue tables.
//
// Why in-plane triangle lists: the reference sums, per accepted triangle,
//   B = sum_x Re(F1(x) F2^(s2)(x) F3^(s3)(x))            (barbie.c:329-337)
// over the NN^2 pixels of the unnormalised backward 2D DFTs
//   F_{p,r}(x) = sum_{k in ring r} Delta(k, p) e^{+i k.x}    (funcs.c:88-109).
// Summing the exponentials over the pixels first gives NN^2 when
// k1 + k2 + k3 = 0 (mod NN) and 0 otherwise, so
//   B = NN^2 Re sum_{k1+k2+k3 = 0 mod NN, k_i in ring r_i} M1(k1) M2'(k2) M3'(k3),
// with M'(k) = Delta(k,|p|) for p >= 0 and conj(Delta(-k,|p|)) for p < 0. The
// closed in-plane triangles of a ring triplet are exactly the ones calCR counts
// (funcs.c:396-399 computes NN^2 times their number), so they depend only on
// the geometry and are listed once per plan.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "beam_internal.h"

namespace beam {

// ---------------------------------------------------------------------------
// In-plane triangle enumeration: for ring triplet u = (r1, r2, r3) and each mode
// k2 of ring r2 (one thread each), count or list the modes k1 of ring r1 for
// which k3 = -(k1 + k2) mod NN lies in ring r3. Triangles are emitted k2-major,
// k1 in ring order, so the list order is deterministic.
// ---------------------------------------------------------------------------
struct TripletRef {
  int r1, r2, r3;
  int m1, n1, m2, n2, m3;  // first mode and mode count of rings r1, r2; first mode of r3
  long long k2base;        // first per-k2 counter of this triplet
};

__global__ void k_tri_count(const TripletRef *trip, const int16_t *__restrict__ mode_ij,
                            const int16_t *__restrict__ ringmap, int NN, int *__restrict__ cnt) {
  const TripletRef t = trip[blockIdx.y];
  int k2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (k2 >= t.n2) return;
  int i2 = mode_ij[2 * (t.m2 + k2)], j2 = mode_ij[2 * (t.m2 + k2) + 1];
  int n = 0;
  for (int k1 = 0; k1 < t.n1; ++k1) {
    int i1 = mode_ij[2 * (t.m1 + k1)], j1 = mode_ij[2 * (t.m1 + k1) + 1];
    int i3 = (2 * NN - i1 - i2) % NN, j3 = (2 * NN - j1 - j2) % NN;
    n += (ringmap[i3 * NN + j3] == t.r3);
  }
  cnt[t.k2base + k2] = n;
}

__global__ void k_tri_write(const TripletRef *trip, const int16_t *__restrict__ mode_ij,
                            const int16_t *__restrict__ ringmap, const int16_t *__restrict__ pixlocal, int NN,
                            const long long *__restrict__ offs, ushort4 *__restrict__ out) {
  const TripletRef t = trip[blockIdx.y];
  int k2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (k2 >= t.n2) return;
  int i2 = mode_ij[2 * (t.m2 + k2)], j2 = mode_ij[2 * (t.m2 + k2) + 1];
  long long at = offs[t.k2base + k2];
  for (int k1 = 0; k1 < t.n1; ++k1) {
    int i1 = mode_ij[2 * (t.m1 + k1)], j1 = mode_ij[2 * (t.m1 + k1) + 1];
    int i3 = (2 * NN - i1 - i2) % NN, j3 = (2 * NN - j1 - j2) % NN;
    if (ringmap[i3 * NN + j3] == t.r3)
      out[at++] = make_ushort4((unsigned short)k1, (unsigned short)k2, (unsigned short)pixlocal[i3 * NN + j3], 0);
  }
}

// Count (and optionally list) the in-plane triangles of the given triplets.
// mode tables (ring_first, mode_ij) must cover every ring the triplets use.
static int enumerate_in_plane(beam_gpu_plan *p, const std::vector<int> &rps, const std::vector<int32_t> &ring_first,
                              const int16_t *d_mode_ij, const int16_t *d_ringmap, const int16_t *d_pixlocal,
                              std::vector<long long> &tri_first, ushort4 **d_list, long long *n_terms) {
  cudaStream_t s = p->ctx->stream;
  const beam_geom &g = p->geom;
  std::vector<TripletRef> refs(rps.size());
  long long k2total = 0;
  int max_n2 = 1;
  for (size_t u = 0; u < rps.size(); ++u) {
    int rp = rps[u];
    TripletRef &t = refs[u];
    t.r1 = g.rp[3 * rp];
    t.r2 = g.rp[3 * rp + 1];
    t.r3 = g.rp[3 * rp + 2];
    t.m1 = ring_first[t.r1];
    t.n1 = ring_first[t.r1 + 1] - t.m1;
    t.m2 = ring_first[t.r2];
    t.n2 = ring_first[t.r2 + 1] - t.m2;
    t.m3 = ring_first[t.r3];
    t.k2base = k2total;
    k2total += t.n2;
    max_n2 = std::max(max_n2, t.n2);
  }
  tri_first.assign(rps.size() + 1, 0);
  if (n_terms) *n_terms = 0;
  if (rps.empty()) return BEAM_OK;
  TripletRef *d_refs = nullptr;
  int *d_cnt = nullptr;
  long long *d_offs = nullptr;
  int rc = BEAM_OK;
  std::vector<int> cnt(k2total);
  std::vector<long long> offs(k2total);
  BEAM_CUDA(cudaMalloc(&d_refs, sizeof(TripletRef) * refs.size()));
  BEAM_CUDA(cudaMalloc(&d_cnt, sizeof(int) * k2total));
  BEAM_CUDA(cudaMemcpyAsync(d_refs, refs.data(), sizeof(TripletRef) * refs.size(), cudaMemcpyHostToDevice, s));
  for (size_t y0 = 0; y0 < refs.size(); y0 += 65535) {
    dim3 grid((max_n2 + 127) / 128, (unsigned)std::min<size_t>(65535, refs.size() - y0));
    k_tri_count<<<grid, 128, 0, s>>>(d_refs + y0, d_mode_ij, d_ringmap, (int)g.NN, d_cnt);
  }
  BEAM_CUDA(cudaGetLastError());
  BEAM_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * k2total, cudaMemcpyDeviceToHost, s));
  BEAM_CUDA(cudaStreamSynchronize(s));
  long long run = 0;
  for (size_t u = 0; u < refs.size(); ++u) {
    tri_first[u] = run;
    for (int k = 0; k < refs[u].n2; ++k) {
      offs[refs[u].k2base + k] = run;
      run += cnt[refs[u].k2base + k];
    }
  }
  tri_first[refs.size()] = run;
  if (n_terms) *n_terms = run;
  if (d_list) {
    rc = dev_alloc(p, d_list, (size_t)run);
    if (rc == BEAM_OK) {
      BEAM_CUDA(cudaMalloc(&d_offs, sizeof(long long) * k2total));
      BEAM_CUDA(cudaMemcpyAsync(d_offs, offs.data(), sizeof(long long) * k2total, cudaMemcpyHostToDevice, s));
      for (size_t y0 = 0; y0 < refs.size(); y0 += 65535) {
        dim3 grid((max_n2 + 127) / 128, (unsigned)std::min<size_t>(65535, refs.size() - y0));
        k_tri_write<<<grid, 128, 0, s>>>(d_refs + y0, d_mode_ij, d_ringmap, d_pixlocal, (int)g.NN, d_offs, *d_list);
      }
      BEAM_CUDA(cudaGetLastError());
      BEAM_CUDA(cudaStreamSynchronize(s));
    }
  }
  cudaFree(d_refs);
  cudaFree(d_cnt);
  cudaFree(d_offs);
  return rc;
}

// Mode table of the given rings: modes (i, j) of each ring in row-major pixel
// order; pixlocal[i*NN+j] = index within its ring (-1 outside the listed rings).
static void build_modes(const beam_geom &g, const std::vector<char> &ring_on, std::vector<int32_t> &ring_first,
                        std::vector<int16_t> &mode_ij, std::vector<int16_t> &pixlocal) {
  long NN = g.NN, Nr = g.Nr;
  std::vector<std::vector<int32_t>> per(Nr);
  for (long x = 0; x < NN * NN; ++x) {
    int r = g.ringmap[x];
    if (r >= 0 && ring_on[r]) per[r].push_back((int32_t)x);
  }
  ring_first.assign(Nr + 1, 0);
  mode_ij.clear();
  pixlocal.assign(NN * NN, -1);
  int at = 0;
  for (long r = 0; r < Nr; ++r) {
    ring_first[r] = at;
    for (size_t k = 0; k < per[r].size(); ++k) {
      int32_t x = per[r][k];
      mode_ij.push_back((int16_t)(x / NN));
      mode_ij.push_back((int16_t)(x % NN));
      pixlocal[x] = (int16_t)k;
    }
    at += (int)per[r].size();
  }
  ring_first[Nr] = at;
}

template <typename T>
static int upload(beam_gpu_plan *p, T **dst, const std::vector<T> &src) {
  BEAM_TRY(dev_alloc(p, dst, src.size()));
  if (!src.empty()) BEAM_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
  return BEAM_OK;
}

int build_plan_tables(beam_gpu_plan *p) {
  const beam_geom &g = p->geom;
  DevPlan &d = p->d;
  const long NN = g.NN, Nr = g.Nr;
  const long long ntri = g.ntri;

  // rings and planes in use
  std::vector<char> ring_on(Nr, 0);
  std::vector<long long> per_rp(g.nrp, 0);
  int Q = 1;
  for (long long t = 0; t < ntri; ++t) {
    int rp = g.t_rp[t];
    per_rp[rp]++;
    for (int k = 0; k < 3; ++k) ring_on[g.rp[3 * rp + k]] = 1;
    int p1 = g.t_p1[t], p2 = g.t_p2[t], p3 = -p1 - p2;
    Q = std::max(Q, 1 + std::max(p1, std::max(std::abs(p2), std::abs(p3))));
  }
  // bulk copies move whole 16-byte units: rows, their starts and lengths are
  // kept in multiples of A complex values (1 for complex128, 2 for complex64)
  const int A = (p->cfg.precision == BEAM_PREC_MIXED) ? 2 : 1;
  auto floorA = [A](int v) { return v - (((v % A) + A) % A); };
  auto ceilA = [A, &floorA](int v) { return floorA(v + A - 1); };
  d.Q = Q;
  d.W = ceilA(2 * Q - 1);

  std::vector<int16_t> pixlocal;
  build_modes(g, ring_on, p->ring_first, p->mode_ij, pixlocal);
  d.n_modes = (int)(p->mode_ij.size() / 2);
  for (long r = 0; r < Nr; ++r)
    if (p->ring_first[r + 1] - p->ring_first[r] > 32767) {
      set_detail("a ring holds more than 32767 modes");
      return BEAM_EINVAL;
    }
  std::vector<int32_t> mode_neg(d.n_modes);
  for (int m = 0; m < d.n_modes; ++m) {
    int i = p->mode_ij[2 * m], j = p->mode_ij[2 * m + 1];
    int ni = (int)((NN - i) % NN), nj = (int)((NN - j) % NN);
    int r = g.ringmap[ni * NN + nj];
    mode_neg[m] = p->ring_first[r] + pixlocal[ni * NN + nj];
  }
  std::vector<int16_t> ringmap(g.ringmap, g.ringmap + NN * NN);
  BEAM_TRY(upload(p, &d.mode_ij, p->mode_ij));
  BEAM_TRY(upload(p, &d.mode_neg, mode_neg));
  BEAM_TRY(upload(p, &d.ringmap, ringmap));
  BEAM_TRY(upload(p, &d.pixlocal, pixlocal));

  // used ring triplets and their combos (accepted triangles in loop order)
  std::vector<int> u_of_rp(g.nrp, -1);
  p->used_rp.clear();
  for (long rp = 0; rp < g.nrp; ++rp)
    if (per_rp[rp]) {
      u_of_rp[rp] = (int)p->used_rp.size();
      p->used_rp.push_back((int)rp);
    }
  d.n_used = (int)p->used_rp.size();
  d.n_combo = ntri;
  std::vector<int32_t> u_cfirst(d.n_used + 1, 0), u_ncombo(d.n_used, 0);
  for (long long t = 0; t < ntri; ++t) u_ncombo[u_of_rp[g.t_rp[t]]]++;
  for (int u = 0; u < d.n_used; ++u) u_cfirst[u + 1] = u_cfirst[u] + u_ncombo[u];
  std::vector<int32_t> combo_p1(ntri), combo_p2(ntri), combo_u(ntri), combo_tid(ntri);
  {
    std::vector<int32_t> fill(u_cfirst.begin(), u_cfirst.end() - 1);
    for (long long t = 0; t < ntri; ++t) {
      int u = u_of_rp[g.t_rp[t]];
      int c = fill[u]++;
      combo_p1[c] = g.t_p1[t];
      combo_p2[c] = g.t_p2[t];
      combo_u[c] = u;
      combo_tid[c] = (int32_t)t;
    }
  }

  // bin order (stable in loop order)
  d.n_bins = g.n_k1bin * g.n_mtbin * g.n_mtbin;
  std::vector<int32_t> bin_first(d.n_bins + 1, 0);
  for (long long t = 0; t < ntri; ++t) bin_first[g.t_bin[t] + 1]++;
  for (int b = 0; b < d.n_bins; ++b) bin_first[b + 1] += bin_first[b];
  p->bin_pos.assign(ntri, 0);
  p->loop_of_bin.assign(ntri, 0);
  {
    std::vector<int32_t> fill(bin_first.begin(), bin_first.end() - 1);
    for (long long t = 0; t < ntri; ++t) {
      int at = fill[g.t_bin[t]]++;
      p->bin_pos[t] = at;
      p->loop_of_bin[at] = (int32_t)t;
    }
  }
  std::vector<int32_t> combo_out(ntri);
  for (long long c = 0; c < ntri; ++c) combo_out[c] = p->bin_pos[combo_tid[c]];

  // in-plane triangle lists (GPU)
  BEAM_TRY(enumerate_in_plane(p, p->used_rp, p->ring_first, d.mode_ij, d.ringmap, d.pixlocal, p->tri_first,
                              &d.tri_list, &d.n_terms));

  // epilogue tables in bin order
  std::vector<double> ep_px(ntri), ep_pz(ntri);
  std::vector<int32_t> ep_cnt(ntri);
  for (long long i = 0; i < ntri; ++i) {
    long long t = p->loop_of_bin[i];
    ep_px[i] = g.t_px[t];
    ep_pz[i] = g.t_pz[t];
    int u = u_of_rp[g.t_rp[t]];
    ep_cnt[i] = (int32_t)(p->tri_first[u + 1] - p->tri_first[u]);
  }

  // work items: split large (triplet) work along its triangle list
  int n_sms = std::max(1, p->ctx->num_sms);
  long double total = 0;
  for (int u = 0; u < d.n_used; ++u)
    total += (long double)u_ncombo[u] * (long double)(p->tri_first[u + 1] - p->tri_first[u]);
  long double target = std::max<long double>(total / (n_sms * 6.0L), 1.0L);
  std::vector<TriItem> items;
  std::vector<int32_t> u_nsplit(d.n_used, 1);
  std::vector<long long> u_part(d.n_used + 1, 0);
  std::vector<long double> item_work;
  const int max_combos = TRI_THREADS * TRI_MAX_SLOTS;
  int max_row = 1;
  for (int u = 0; u < d.n_used; ++u) {
    long long nt = p->tri_first[u + 1] - p->tri_first[u];
    long double w = (long double)u_ncombo[u] * (long double)nt;
    int ncg = (u_ncombo[u] + max_combos - 1) / max_combos;  // combo groups
    long long ns = (long long)std::ceil((double)(w / (target * ncg)));
    ns = std::max<long long>(1, std::min<long long>(ns, std::max<long long>(1, nt / (4 * TRI_CHUNK))));
    u_nsplit[u] = (int)ns;
    u_part[u + 1] = u_part[u] + ns * (long long)u_ncombo[u];
    int rp = p->used_rp[u];
    int r1 = g.rp[3 * rp], r2 = g.rp[3 * rp + 1], r3 = g.rp[3 * rp + 2];
    for (int cg = 0; cg < ncg; ++cg) {
      int c0 = u_cfirst[u] + cg * max_combos, c1 = std::min(u_cfirst[u + 1], c0 + max_combos);
      int p1lo = 1 << 30, p1hi = -(1 << 30), p2lo = 1 << 30, p2hi = -(1 << 30), p3lo = 1 << 30, p3hi = -(1 << 30);
      for (int c = c0; c < c1; ++c) {
        int a = combo_p1[c], b = combo_p2[c], e = -a - b;
        p1lo = std::min(p1lo, a); p1hi = std::max(p1hi, a);
        p2lo = std::min(p2lo, b); p2hi = std::max(p2hi, b);
        p3lo = std::min(p3lo, e); p3hi = std::max(p3hi, e);
      }
      for (long long s = 0; s < ns; ++s) {
        TriItem it;
        it.u = u;
        it.split = (int)s;
        it.c0 = c0;
        it.c1 = c1;
        it.t0 = p->tri_first[u] + nt * s / ns;
        it.t1 = p->tri_first[u] + nt * (s + 1) / ns;
        it.m1 = p->ring_first[r1];
        it.m2 = p->ring_first[r2];
        it.m3 = p->ring_first[r3];
        // column ranges of the signed-plane rows (column of plane q is q + Q - 1)
        it.p1lo = floorA(p1lo + Q - 1); it.L1 = ceilA(p1hi + Q) - it.p1lo;
        it.p2lo = floorA(p2lo + Q - 1); it.L2 = ceilA(p2hi + Q) - it.p2lo;
        it.p3lo = floorA(p3lo + Q - 1); it.L3 = ceilA(p3hi + Q) - it.p3lo;
        max_row = std::max(max_row, it.L1 + it.L2 + it.L3);
        items.push_back(it);
        item_work.push_back((long double)(c1 - c0) * (long double)(it.t1 - it.t0));
      }
    }
  }
  // largest first, so the tail of the launch holds the small items
  std::vector<int> order(items.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return item_work[a] > item_work[b]; });
  std::vector<TriItem> sorted(items.size());
  for (size_t k = 0; k < order.size(); ++k) sorted[k] = items[order[k]];
  d.n_items = (int)sorted.size();
  d.max_row = max_row;
  {
    // two pipeline stages of `chunk` triangle rows must fit the opt-in shared memory
    size_t elem = (A == 2) ? 8 : 16;
    size_t budget = p->ctx->smem_optin > 4096 ? p->ctx->smem_optin - 4096 : 48 * 1024;
    size_t fit = budget / (2 * (size_t)max_row * elem);
    if (fit < 1) {
      set_detail("signed-plane rows too long for shared memory");
      return BEAM_EINVAL;
    }
    d.chunk = (int)std::min<size_t>(TRI_CHUNK, fit);
  }
  d.n_part = u_part[d.n_used];
  u_part.pop_back();
  u_cfirst.pop_back();

  BEAM_TRY(upload(p, &d.items, sorted));
  BEAM_TRY(upload(p, &d.combo_p1, combo_p1));
  BEAM_TRY(upload(p, &d.combo_p2, combo_p2));
  BEAM_TRY(upload(p, &d.combo_u, combo_u));
  BEAM_TRY(upload(p, &d.combo_out, combo_out));
  BEAM_TRY(upload(p, &d.u_cfirst, u_cfirst));
  BEAM_TRY(upload(p, &d.u_ncombo, u_ncombo));
  BEAM_TRY(upload(p, &d.u_nsplit, u_nsplit));
  BEAM_TRY(upload(p, &d.u_part, u_part));
  BEAM_TRY(upload(p, &d.bin_first, bin_first));
  BEAM_TRY(upload(p, &d.ep_px, ep_px));
  BEAM_TRY(upload(p, &d.ep_pz, ep_pz));
  BEAM_TRY(upload(p, &d.ep_cnt, ep_cnt));

  // per-realization buffers
  BEAM_TRY(dev_alloc(p, &d.staging, (size_t)d.n_modes * Q * 2));
  if (p->cfg.precision == BEAM_PREC_MIXED)
    BEAM_TRY(dev_alloc(p, &d.S32, (size_t)d.n_modes * d.W * 2));
  else
    BEAM_TRY(dev_alloc(p, &d.S64, (size_t)d.n_modes * d.W * 2));
  BEAM_TRY(dev_alloc(p, &d.part, (size_t)d.n_part));
  BEAM_TRY(dev_alloc(p, &d.B, (size_t)ntri));
  BEAM_TRY(dev_alloc(p, &d.bins, (size_t)3 * d.n_bins * BEAM_NPOLES));
  BEAM_TRY(dev_alloc(p, &d.bin_count, (size_t)d.n_bins));
  BEAM_TRY(dev_alloc(p, &d.status, 1));
  BEAM_CUDA(cudaMemset(d.status, 0, sizeof(int)));
  BEAM_CUDA(cudaMallocHost(&p->h_staging, sizeof(double) * 2 * std::max<size_t>(1, (size_t)d.n_modes * Q)));
  BEAM_CUDA(cudaMallocHost(&p->h_bins, sizeof(double) * 3 * std::max(1, d.n_bins) * BEAM_NPOLES));
  BEAM_CUDA(cudaMallocHost(&p->h_count, sizeof(long long) * std::max(1, d.n_bins)));
  return BEAM_OK;
}

void free_plan_tables(beam_gpu_plan *p) {
  DevPlan &d = p->d;
  void *ptrs[] = {d.mode_ij, d.mode_neg, d.ringmap, d.pixlocal, d.tri_list, d.combo_p1, d.combo_p2, d.combo_u,
                  d.combo_out, d.u_cfirst, d.u_ncombo, d.u_nsplit, d.u_part, d.items, d.part, d.staging, d.S64,
                  d.S32, d.B, d.bin_first, d.ep_px, d.ep_pz, d.ep_cnt, d.bins, d.bin_count, d.status};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (p->h_staging) cudaFreeHost(p->h_staging);
  if (p->h_bins) cudaFreeHost(p->h_bins);
  if (p->h_count) cudaFreeHost(p->h_count);
  p->h_staging = nullptr;
  p->h_bins = nullptr;
  p->h_count = nullptr;
  d = DevPlan();
}

// Exact triangle counts of every closed ring triplet (calCR's Num / NN^2).
int count_closed_triangles(beam_gpu_plan *p, std::vector<long long> &counts) {
  const beam_geom &g = p->geom;
  std::vector<char> all(g.Nr, 1);
  std::vector<int32_t> ring_first;
  std::vector<int16_t> mode_ij, pixlocal;
  build_modes(g, all, ring_first, mode_ij, pixlocal);
  int16_t *d_mode = nullptr;
  BEAM_CUDA(cudaMalloc(&d_mode, sizeof(int16_t) * std::max<size_t>(1, mode_ij.size())));
  BEAM_CUDA(cudaMemcpy(d_mode, mode_ij.data(), sizeof(int16_t) * mode_ij.size(), cudaMemcpyHostToDevice));
  std::vector<int> rps(g.nrp);
  std::iota(rps.begin(), rps.end(), 0);
  std::vector<long long> first;
  size_t before = p->device_bytes;
  int rc = enumerate_in_plane(p, rps, ring_first, d_mode, p->d.ringmap, nullptr, first, nullptr, nullptr);
  p->device_bytes = before;
  cudaFree(d_mode);
  if (rc != BEAM_OK) return rc;
  counts.resize(g.nrp);
  for (long k = 0; k < g.nrp; ++k) counts[k] = first[k + 1] - first[k];
  return BEAM_OK;
}

}  // namespace beam
