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
#include <chrono>
#include <cstring>
#include <numeric>
#include <thread>

#include "beam_internal.h"

namespace beam {

// ---------------------------------------------------------------------------
// In-plane triangle enumeration: for ring triplet u = (r1, r2, r3) and each mode
// k2 of ring r2 (one thread each), count or list the modes k1 of ring r1 for
// which k3 = -(k1 + k2) mod NN lies in ring r3. Triangles are emitted k2-major,
// k1 in ring order, so the list order is deterministic.
//
// Which two of the triplet's rings play "r2" and "r3" here is the caller's
// choice (swap): the run leg ("r2", whose mode a run of the list shares and
// whose plane is -p1 - p(tile)) and the tile leg ("r3"). The sum is symmetric
// in the two; the plan takes as run leg the ring whose runs are longer.
// ---------------------------------------------------------------------------
struct TripletRef {
  int r1, r2, r3;
  int m1, n1, m2, n2, m3;  // first mode and mode count of rings r1, r2; first mode of r3
  long long k2base;        // first per-k2 counter of this triplet
  long long k3base;        // first per-k3 counter (k_tri_count_both)
};

// (NN - u - v) mod NN for u, v in [0, NN), without a division
__device__ __forceinline__ int neg_sum_mod(int u, int v, int NN) {
  int w = NN - u - v;
  w += (w < 0) ? NN : 0;
  return w >= NN ? w - NN : w;
}

// Counts in both orientations at once: per mode k2 of ring r2 the triangles
// sharing it (one thread each, as k_tri_count), and per mode k3 of ring r3 the
// triangles sharing that, by atomic increments (integer counts: the order does
// not matter).
__global__ void k_tri_count_both(const TripletRef *trip, const int16_t *__restrict__ mode_ij,
                                 const int16_t *__restrict__ ringmap, const int16_t *__restrict__ pixlocal, int NN,
                                 int *__restrict__ cnt2, int *__restrict__ cnt3) {
  const TripletRef t = trip[blockIdx.y];
  int k2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (k2 >= t.n2) return;
  int i2 = mode_ij[2 * (t.m2 + k2)], j2 = mode_ij[2 * (t.m2 + k2) + 1];
  int n = 0;
  for (int k1 = 0; k1 < t.n1; ++k1) {
    int i1 = mode_ij[2 * (t.m1 + k1)], j1 = mode_ij[2 * (t.m1 + k1) + 1];
    const int pix = neg_sum_mod(i1, i2, NN) * NN + neg_sum_mod(j1, j2, NN);
    if (ringmap[pix] == t.r3) {
      ++n;
      atomicAdd(&cnt3[t.k3base + pixlocal[pix]], 1);
    }
  }
  cnt2[t.k2base + k2] = n;
}

__global__ void k_tri_count(const TripletRef *trip, const int16_t *__restrict__ mode_ij,
                            const int16_t *__restrict__ ringmap, int NN, int *__restrict__ cnt) {
  const TripletRef t = trip[blockIdx.y];
  int k2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (k2 >= t.n2) return;
  int i2 = mode_ij[2 * (t.m2 + k2)], j2 = mode_ij[2 * (t.m2 + k2) + 1];
  int n = 0;
  for (int k1 = 0; k1 < t.n1; ++k1) {
    int i1 = mode_ij[2 * (t.m1 + k1)], j1 = mode_ij[2 * (t.m1 + k1) + 1];
    n += (ringmap[neg_sum_mod(i1, i2, NN) * NN + neg_sum_mod(j1, j2, NN)] == t.r3);
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
    const int pix = neg_sum_mod(i1, i2, NN) * NN + neg_sum_mod(j1, j2, NN);
    if (ringmap[pix] == t.r3)
      out[at++] = make_ushort4((unsigned short)k1, (unsigned short)k2, (unsigned short)pixlocal[pix], 0);
  }
}

// One copy descriptor per chunk from the chunk table, the triangle list and
// the piece table.
__global__ void k_build_desc(const TriChunk *__restrict__ chunks, long long n, const ushort4 *__restrict__ list,
                             const int2 *__restrict__ pieces, TriDesc *__restrict__ out) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const TriChunk k = chunks[c];
  const int nt = chunk_nt(k.packed), npc = chunk_npc(k.packed);
  TriDesc d;
  for (int j = 0; j < TRI_CHUNK; ++j) {
    ushort4 e = j < nt ? list[k.t0 + j] : make_ushort4(0, 0, 0, 0);
    d.xz[j][0] = e.x;
    d.xz[j][1] = e.z;
  }
  for (int j = 0; j < TRI_PIECES; ++j) d.y[j] = j < npc ? (uint16_t)pieces[k.pc0 + j].y : (uint16_t)0;
  d.packed = k.packed;
  d.pad = 0;
  out[c] = d;
}

// Count (and optionally list) the in-plane triangles of the given triplets.
// mode tables (ring_first, mode_ij) must cover every ring the triplets use.
static int enumerate_in_plane(beam_gpu_plan *p, const std::vector<int> &rps, const std::vector<int32_t> &ring_first,
                              const int16_t *d_mode_ij, const int16_t *d_ringmap, const int16_t *d_pixlocal,
                              std::vector<long long> &tri_first, ushort4 **d_list, long long *n_terms,
                              std::vector<int> *k2cnt, const std::vector<char> *swap = nullptr,
                              const std::vector<int> *given = nullptr) {
  cudaStream_t s = p->ctx->stream;
  const beam_geom &g = p->geom;
  std::vector<TripletRef> refs(rps.size());
  long long k2total = 0;
  int max_n2 = 1;
  for (size_t u = 0; u < rps.size(); ++u) {
    int rp = rps[u];
    TripletRef &t = refs[u];
    const bool sw = swap && (*swap)[u];
    t.r1 = g.rp[3 * rp];
    t.r2 = g.rp[3 * rp + (sw ? 2 : 1)];
    t.r3 = g.rp[3 * rp + (sw ? 1 : 2)];
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
  // a failed CUDA call records its error and skips the rest; the buffers are
  // freed on every path
  auto cuda_ok = [&](cudaError_t e, const char *what) {
    if (rc == BEAM_OK && e != cudaSuccess) {
      set_detail(std::string(what) + ": " + cudaGetErrorString(e));
      rc = BEAM_ECUDA;
    }
    return rc == BEAM_OK;
  };
  if (given) {  // counts from an earlier pass in the same orientation
    if ((long long)given->size() != k2total) {
      set_detail("in-plane triangle counts of another orientation");
      return BEAM_EINVAL;
    }
    cnt = *given;
  }
  if (cuda_ok(cudaMalloc(&d_refs, sizeof(TripletRef) * refs.size()), "cudaMalloc(triplets)") && given) {
    cuda_ok(cudaMemcpyAsync(d_refs, refs.data(), sizeof(TripletRef) * refs.size(), cudaMemcpyHostToDevice, s),
            "cudaMemcpyAsync(triplets)");
  } else if (rc == BEAM_OK && cuda_ok(cudaMalloc(&d_cnt, sizeof(int) * k2total), "cudaMalloc(counts)") &&
      cuda_ok(cudaMemcpyAsync(d_refs, refs.data(), sizeof(TripletRef) * refs.size(), cudaMemcpyHostToDevice, s),
              "cudaMemcpyAsync(triplets)")) {
    for (size_t y0 = 0; y0 < refs.size(); y0 += 65535) {
      dim3 grid((max_n2 + 127) / 128, (unsigned)std::min<size_t>(65535, refs.size() - y0));
      k_tri_count<<<grid, 128, 0, s>>>(d_refs + y0, d_mode_ij, d_ringmap, (int)g.NN, d_cnt);
    }
    if (cuda_ok(cudaGetLastError(), "k_tri_count") &&
        cuda_ok(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * k2total, cudaMemcpyDeviceToHost, s),
                "cudaMemcpyAsync(counts)"))
      cuda_ok(cudaStreamSynchronize(s), "k_tri_count");
  }
  if (rc == BEAM_OK) {
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
    if (k2cnt) *k2cnt = cnt;
    if (d_list) {
      rc = dev_alloc(p, d_list, (size_t)run);
      if (rc == BEAM_OK && cuda_ok(cudaMalloc(&d_offs, sizeof(long long) * k2total), "cudaMalloc(offsets)") &&
          cuda_ok(cudaMemcpyAsync(d_offs, offs.data(), sizeof(long long) * k2total, cudaMemcpyHostToDevice, s),
                  "cudaMemcpyAsync(offsets)")) {
        for (size_t y0 = 0; y0 < refs.size(); y0 += 65535) {
          dim3 grid((max_n2 + 127) / 128, (unsigned)std::min<size_t>(65535, refs.size() - y0));
          k_tri_write<<<grid, 128, 0, s>>>(d_refs + y0, d_mode_ij, d_ringmap, d_pixlocal, (int)g.NN, d_offs, *d_list);
        }
        if (cuda_ok(cudaGetLastError(), "k_tri_write")) cuda_ok(cudaStreamSynchronize(s), "k_tri_write");
      }
    }
  }
  cudaFree(d_refs);
  cudaFree(d_cnt);
  cudaFree(d_offs);
  return rc;
}

// In-plane triangle counts of the used triplets in both orientations (run leg
// r2 or r3): c2 per mode of r2 and c3 per mode of r3, triplet after triplet.
static int count_both_orientations(beam_gpu_plan *p, const int16_t *d_mode_ij, const int16_t *d_ringmap,
                                   const int16_t *d_pixlocal, std::vector<int> &c2, std::vector<int> &c3) {
  cudaStream_t s = p->ctx->stream;
  const beam_geom &g = p->geom;
  const std::vector<int> &rps = p->used_rp;
  std::vector<TripletRef> refs(rps.size());
  long long tot2 = 0, tot3 = 0;
  int max_n2 = 1;
  for (size_t u = 0; u < rps.size(); ++u) {
    const int rp = rps[u];
    TripletRef &t = refs[u];
    t.r1 = g.rp[3 * rp];
    t.r2 = g.rp[3 * rp + 1];
    t.r3 = g.rp[3 * rp + 2];
    t.m1 = p->ring_first[t.r1];
    t.n1 = p->ring_first[t.r1 + 1] - t.m1;
    t.m2 = p->ring_first[t.r2];
    t.n2 = p->ring_first[t.r2 + 1] - t.m2;
    t.m3 = p->ring_first[t.r3];
    t.k2base = tot2;
    t.k3base = tot3;
    tot2 += t.n2;
    tot3 += p->ring_first[t.r3 + 1] - t.m3;
    max_n2 = std::max(max_n2, t.n2);
  }
  c2.assign(tot2, 0);
  c3.assign(tot3, 0);
  if (rps.empty()) return BEAM_OK;
  TripletRef *d_refs = nullptr;
  int *d2 = nullptr, *d3 = nullptr;
  int rc = BEAM_OK;
  auto cuda_ok = [&](cudaError_t e, const char *what) {
    if (rc == BEAM_OK && e != cudaSuccess) {
      set_detail(std::string(what) + ": " + cudaGetErrorString(e));
      rc = BEAM_ECUDA;
    }
    return rc == BEAM_OK;
  };
  if (cuda_ok(cudaMalloc(&d_refs, sizeof(TripletRef) * refs.size()), "cudaMalloc(triplets)") &&
      cuda_ok(cudaMalloc(&d2, sizeof(int) * std::max<long long>(1, tot2)), "cudaMalloc(counts)") &&
      cuda_ok(cudaMalloc(&d3, sizeof(int) * std::max<long long>(1, tot3)), "cudaMalloc(counts)") &&
      cuda_ok(cudaMemsetAsync(d3, 0, sizeof(int) * std::max<long long>(1, tot3), s), "cudaMemsetAsync(counts)") &&
      cuda_ok(cudaMemcpyAsync(d_refs, refs.data(), sizeof(TripletRef) * refs.size(), cudaMemcpyHostToDevice, s),
              "cudaMemcpyAsync(triplets)")) {
    for (size_t y0 = 0; y0 < refs.size(); y0 += 65535) {
      dim3 grid((max_n2 + 127) / 128, (unsigned)std::min<size_t>(65535, refs.size() - y0));
      k_tri_count_both<<<grid, 128, 0, s>>>(d_refs + y0, d_mode_ij, d_ringmap, d_pixlocal, (int)g.NN, d2, d3);
    }
    if (cuda_ok(cudaGetLastError(), "k_tri_count_both") &&
        cuda_ok(cudaMemcpyAsync(c2.data(), d2, sizeof(int) * tot2, cudaMemcpyDeviceToHost, s), "counts") &&
        cuda_ok(cudaMemcpyAsync(c3.data(), d3, sizeof(int) * tot3, cudaMemcpyDeviceToHost, s), "counts"))
      cuda_ok(cudaStreamSynchronize(s), "k_tri_count_both");
  }
  cudaFree(d_refs);
  cudaFree(d2);
  cudaFree(d3);
  return rc;
}

// Stable counting sort of n items by key(t) in [0, nb), on up to 16 host
// threads: pos[t] is item t's place in key order (ties in index order), first
// (nb + 1 entries) each key's first place. Each thread counts its own range of
// items; a key's places go to the ranges in order, so the result is the one
// pass in index order gives.
template <typename K>
static void stable_bucket_sort(long long n, int nb, const K &key, std::vector<int32_t> &pos,
                               std::vector<int32_t> &first) {
  const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::vector<int32_t>> cnt(nt, std::vector<int32_t>(nb, 0));
  host_parallel(nt, [&](int k) {
    for (long long t = n * k / nt; t < n * (k + 1) / nt; ++t) cnt[k][key(t)]++;
  });
  first.assign(nb + 1, 0);
  for (int b = 0; b < nb; ++b) {
    int32_t at = first[b];
    for (int k = 0; k < nt; ++k) {
      const int32_t c = cnt[k][b];
      cnt[k][b] = at;  // thread k's first place in key b
      at += c;
    }
    first[b + 1] = at;
  }
  pos.assign(n, 0);
  host_parallel(nt, [&](int k) {
    for (long long t = n * k / nt; t < n * (k + 1) / nt; ++t) pos[t] = cnt[k][key(t)]++;
  });
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

// Tiles, pieces, chunks and CTA work items of the triangle-sum kernel.
//  * tiles: per ring triplet, its combos (p1, p2) placed on a grid of
//    TRI_P1 planes p1 x 32 planes p3 (p3 = -p1-p2); a CTA takes the tiles of
//    one p3 window and up to TRI_WARPS consecutive p1 blocks, so it stages
//    one z segment of 32 planes and x/y segments of at most
//    TRI_WARPS * TRI_P1 + 32 planes;
//  * runs: consecutive list entries sharing k2 (k2cnt, list order); a
//    triplet's runs are split into `ns` contiguous ranges of about equal size
//    when its work is large, so its CTAs share the triangle list;
//  * pieces: runs cut to at most TRI_CHUNK triangles; chunks: whole pieces
//    packed up to TRI_CHUNK triangles.
// A = 16-byte unit of complex values (1 or 2); u_part receives the first
// partial-sum slot of each triplet (ns_u * ncombo_u slots each). Triplets
// that another shard sums (own[u] == 0) get no tiles, chunks or items and one
// split of partial sums that stay zero, so their triangles come out as B = 0.
static int build_work(beam_gpu_plan *p, const std::vector<int32_t> &u_cfirst, const std::vector<int32_t> &u_ncombo,
                      const std::vector<int32_t> &combo_p1, const std::vector<int32_t> &combo_p2,
                      const std::vector<int> &k2cnt, const std::vector<char> &own, const std::vector<char> &u_swap,
                      int A, std::vector<int32_t> &u_nsplit, std::vector<long long> &u_part) {
  const beam_geom &g = p->geom;
  DevPlan &d = p->d;
  auto floorA = [A](int v) { return v - (((v % A) + A) % A); };
  auto ceilA = [&](int v) { return floorA(v + A - 1); };
  struct Slot {
    long long gkey, tkey;
    int a, lane, c;
  };
  struct Group {
    int tile0, ntiles;
    int p1lo, p1hi, p3lo, p3hi, p2lo, p2hi;  // over accepted combos
    int tp1lo, tp1hi;                        // first plane p1 of the tiles
    int w3lo, w3hi;                          // int8: first plane p3 of the group's first and last window
  };
  std::vector<TriTile> tiles;
  std::vector<int32_t> tile_combo;
  std::vector<std::vector<Group>> groups(d.n_used);
  std::vector<long long> k2base(d.n_used + 1, 0);
  for (int u = 0; u < d.n_used; ++u) {
    int ry = g.rp[3 * p->used_rp[u] + (u_swap[u] ? 2 : 1)];  // the run leg's ring
    k2base[u + 1] = k2base[u] + (p->ring_first[ry + 1] - p->ring_first[ry]);
  }
  // Origin of each triplet's block grid: p1 blocks start at 8 b - o1 (o1 in
  // {0, 4}: the mixed consumer reads a block's planes as aligned float4s),
  // p3 blocks at p3min - o3 + 8 b (o3 in 0..7; on the mixed path only those
  // that put p3 blocks on multiples of 4, for the same reason). The origin with the fewest
  // non-empty blocks is kept: fewer MMA cells without a combo. Triplets are
  // searched in parallel; each block is marked with the number of the origin
  // being counted, so the marks need no clearing between origins.
  // Block geometry: TRI_P1 planes p1 x BW planes p3, NBT blocks per tile. The
  // int8 path's tile is one window of I8_BW planes p3 x up to two p1 blocks
  // (a group is one window); the others pack any four 8 x 8 blocks of a
  // 32-plane p3 window.
  const bool i8 = p->cfg.precision == BEAM_PREC_INT8;
  const int BW = i8 ? I8_BW : TRI_BW, NBT = i8 ? I8_NBT : TRI_BLOCKS;
  struct Origin {
    int p3min, o1, o3;
  };
  std::vector<Origin> org(d.n_used, Origin{0, 0, 0});
  {
    auto search = [&](int u) {
      const int cf = u_cfirst[u], nc = u_ncombo[u];
      int p3min = 1 << 30, p3max = -(1 << 30), p1max = 0;
      for (int c = cf; c < cf + nc; ++c) {
        p3min = std::min(p3min, -combo_p1[c] - combo_p2[c]);
        p3max = std::max(p3max, -combo_p1[c] - combo_p2[c]);
        p1max = std::max(p1max, combo_p1[c]);
      }
      Origin o{p3min, 0, 0};
      const int nb1 = (p1max + 4) / TRI_P1 + 1, nb3 = (p3max - p3min + BW - 1) / BW + 1;
      std::vector<uint8_t> mark((size_t)nb1 * nb3, 0);
      int best = 1 << 30;
      uint8_t stamp = 0;
      const bool f4 = (A == 4) && !i8;  // the mixed consumer's aligned float4 reads
      const int a3first = f4 ? ((p3min % 4) + 4) % 4 : 0, a3step = f4 ? 4 : 1;
      for (int a1 = 0; a1 < TRI_P1; a1 += 4)
        for (int a3 = a3first; a3 < BW; a3 += a3step) {
          ++stamp;
          int nblocks = 0;
          for (int c = cf; c < cf + nc; ++c) {
            const int p1 = combo_p1[c], p3 = -p1 - combo_p2[c];
            uint8_t &m = mark[(size_t)((p1 + a1) / TRI_P1) * nb3 + (p3 - p3min + a3) / BW];
            nblocks += (m != stamp);
            m = stamp;
          }
          if (nblocks < best) best = nblocks, o.o1 = a1, o.o3 = a3;
        }
      org[u] = o;
    };
    const int nt = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    host_parallel(nt, [&](int k) {
      for (int u = k; u < d.n_used; u += nt)
        if (own[u] && u_ncombo[u] > 0) search(u);
    });
  }
  // tiles and groups, per triplet on up to 16 host threads (each triplet's
  // tiles in local lists, joined in triplet order below: the same tables as
  // one pass in triplet order)
  std::vector<std::vector<TriTile>> u_tiles(d.n_used);
  std::vector<std::vector<int32_t>> u_tc(d.n_used);
  std::vector<char> too_big(d.n_used, 0);
  auto tile_triplet = [&](int u) {
    std::vector<TriTile> &tiles = u_tiles[u];
    std::vector<int32_t> &tile_combo = u_tc[u];
    int cf = u_cfirst[u], nc = u_ncombo[u];
    const int p3min = org[u].p3min, o1 = org[u].o1, o3 = org[u].o3;
    std::vector<Slot> slots(nc);
    for (int k = 0; k < nc; ++k) {
      int c = cf + k, p1 = combo_p1[c], p3 = -p1 - combo_p2[c];
      long long bp1 = (p1 + o1) / TRI_P1, b3 = (p3 - p3min + o3) / BW;
      // a group is one window of 32 planes p3 over up to TRI_WARPS blocks of
      // planes p1; its non-empty TRI_P1 x TRI_BW blocks are packed four to a
      // tile (int8: one I8_BW window over up to 2 TRI_WARPS p1 blocks, two to a tile)
      // (int8: I8_GROUP_WINDOWS windows over up to TRI_WARPS p1 blocks, a tile being two p1
      // blocks of one window, the blocks window-major)
      const long long gkey =
          i8 ? (b3 / I8_GROUP_WINDOWS) * 1000000 + bp1 / TRI_WARPS : (b3 / TRI_BLOCKS) * 1000000 + bp1 / TRI_WARPS;
      const long long tkey = i8 ? b3 * 1000000 + bp1 : bp1 * 1000000 + b3;
      slots[k] = Slot{gkey, tkey, (p1 + o1) % TRI_P1, (p3 - p3min + o3) % BW, c};
    }
    std::sort(slots.begin(), slots.end(), [](const Slot &x, const Slot &y) {
      return x.gkey != y.gkey ? x.gkey < y.gkey : (x.tkey != y.tkey ? x.tkey < y.tkey : x.c < y.c);
    });
    for (size_t k = 0; k < slots.size();) {
      Group gr{(int)tiles.size(), 0, 1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30),
               1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
      long long gk = slots[k].gkey;
      while (k < slots.size() && slots[k].gkey == gk && (!i8 || gr.ntiles < I8_MAX_TILES)) {
        TriTile tl;
        tiles.push_back(tl);
        tile_combo.resize(tiles.size() * TRI_P1 * 32, -1);
        int32_t *tc = tile_combo.data() + (tiles.size() - 1) * TRI_P1 * 32;
        int nb = 0;
        for (; nb < NBT && k < slots.size() && slots[k].gkey == gk &&
               (!i8 || nb == 0 || slots[k].tkey / 1000000 == slots[k - 1].tkey / 1000000);
             ++nb) {
          long long bk = slots[k].tkey;
          int bp1 = (int)(bk / 1000000), b3 = (int)(bk % 1000000);
          if (i8) std::swap(bp1, b3);
          tl.p1_0[nb] = bp1 * TRI_P1 - o1;
          tl.p3_0[nb] = p3min - o3 + b3 * BW;
          gr.w3lo = std::min(gr.w3lo, tl.p3_0[nb]);
          gr.w3hi = std::max(gr.w3hi, tl.p3_0[nb]);
          for (; k < slots.size() && slots[k].tkey == bk && slots[k].gkey == gk; ++k) {
            const Slot &s = slots[k];
            tc[s.a * 32 + nb * BW + s.lane] = s.c;
            int p1 = combo_p1[s.c], p2 = combo_p2[s.c], p3 = -p1 - p2;
            gr.p1lo = std::min(gr.p1lo, p1); gr.p1hi = std::max(gr.p1hi, p1);
            gr.p2lo = std::min(gr.p2lo, p2); gr.p2hi = std::max(gr.p2hi, p2);
            gr.p3lo = std::min(gr.p3lo, p3); gr.p3hi = std::max(gr.p3hi, p3);
          }
          gr.tp1lo = std::min(gr.tp1lo, tl.p1_0[nb]);
          gr.tp1hi = std::max(gr.tp1hi, tl.p1_0[nb]);
        }
        tl.nblk = nb;
        for (int n = nb; n < TRI_BLOCKS; ++n) {  // unused blocks repeat the first one (no combos)
          tl.p1_0[n] = tl.p1_0[0];
          tl.p3_0[n] = tl.p3_0[0];
        }
        tiles.back() = tl;
        gr.ntiles++;
      }
      if (gr.ntiles > (i8 ? I8_MAX_TILES : TRI_WARPS)) too_big[u] = 1;
      groups[u].push_back(gr);
    }
  };
  {
    const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    host_parallel(nt, [&](int k) {
      for (int u = k; u < d.n_used; u += nt)
        if (own[u]) tile_triplet(u);
    });
    for (int u = 0; u < d.n_used; ++u) {
      if (too_big[u]) {
        set_detail("tile group larger than a CTA");
        return BEAM_EINVAL;
      }
      const int base = (int)tiles.size();
      for (Group &gr : groups[u]) gr.tile0 += base;
      tiles.insert(tiles.end(), u_tiles[u].begin(), u_tiles[u].end());
      tile_combo.insert(tile_combo.end(), u_tc[u].begin(), u_tc[u].end());
      std::vector<TriTile>().swap(u_tiles[u]);
      std::vector<int32_t>().swap(u_tc[u]);
    }
  }
  // splits, pieces, chunks, items
  double total = 0.0;
  for (int u = 0; u < d.n_used; ++u)
    for (const Group &gr : groups[u]) total += (double)gr.ntiles * 256.0 * (double)(p->tri_first[u + 1] - p->tri_first[u]);
  const double target = std::max(1.0, total / (std::max(1, p->ctx->num_sms) * p->balance));
  // Splits per triplet: by work (load balance: about `balance` items' worth of
  // work per SM) and by list length (no CTA walks more than about tau_max
  // triangles: a CTA's time grows with its list, not its tiles). Each split
  // keeps a partial sum per combo, so tau_max starts at the plan's tau0
  // (TRI_TAU_MAX mixed, twice that FP64, unless tuned) and doubles while the partial sums would pass
  // max(PART_PER_COMBO x combos, PART_MIN) slots per realization.
  constexpr long long PART_PER_COMBO = 4, PART_MIN = 64LL << 20;
  std::vector<long long> nruns(d.n_used, 0);
  std::vector<double> wmaxu(d.n_used, 0.0);
  long long max_nt = 1;
  for (int u = 0; u < d.n_used; ++u) {
    if (!own[u]) continue;
    const long long nt = p->tri_first[u + 1] - p->tri_first[u];
    max_nt = std::max(max_nt, nt);
    for (long long k = k2base[u]; k < k2base[u + 1]; ++k) nruns[u] += (k2cnt[k] > 0);
    for (const Group &gr : groups[u]) wmaxu[u] = std::max(wmaxu[u], (double)gr.ntiles * 256.0 * (double)nt);
  }
  p->n_run_combos = 0;
  for (int u = 0; u < d.n_used; ++u) p->n_run_combos += nruns[u] * (long long)u_ncombo[u];
  auto splits = [&](int u, long long tau_max) {
    const long long nt = p->tri_first[u + 1] - p->tri_first[u];
    double want = std::max(std::ceil(wmaxu[u] / target), std::ceil((double)nt / (double)tau_max));
    return (int)std::min<double>(std::max(1.0, want), (double)std::max<long long>(1, nruns[u]));
  };
  long long tau_max = std::max<long long>(16, p->tau0);
  for (;;) {
    long long slots = 0;
    for (int u = 0; u < d.n_used; ++u) slots += own[u] ? (long long)splits(u, tau_max) * u_ncombo[u] : u_ncombo[u];
    if (slots <= std::max(PART_PER_COMBO * (long long)combo_p1.size(), PART_MIN) || tau_max >= max_nt) break;
    tau_max *= 2;
  }
  std::vector<TriChunk> chunks;
  std::vector<int2> pieces;
  std::vector<TriItem> items;
  std::vector<double> work;
  u_nsplit.assign(d.n_used, 1);
  u_part.assign(d.n_used + 1, 0);
  for (int u = 0; u < d.n_used; ++u) {
    if (!own[u]) {
      u_part[u + 1] = u_part[u] + u_ncombo[u];
      continue;
    }
    const long long nt = p->tri_first[u + 1] - p->tri_first[u];
    std::vector<int2> runs;  // (length, k2)
    for (long long k = k2base[u]; k < k2base[u + 1]; ++k)
      for (int left = k2cnt[k]; left > 0;) {  // int8: runs of at most I8_RUN_MAX (exact int32 sums)
        const int len = i8 ? std::min(left, I8_RUN_MAX) : left;
        runs.push_back(make_int2(len, (int)(k - k2base[u])));
        left -= len;
      }
    int ns = splits(u, tau_max);
    u_nsplit[u] = ns;
    u_part[u + 1] = u_part[u] + (long long)ns * u_ncombo[u];
    int rp = p->used_rp[u];
    const int ly = u_swap[u] ? 2 : 1, lz = u_swap[u] ? 1 : 2;  // run leg and tile leg
    int m1 = p->ring_first[g.rp[3 * rp]], m2 = p->ring_first[g.rp[3 * rp + ly]],
        m3 = p->ring_first[g.rp[3 * rp + lz]];
    size_t r = 0;
    long long t = p->tri_first[u], done = 0;
    for (int s = 0; s < ns; ++s) {
      long long goal = nt * (s + 1) / ns;
      int ch0 = (int)chunks.size();
      // chunk under construction: triangles, pieces, piece lengths and the
      // run-continuation flags
      long long ct0 = t;
      int cpc0 = (int)pieces.size(), cnt_ = 0, cnpc = 0, clens = 0, cflags = 0;
      long long tsplit = 0;
      auto close_chunk = [&]() {
        chunks.push_back(TriChunk{ct0, cpc0, chunk_pack(cnt_, cnpc, clens, cflags)});
        tsplit += cnt_;
        ct0 = t;
        cpc0 = (int)pieces.size();
        cnt_ = cnpc = clens = cflags = 0;
      };
      while (r < runs.size() && (done < goal || s == ns - 1)) {
        // A run that does not fit the chunk's room goes on in the next chunk:
        // its part here is a whole number of groups of 4 triangles (the FP64
        // consumer's MMA depth), so only a run's last part can be ragged.
        int left = runs[r].x;
        bool cont = false;
        while (left > 0) {
          // int8: one run per chunk (a chunk is one MMA depth of 16 triangles)
          if (cnpc == TRI_PIECES || TRI_CHUNK - cnt_ < std::min(left, 4) || (i8 && cnt_ > 0)) close_chunk();
          const int room = TRI_CHUNK - cnt_;  // >= 4 whenever the run does not fit
          const int len = left <= room ? left : (room / 4) * 4;
          const bool more = len < left;
          pieces.push_back(make_int2(len, runs[r].y));
          clens |= len << (5 * cnpc);
          if (cnpc == 0 && cont) cflags |= CHUNK_CONT_IN;
          cnt_ += len;
          cnpc += 1;
          t += len;
          left -= len;
          cont = more;
          if (more) {
            cflags |= CHUNK_CONT_OUT;
            close_chunk();
          }
        }
        done += runs[r].x;
        ++r;
      }
      if (cnt_ > 0) close_chunk();
      int ch1 = (int)chunks.size();
      for (const Group &gr : groups[u]) {
        TriItem it;
        it.u = u;
        it.split = s;
        it.ch0 = ch0;
        it.ch1 = ch1;
        it.tile0 = gr.tile0;
        it.ntiles = gr.ntiles;
        it.m1 = m1;
        it.m2 = m2;
        it.m3 = m3;
        // staged columns: x over the tiles' full p1 blocks (read warp-wide),
        // z over the accepted p3, y over the accepted p2 widened by TRI_P1 - 1
        // (a lane reads y for all TRI_P1 planes p1 of its tile)
        const int cb = d.colbase, ext = TRI_P1 - 1;
        it.colx = floorA(gr.tp1lo + cb); it.Lx = ceilA(gr.tp1hi + ext + cb + 1) - it.colx;
        it.colz = floorA(gr.p3lo + cb); it.Lz = ceilA(gr.p3hi + cb + 1) - it.colz;
        if (i8) {  // the group's windows (rows outside the mode rows read column 0)
          it.colz = std::max(0, floorA(gr.w3lo + cb));
          it.Lz = std::min(d.W, ceilA(gr.w3hi + I8_BW + cb)) - it.colz;
        }
        it.rx = g.rp[3 * rp];
        it.rz = g.rp[3 * rp + lz];
        it.coly = floorA(gr.p2lo - ext + cb); it.Ly = ceilA(gr.p2hi + ext + cb + 1) - it.coly;
        if (it.colx < 0 || it.colx + it.Lx > d.W || it.colz < 0 || it.colz + it.Lz > d.W || it.coly < 0 ||
            it.coly + it.Ly > d.W)
          return set_detail("staged columns outside the mode rows"), BEAM_EINVAL;
        items.push_back(it);
        work.push_back((double)gr.ntiles * 256.0 * (double)tsplit);
      }
    }
  }
  // consistency: every owned combo in exactly one tile slot, every owned
  // triangle in exactly one chunk
  {
    std::vector<char> seen(combo_p1.size(), 0);
    long long owned_terms = 0;
    for (int u = 0; u < d.n_used; ++u) {
      if (own[u]) {
        owned_terms += p->tri_first[u + 1] - p->tri_first[u];
        continue;
      }
      for (int c = u_cfirst[u]; c < u_cfirst[u] + u_ncombo[u]; ++c) seen[c] = 2;
    }
    if (A == 4 && !i8)  // the mixed consumer's float4 reads of x and z
      for (const TriTile &tl : tiles)
        for (int n = 0; n < TRI_BLOCKS; ++n)
          if ((tl.p1_0[n] & 3) || (tl.p3_0[n] & 3)) return set_detail("mixed tile block off a 4-plane boundary"), BEAM_EINVAL;
    for (int32_t c : tile_combo)
      if (c >= 0) {
        if (seen[c]) return set_detail("combo placed twice or outside its shard"), BEAM_EINVAL;
        seen[c] = 1;
      }
    for (char v : seen)
      if (!v) return set_detail("combo without a tile"), BEAM_EINVAL;
    long long covered = 0, piece_sum = 0;
    for (size_t c = 0; c < chunks.size(); ++c) {
      const TriChunk &k = chunks[c];
      if (chunk_cont_out(k.packed)) {
        // the next chunk carries the run on: same run mode, no piece after it here
        if (c + 1 >= chunks.size() || !chunk_cont_in(chunks[c + 1].packed) ||
            pieces[chunks[c + 1].pc0].y != pieces[k.pc0 + chunk_npc(k.packed) - 1].y)
          return set_detail("run continuation"), BEAM_EINVAL;
      }
      if (chunk_cont_in(k.packed) && (c == 0 || !chunk_cont_out(chunks[c - 1].packed)))
        return set_detail("run continuation"), BEAM_EINVAL;
    }
    for (const TriChunk &k : chunks) {
      int nt = chunk_nt(k.packed), npc = chunk_npc(k.packed), lsum = 0;
      covered += nt;
      for (int j = 0; j < npc; ++j) {
        piece_sum += pieces[k.pc0 + j].x;
        lsum += chunk_len(k.packed, j);
        if (chunk_len(k.packed, j) != pieces[k.pc0 + j].x) return set_detail("packed piece length"), BEAM_EINVAL;
      }
      if (lsum != nt) return set_detail("chunk length"), BEAM_EINVAL;
    }
    if (covered != owned_terms || piece_sum != owned_terms)
      return set_detail("chunks do not cover the triangle lists"), BEAM_EINVAL;
  }
  // grouped by tile count (one launch per count, CTAs of that many warps),
  // largest work first within a group so each launch ends on small items
  std::vector<int> order(items.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return items[a].ntiles != items[b].ntiles ? items[a].ntiles < items[b].ntiles : work[a] > work[b];
  });
  std::vector<TriItem> sorted(items.size());
  for (size_t k = 0; k < order.size(); ++k) sorted[k] = items[order[k]];
  // the persistent kernel's order: every item by decreasing work (ties: class order)
  std::vector<int32_t> q_order(items.size());
  std::iota(q_order.begin(), q_order.end(), 0);
  std::stable_sort(q_order.begin(), q_order.end(), [&](int x, int y) { return work[order[x]] > work[order[y]]; });
  size_t elem = (A == 1) ? 16 : 8;
  size_t budget = p->ctx->smem_optin > 4096 ? p->ctx->smem_optin - 4096 : 48 * 1024;
  for (int n = 0; n <= TRI_CLASSES + 1; ++n) d.class_first[n] = 0;
  for (int n = 0; n <= TRI_CLASSES; ++n) d.class_stage[n] = 0;
  for (const TriItem &it : sorted) {
    d.class_first[it.ntiles + 1]++;
    const bool f64 = (A == 1);
    int stage = TRI_CHUNK * (stage_pitch(it.Lx, f64) + stage_pitch(it.Lz, f64)) + TRI_PIECES * it.Ly;
    if (i8) stage = i8_stage_bytes(it);  // in bytes
    d.class_stage[it.ntiles] = std::max(d.class_stage[it.ntiles], stage);
  }
  if (i8) elem = 1;
  for (int n = 0; n <= TRI_CLASSES; ++n) d.class_first[n + 1] += d.class_first[n];
  for (int n = 1; n <= TRI_CLASSES; ++n)
    if ((size_t)(i8 ? I8_STAGES : TRI_STAGES) * d.class_stage[n] * elem + (i8 ? (size_t)n * 8 * 32 * sizeof(double) : 0) >
        budget) {
      set_detail("staged mode rows do not fit shared memory");
      return BEAM_EINVAL;
    }
  d.n_tiles = (int)tiles.size();
  d.n_chunks = (long long)chunks.size();
  d.n_pieces = (long long)pieces.size();
  d.n_items = (int)sorted.size();
  BEAM_TRY(upload(p, &d.tiles, tiles));
  BEAM_TRY(upload(p, &d.tile_combo, tile_combo));
  BEAM_TRY(upload(p, &d.chunks, chunks));
  BEAM_TRY(upload(p, &d.pieces, pieces));
  BEAM_TRY(upload(p, &d.items, sorted));
  BEAM_TRY(upload(p, &d.q_order, q_order));
  // per-chunk copy descriptors; the list, chunk and piece tables are then no longer needed
  BEAM_TRY(dev_alloc(p, &d.descs, (size_t)d.n_chunks));
  if (d.n_chunks) {
    k_build_desc<<<(unsigned)((d.n_chunks + 255) / 256), 256, 0, p->ctx->stream>>>(d.chunks, d.n_chunks, d.tri_list,
                                                                                   d.pieces, d.descs);
    BEAM_CUDA(cudaGetLastError());
    BEAM_CUDA(cudaStreamSynchronize(p->ctx->stream));
  }
  cudaFree(d.chunks);
  cudaFree(d.pieces);
  cudaFree(d.tri_list);
  p->device_bytes -= sizeof(TriChunk) * d.n_chunks + sizeof(int2) * d.n_pieces + sizeof(ushort4) * d.n_terms;
  d.chunks = nullptr;
  d.pieces = nullptr;
  d.tri_list = nullptr;
  return BEAM_OK;
}

int build_plan_tables(beam_gpu_plan *p) {
  const beam_geom &g = p->geom;
  DevPlan &d = p->d;
  const long NN = g.NN, Nr = g.Nr;
  const long long ntri = g.ntri;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return (float)std::chrono::duration<double, std::milli>(b - a).count();
  };
  const auto t0 = now();

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
  // kept in multiples of A complex values (1 for complex128; 4 for the mixed
  // path, whose rows hold blocks of 4 real parts then their 4 imaginary parts,
  // so a copied segment starts and ends on a whole block; 4 for the int8
  // path, whose slice sub-rows hold 4 bytes per column)
  const bool i8 = p->cfg.precision == BEAM_PREC_INT8;
  const int A = (p->cfg.precision == BEAM_PREC_MIXED || i8) ? 4 : 1;
  auto floorA = [A](int v) { return v - (((v % A) + A) % A); };
  auto ceilA = [A, &floorA](int v) { return floorA(v + A - 1); };
  d.Q = Q;
  // plane 0 at a column that is a multiple of A (the mixed consumer reads a
  // tile's 8 planes p1, which start at multiples of 8, as aligned float4s)
  d.colbase = ceilA(Q - 1 + TRI_PAD);
  d.W = ceilA(d.colbase + Q + TRI_PAD);

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
  std::vector<int32_t> u_cfirst, u_ncombo(d.n_used, 0);
  std::vector<int32_t> combo_p1(ntri), combo_p2(ntri), combo_u(ntri), combo_tid(ntri);
  {
    // combos grouped by triplet, loop order within a triplet
    std::vector<int32_t> at;
    stable_bucket_sort(ntri, d.n_used, [&](long long t) { return u_of_rp[g.t_rp[t]]; }, at, u_cfirst);
    for (int u = 0; u < d.n_used; ++u) u_ncombo[u] = u_cfirst[u + 1] - u_cfirst[u];
    const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    host_parallel(nt, [&](int k) {
      for (long long t = ntri * k / nt; t < ntri * (k + 1) / nt; ++t) {
        const int c = at[t];
        combo_p1[c] = g.t_p1[t];
        combo_p2[c] = g.t_p2[t];
        combo_u[c] = u_of_rp[g.t_rp[t]];
        combo_tid[c] = (int32_t)t;
      }
    });
  }

  // bin order (stable in loop order)
  d.n_bins = g.n_k1bin * g.n_mtbin * g.n_mtbin;
  std::vector<int32_t> bin_first;
  stable_bucket_sort(ntri, d.n_bins, [&](long long t) { return g.t_bin[t]; }, p->bin_pos, bin_first);
  p->loop_of_bin.assign(ntri, 0);
  for (long long t = 0; t < ntri; ++t) p->loop_of_bin[p->bin_pos[t]] = (int32_t)t;
  std::vector<int32_t> combo_out(ntri);
  for (long long c = 0; c < ntri; ++c) combo_out[c] = p->bin_pos[combo_tid[c]];

  // Run leg of each used triplet: of rings r2 and r3, the one with fewer
  // distinct modes in the triplet's in-plane list, so its runs are longer and
  // the product with the run leg (once per run and accepted triangle) is paid
  // fewer times. At NN=384 this lengthens the mean run (weighted by work) from
  // 17 to 50 triangles. Both orientations are counted on the GPU.
  std::vector<char> u_swap(d.n_used, 0);
  std::vector<int> chosen;  // the counts of the chosen orientation, triplet by triplet
  {
    std::vector<int> c2, c3;
    BEAM_TRY(count_both_orientations(p, d.mode_ij, d.ringmap, d.pixlocal, c2, c3));
    size_t a2 = 0, a3 = 0;
    for (int u = 0; u < d.n_used; ++u) {
      const int rp = p->used_rp[u], r2 = g.rp[3 * rp + 1], r3 = g.rp[3 * rp + 2];
      const int n2 = p->ring_first[r2 + 1] - p->ring_first[r2], n3 = p->ring_first[r3 + 1] - p->ring_first[r3];
      long long runs2 = 0, runs3 = 0;
      for (int k = 0; k < n2; ++k) runs2 += (c2[a2 + k] > 0);
      for (int k = 0; k < n3; ++k) runs3 += (c3[a3 + k] > 0);
      u_swap[u] = runs3 < runs2;
      const std::vector<int> &src = u_swap[u] ? c3 : c2;
      const size_t at = u_swap[u] ? a3 : a2;
      chosen.insert(chosen.end(), src.begin() + at, src.begin() + at + (u_swap[u] ? n3 : n2));
      a2 += n2;
      a3 += n3;
    }
  }
  // the tile axis of a triplet is the tile leg's plane; combo_p2 below holds
  // the run leg's plane (p3 for a swapped triplet), the tile's p3 = -p1 - it
  for (long long c = 0; c < ntri; ++c)
    if (u_swap[combo_u[c]]) combo_p2[c] = -combo_p1[c] - combo_p2[c];

  // in-plane triangle lists (GPU), run-leg-major: k2cnt holds each run's length
  std::vector<int> k2cnt;
  BEAM_TRY(enumerate_in_plane(p, p->used_rp, p->ring_first, d.mode_ij, d.ringmap, d.pixlocal, p->tri_first,
                              &d.tri_list, &d.n_terms, &k2cnt, &u_swap, &chosen));

  // epilogue tables in bin order
  std::vector<double> ep_px(ntri), ep_pz(ntri), ep_ana(ntri);
  std::vector<int32_t> ep_cnt(ntri);
  {
    const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    host_parallel(nt, [&](int k) {
      for (long long i = ntri * k / nt; i < ntri * (k + 1) / nt; ++i) {
        long long t = p->loop_of_bin[i];
        ep_px[i] = g.t_px[t];
        ep_pz[i] = g.t_pz[t];
        ep_ana[i] = g.t_ana[t];
        int u = u_of_rp[g.t_rp[t]];
        ep_cnt[i] = (int32_t)(p->tri_first[u + 1] - p->tri_first[u]);
      }
    });
  }

  // ring triplets this shard sums: longest-processing-time assignment by
  // work = accepted triangles x in-plane triangles
  std::vector<char> own(d.n_used, 1);
  p->u_owner.assign(d.n_used, 0);
  if (p->cfg.shard_count > 1) {
    std::vector<double> uwork(d.n_used);
    for (int u = 0; u < d.n_used; ++u)
      uwork[u] = (double)u_ncombo[u] * (double)(p->tri_first[u + 1] - p->tri_first[u]);
    beam_shard_assign(uwork.data(), d.n_used, p->cfg.shard_count, p->u_owner.data());
    for (int u = 0; u < d.n_used; ++u) own[u] = (p->u_owner[u] == p->cfg.shard_index);
  }

  // work decomposition of the triangle-sum kernel
  const auto t1 = now();
  p->build_ms[1] = ms(t0, t1);
  std::vector<int32_t> u_nsplit;
  std::vector<long long> u_part;
  BEAM_TRY(build_work(p, u_cfirst, u_ncombo, combo_p1, combo_p2, k2cnt, own, u_swap, A, u_nsplit, u_part));
  const auto t2 = now();
  p->build_ms[2] = ms(t1, t2);
  d.n_part = u_part[d.n_used];
  u_part.pop_back();
  u_cfirst.pop_back();

  BEAM_TRY(upload(p, &d.combo_u, combo_u));
  BEAM_TRY(upload(p, &d.combo_out, combo_out));
  BEAM_TRY(upload(p, &d.u_cfirst, u_cfirst));
  BEAM_TRY(upload(p, &d.u_ncombo, u_ncombo));
  BEAM_TRY(upload(p, &d.u_nsplit, u_nsplit));
  BEAM_TRY(upload(p, &d.u_part, u_part));
  BEAM_TRY(upload(p, &d.bin_first, bin_first));
  {
    // epilogue chunks: each bin cut into ranges of at most EP_CHUNK triangles
    std::vector<int32_t> chunk_first, bin_chunk(d.n_bins + 1, 0);
    for (int b = 0; b < d.n_bins; ++b) {
      bin_chunk[b] = (int32_t)chunk_first.size();
      for (int32_t t = bin_first[b]; t < bin_first[b + 1]; t += EP_CHUNK) chunk_first.push_back(t);
    }
    bin_chunk[d.n_bins] = (int32_t)chunk_first.size();
    d.n_epchunks = (int)chunk_first.size();
    chunk_first.push_back(bin_first[d.n_bins]);
    // chunk c covers [chunk_first[c], chunk_first[c+1]): bins are contiguous in
    // bin order, so a bin's last chunk ends where the next non-empty bin begins
    BEAM_TRY(upload(p, &d.ep_chunk_first, chunk_first));
    BEAM_TRY(upload(p, &d.bin_chunk, bin_chunk));
  }
  BEAM_TRY(upload(p, &d.ep_px, ep_px));
  BEAM_TRY(upload(p, &d.ep_pz, ep_pz));
  BEAM_TRY(upload(p, &d.ep_ana, ep_ana));
  BEAM_TRY(upload(p, &d.ep_cnt, ep_cnt));

  d.elem = (p->cfg.precision == BEAM_PREC_MIXED) ? sizeof(float2) : (i8 ? 48 : sizeof(double2));
  d.i8 = i8 ? 1 : 0;
  d.n_rings = (int)Nr;
  if (i8) BEAM_TRY(upload(p, &d.ring_first, p->ring_first));
  p->build_ms[3] = ms(t2, now());
  return BEAM_OK;
}

void free_plan_tables(beam_gpu_plan *p) {
  DevPlan &d = p->d;
  void *ptrs[] = {d.mode_ij,  d.mode_neg, d.ringmap, d.pixlocal,   d.tri_list, d.combo_u, d.combo_out,
                  d.u_cfirst, d.u_ncombo, d.u_nsplit, d.u_part,    d.tiles,    d.tile_combo, d.chunks,
                  d.pieces,   d.descs,    d.items,    d.q_order,   d.bin_first, d.ep_px,  d.ep_pz,   d.ep_cnt,
                  d.ep_chunk_first, d.bin_chunk, d.ep_ana, d.ring_first};
  for (void *q : ptrs)
    if (q) cudaFree(q);
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
  const cudaError_t ce = cudaMemcpy(d_mode, mode_ij.data(), sizeof(int16_t) * mode_ij.size(), cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    cudaFree(d_mode);
    set_detail(std::string("cudaMemcpy(mode table): ") + cudaGetErrorString(ce));
    return BEAM_ECUDA;
  }
  std::vector<int> rps(g.nrp);
  std::iota(rps.begin(), rps.end(), 0);
  std::vector<long long> first;
  size_t before = p->device_bytes;
  int rc = enumerate_in_plane(p, rps, ring_first, d_mode, p->d.ringmap, nullptr, first, nullptr, nullptr, nullptr);
  p->device_bytes = before;
  cudaFree(d_mode);
  if (rc != BEAM_OK) return rc;
  counts.resize(g.nrp);
  for (long k = 0; k < g.nrp; ++k) counts[k] = first[k + 1] - first[k];
  return BEAM_OK;
}

}  // namespace beam
