// Plane-ring transforms and the reference-literal pixel-sum method.
//
// k_plane_ring_dft computes, for a (plane p, ring r) pair, the unnormalised
// backward 2D DFT of the ring-masked plane (Df, funcs.c:88-109):
//   F[x][y] = sum_{(i,j) in ring r} D(i,j,p) exp(+2 pi i (i x + j y)/NN),
// with D(0,0,0) = 0. A ring's modes occupy few rows i, so the transform is
// taken as two separable direct sums over the non-zero entries only:
//   G[i][y] = sum_j D(i,j,p) w^(j y)      (rows of the ring)
//   F[x][y] = sum_i G[i][y]  w^(i x)      (non-zero rows only)
// with w^k read from a table of exp(+2 pi i k/NN). One CTA produces a block of
// PR_YB output columns of one (plane, ring) array.
//
// The pixel method then sums Re(F1 F2^(s2) F3^(s3)) over all NN^2 pixels per
// accepted triangle (barbie.c:329-337), with the whole plane-ring cache held in
// device memory instead of the reference's per-(plane,ring) files.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "beam_internal.h"

namespace beam {

constexpr int PR_YB = 16;        // output columns per CTA
constexpr int PR_THREADS = 256;

struct RingRows {                // non-zero rows of one ring in the all-ring mode table
  int first_row, n_rows;         // into row_i / row_mode
};

struct PixelPath {
  // all-ring mode table and per-ring row lists
  std::vector<int32_t> ring_first;  // [Nr+1]
  int16_t *mode_ij = nullptr;       // [modes][2]
  int32_t *row_i = nullptr;         // [rows] row index i
  int32_t *row_mode = nullptr;      // [rows+1] first mode of each row (sentinel at end)
  RingRows *ring_rows = nullptr;    // [Nr]
  std::vector<RingRows> h_ring_rows;
  double2 *tw = nullptr;            // [NN] exp(+2 pi i k/NN)
  int max_rows = 0;
  // pixel method (only when the plan's method is BEAM_METHOD_PIXEL)
  double *r2c = nullptr;            // device copy of the r2c buffer
  int n_slots = 0;                  // (plane, ring) arrays in the cache
  int32_t *slot_plane = nullptr, *slot_ring = nullptr;
  double *cache = nullptr;          // [n_slots][NN*NN] complex128
  // plane-pair groups
  int n_pairs = 0;
  int32_t *pair_first = nullptr;    // [n_pairs+1] into the pair-ordered triangle arrays
  int32_t *pair_row_first = nullptr;// [n_pairs+1] into pair_rows
  int32_t *pair_rows = nullptr;     // cache slot of each row used by the pair
  int32_t *tri_rows = nullptr;      // [ntri] packed (ra | rb<<10 | rc<<20) local rows
  int32_t *tri_sign = nullptr;      // [ntri] bit0: conj leg 2, bit1: conj leg 3
  int32_t *tri_out = nullptr;       // [ntri] bin-order output position
  int max_pair_rows = 0;
  int xtile = 0;
};

static PixelPath *pix_of(const beam_gpu_plan *p) { return p->pix; }

bool pixel_method(const beam_gpu_plan *p) { return p->cfg.method == BEAM_METHOD_PIXEL; }

template <typename C>
struct PrOut;
template <>
struct PrOut<double2> {
  static __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
};
template <>
struct PrOut<float2> {
  static __device__ __forceinline__ float2 make(double a, double b) { return make_float2((float)a, (float)b); }
};

// grid.x: column block, grid.y: (plane, ring) job
template <typename C>
__global__ void __launch_bounds__(PR_THREADS)
    k_plane_ring_dft(const double2 *__restrict__ r2c, int NN, const int32_t *__restrict__ job_plane,
                     const int32_t *__restrict__ job_ring, const RingRows *__restrict__ ring_rows,
                     const int32_t *__restrict__ row_i, const int32_t *__restrict__ row_mode,
                     const int16_t *__restrict__ mode_ij, const double2 *__restrict__ tw, C *__restrict__ out,
                     long long out_stride) {
  extern __shared__ __align__(16) unsigned char pr_smem[];
  double2 *s_tw = reinterpret_cast<double2 *>(pr_smem);  // [NN]
  double2 *s_g = s_tw + NN;                               // [n_rows][PR_YB]
  const int job = blockIdx.y;
  const int p = job_plane[job], r = job_ring[job];
  const RingRows rr = ring_rows[r];
  const int y0 = blockIdx.x * PR_YB;
  const int NH = NN / 2 + 1;
  for (int k = threadIdx.x; k < NN; k += PR_THREADS) s_tw[k] = tw[k];
  __syncthreads();
  // rows: G[s][yy] = sum over the row's modes of D(i,j,p) w^(j y)
  for (int e = threadIdx.x; e < rr.n_rows * PR_YB; e += PR_THREADS) {
    int s = e / PR_YB, yy = e % PR_YB, y = y0 + yy;
    double gr = 0.0, gi = 0.0;
    if (y < NN) {
      int row = rr.first_row + s;
      for (int m = row_mode[row]; m < row_mode[row + 1]; ++m) {
        int i = mode_ij[2 * m], j = mode_ij[2 * m + 1];
        double2 d = r2c[((size_t)i * NN + j) * NH + p];
        if (p == 0 && i == 0 && j == 0) d = make_double2(0.0, 0.0);
        double2 w = s_tw[(int)(((long long)j * y) % NN)];
        gr += d.x * w.x - d.y * w.y;
        gi += d.x * w.y + d.y * w.x;
      }
    }
    s_g[s * PR_YB + yy] = make_double2(gr, gi);
  }
  __syncthreads();
  // columns: F[x][y] = sum_s G[s][y] w^(i_s x)
  C *o = out + (long long)job * out_stride;
  for (int e = threadIdx.x; e < NN * PR_YB; e += PR_THREADS) {
    int x = e / PR_YB, yy = e % PR_YB, y = y0 + yy;
    if (y >= NN) continue;
    double fr = 0.0, fi = 0.0;
    for (int s = 0; s < rr.n_rows; ++s) {
      int i = row_i[rr.first_row + s];
      double2 w = s_tw[(int)(((long long)i * x) % NN)];
      double2 g = s_g[s * PR_YB + yy];
      fr += g.x * w.x - g.y * w.y;
      fi += g.x * w.y + g.y * w.x;
    }
    o[(size_t)x * NN + y] = PrOut<C>::make(fr, fi);
  }
}

static int build_transform_tables(beam_gpu_plan *p, PixelPath *px) {
  const beam_geom &g = p->geom;
  const long NN = g.NN, Nr = g.Nr;
  std::vector<std::vector<int32_t>> per(Nr);
  for (long x = 0; x < NN * NN; ++x)
    if (g.ringmap[x] >= 0) per[g.ringmap[x]].push_back((int32_t)x);
  px->ring_first.assign(Nr + 1, 0);
  std::vector<int16_t> mode_ij;
  std::vector<int32_t> row_i, row_mode;
  px->h_ring_rows.assign(Nr, RingRows{0, 0});
  int m = 0;
  for (long r = 0; r < Nr; ++r) {
    px->ring_first[r] = m;
    px->h_ring_rows[r].first_row = (int)row_i.size();
    int last_i = -1;
    for (int32_t x : per[r]) {
      int i = (int)(x / NN), j = (int)(x % NN);
      if (i != last_i) {
        row_i.push_back(i);
        row_mode.push_back(m);
        last_i = i;
      }
      mode_ij.push_back((int16_t)i);
      mode_ij.push_back((int16_t)j);
      ++m;
    }
    px->h_ring_rows[r].n_rows = (int)row_i.size() - px->h_ring_rows[r].first_row;
    px->max_rows = std::max(px->max_rows, px->h_ring_rows[r].n_rows);
  }
  px->ring_first[Nr] = m;
  row_mode.push_back(m);
  std::vector<double2> tw(NN);
  for (long k = 0; k < NN; ++k) {
    double a = 2.0 * M_PI * (double)k / (double)NN;
    tw[k] = make_double2(std::cos(a), std::sin(a));
  }
  auto up = [&](auto **dst, const auto &src) -> int {
    using T = typename std::remove_reference<decltype(src)>::type::value_type;
    BEAM_TRY(dev_alloc(p, reinterpret_cast<T **>(dst), src.size()));
    if (!src.empty()) BEAM_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
    return BEAM_OK;
  };
  BEAM_TRY(up(&px->mode_ij, mode_ij));
  BEAM_TRY(up(&px->row_i, row_i));
  BEAM_TRY(up(&px->row_mode, row_mode));
  BEAM_TRY(up(&px->ring_rows, px->h_ring_rows));
  BEAM_TRY(up(&px->tw, tw));
  return BEAM_OK;
}

static PixelPath *ensure_pix(beam_gpu_plan *p, int *rc) {
  PixelPath *px = pix_of(p);
  *rc = BEAM_OK;
  if (px) return px;
  px = new PixelPath();
  p->pix = px;
  *rc = build_transform_tables(p, px);
  return px;
}

template <typename C>
static int launch_dft(beam_gpu_plan *p, PixelPath *px, const double *r2c_dev, const int32_t *d_plane,
                      const int32_t *d_ring, int n, C *out, long long stride) {
  if (n == 0) return BEAM_OK;
  const int NN = (int)p->geom.NN;
  size_t smem = sizeof(double2) * ((size_t)NN + (size_t)std::max(1, px->max_rows) * PR_YB);
  BEAM_CUDA(cudaFuncSetAttribute(k_plane_ring_dft<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int j0 = 0; j0 < n; j0 += 65535) {
    int nj = std::min(65535, n - j0);
    dim3 grid((NN + PR_YB - 1) / PR_YB, nj);
    k_plane_ring_dft<C><<<grid, PR_THREADS, smem, p->ctx->stream>>>(
        (const double2 *)r2c_dev, NN, d_plane + j0, d_ring + j0, px->ring_rows, px->row_i, px->row_mode, px->mode_ij,
        px->tw, out + (long long)j0 * stride, stride);
  }
  BEAM_CUDA(cudaGetLastError());
  return BEAM_OK;
}

int plane_rings(beam_gpu_plan *p, const double *r2c, int on_device, const int *planes, const int *rings, int n,
                double *out, int out_on_device) {
  const beam_geom &g = p->geom;
  for (int k = 0; k < n; ++k)
    if (planes[k] < 0 || planes[k] >= g.Nmax || planes[k] > g.NN / 2 || rings[k] < 0 || rings[k] >= g.Nr)
      return BEAM_EINVAL;
  int rc;
  PixelPath *px = ensure_pix(p, &rc);
  if (rc != BEAM_OK) return rc;
  cudaStream_t s = p->ctx->stream;
  const size_t n2 = (size_t)g.NN * g.NN, rbytes = sizeof(double) * (size_t)g.NN * g.NN * (g.NN + 2);
  double *d_r2c = nullptr, *d_out = nullptr;
  int32_t *d_jobs = nullptr;
  // a failed CUDA call records its error and skips the rest; the temporary
  // buffers are freed on every path
  auto cuda_ok = [&](cudaError_t e, const char *what) {
    if (rc == BEAM_OK && e != cudaSuccess) {
      set_detail(std::string(what) + ": " + cudaGetErrorString(e));
      rc = BEAM_ECUDA;
    }
    return rc == BEAM_OK;
  };
  if (!on_device && cuda_ok(cudaMalloc(&d_r2c, rbytes), "cudaMalloc(r2c)"))
    cuda_ok(cudaMemcpyAsync(d_r2c, r2c, rbytes, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(r2c)");
  if (rc == BEAM_OK && !out_on_device)
    cuda_ok(cudaMalloc(&d_out, sizeof(double) * 2 * n2 * std::max(1, n)), "cudaMalloc(out)");
  if (rc == BEAM_OK && cuda_ok(cudaMalloc(&d_jobs, sizeof(int32_t) * 2 * std::max(1, n)), "cudaMalloc(jobs)") &&
      cuda_ok(cudaMemcpyAsync(d_jobs, planes, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(planes)"))
    cuda_ok(cudaMemcpyAsync(d_jobs + n, rings, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(rings)");
  if (rc == BEAM_OK) {
    size_t before = p->device_bytes;
    rc = launch_dft<double2>(p, px, on_device ? r2c : d_r2c, d_jobs, d_jobs + n, n,
                             (double2 *)(out_on_device ? out : d_out), (long long)n2);
    p->device_bytes = before;
  }
  if (rc == BEAM_OK && !out_on_device)
    cuda_ok(cudaMemcpyAsync(out, d_out, sizeof(double) * 2 * n2 * n, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync(out)");
  const cudaError_t se = cudaStreamSynchronize(s);  // before the buffers are freed, on every path
  cuda_ok(se, "cudaStreamSynchronize");
  cudaFree(d_r2c);
  cudaFree(d_out);
  cudaFree(d_jobs);
  return rc;
}

// ------------------------------------------------------------- pixel method
// One CTA per plane pair (p1, p2): the rows (cache arrays) the pair's triangles
// use are staged PIX_X pixels at a time; each thread owns triangles of the pair
// and accumulates Re(a * b^(s2) * c^(s3)) over the staged pixels.
constexpr int PIX_THREADS = 256;
constexpr int PIX_SLOTS = 8;

__global__ void __launch_bounds__(PIX_THREADS)
    k_pixel_sums(const double2 *__restrict__ cache, long long n2, int xtile, const int32_t *__restrict__ pair_first,
                 const int32_t *__restrict__ pair_row_first, const int32_t *__restrict__ pair_rows,
                 const int32_t *__restrict__ tri_rows, const int32_t *__restrict__ tri_sign,
                 const int32_t *__restrict__ tri_out, double *__restrict__ B) {
  extern __shared__ __align__(16) unsigned char px_smem[];
  double2 *tile = reinterpret_cast<double2 *>(px_smem);  // [rows][xtile]
  const int pr = blockIdx.x;
  const int rf = pair_row_first[pr], nrows = pair_row_first[pr + 1] - rf;
  const int t0 = pair_first[pr], t1 = pair_first[pr + 1];
  for (int tb = t0; tb < t1; tb += PIX_THREADS * PIX_SLOTS) {
    double acc[PIX_SLOTS];
    int ra[PIX_SLOTS], rb[PIX_SLOTS], rc[PIX_SLOTS];
    double s2[PIX_SLOTS], s3[PIX_SLOTS];
#pragma unroll
    for (int k = 0; k < PIX_SLOTS; ++k) {
      int t = tb + threadIdx.x + k * PIX_THREADS;
      acc[k] = 0.0;
      ra[k] = rb[k] = rc[k] = 0;
      s2[k] = s3[k] = 1.0;
      if (t < t1) {
        int packed = tri_rows[t], sg = tri_sign[t];
        ra[k] = packed & 1023;
        rb[k] = (packed >> 10) & 1023;
        rc[k] = (packed >> 20) & 1023;
        s2[k] = (sg & 1) ? -1.0 : 1.0;
        s3[k] = (sg & 2) ? -1.0 : 1.0;
      }
    }
    for (long long x0 = 0; x0 < n2; x0 += xtile) {
      int nx = (int)(xtile < n2 - x0 ? xtile : n2 - x0);
      __syncthreads();
      for (int e = threadIdx.x; e < nrows * nx; e += PIX_THREADS) {
        int rr = e / nx, xx = e % nx;
        tile[rr * xtile + xx] = cache[(long long)pair_rows[rf + rr] * n2 + x0 + xx];
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < PIX_SLOTS; ++k) {
        int t = tb + threadIdx.x + k * PIX_THREADS;
        if (t >= t1) continue;
        const double2 *A = tile + ra[k] * xtile, *Bv = tile + rb[k] * xtile, *Cv = tile + rc[k] * xtile;
        double a = acc[k];
        for (int xx = 0; xx < nx; ++xx) {
          double2 u = A[xx], v = Bv[xx], w = Cv[xx];
          double vi = s2[k] * v.y, wi = s3[k] * w.y;
          double ur = u.x * v.x - u.y * vi, ui = u.x * vi + u.y * v.x;
          a += ur * w.x - ui * wi;
        }
        acc[k] = a;
      }
    }
#pragma unroll
    for (int k = 0; k < PIX_SLOTS; ++k) {
      int t = tb + threadIdx.x + k * PIX_THREADS;
      if (t < t1) B[tri_out[t]] = acc[k];
    }
  }
}

int build_pixel_path(beam_gpu_plan *p) {
  int rc;
  PixelPath *px = ensure_pix(p, &rc);
  if (rc != BEAM_OK) return rc;
  const beam_geom &g = p->geom;
  const long long ntri = g.ntri;
  const long NN = g.NN;
  // cache slots for every (|p|, ring) a leg uses
  std::map<long long, int> slot_of;
  std::vector<int32_t> sp, sr;
  auto slot = [&](int plane, int ring) {
    long long key = (long long)plane * 4096 + ring;
    auto it = slot_of.find(key);
    if (it != slot_of.end()) return it->second;
    int s = (int)sp.size();
    slot_of[key] = s;
    sp.push_back(plane);
    sr.push_back(ring);
    return s;
  };
  // group triangles by plane pair (p1, p2), loop order within a pair
  std::map<long long, std::vector<long long>> pairs;
  for (long long t = 0; t < ntri; ++t) pairs[(long long)g.t_p1[t] * 100000 + (g.t_p2[t] + 50000)].push_back(t);
  std::vector<int32_t> pair_first(1, 0), pair_row_first(1, 0), pair_rows, tri_rows, tri_sign, tri_out;
  int max_rows = 1;
  for (auto &kv : pairs) {
    std::map<int, int> local;
    std::vector<int32_t> rows;
    auto lrow = [&](int s) {
      auto it = local.find(s);
      if (it != local.end()) return it->second;
      int l = (int)rows.size();
      local[s] = l;
      rows.push_back(s);
      return l;
    };
    for (long long t : kv.second) {
      int rp = g.t_rp[t];
      int r1 = g.rp[3 * rp], r2 = g.rp[3 * rp + 1], r3 = g.rp[3 * rp + 2];
      int p1 = g.t_p1[t], p2 = g.t_p2[t], p3 = -p1 - p2;
      int a = lrow(slot(p1, r1)), b = lrow(slot(std::abs(p2), r2)), c = lrow(slot(std::abs(p3), r3));
      tri_rows.push_back(a | (b << 10) | (c << 20));
      tri_sign.push_back((p2 < 0 ? 1 : 0) | (p3 < 0 ? 2 : 0));
      tri_out.push_back(p->bin_pos[t]);
    }
    if (rows.size() > 1023) {
      set_detail("a plane pair uses more than 1023 cache arrays");
      return BEAM_EINVAL;
    }
    max_rows = std::max(max_rows, (int)rows.size());
    pair_rows.insert(pair_rows.end(), rows.begin(), rows.end());
    pair_first.push_back((int32_t)tri_rows.size());
    pair_row_first.push_back((int32_t)pair_rows.size());
  }
  px->n_pairs = (int)pairs.size();
  px->n_slots = (int)sp.size();
  px->max_pair_rows = max_rows;
  size_t budget = p->ctx->smem_optin > 4096 ? p->ctx->smem_optin - 4096 : 48 * 1024;
  int xt = (int)std::min<size_t>(512, budget / (sizeof(double2) * max_rows));
  xt = (xt / 32) * 32;
  if (xt < 32) {
    set_detail("plane pair rows do not fit shared memory");
    return BEAM_EINVAL;
  }
  px->xtile = xt;
  auto up = [&](int32_t **dst, const std::vector<int32_t> &src) -> int {
    BEAM_TRY(dev_alloc(p, dst, src.size()));
    if (!src.empty()) BEAM_CUDA(cudaMemcpy(*dst, src.data(), sizeof(int32_t) * src.size(), cudaMemcpyHostToDevice));
    return BEAM_OK;
  };
  BEAM_TRY(up(&px->slot_plane, sp));
  BEAM_TRY(up(&px->slot_ring, sr));
  BEAM_TRY(up(&px->pair_first, pair_first));
  BEAM_TRY(up(&px->pair_row_first, pair_row_first));
  BEAM_TRY(up(&px->pair_rows, pair_rows));
  BEAM_TRY(up(&px->tri_rows, tri_rows));
  BEAM_TRY(up(&px->tri_sign, tri_sign));
  BEAM_TRY(up(&px->tri_out, tri_out));
  BEAM_TRY(dev_alloc(p, &px->r2c, (size_t)NN * NN * (NN + 2)));
  BEAM_TRY(dev_alloc(p, &px->cache, (size_t)px->n_slots * NN * NN * 2));
  return BEAM_OK;
}

int pixel_triangle_sums(beam_gpu_plan *p, const double *r2c, int on_device) {
  PixelPath *px = pix_of(p);
  if (!px || !px->cache) return BEAM_EINVAL;
  cudaStream_t s = p->ctx->stream;
  const long long NN = p->geom.NN, n2 = NN * NN;
  const double *src = r2c;
  if (!on_device) {
    BEAM_CUDA(cudaMemcpyAsync(px->r2c, r2c, sizeof(double) * NN * NN * (NN + 2), cudaMemcpyHostToDevice, s));
    src = px->r2c;
  }
  RunSlot *slot = p->main;
  BEAM_TRY(launch_dft<double2>(p, px, src, px->slot_plane, px->slot_ring, px->n_slots, (double2 *)px->cache, n2));
  slot->launches += (px->n_slots + 65534) / 65535;
  mark(slot, 1);
  if (px->n_pairs == 0) {
    mark(slot, 2);
    mark(slot, 3);
    return BEAM_OK;
  }
  size_t smem = sizeof(double2) * (size_t)px->max_pair_rows * px->xtile;
  BEAM_CUDA(cudaFuncSetAttribute(k_pixel_sums, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_pixel_sums<<<px->n_pairs, PIX_THREADS, smem, s>>>((const double2 *)px->cache, n2, px->xtile, px->pair_first,
                                                      px->pair_row_first, px->pair_rows, px->tri_rows, px->tri_sign,
                                                      px->tri_out, slot->B);
  BEAM_CUDA(cudaGetLastError());
  slot->launches++;
  mark(slot, 2);
  mark(slot, 3);
  return BEAM_OK;
}

void free_pixel_path(beam_gpu_plan *p) {
  PixelPath *px = pix_of(p);
  if (!px) return;
  void *ptrs[] = {px->mode_ij, px->row_i, px->row_mode, px->ring_rows, px->tw, px->r2c, px->slot_plane,
                  px->slot_ring, px->cache, px->pair_first, px->pair_row_first, px->pair_rows, px->tri_rows,
                  px->tri_sign, px->tri_out};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  p->pix = nullptr;
  delete px;
}

// ----------------------------------------------- allocation-free plane rings
// beam_gpu_plane_rings_noalloc: the same transform kernel, with its tables in
// a fixed scratch array of the library's device image instead of cudaMalloc'd
// buffers. The tables are assembled in a static host buffer (one call at a
// time, under a mutex), copied into the scratch array on the caller's stream
// and read by the kernel from there.
static __device__ __align__(256) unsigned char g_noalloc_scratch[BEAM_NOALLOC_SCRATCH_BYTES];
alignas(16) static unsigned char g_noalloc_host[BEAM_NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mutex;

// Device address of the scratch array in the current device's context, looked
// up on every call (no allocation; a cached address would go stale after
// cudaDeviceReset or under another context of the same device).
static int noalloc_scratch(void **ptr) {
  void *a = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
  if (e != cudaSuccess || !a) {
    set_detail(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    return BEAM_ECUDA;
  }
  *ptr = a;
  return BEAM_OK;
}

static size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// Visit the pixels of ring r in row-major order: fn(i, j) for every (i, j)
// with low <= |k| < high. Only rows and columns with |i|, |j| < high can hold
// ring pixels, so the scan covers those alone.
template <typename F>
static void noalloc_ring_pixels(long NN, double low, double high, const F &fn) {
  const long lim = std::min(NN / 2, (long)std::ceil(high));  // |i|, |j| <= lim covers |k| < high
  for (long i = 0; i < NN; ++i) {
    if (i > lim && i < NN - lim) i = NN - lim;
    const int ia = (int)((i > NN / 2) ? (i - NN) : i);
    for (long j = 0; j < NN; ++j) {
      if (j > lim && j < NN - lim) j = NN - lim;
      const int ja = (int)((j > NN / 2) ? (j - NN) : j);
      const double kk = sqrt(1. * (ia * ia + ja * ja));
      if (kk >= low && kk < high) fn(i, j);
    }
  }
}

}  // namespace beam

extern "C" int beam_gpu_plane_rings_noalloc(long NN, long Nmax, long Nr, const double *r2c_dev, const int *planes,
                                            const int *rings, int n, double *out_dev, void *stream) {
  using namespace beam;
  if (NN < 4 || NN % 2 || NN > 4096 || Nmax < 1 || Nmax > NN / 2 || Nr < 10 || Nr % 10 || Nr > 1000 || n < 0 ||
      (n > 0 && (!r2c_dev || !planes || !rings || !out_dev))) {
    set_detail("invalid arguments (NN even, 1 <= Nmax <= NN/2, Nr a multiple of 10, device buffers)");
    return BEAM_EINVAL;
  }
  if (n > 0 && (((uintptr_t)r2c_dev & 15) || ((uintptr_t)out_dev & 15))) {
    set_detail("device buffers must be 16-byte aligned");
    return BEAM_EINVAL;
  }
  if (n > BEAM_NOALLOC_MAX_JOBS) {
    set_detail("more than BEAM_NOALLOC_MAX_JOBS (plane, ring) pairs in one call");
    return BEAM_EINVAL;
  }
  for (int k = 0; k < n; ++k)
    if (planes[k] < 0 || planes[k] >= Nmax || rings[k] < 0 || rings[k] >= Nr) {
      set_detail("plane or ring out of range");
      return BEAM_EINVAL;
    }
  if (n == 0) return BEAM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The tables travel from a static host buffer that the next call rewrites;
  // a captured copy would read it at replay time, after that rewrite. So a
  // capturing stream is refused before any other CUDA call.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BEAM_CUDA(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone) {
    set_detail("the allocation-free plane-ring call cannot be captured into a CUDA graph (its tables are staged "
               "from a host buffer that later calls rewrite)");
    return BEAM_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  int dev = 0;
  BEAM_CUDA(cudaGetDevice(&dev));
  int smem_optin = 0;
  BEAM_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  void *scratch = nullptr;
  BEAM_TRY(noalloc_scratch(&scratch));

  // ring edges and, for the requested rings, their non-zero rows and modes in
  // row-major order (the order beam_gpu_plane_rings uses)
  double low[1000], high[1000], avg[1000];
  if (beam_ring_edges(Nr, Nmax, low, high, avg) != BEAM_OK) return BEAM_EINVAL;
  bool want[1000] = {};
  for (int k = 0; k < n; ++k) want[rings[k]] = true;
  size_t off_tw = 0;
  size_t off_jobs = align16(off_tw + sizeof(double2) * NN);
  size_t off_rr = align16(off_jobs + sizeof(int32_t) * 2 * n);
  size_t off_rows = align16(off_rr + sizeof(RingRows) * Nr);
  unsigned char *h = g_noalloc_host;
  // count rows and modes first, to lay the tables out and check the limits
  long nrows = 0, nmodes = 0;
  int max_rows = 1;
  for (long r = 0; r < Nr; ++r) {
    if (!want[r]) continue;
    long rows = 0, last_i = -1;
    noalloc_ring_pixels(NN, low[r], high[r], [&](long i, long) {
      ++nmodes;
      if (i != last_i) ++rows, last_i = i;
    });
    nrows += rows;
    max_rows = std::max(max_rows, (int)rows);
  }
  size_t off_rmode = align16(off_rows + sizeof(int32_t) * nrows);
  size_t off_mode = align16(off_rmode + sizeof(int32_t) * (nrows + 1));
  size_t total = align16(off_mode + sizeof(int16_t) * 2 * nmodes);
  if (total > BEAM_NOALLOC_SCRATCH_BYTES) {
    set_detail("the requested rings need " + std::to_string(total) + " bytes of tables; the allocation-free path holds " +
               std::to_string((size_t)BEAM_NOALLOC_SCRATCH_BYTES));
    return BEAM_EINVAL;
  }
  const size_t smem = sizeof(double2) * ((size_t)NN + (size_t)max_rows * PR_YB);
  if (smem > (size_t)smem_optin) {
    set_detail("the widest requested ring needs " + std::to_string(smem) + " bytes of shared memory per block; "
               "the device allows " + std::to_string(smem_optin));
    return BEAM_EINVAL;
  }
  double2 *tw = reinterpret_cast<double2 *>(h + off_tw);
  for (long k = 0; k < NN; ++k) {
    double a = 2.0 * M_PI * (double)k / (double)NN;
    tw[k] = make_double2(std::cos(a), std::sin(a));
  }
  int32_t *jp = reinterpret_cast<int32_t *>(h + off_jobs);
  for (int k = 0; k < n; ++k) {
    jp[k] = planes[k];
    jp[n + k] = rings[k];
  }
  RingRows *rr = reinterpret_cast<RingRows *>(h + off_rr);
  int32_t *row_i = reinterpret_cast<int32_t *>(h + off_rows);
  int32_t *row_mode = reinterpret_cast<int32_t *>(h + off_rmode);
  int16_t *mode_ij = reinterpret_cast<int16_t *>(h + off_mode);
  long at_row = 0, at_mode = 0;
  for (long r = 0; r < Nr; ++r) {
    rr[r] = RingRows{(int)at_row, 0};
    if (!want[r]) continue;
    long last_i = -1;
    noalloc_ring_pixels(NN, low[r], high[r], [&](long i, long j) {
      if (i != last_i) {
        row_i[at_row] = (int32_t)i;
        row_mode[at_row] = (int32_t)at_mode;
        ++at_row;
        last_i = i;
      }
      mode_ij[2 * at_mode] = (int16_t)i;
      mode_ij[2 * at_mode + 1] = (int16_t)j;
      ++at_mode;
    });
    rr[r].n_rows = (int)at_row - rr[r].first_row;
  }
  row_mode[at_row] = (int32_t)at_mode;

  // The attribute first: a refusal leaves nothing queued. Its error is also
  // cleared here, so it cannot surface in a later call's launch check.
  cudaError_t ea = cudaFuncSetAttribute(k_plane_ring_dft<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem);
  if (ea != cudaSuccess) {
    (void)cudaGetLastError();
    set_detail(std::string("cudaFuncSetAttribute(shared memory): ") + cudaGetErrorString(ea));
    return BEAM_ECUDA;
  }
  unsigned char *d = static_cast<unsigned char *>(scratch);
  // From pageable memory the driver stages the tables before this returns
  // (so the next call may rewrite the host buffer); it may first wait for
  // the stream's earlier work.
  BEAM_CUDA(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, st));
  dim3 grid((unsigned)((NN + PR_YB - 1) / PR_YB), (unsigned)n);
  k_plane_ring_dft<double2><<<grid, PR_THREADS, smem, st>>>(
      reinterpret_cast<const double2 *>(r2c_dev), (int)NN, reinterpret_cast<const int32_t *>(d + off_jobs),
      reinterpret_cast<const int32_t *>(d + off_jobs) + n, reinterpret_cast<const RingRows *>(d + off_rr),
      reinterpret_cast<const int32_t *>(d + off_rows), reinterpret_cast<const int32_t *>(d + off_rmode),
      reinterpret_cast<const int16_t *>(d + off_mode), reinterpret_cast<const double2 *>(d + off_tw),
      reinterpret_cast<double2 *>(out_dev), (long long)NN * NN);
  BEAM_CUDA(cudaGetLastError());
  return BEAM_OK;
}
