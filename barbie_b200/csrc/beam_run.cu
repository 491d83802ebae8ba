// Per-realization kernels of libbeam_gpu (sm_100a):
//   k_build_modes  gather the ring modes of the planes in use from the r2c
//                  buffer into signed-plane rows S[m][q + Q-1] (conjugate of the
//                  mirrored mode for q < 0)                      (funcs.c:94-106)
//   k_triangle     per accepted triangle, the in-plane closed-triangle sum
//                  Re sum M1(k1) M2'(k2) M3'(k3)                 (barbie.c:329-337)
//   k_reduce       sum the triangle-range splits, scale by NN^2, bin order
//   k_epilogue     cal_coeff weights, bins, normalisation        (barbie.c:343-363,
//                                                               383-392; funcs.c:708-745)
#include <cstring>

#include "beam_internal.h"

namespace beam {

// ------------------------------------------------------------------ helpers
template <typename C>
struct CplxOf;
template <>
struct CplxOf<double2> {
  static __device__ __forceinline__ double2 make(double re, double im) { return make_double2(re, im); }
};
template <>
struct CplxOf<float2> {
  static __device__ __forceinline__ float2 make(double re, double im) { return make_float2((float)re, (float)im); }
};

__device__ __forceinline__ long long lmin(long long a, long long b) { return a < b ? a : b; }

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for a barrier phase for at most ~2 s of wall time.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  unsigned long long start = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - start > 2000000000ull) return false;
  return true;
}

// 1D bulk copy global -> shared (TMA engine), completion counted on bar.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// ------------------------------------------------------------- mode gather
// S[m][w] for signed plane q = w - (Q-1): Delta(k_m, q) for q >= 0 (zero for
// k_perp = 0 on plane 0, funcs.c:102-106) and conj(Delta(-k_m, -q)) for q < 0,
// the conjugate plane the reference reads as sign_2/sign_3 = -1 (barbie.c:332).
// rows: either staged rows [n_modes][Q] (row of mode m at m*Q) or the full r2c
// buffer (row of mode m at (i*NN + j)*(NN/2+1)).
template <typename C>
__global__ void k_build_modes(const double2 *__restrict__ src, int staged, const int16_t *__restrict__ mode_ij,
                              const int32_t *__restrict__ mode_neg, int n_modes, int Q, int W, int NN,
                              C *__restrict__ S) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_modes * W) return;
  int m = (int)(idx / W), w = (int)(idx % W);
  int q = w - (Q - 1);
  C v = CplxOf<C>::make(0.0, 0.0);
  if (w < 2 * Q - 1) {
    int mm = q >= 0 ? m : mode_neg[m];
    int aq = q >= 0 ? q : -q;
    size_t row = staged ? (size_t)mm * Q
                        : ((size_t)mode_ij[2 * mm] * NN + (size_t)mode_ij[2 * mm + 1]) * (size_t)(NN / 2 + 1);
    double2 a = src[row + aq];
    bool origin = (mode_ij[2 * m] == 0 && mode_ij[2 * m + 1] == 0);
    if (q == 0 && origin) a = make_double2(0.0, 0.0);
    v = CplxOf<C>::make(a.x, q >= 0 ? a.y : -a.y);
  }
  S[idx] = v;
}

// ------------------------------------------------------------ triangle sums
// One CTA per work item (ring triplet u, combo range, in-plane triangle range).
// Threads own combos (plane pairs p1, p2; p3 = -p1-p2); the CTA walks the
// triangle list in chunks of TRI_CHUNK. For each triangle one lane of warp 0
// bulk-copies the three signed-plane row segments it needs (rings r1, r2, r3
// over the item's plane ranges) into a double-buffered shared stage; every
// thread then adds Re(x*y*z) for each of its combos.
template <typename C>
struct TriMath;
template <>
struct TriMath<double2> {
  typedef double chunk_t;
  static __device__ __forceinline__ double term(double2 x, double2 y, double2 z) {
    double ur = fma(x.x, y.x, -x.y * y.y);
    double ui = fma(x.x, y.y, x.y * y.x);
    return fma(ur, z.x, -ui * z.y);
  }
};
template <>
struct TriMath<float2> {
  typedef float chunk_t;
  static __device__ __forceinline__ float term(float2 x, float2 y, float2 z) {
    float ur = fmaf(x.x, y.x, -x.y * y.y);
    float ui = fmaf(x.x, y.y, x.y * y.x);
    return fmaf(ur, z.x, -ui * z.y);
  }
};

struct TriArgs {
  const TriItem *items;
  const ushort4 *list;
  const void *S;
  int W;
  int Q;
  const int32_t *combo_p1, *combo_p2;
  const int32_t *u_cfirst, *u_ncombo;
  const long long *u_part;
  double *part;
  int *status;
  int stage_elems;  // chunk * max_row
  int chunk;        // in-plane triangles per stage (<= TRI_CHUNK)
};

template <typename C>
__device__ __forceinline__ void tri_issue(const TriArgs &a, const TriItem &it, const C *S, C *stage, uint32_t bar,
                                          long long tbeg, int n, int row) {
  int lane = threadIdx.x & 31;
  if (lane == 0) mbar_expect_tx(bar, (uint32_t)(n * row * sizeof(C)));
  __syncwarp();
  if (lane < n) {
    ushort4 e = a.list[tbeg + lane];
    C *dst = stage + lane * row;
    const C *s1 = S + (size_t)(it.m1 + e.x) * a.W + it.p1lo;
    const C *s2 = S + (size_t)(it.m2 + e.y) * a.W + it.p2lo;
    const C *s3 = S + (size_t)(it.m3 + e.z) * a.W + it.p3lo;
    bulk_g2s(smem_addr(dst), s1, (uint32_t)(it.L1 * sizeof(C)), bar);
    bulk_g2s(smem_addr(dst + it.L1), s2, (uint32_t)(it.L2 * sizeof(C)), bar);
    bulk_g2s(smem_addr(dst + it.L1 + it.L2), s3, (uint32_t)(it.L3 * sizeof(C)), bar);
  }
}

template <typename C, int SLOTS>
__device__ __forceinline__ void tri_body(const TriArgs &a, const TriItem &it, C *stages, uint64_t *bars,
                                         int *s_fail) {
  typedef typename TriMath<C>::chunk_t chunk_t;
  const C *S = static_cast<const C *>(a.S);
  const int tid = threadIdx.x;
  const int row = it.L1 + it.L2 + it.L3;
  int o1[SLOTS], o2[SLOTS], o3[SLOTS];
  double acc[SLOTS];
  int nsl = 0;
#pragma unroll
  for (int k = 0; k < SLOTS; ++k) {
    int c = it.c0 + tid + k * TRI_THREADS;
    acc[k] = 0.0;
    o1[k] = o2[k] = o3[k] = 0;
    if (c < it.c1) {
      int p1 = a.combo_p1[c], p2 = a.combo_p2[c], p3 = -p1 - p2;
      o1[k] = p1 + a.Q - 1 - it.p1lo;
      o2[k] = it.L1 + p2 + a.Q - 1 - it.p2lo;
      o3[k] = it.L1 + it.L2 + p3 + a.Q - 1 - it.p3lo;
      nsl = k + 1;
    }
  }
  const long long nt = it.t1 - it.t0;
  const int CH = a.chunk;
  const int nch = (int)((nt + CH - 1) / CH);
  const uint32_t bar0 = smem_addr(&bars[0]), bar1 = smem_addr(&bars[1]);
  if (tid < 32) {
    tri_issue<C>(a, it, S, stages, bar0, it.t0, (int)lmin(CH, nt), row);
    if (nch > 1)
      tri_issue<C>(a, it, S, stages + a.stage_elems, bar1, it.t0 + CH, (int)lmin(CH, nt - CH), row);
  }
  for (int c = 0; c < nch; ++c) {
    const int s = c & 1;
    const uint32_t bar = s ? bar1 : bar0;
    bool ok = mbar_wait_bounded(bar, (uint32_t)((c >> 1) & 1));
    if (!ok) *s_fail = 1;
    __syncthreads();
    if (*s_fail) {
      // give the copies still in flight into the other stage time to land
      if (c + 1 < nch) mbar_wait_bounded(s ? bar0 : bar1, (uint32_t)(((c + 1) >> 1) & 1));
      if (tid == 0) atomicOr(a.status, DEV_TIMEOUT);
      return;
    }
    const C *st = stages + s * a.stage_elems;
    const int n = (int)lmin(CH, nt - (long long)c * CH);
    chunk_t cs[SLOTS];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) cs[k] = 0;
    for (int tt = 0; tt < n; ++tt) {
      const C *r = st + tt * row;
#pragma unroll
      for (int k = 0; k < SLOTS; ++k)
        if (k < nsl) cs[k] += TriMath<C>::term(r[o1[k]], r[o2[k]], r[o3[k]]);
    }
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) acc[k] += (double)cs[k];
    __syncthreads();
    if (c + 2 < nch && tid < 32)
      tri_issue<C>(a, it, S, stages + s * a.stage_elems, bar, it.t0 + (long long)(c + 2) * CH,
                   (int)lmin(CH, nt - (long long)(c + 2) * CH), row);
  }
  const int nc = a.u_ncombo[it.u];
  double *out = a.part + a.u_part[it.u] + (long long)it.split * nc - a.u_cfirst[it.u];
#pragma unroll
  for (int k = 0; k < SLOTS; ++k)
    if (k < nsl) {
      int c = it.c0 + tid + k * TRI_THREADS;
      if (c < it.c1) out[c] = acc[k];
    }
}

template <typename C>
__global__ void __launch_bounds__(TRI_THREADS) k_triangle(TriArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bars[2];
  __shared__ int s_fail;
  const TriItem it = a.items[blockIdx.x];
  if (threadIdx.x == 0) {
    mbar_init(smem_addr(&bars[0]), 1);
    mbar_init(smem_addr(&bars[1]), 1);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  C *stages = reinterpret_cast<C *>(smem_raw);
  const int slots = (it.c1 - it.c0 + TRI_THREADS - 1) / TRI_THREADS;
  if (slots <= 1)
    tri_body<C, 1>(a, it, stages, bars, &s_fail);
  else if (slots <= 2)
    tri_body<C, 2>(a, it, stages, bars, &s_fail);
  else if (slots <= 4)
    tri_body<C, 4>(a, it, stages, bars, &s_fail);
  else if (slots <= 8)
    tri_body<C, 8>(a, it, stages, bars, &s_fail);
  else
    tri_body<C, 16>(a, it, stages, bars, &s_fail);
}

// Sum the splits of each combo in split order, scale by NN^2 and store the
// triangle's B at its bin-order position.
__global__ void k_reduce(long long n_combo, const int32_t *__restrict__ combo_u, const int32_t *__restrict__ u_cfirst,
                         const int32_t *__restrict__ u_ncombo, const int32_t *__restrict__ u_nsplit,
                         const long long *__restrict__ u_part, const int32_t *__restrict__ combo_out,
                         const double *__restrict__ part, double nn2, double *__restrict__ B) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_combo) return;
  int u = combo_u[c];
  int nc = u_ncombo[u], ns = u_nsplit[u];
  const double *p = part + u_part[u] + (c - u_cfirst[u]);
  double s = 0.0;
  for (int k = 0; k < ns; ++k) s += p[(long long)k * nc];
  B[combo_out[c]] = nn2 * s;
}

// ----------------------------------------------------------------- epilogue
// Orientation weights bs[] and norms norm[] of the 16 (l,m) multipoles for a
// triangle orientation (px, pz) -- the polynomials of funcs.c:708-745, written
// in z = pz^2, x = px^2, w = z - 1, u = 1 - z.
__device__ __forceinline__ void orientation_weights(double px, double pz, double *bs, double *nm) {
  const double z = pz * pz, x = px * px, w = z - 1.0, u = 1.0 - z;
  const double xz = px * pz;
  const double c2 = 2.0 * x + w;                     // 2px^2 + pz^2 - 1
  const double c4 = 8.0 * x * x + 8.0 * x * w + w * w;
  const double s23 = 0.816496580927726;              // sqrt(2/3)
  bs[0] = 1.0;
  bs[1] = 2.0 * (3.0 * z - 1.0);
  bs[2] = -s23 * xz;
  bs[3] = 2.0 * s23 * c2;
  bs[4] = 8.0 * (3.0 - 30.0 * z + 35.0 * z * z);
  bs[5] = -4.0 * xz * (7.0 * z - 3.0) * 0.4472135954999579;            // 1/sqrt(5)
  bs[6] = 4.0 * 0.6324555320336759 * c2 * (7.0 * z - 1.0);             // sqrt(0.4)
  bs[7] = -4.0 * xz * (4.0 * x + 3.0 * w) * 0.1690308509457033;        // 1/sqrt(35)
  bs[8] = 8.0 * 0.2390457218668787 * c4;                               // sqrt(2/35)
  bs[9] = 16.0 * (-5.0 + z * (105.0 + z * (-315.0 + 231.0 * z)));
  bs[10] = -8.0 * 0.3086066999241838 * xz * (5.0 - 30.0 * z + 33.0 * z * z);  // sqrt(2/21)
  bs[11] = 32.0 * c2 * (1.0 - 18.0 * z + 33.0 * z * z) * 0.09759000729485332;  // 1/sqrt(105)
  bs[12] = -16.0 * xz * (4.0 * x + 3.0 * w) * (11.0 * z - 3.0) * 0.09759000729485332;
  bs[13] = 16.0 * 0.5345224838248488 * (11.0 * z - 1.0) * c4 / 3.0;   // sqrt(2/7)
  bs[14] = -16.0 * xz * (16.0 * x * x + 20.0 * x * w + 5.0 * w * w) / (3.0 * 8.774964387392123);  // sqrt(77)
  bs[15] = 32.0 * (32.0 * x * x * x + 48.0 * x * x * w + 18.0 * x * w * w + w * w * w) * 0.06579516949597690;  // 1/sqrt(231)
  const double l2 = 3.0 * z - 1.0, l4 = 3.0 - 30.0 * z + 35.0 * z * z;
  const double l6 = -5.0 + z * (105.0 + z * (-315.0 + 231.0 * z));
  const double a5 = pz * (7.0 * z - 3.0), a6 = 7.0 * z - 1.0;
  const double a10 = pz * (5.0 - 30.0 * z + 33.0 * z * z), a11 = 1.0 - 18.0 * z + 33.0 * z * z;
  const double a12 = pz * (11.0 * z - 3.0), a13 = 11.0 * z - 1.0;
  const double u2 = u * u, u3 = u2 * u, u4 = u2 * u2;
  nm[0] = 1.0;
  nm[1] = l2 * l2;
  nm[2] = z * u;
  nm[3] = u2;
  nm[4] = l4 * l4;
  nm[5] = u * a5 * a5;
  nm[6] = u2 * a6 * a6;
  nm[7] = z * u3;
  nm[8] = u4;
  nm[9] = l6 * l6;
  nm[10] = u * a10 * a10;
  nm[11] = u2 * a11 * a11;
  nm[12] = u3 * a12 * a12;
  nm[13] = u4 * a13 * a13;
  nm[14] = z * u4 * u;
  nm[15] = u3 * u3;
}

constexpr int EP_THREADS = 128;

// One CTA per (k1, t, mu) bin over its triangles (bin order = loop order within
// the bin). B == 0 drops the triangle's count (barbie.c:355-357). Reduction
// order is fixed, so results are run-to-run identical.
__global__ void __launch_bounds__(EP_THREADS) k_epilogue(const int32_t *__restrict__ bin_first,
                                                         const double *__restrict__ B,
                                                         const double *__restrict__ px,
                                                         const double *__restrict__ pz,
                                                         const int32_t *__restrict__ cnt, double nn2, double vol,
                                                         int n_bins, double *__restrict__ bins,
                                                         long long *__restrict__ bin_count) {
  __shared__ double red[2 * BEAM_NPOLES][EP_THREADS];
  __shared__ long long redc[EP_THREADS];
  const int b = blockIdx.x, tid = threadIdx.x;
  double sb[BEAM_NPOLES], sn[BEAM_NPOLES];
#pragma unroll
  for (int k = 0; k < BEAM_NPOLES; ++k) sb[k] = sn[k] = 0.0;
  long long sc = 0;
  for (int i = bin_first[b] + tid; i < bin_first[b + 1]; i += EP_THREADS) {
    double Bv = B[i];
    double bs[BEAM_NPOLES], nm[BEAM_NPOLES];
    orientation_weights(px[i], pz[i], bs, nm);
    bool nz = (Bv != 0.0);
    double num = nz ? nn2 * (double)cnt[i] : 0.0;
    sc += nz ? (long long)cnt[i] : 0;
#pragma unroll
    for (int k = 0; k < BEAM_NPOLES; ++k) {
      sb[k] += Bv * bs[k];
      sn[k] += num * nm[k];
    }
  }
#pragma unroll
  for (int k = 0; k < BEAM_NPOLES; ++k) {
    red[k][tid] = sb[k];
    red[BEAM_NPOLES + k][tid] = sn[k];
  }
  redc[tid] = sc;
  __syncthreads();
  for (int s = EP_THREADS / 2; s > 0; s >>= 1) {
    if (tid < s) {
#pragma unroll
      for (int k = 0; k < 2 * BEAM_NPOLES; ++k) red[k][tid] += red[k][tid + s];
      redc[tid] += redc[tid + s];
    }
    __syncthreads();
  }
  if (tid < BEAM_NPOLES) {
    double vbs = red[tid][0], vn = red[BEAM_NPOLES + tid][0];
    bins[(size_t)b * BEAM_NPOLES + tid] = vbs;
    bins[((size_t)n_bins + b) * BEAM_NPOLES + tid] = vn;
    bins[((size_t)2 * n_bins + b) * BEAM_NPOLES + tid] = vbs / (vol * vn);
  }
  if (tid == 0) bin_count[b] = redc[0];
}

// ------------------------------------------------------------ host drivers
int upload_modes_host(beam_gpu_plan *p, const double *r2c) {
  DevPlan &d = p->d;
  const long NN = p->geom.NN, NH = NN / 2 + 1;
  const int Q = d.Q;
  for (int m = 0; m < d.n_modes; ++m) {
    size_t row = ((size_t)p->mode_ij[2 * m] * NN + (size_t)p->mode_ij[2 * m + 1]) * (size_t)NH;
    std::memcpy(p->h_staging + (size_t)2 * m * Q, r2c + 2 * row, sizeof(double) * 2 * Q);
  }
  cudaStream_t s = p->ctx->stream;
  BEAM_CUDA(cudaMemcpyAsync(d.staging, p->h_staging, sizeof(double) * 2 * (size_t)d.n_modes * Q,
                            cudaMemcpyHostToDevice, s));
  long long n = (long long)d.n_modes * d.W;
  if (n == 0) return BEAM_OK;
  int blocks = (int)((n + 255) / 256);
  if (d.S64)
    k_build_modes<double2><<<blocks, 256, 0, s>>>((const double2 *)d.staging, 1, d.mode_ij, d.mode_neg, d.n_modes,
                                                   Q, d.W, (int)NN, (double2 *)d.S64);
  else
    k_build_modes<float2><<<blocks, 256, 0, s>>>((const double2 *)d.staging, 1, d.mode_ij, d.mode_neg, d.n_modes, Q,
                                                  d.W, (int)NN, (float2 *)d.S32);
  BEAM_CUDA(cudaGetLastError());
  return BEAM_OK;
}

int upload_modes_device(beam_gpu_plan *p, const double *r2c_dev) {
  DevPlan &d = p->d;
  cudaStream_t s = p->ctx->stream;
  long long n = (long long)d.n_modes * d.W;
  if (n == 0) return BEAM_OK;
  int blocks = (int)((n + 255) / 256);
  if (d.S64)
    k_build_modes<double2><<<blocks, 256, 0, s>>>((const double2 *)r2c_dev, 0, d.mode_ij, d.mode_neg, d.n_modes, d.Q,
                                                   d.W, (int)p->geom.NN, (double2 *)d.S64);
  else
    k_build_modes<float2><<<blocks, 256, 0, s>>>((const double2 *)r2c_dev, 0, d.mode_ij, d.mode_neg, d.n_modes, d.Q,
                                                  d.W, (int)p->geom.NN, (float2 *)d.S32);
  BEAM_CUDA(cudaGetLastError());
  return BEAM_OK;
}

static size_t tri_smem_bytes(const DevPlan &d, size_t elem) { return 2 * (size_t)d.chunk * d.max_row * elem; }

int run_triangle_sums(beam_gpu_plan *p) {
  DevPlan &d = p->d;
  cudaStream_t s = p->ctx->stream;
  if (d.n_combo == 0) {
    for (int k = 1; k <= 3; ++k) mark(p, k);
    return BEAM_OK;
  }
  TriArgs a;
  a.items = d.items;
  a.list = d.tri_list;
  a.W = d.W;
  a.Q = d.Q;
  a.combo_p1 = d.combo_p1;
  a.combo_p2 = d.combo_p2;
  a.u_cfirst = d.u_cfirst;
  a.u_ncombo = d.u_ncombo;
  a.u_part = d.u_part;
  a.part = d.part;
  a.status = d.status;
  a.stage_elems = d.chunk * d.max_row;
  a.chunk = d.chunk;
  mark(p, 1);
  if (d.S64) {
    a.S = d.S64;
    size_t smem = tri_smem_bytes(d, sizeof(double2));
    BEAM_CUDA(cudaFuncSetAttribute(k_triangle<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_triangle<double2><<<d.n_items, TRI_THREADS, smem, s>>>(a);
  } else {
    a.S = d.S32;
    size_t smem = tri_smem_bytes(d, sizeof(float2));
    BEAM_CUDA(cudaFuncSetAttribute(k_triangle<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_triangle<float2><<<d.n_items, TRI_THREADS, smem, s>>>(a);
  }
  BEAM_CUDA(cudaGetLastError());
  mark(p, 2);
  double nn2 = (double)p->geom.NN * (double)p->geom.NN;
  k_reduce<<<(unsigned)((d.n_combo + 255) / 256), 256, 0, s>>>(d.n_combo, d.combo_u, d.u_cfirst, d.u_ncombo,
                                                               d.u_nsplit, d.u_part, d.combo_out, d.part, nn2, d.B);
  BEAM_CUDA(cudaGetLastError());
  mark(p, 3);
  return BEAM_OK;
}

int run_epilogue(beam_gpu_plan *p) {
  DevPlan &d = p->d;
  cudaStream_t s = p->ctx->stream;
  if (d.n_bins == 0) return BEAM_OK;
  double nn2 = (double)p->geom.NN * (double)p->geom.NN;
  k_epilogue<<<d.n_bins, EP_THREADS, 0, s>>>(d.bin_first, d.B, d.ep_px, d.ep_pz, d.ep_cnt, nn2, p->geom.vol,
                                             d.n_bins, d.bins, d.bin_count);
  BEAM_CUDA(cudaGetLastError());
  return BEAM_OK;
}

int check_status(beam_gpu_plan *p) {
  int st = 0;
  BEAM_CUDA(cudaMemcpyAsync(&st, p->d.status, sizeof(int), cudaMemcpyDeviceToHost, p->ctx->stream));
  BEAM_CUDA(cudaStreamSynchronize(p->ctx->stream));
  if (st & DEV_TIMEOUT) {
    set_detail("a bounded device wait in the triangle-sum kernel gave up");
    cudaMemsetAsync(p->d.status, 0, sizeof(int), p->ctx->stream);
    return BEAM_ETIMEDOUT;
  }
  if (st) {
    set_detail("device reported a bad index");
    cudaMemsetAsync(p->d.status, 0, sizeof(int), p->ctx->stream);
    return BEAM_ECUDA;
  }
  return BEAM_OK;
}

}  // namespace beam
