// Per-realization kernels of libbeam_gpu (sm_100a) other than the triangle sums
// (beam_triangle.cu):
//   k_build_modes  gather the ring modes of the planes in use from the r2c
//                  buffer into signed-plane rows (conjugate of the mirrored mode
//                  for negative planes)                          (funcs.c:94-106)
//   k_epilogue     cal_coeff weights, bins, normalisation        (barbie.c:343-363,
//                                                               383-392; funcs.c:708-745)
#include <algorithm>
#include <cstring>
#include <new>
#include <type_traits>

#include "beam_device.cuh"
#include "beam_internal.h"

namespace beam {

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

// ------------------------------------------------------------- mode gather
// Row of mode m: column colbase + q holds plane q = -(Q-1)..Q-1: Delta(k_m, q)
// for q >= 0 (zero for k_perp = 0 on plane 0, funcs.c:102-106) and
// conj(Delta(-k_m, -q)) for q < 0, the conjugate plane the reference reads with
// sign_2/sign_3 = -1 (barbie.c:332); other columns are zero.
// srcs[r] for realization r = blockIdx.y: its staged rows [n_modes][Q]
// (staged = 1) or its full r2c buffer; S rows of realization r start at
// r * n_modes * W. FP64 rows are complex128[W]; the mixed path's rows are
// blocked by 4 columns (mixed_re: 4 real parts, then their 4 imaginary
// parts), so its consumer loads 4 planes' real or imaginary parts at once
// and multiplies pairs of planes with packed FP32 FMAs.
// real_stride: elements of C from one realization's rows to the next's.
template <typename C>
__global__ void k_build_modes(const double *const *__restrict__ srcs, int staged, const int16_t *__restrict__ mode_ij,
                              const int32_t *__restrict__ mode_neg, int n_modes, int Q, int W, int colbase, int NN,
                              C *__restrict__ S, long long real_stride) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_modes * W) return;
  const double2 *src = reinterpret_cast<const double2 *>(srcs[blockIdx.y]);
  S += (size_t)blockIdx.y * real_stride;
  int m = (int)(idx / W), w = (int)(idx % W);
  int q = w - colbase;
  C v = CplxOf<C>::make(0.0, 0.0);
  if (q > -Q && q < Q) {
    int mm = q >= 0 ? m : mode_neg[m];
    int aq = q >= 0 ? q : -q;
    size_t row = staged ? (size_t)mm * Q
                        : ((size_t)mode_ij[2 * mm] * NN + (size_t)mode_ij[2 * mm + 1]) * (size_t)(NN / 2 + 1);
    double2 a = src[row + aq];
    bool origin = (mode_ij[2 * m] == 0 && mode_ij[2 * m + 1] == 0);
    if (q == 0 && origin) a = make_double2(0.0, 0.0);
    v = CplxOf<C>::make(a.x, q >= 0 ? a.y : -a.y);
  }
  if constexpr (std::is_same<C, float2>::value) {
    float *row = reinterpret_cast<float *>(S) + (size_t)m * 2 * W;
    row[mixed_re(w)] = v.x;
    row[mixed_re(w) + 4] = v.y;
  } else {
    S[idx] = v;
  }
}

// ------------------------------------------------------- int8 slice rows
// Scale exponent e(r, c) of ring r on the plane of column c: the smallest e
// with max |Re|, |Im| over the ring's modes there below 2^e (0 for a column
// of zeros). CTA: 32 columns x 8 strides over the ring's modes, one ring
// (blockIdx.x / ceil(W / 32)); realization blockIdx.y.
__global__ void k_ring_scale(const double2 *__restrict__ S, long long real_stride, const int32_t *__restrict__ ring_first,
                             int W, int32_t *__restrict__ scale, long long scale_stride) {
  __shared__ double s_max[8][32];
  const int cblocks = (W + 31) / 32;
  const int r = blockIdx.x / cblocks, c = (blockIdx.x % cblocks) * 32 + (threadIdx.x & 31), k = threadIdx.x >> 5;
  S += (size_t)blockIdx.y * real_stride;
  double mx = 0.0;
  if (c < W)
    for (int m = ring_first[r] + k; m < ring_first[r + 1]; m += 8) {
      const double2 v = S[(size_t)m * W + c];
      mx = fmax(mx, fmax(fabs(v.x), fabs(v.y)));
    }
  s_max[k][threadIdx.x & 31] = mx;
  __syncthreads();
  if (k == 0 && c < W) {
    for (int j = 1; j < 8; ++j) mx = fmax(mx, s_max[j][threadIdx.x]);
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);  // mx = f 2^e with f in [0.5, 1)
    scale[(size_t)blockIdx.y * scale_stride + (size_t)r * W + c] = e;
  }
}

// The five slices of v against 2^e (|v| < 2^e): a0 = floor(v 2^(7-e)) in
// [-128, 127], then a1..a4 = the next four base-256 digits of the remainder
// in [0, 1), each step exact in FP64. Byte k of the result's low and high
// words is slice k (slices 0-3 in lo, 4 in hi).
__device__ __forceinline__ void slice5(double v, int e, uint32_t &lo, uint32_t &hi) {
  double u = ldexp(v, 7 - e);
  double a = floor(u);
  double rem = u - a;
  lo = (uint32_t)((int)a & 0xff);
  hi = 0;
#pragma unroll
  for (int k = 1; k < I8_SLICES; ++k) {
    rem *= 256.0;
    a = floor(rem);
    rem -= a;
    if (k < 4) lo |= (uint32_t)a << (8 * k);
    else hi = (uint32_t)a;
  }
}

// Slice tables of every mode (realization blockIdx.y). The x table holds per
// (mode, column) I8_XW words: word s = slice s of (Re, -Im, Im, Re) as bytes
// 0-3 (the x leg's two operand orders); the z table I8_ZW words: (Re, Im)
// pairs of slices (0, 1), (2, 3) and (4) (the z leg's operand). The slices of
// -Im are those of the negated value, not negated slices (slices 1-4 are
// unsigned).
__global__ void k_build_slices(const double2 *__restrict__ S, long long real_stride, const int32_t *__restrict__ ring_first,
                               int n_rings, int n_modes, int W, const int32_t *__restrict__ scale, long long scale_stride,
                               uint32_t *__restrict__ xtab, uint32_t *__restrict__ ztab, long long tab_stride) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_modes * W) return;
  const int m = (int)(idx / W), c = (int)(idx % W);
  int lo = 0, hi = n_rings;  // ring of mode m: ring_first[r] <= m < ring_first[r + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (ring_first[mid] <= m) lo = mid; else hi = mid;
  }
  const double2 v = S[(size_t)blockIdx.y * real_stride + idx];
  const int e = scale[(size_t)blockIdx.y * scale_stride + (size_t)lo * W + c];
  uint32_t re0, re4, im0, im4, ni0, ni4;
  slice5(v.x, e, re0, re4);
  slice5(v.y, e, im0, im4);
  slice5(-v.y, e, ni0, ni4);
  uint32_t *xo = xtab + (size_t)blockIdx.y * tab_stride + (size_t)idx * I8_XW;
#pragma unroll
  for (int k = 0; k < I8_XW; ++k) {
    const uint32_t r = k < 4 ? (re0 >> (8 * k)) & 0xff : re4, i = k < 4 ? (im0 >> (8 * k)) & 0xff : im4,
                   n = k < 4 ? (ni0 >> (8 * k)) & 0xff : ni4;
    xo[k] = r | (n << 8) | (i << 16) | (r << 24);
  }
  uint32_t *zo = ztab + (size_t)blockIdx.y * tab_stride + (size_t)idx * I8_ZW;
  zo[0] = (re0 & 0xff) | ((im0 & 0xff) << 8) | (((re0 >> 8) & 0xff) << 16) | (((im0 >> 8) & 0xff) << 24);
  zo[1] = ((re0 >> 16) & 0xff) | (((im0 >> 16) & 0xff) << 8) | ((re0 >> 24) << 16) | ((im0 >> 24) << 24);
  zo[2] = re4 | (im4 << 8);
}

// Scales and slice rows of realizations [0, n) from their FP64 rows.
int build_slices(beam_gpu_plan *p, RunSlot *s, int n) {
  const DevPlan &d = p->d;
  cudaStream_t st = s->lane->stream;
  const long long real_bytes = (long long)mode_data_bytes(d);
  const double2 *S = (const double2 *)s->S;
  uint32_t *xtab = (uint32_t *)((unsigned char *)s->S + i8_fp64_bytes(d));
  uint32_t *ztab = (uint32_t *)((unsigned char *)s->S + i8_fp64_bytes(d) + i8_xtab_bytes(d));
  int32_t *scale = (int32_t *)((unsigned char *)s->S + i8_fp64_bytes(d) + i8_slice_bytes(d));
  const int cblocks = (d.W + 31) / 32;
  k_ring_scale<<<dim3((unsigned)(d.n_rings * cblocks), (unsigned)n), 256, 0, st>>>(
      S, real_bytes / 16, d.ring_first, d.W, scale, real_bytes / 4);
  BEAM_CUDA(cudaGetLastError());
  const long long per = (long long)d.n_modes * d.W;
  k_build_slices<<<dim3((unsigned)((per + 255) / 256), (unsigned)n), 256, 0, st>>>(
      S, real_bytes / 16, d.ring_first, d.n_rings, d.n_modes, d.W, scale, real_bytes / 4, xtab, ztab, real_bytes / 4);
  BEAM_CUDA(cudaGetLastError());
  s->launches += 2;
  return BEAM_OK;
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
constexpr int EP_VALS = 3 * BEAM_NPOLES + 1;  // bs[16], norm[16], analytic[16], count per chunk

// Epilogue, pass 1: one CTA per chunk of at most EP_CHUNK triangles of one
// (k1, t, mu) bin (blockIdx.x) and realization (blockIdx.y), in bin order
// (loop order within the bin). Each triangle adds B * bs[ii], Num * norm[ii]
// and Biana * Num * bs[ii] with its cal_coeff weights; B == 0 drops the
// triangle's Num, Biana and count (barbie.c:355-361). The CTA writes its
// chunk's EP_VALS sums. Every reduction has a
// fixed order, so results are run-to-run identical and do not depend on the
// batch a realization runs in.
// 3 CTAs per SM: at most 170 registers per thread for the 49 running sums (216 unbounded, 2 CTAs
// per SM; the epilogue 0.138 -> 0.114 ms at NN=384, bit-identical)
__global__ void __launch_bounds__(EP_THREADS, 3) k_ep_chunks(const int32_t *__restrict__ chunk_first, int n_chunks,
                                                          const double *__restrict__ B, long long b_stride,
                                                          const double *__restrict__ px,
                                                          const double *__restrict__ pz,
                                                          const double *__restrict__ ana,
                                                          const int32_t *__restrict__ cnt, double nn2,
                                                          double *__restrict__ part) {
  __shared__ double red[EP_THREADS / 32][EP_VALS];
  const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  B += (size_t)blockIdx.y * b_stride;
  part += ((size_t)blockIdx.y * n_chunks + c) * EP_VALS;
  double v[EP_VALS];
#pragma unroll
  for (int k = 0; k < EP_VALS; ++k) v[k] = 0.0;
  for (int i = chunk_first[c] + tid; i < chunk_first[c + 1]; i += EP_THREADS) {
    double Bv = B[i];
    double bs[BEAM_NPOLES], nm[BEAM_NPOLES];
    orientation_weights(px[i], pz[i], bs, nm);
    bool nz = (Bv != 0.0);
    double num = nz ? nn2 * (double)cnt[i] : 0.0;
    double an = nz ? ana[i] : 0.0;
    v[3 * BEAM_NPOLES] += nz ? (double)cnt[i] : 0.0;
#pragma unroll
    for (int k = 0; k < BEAM_NPOLES; ++k) {
      v[k] += Bv * bs[k];
      v[BEAM_NPOLES + k] += num * nm[k];
      v[2 * BEAM_NPOLES + k] += an * num * bs[k];
    }
  }
  // fixed-order reduction: within each warp by halving, then warps in order
#pragma unroll
  for (int k = 0; k < EP_VALS; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < EP_VALS; ++k) red[warp][k] = v[k];
  __syncthreads();
  if (tid < EP_VALS) {
    double t = red[0][tid];
#pragma unroll
    for (int w = 1; w < EP_THREADS / 32; ++w) t += red[w][tid];
    part[tid] = t;
  }
}

// Epilogue, pass 2: bin sums over the bin's chunks in order, the
// normalisation out = bs / (vol * norm) (barbie.c:390), the analytic sum and
// the exact count.
// One thread per (bin, pole); realization blockIdx.y.
__global__ void k_ep_bins(const int32_t *__restrict__ bin_chunk, int n_bins, int n_chunks,
                          const double *__restrict__ part, double vol, double *__restrict__ bins,
                          long long *__restrict__ bin_count) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_bins * BEAM_NPOLES) return;
  const int b = idx / BEAM_NPOLES, k = idx % BEAM_NPOLES;
  part += (size_t)blockIdx.y * n_chunks * EP_VALS;
  bins += (size_t)blockIdx.y * BIN_SECTIONS * n_bins * BEAM_NPOLES;
  bin_count += (size_t)blockIdx.y * n_bins;
  double vbs = 0.0, vn = 0.0, va = 0.0, vc = 0.0;
  for (int c = bin_chunk[b]; c < bin_chunk[b + 1]; ++c) {
    vbs += part[(size_t)c * EP_VALS + k];
    vn += part[(size_t)c * EP_VALS + BEAM_NPOLES + k];
    va += part[(size_t)c * EP_VALS + 2 * BEAM_NPOLES + k];
    vc += part[(size_t)c * EP_VALS + 3 * BEAM_NPOLES];
  }
  bins[(size_t)b * BEAM_NPOLES + k] = vbs;
  bins[((size_t)n_bins + b) * BEAM_NPOLES + k] = vn;
  bins[((size_t)2 * n_bins + b) * BEAM_NPOLES + k] = vbs / (vol * vn);
  bins[((size_t)3 * n_bins + b) * BEAM_NPOLES + k] = va;
  if (k == 0) bin_count[b] = (long long)vc;  // a sum of integers below 2^53: exact
}

// ------------------------------------------------------------ host drivers
int lane_create(Lane *l, int priority) {
  cudaError_t e = cudaStreamCreateWithPriority(&l->stream, cudaStreamNonBlocking, priority);
  for (int k = 0; k < TRI_CLASSES && e == cudaSuccess; ++k) {
    e = cudaStreamCreateWithPriority(&l->side[k], cudaStreamNonBlocking, priority);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&l->join[k], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&l->fork, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    set_detail(std::string("stream/event creation: ") + cudaGetErrorString(e));
    lane_destroy(l);
    return BEAM_ECUDA;
  }
  return BEAM_OK;
}

void lane_destroy(Lane *l) {
  for (int k = 0; k < TRI_CLASSES; ++k) {
    if (l->side[k]) cudaStreamDestroy(l->side[k]);
    if (l->join[k]) cudaEventDestroy(l->join[k]);
  }
  if (l->fork) cudaEventDestroy(l->fork);
  if (l->stream) cudaStreamDestroy(l->stream);
  *l = Lane();
}

// Sizes of a slot's device buffers, in the order slot_alloc allocates them.
struct SlotSizes {
  size_t staging, src, S, part, B, bins, count, ep;
};
static SlotSizes slot_sizes(const beam_gpu_plan *p, int cap) {
  const DevPlan &d = p->d;
  const size_t c = (size_t)cap;
  SlotSizes z;
  z.staging = sizeof(double) * 2 * c * (size_t)d.n_modes * d.Q;
  z.src = sizeof(double *) * 2 * c;
  z.S = c * mode_data_bytes(d);
  z.part = sizeof(double) * c * (size_t)d.n_part;
  z.B = sizeof(double) * c * (size_t)std::max<long long>(1, d.n_combo);
  z.bins = sizeof(double) * c * BIN_SECTIONS * (size_t)d.n_bins * BEAM_NPOLES;
  z.count = sizeof(long long) * c * (size_t)d.n_bins;
  z.ep = sizeof(double) * c * (size_t)std::max(1, d.n_epchunks) * EP_VALS;
  return z;
}

size_t slot_bytes(const beam_gpu_plan *p, int cap) {
  SlotSizes z = slot_sizes(p, cap);
  return z.staging + z.src + z.S + z.part + z.B + z.bins + z.count + z.ep + sizeof(int);
}

void slot_destroy(RunSlot *s) {
  if (!s) return;
  if (s->lane && s->lane->stream) cudaStreamSynchronize(s->lane->stream);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  void *dev[] = {s->staging, (void *)s->src, s->S, s->part, s->B, s->bins, s->bin_count, s->ep_part, s->status};
  for (void *q : dev)
    if (q) cudaFree(q);
  void *host[] = {s->h_staging, (void *)s->h_src, s->h_bins, s->h_count, s->h_status};
  for (void *q : host)
    if (q) cudaFreeHost(q);
  for (int k = 0; k < 5; ++k)
    if (s->ev[k]) cudaEventDestroy(s->ev[k]);
  if (s->done) cudaEventDestroy(s->done);
  lane_destroy(&s->own);
  delete s;
}

static int slot_alloc(beam_gpu_plan *p, RunSlot *s) {
  const DevPlan &d = p->d;
  const int cap = s->cap;
  SlotSizes z = slot_sizes(p, cap);
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->staging, z.staging));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->src, z.src));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->S, z.S));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->part, z.part));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->B, z.B));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->bins, z.bins));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->bin_count, z.count));
  BEAM_TRY(dev_alloc(&s->bytes, (unsigned char **)&s->ep_part, z.ep));
  BEAM_TRY(dev_alloc(&s->bytes, &s->status, 2));  // status word, persistent kernel's work counter
  BEAM_CUDA(cudaMallocHost(&s->h_staging, std::max<size_t>(16, z.staging)));
  BEAM_CUDA(cudaMallocHost((void **)&s->h_src, z.src));
  BEAM_CUDA(cudaMallocHost(&s->h_bins, std::max<size_t>(16, z.bins)));
  BEAM_CUDA(cudaMallocHost(&s->h_count, std::max<size_t>(16, z.count)));
  BEAM_CUDA(cudaMallocHost(&s->h_status, sizeof(int)));
  *s->h_status = 0;
  for (int k = 0; k < 5; ++k) BEAM_CUDA(cudaEventCreate(&s->ev[k]));
  BEAM_CUDA(cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming));
  // staged sources are fixed: realization r reads staging rows r
  for (int r = 0; r < cap; ++r) {
    s->h_src[r] = s->staging + (size_t)2 * r * d.n_modes * d.Q;
    s->h_src[cap + r] = nullptr;
  }
  cudaStream_t st = s->lane->stream;
  BEAM_CUDA(cudaMemcpyAsync((void *)s->src, s->h_src, z.src, cudaMemcpyHostToDevice, st));
  // partial sums that no CTA writes (ring triplets of other shards) stay zero
  BEAM_CUDA(cudaMemsetAsync(s->part, 0, z.part, st));
  BEAM_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
  BEAM_CUDA(cudaStreamSynchronize(st));
  return BEAM_OK;
}

int slot_create(beam_gpu_plan *p, int cap, Lane *lane, RunSlot **out, int priority) {
  *out = nullptr;
  if (cap < 1 || cap > 65535) {
    set_detail("slot capacity must be 1..65535 realizations");
    return BEAM_EINVAL;
  }
  RunSlot *s = new (std::nothrow) RunSlot();
  if (!s) return BEAM_ENOMEM;
  s->cap = cap;
  int rc = BEAM_OK;
  if (lane) {
    s->lane = lane;
  } else {
    rc = lane_create(&s->own, priority);
    s->lane = &s->own;
  }
  if (rc == BEAM_OK) rc = slot_alloc(p, s);
  if (rc != BEAM_OK) {
    slot_destroy(s);
    return rc;
  }
  *out = s;
  return BEAM_OK;
}

// Copy the plan's mode rows [m0, m1) of one host r2c buffer into the slot's
// pinned staging rows of realization r (funcs.c:94-106 reads the same elements).
void gather_host(const beam_gpu_plan *p, RunSlot *s, int r, const double *r2c, int m0, int m1) {
  const DevPlan &d = p->d;
  const long NN = p->geom.NN, NH = NN / 2 + 1;
  const int Q = d.Q;
  double *dst = s->h_staging + (size_t)2 * r * d.n_modes * Q;
  if (m1 < 0 || m1 > d.n_modes) m1 = d.n_modes;
  for (int m = m0; m < m1; ++m) {
    size_t row = ((size_t)p->mode_ij[2 * m] * NN + (size_t)p->mode_ij[2 * m + 1]) * (size_t)NH;
    std::memcpy(dst + (size_t)2 * m * Q, r2c + 2 * row, sizeof(double) * 2 * Q);
  }
}

// Realization 0's mode rows gathered by the device straight from a page-locked
// host r2c buffer (r2c_mapped: its device-side address) into the slot's
// staging rows: each needed row crosses the bus once, with no host-side gather.
__global__ void k_gather_rows(const double2 *__restrict__ r2c_mapped, const int16_t *__restrict__ mode_ij,
                              int n_modes, int Q, int NN, double2 *__restrict__ staging) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_modes * Q) return;
  int m = (int)(idx / Q), q = (int)(idx % Q);
  size_t row = ((size_t)mode_ij[2 * m] * NN + (size_t)mode_ij[2 * m + 1]) * (size_t)(NN / 2 + 1);
  staging[idx] = r2c_mapped[row + q];
}

int gather_mapped(beam_gpu_plan *p, RunSlot *s, const double *r2c_mapped) {
  const DevPlan &d = p->d;
  long long n = (long long)d.n_modes * d.Q;
  if (n == 0) return BEAM_OK;
  k_gather_rows<<<(unsigned)((n + 255) / 256), 256, 0, s->lane->stream>>>(
      (const double2 *)r2c_mapped, d.mode_ij, d.n_modes, d.Q, (int)p->geom.NN, (double2 *)s->staging);
  BEAM_CUDA(cudaGetLastError());
  s->launches++;
  return BEAM_OK;
}

// Mode rows of realizations [0, n): from the pinned staging rows (staged) or
// from the device r2c buffers the caller put in h_src[cap + r].
int upload_modes(beam_gpu_plan *p, RunSlot *s, int n, bool staged, bool staged_on_device) {
  const DevPlan &d = p->d;
  cudaStream_t st = s->lane->stream;
  if (staged && !staged_on_device) {
    BEAM_CUDA(cudaMemcpyAsync(s->staging, s->h_staging, sizeof(double) * 2 * (size_t)n * d.n_modes * d.Q,
                              cudaMemcpyHostToDevice, st));
  } else if (!staged) {
    BEAM_CUDA(cudaMemcpyAsync((void *)(s->src + s->cap), s->h_src + s->cap, sizeof(double *) * n,
                              cudaMemcpyHostToDevice, st));
  }
  long long per = (long long)d.n_modes * d.W;
  if (per == 0) return BEAM_OK;
  dim3 grid((unsigned)((per + 255) / 256), (unsigned)n);
  const double *const *srcs = staged ? s->src : s->src + s->cap;
  if (d.elem == sizeof(float2))
    k_build_modes<float2><<<grid, 256, 0, st>>>(srcs, staged ? 1 : 0, d.mode_ij, d.mode_neg, d.n_modes, d.Q, d.W,
                                                d.colbase, (int)p->geom.NN, (float2 *)s->S, per);
  else
    k_build_modes<double2><<<grid, 256, 0, st>>>(srcs, staged ? 1 : 0, d.mode_ij, d.mode_neg, d.n_modes, d.Q, d.W,
                                                 d.colbase, (int)p->geom.NN, (double2 *)s->S,
                                                 (long long)(mode_data_bytes(d) / sizeof(double2)));
  BEAM_CUDA(cudaGetLastError());
  s->launches++;
  if (d.i8) BEAM_TRY(build_slices(p, s, n));
  return BEAM_OK;
}

int run_epilogue(beam_gpu_plan *p, RunSlot *s, int n) {
  const DevPlan &d = p->d;
  if (d.n_bins == 0) return BEAM_OK;
  double nn2 = (double)p->geom.NN * (double)p->geom.NN;
  long long b_stride = std::max<long long>(1, d.n_combo);
  cudaStream_t st = s->lane->stream;
  if (d.n_epchunks > 0) {
    k_ep_chunks<<<dim3((unsigned)d.n_epchunks, (unsigned)n), EP_THREADS, 0, st>>>(
        d.ep_chunk_first, d.n_epchunks, s->B, b_stride, d.ep_px, d.ep_pz, d.ep_ana, d.ep_cnt, nn2, s->ep_part);
    BEAM_CUDA(cudaGetLastError());
    s->launches++;
  }
  const int threads = 256, cells = d.n_bins * BEAM_NPOLES;
  k_ep_bins<<<dim3((unsigned)((cells + threads - 1) / threads), (unsigned)n), threads, 0, st>>>(
      d.bin_chunk, d.n_bins, d.n_epchunks, s->ep_part, p->geom.vol, s->bins, s->bin_count);
  BEAM_CUDA(cudaGetLastError());
  s->launches++;
  return BEAM_OK;
}

// Queue the copies of realizations [0, n)'s bins, counts and the status word
// to the slot's pinned host buffers, then the slot's `done` event.
int fetch_results(beam_gpu_plan *p, RunSlot *s, int n) {
  const DevPlan &d = p->d;
  cudaStream_t st = s->lane->stream;
  size_t nb = (size_t)d.n_bins;
  if (nb) {
    BEAM_CUDA(cudaMemcpyAsync(s->h_bins, s->bins, sizeof(double) * n * BIN_SECTIONS * nb * BEAM_NPOLES, cudaMemcpyDeviceToHost,
                              st));
    BEAM_CUDA(cudaMemcpyAsync(s->h_count, s->bin_count, sizeof(long long) * n * nb, cudaMemcpyDeviceToHost, st));
  }
  BEAM_CUDA(cudaMemcpyAsync(s->h_status, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  BEAM_CUDA(cudaEventRecord(s->done, st));
  return BEAM_OK;
}

// Wait for the slot's last queued run and turn the device status word into an
// error code (clearing it for the next run).
int check_status(RunSlot *s) {
  BEAM_CUDA(cudaEventSynchronize(s->done));
  int st = *s->h_status;
  if (st == 0) return BEAM_OK;
  *s->h_status = 0;
  cudaMemsetAsync(s->status, 0, sizeof(int), s->lane->stream);
  if (st & DEV_TIMEOUT) {
    set_detail("a bounded device wait in the triangle-sum kernel gave up");
    return BEAM_ETIMEDOUT;
  }
  set_detail("device reported a bad index");
  return BEAM_ECUDA;
}

// Bins of realization r from the slot's pinned copies (after check_status).
int copy_result(const beam_gpu_plan *p, const RunSlot *s, int r, beam_result *res) {
  if (!res) return BEAM_OK;
  size_t nb = (size_t)p->d.n_bins, n = nb * BEAM_NPOLES;
  const double *h = s->h_bins + (size_t)r * BIN_SECTIONS * n;
  if (res->bs) std::memcpy(res->bs, h, sizeof(double) * n);
  if (res->norm) std::memcpy(res->norm, h + n, sizeof(double) * n);
  if (res->out) std::memcpy(res->out, h + 2 * n, sizeof(double) * n);
  if (res->ana_sum) std::memcpy(res->ana_sum, h + 3 * n, sizeof(double) * n);
  if (res->ana)
    for (size_t i = 0; i < n; ++i) res->ana[i] = h[3 * n + i] / h[n + i];  // barbie.c:391
  if (res->count)
    for (size_t b = 0; b < nb; ++b) res->count[b] = (int64_t)s->h_count[(size_t)r * nb + b];
  return BEAM_OK;
}

// One host-input run of realizations [0, n) whose staging rows are gathered:
// H2D of the rows, mode build, triangle sums, epilogue and D2H of the bins,
// captured once per n into a CUDA graph and replayed.
int slot_run_graph(beam_gpu_plan *p, RunSlot *s, int n) {
  cudaStream_t st = s->lane->stream;
  if (!s->graph || s->graph_n != n) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->graph_n = 0;
    BEAM_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    s->launches = 0;
    s->capturing = true;
    int rc = upload_modes(p, s, n, true);
    if (rc == BEAM_OK) rc = run_triangle_sums(p, s, n);
    if (rc == BEAM_OK) rc = run_epilogue(p, s, n);
    if (rc == BEAM_OK) rc = fetch_results(p, s, n);
    s->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != BEAM_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) {
      set_detail(std::string("graph capture: ") + cudaGetErrorString(e));
      return BEAM_ECUDA;
    }
    e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      s->graph = nullptr;
      set_detail(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      return BEAM_ECUDA;
    }
    s->graph_n = n;
  }
  s->timed = false;
  BEAM_CUDA(cudaGraphLaunch(s->graph, st));
  // the graph ends with fetch_results; `done` must follow this replay
  BEAM_CUDA(cudaEventRecord(s->done, st));
  return BEAM_OK;
}
}  // namespace beam
