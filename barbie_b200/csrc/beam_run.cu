// Per-realization kernels of libbeam_gpu (sm_100a) other than the triangle sums
// (beam_triangle.cu):
//   k_build_modes  gather the ring modes of the planes in use from the r2c
//                  buffer into signed-plane rows (conjugate of the mirrored mode
//                  for negative planes)                          (funcs.c:94-106)
//   k_epilogue     cal_coeff weights, bins, normalisation        (barbie.c:343-363,
//                                                               383-392; funcs.c:708-745)
#include <cstring>

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
// src: staged rows [n_modes][Q] (staged = 1) or the full r2c buffer.
template <typename C>
__global__ void k_build_modes(const double2 *__restrict__ src, int staged, const int16_t *__restrict__ mode_ij,
                              const int32_t *__restrict__ mode_neg, int n_modes, int Q, int W, int colbase, int NN,
                              C *__restrict__ S) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_modes * W) return;
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
  S[idx] = v;
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
                                                   Q, d.W, d.colbase, (int)NN, (double2 *)d.S64);
  else
    k_build_modes<float2><<<blocks, 256, 0, s>>>((const double2 *)d.staging, 1, d.mode_ij, d.mode_neg, d.n_modes, Q,
                                                  d.W, d.colbase, (int)NN, (float2 *)d.S32);
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
                                                   d.W, d.colbase, (int)p->geom.NN, (double2 *)d.S64);
  else
    k_build_modes<float2><<<blocks, 256, 0, s>>>((const double2 *)r2c_dev, 0, d.mode_ij, d.mode_neg, d.n_modes, d.Q,
                                                  d.W, d.colbase, (int)p->geom.NN, (float2 *)d.S32);
  BEAM_CUDA(cudaGetLastError());
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
