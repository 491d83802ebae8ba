// Power spectrum multipoles of the r2c buffer (beam_gpu_power_multipoles):
// the reference's calpow_mom (funcs.c:860-1074) on the GPU.
//
// Every mode the reference visits -- its half lines, half planes and half cube,
// i.e. each independent Fourier mode of the real field once -- is binned in
// Nbin logarithmic bins of |k| with |Delta|^2 and its Legendre-weighted copies.
// The mode's |k|, mu, P2, P4, P6 and bin are computed in the reference's
// float/double types; this file is compiled without FMA contraction so they
// round as the reference's C does. powf(mu, 4) and powf(mu, 6) are taken as
// mu^2 products in double rounded once to float (the correctly rounded value;
// the reference's libm powf differs from it by one float ulp on about 0.06% of
// modes).
//
// One CTA per plane i sums its modes into per-bin partials in a fixed order
// (tiles of PK_THREADS modes; warp w owns bins w, w + warps, ...); a second
// kernel adds the planes' partials in plane order. HBM-bound: the buffer is
// read once (NN^2 (NN/2+1) complex128).
#include <cmath>
#include <vector>

#include "beam_internal.h"

namespace beam {

constexpr int PK_THREADS = 256;
constexpr int PK_VALS = 9;  // P0, P2, P4, P6 sums, |k| sum, modes, sum P2^2, P4^2, P6^2

struct PkMode {
  int d;  // bin, -1 if the mode is not visited or outside the bins
  double v[PK_VALS];
};

// funcs.c:932-954 for one mode (a, b, c) of the r2c buffer.
__device__ __forceinline__ PkMode pk_mode(double2 z, long a, long b, long c, long NN, int Nbin, float fac, float scale) {
  PkMode r;
  float m = (float)sqrt((double)(fac * a * a + fac * b * b + fac * c * c));
  float mu = (float)((1.0 * c) / (double)(NN * m));
  float P2 = (float)(0.5 * (3. * mu * mu - 1.));
  const double m2 = (double)mu * mu;
  const float mu4 = (float)(m2 * m2), mu6 = (float)(m2 * m2 * m2);
  float P4 = (float)(0.125 * (35.0 * mu4 - 30.0 * mu * mu + 3));
  float P6 = (float)(0.0625 * (231.0 * mu6 - 315.0 * mu4 + 105.0 * mu * mu - 5));
  r.d = (int)floorf((float)(log10((double)(m * NN)) / scale));
  if (r.d < 0 || r.d >= Nbin) {
    r.d = -1;
    return r;
  }
  const double pw = (z.x * z.x) + (z.y * z.y);
  r.v[0] = pw;
  r.v[1] = pw * P2;
  r.v[2] = pw * P4;
  r.v[3] = pw * P6;
  r.v[4] = (double)m;
  r.v[5] = 1.0;
  r.v[6] = (double)(P2 * P2);
  r.v[7] = (double)(P4 * P4);
  r.v[8] = (double)(P6 * P6);
  return r;
}

__global__ void __launch_bounds__(PK_THREADS) k_pk_planes(const double2 *__restrict__ r2c, int NN, int Nbin, float fac,
                                                          float scale, double *__restrict__ part) {
  extern __shared__ double acc[];  // [Nbin][PK_VALS]
  __shared__ int dbin[PK_THREADS];
  __shared__ double val[PK_VALS][PK_THREADS];
  const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long N = NN, NH = N / 2 + 1, half = N / 2;
  for (int q = tid; q < Nbin * PK_VALS; q += PK_THREADS) acc[q] = 0.0;
  const long a_fold = (i > half) ? N - i : i;
  const double2 *plane = r2c + (size_t)i * N * NH;
  for (long e0 = 0; e0 < N * NH; e0 += PK_THREADS) {
    const long e = e0 + tid;
    int d = -1;
    PkMode md;
    if (e < N * NH) {
      const long j = e / NH, k = e % NH;
      long a = -1, b = 0;
      if (k == 0 || k == half) {
        if (j == 0 || j == half) {
          if (i >= 1 && i <= half) a = i, b = j;  // half lines (funcs.c:925-957)
        } else if (j < half) {
          a = a_fold, b = j;  // half planes (funcs.c:961-1000)
        }
      } else {
        a = a_fold, b = (j > half) ? N - j : j;  // half cube (funcs.c:1004-1048)
      }
      if (a >= 0) {
        md = pk_mode(plane[e], a, b, k, N, Nbin, fac, scale);
        d = md.d;
      }
    }
    dbin[tid] = d;
#pragma unroll
    for (int v = 0; v < PK_VALS; ++v) val[v][tid] = d >= 0 ? md.v[v] : 0.0;
    __syncthreads();
    for (int bin = warp; bin < Nbin; bin += PK_THREADS / 32) {
      double s[PK_VALS];
#pragma unroll
      for (int v = 0; v < PK_VALS; ++v) s[v] = 0.0;
      for (int t = lane; t < PK_THREADS; t += 32)
        if (dbin[t] == bin)
#pragma unroll
          for (int v = 0; v < PK_VALS; ++v) s[v] += val[v][t];
#pragma unroll
      for (int v = 0; v < PK_VALS; ++v)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[v] += __shfl_down_sync(0xffffffffu, s[v], o);
      if (lane == 0)
#pragma unroll
        for (int v = 0; v < PK_VALS; ++v) acc[bin * PK_VALS + v] += s[v];
    }
    __syncthreads();
  }
  for (int q = tid; q < Nbin * PK_VALS; q += PK_THREADS) part[(size_t)i * Nbin * PK_VALS + q] = acc[q];
}

// Sum of the planes' partials in plane order.
__global__ void k_pk_total(const double *__restrict__ part, int NN, int Nbin, double *__restrict__ tot) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= Nbin * PK_VALS) return;
  double s = 0.0;
  for (int i = 0; i < NN; ++i) s += part[(size_t)i * Nbin * PK_VALS + q];
  tot[q] = s;
}

}  // namespace beam

using namespace beam;

extern "C" int beam_gpu_power_multipoles(beam_gpu_ctx *ctx, long NN, double LL, int Nbin, const double *r2c,
                                         int r2c_on_device, double *out) {
  if (!ctx || !r2c || !out || NN < 2 || NN % 2 || NN > 4096 || Nbin < 1 || Nbin > 1024 || !(LL > 0)) {
    set_detail("power multipoles: NN even in [2, 4096], 1 <= Nbin <= 1024, LL > 0, non-null buffers");
    return BEAM_EINVAL;
  }
  BEAM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t n_r2c = (size_t)NN * NN * (NN + 2);
  size_t bytes = 0;
  double *d_r2c = nullptr, *part = nullptr, *tot = nullptr;
  auto release = [&]() {
    if (!r2c_on_device && d_r2c) cudaFree(d_r2c);
    if (part) cudaFree(part);
    if (tot) cudaFree(tot);
  };
  int rc = BEAM_OK;
  const double *src = r2c;
  if (!r2c_on_device) {
    rc = dev_alloc(&bytes, &d_r2c, n_r2c);
    if (rc == BEAM_OK && cudaMemcpyAsync(d_r2c, r2c, sizeof(double) * n_r2c, cudaMemcpyHostToDevice, st) != cudaSuccess)
      rc = BEAM_ECUDA;
    src = d_r2c;
  }
  if (rc == BEAM_OK) rc = dev_alloc(&bytes, &part, (size_t)NN * Nbin * PK_VALS);
  if (rc == BEAM_OK) rc = dev_alloc(&bytes, &tot, (size_t)Nbin * PK_VALS);
  if (rc != BEAM_OK) {
    release();
    return rc;
  }
  // the reference's float constants (funcs.c:898-900,922)
  const float fac = 1. / (1. * NN * NN);
  const float scale = log10(0.5 * NN) / Nbin;
  const size_t smem = sizeof(double) * (size_t)Nbin * PK_VALS;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_pk_planes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_pk_planes<<<(unsigned)NN, PK_THREADS, smem, st>>>((const double2 *)src, (int)NN, Nbin, fac, scale, part);
  k_pk_total<<<(unsigned)((Nbin * PK_VALS + 255) / 256), 256, 0, st>>>(part, (int)NN, Nbin, tot);
  std::vector<double> q((size_t)Nbin * PK_VALS);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(q.data(), tot, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  release();
  if (e != cudaSuccess) {
    set_detail(std::string("power multipoles: ") + cudaGetErrorString(e));
    return BEAM_ECUDA;
  }
  // normalisation of funcs.c:1050-1066
  const double norml = 1. / (1. * NN * NN * NN), pi = M_PI;
  for (int d = 0; d < Nbin; ++d) {
    const double *v = &q[(size_t)d * PK_VALS];
    double kmode = v[4], P0 = v[0], P2 = v[1], P4 = v[2], P6 = v[3];
    if (v[5] > 0.0) {
      P0 = norml * P0 / (1.0 * v[5] * pow(LL, 3.));
      kmode = 2. * pi * kmode / (v[5] * LL);
    }
    if (v[6] > 0.0) P2 = norml * P2 / (1.0 * v[6] * pow(LL, 3.));
    if (v[7] > 0.0) P4 = norml * P4 / (1.0 * v[7] * pow(LL, 3.));
    if (v[8] > 0.0) P6 = norml * P6 / (1.0 * v[8] * pow(LL, 3.));
    out[d] = kmode;
    out[Nbin + d] = P0;
    out[2 * Nbin + d] = P2;
    out[3 * Nbin + d] = P4;
    out[4 * Nbin + d] = P6;
    out[5 * Nbin + d] = v[5];
  }
  return BEAM_OK;
}
