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
// Rows (fixed i, j) are contiguous and, among the modes a row contributes,
// |k| -- and so the bin -- never decreases along k. k_pk_rows therefore reads
// 32 consecutive modes of a row per warp step (coalesced), combines equal
// bins with a segmented shuffle scan, and the last lane of each bin's segment
// adds it to the warp's own shared accumulators; each CTA owns a fixed block
// of rows, so the summation order is fixed and independent of the device.
// k_pk_total then adds the CTAs' partials in order. For more than
// PK_FAST_BINS bins the per-plane kernel k_pk_planes (one CTA per plane, a
// warp per bin over tiles of PK_THREADS modes) is used instead. HBM-bound:
// the buffer is read once (NN^2 (NN/2+1) complex128).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "beam_internal.h"

namespace beam {

constexpr int PK_THREADS = 256;
constexpr int PK_VALS = 9;  // P0, P2, P4, P6 sums, |k| sum, modes, sum P2^2, P4^2, P6^2
constexpr int PK_FAST_BINS = 32;
constexpr int PK_ROWS = 64;       // rows per CTA of k_pk_rows (8 warps x 8)
constexpr int PK_ROW_LOADS = 4;   // 32-mode steps of a row loaded ahead by k_pk_rows

struct PkMode {
  int d;  // bin, -1 if the mode is not visited or outside the bins
  double v[PK_VALS];
};

// funcs.c:932-954 for one mode (a, b, c) of the r2c buffer.
__device__ __forceinline__ PkMode pk_mode(double2 z, long a, long b, long c, long NN, int Nbin, float fac, float scale) {
  PkMode r;
  // sqrt and the division are taken in float: the reference rounds their
  // double results to float, which gives the correctly rounded float result
  // (double rounding is innocuous for sqrt and division when the wider format
  // has at least 2p + 2 bits, 53 >= 2 * 24 + 2), i.e. exactly these
  float m = __fsqrt_rn(fac * a * a + fac * b * b + fac * c * c);
  float mu = __fdiv_rn((float)c, NN * m);
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

// the include rules of funcs.c:925-1048 for mode (i, j, k): (a, b) of the
// visited mode, a = -1 if the reference does not visit it
__device__ __forceinline__ long pk_visit(long i, long j, long k, long N, long *b) {
  const long half = N / 2;
  long a = -1;
  *b = 0;
  if (k == 0 || k == half) {
    if (j == 0 || j == half) {
      if (i >= 1 && i <= half) a = i, *b = j;  // half lines (funcs.c:925-957)
    } else if (j < half) {
      a = (i > half) ? N - i : i, *b = j;  // half planes (funcs.c:961-1000)
    }
  } else {
    a = (i > half) ? N - i : i, *b = (j > half) ? N - j : j;  // half cube (funcs.c:1004-1048)
  }
  return a;
}

// Bin edges of the row kernel: t[d] is the smallest float m (|k| in the
// reference's units) whose bin (int)floorf((float)(log10((double)(m * NN)) /
// scale)) (funcs.c:941) is at least d, found on the host with the host's
// log10 by bisection over float bit patterns (the bin is non-decreasing in m).
// A mode is in bin d iff t[d] <= m < t[d+1], d in [0, Nbin).
struct PkEdges {
  float t[PK_FAST_BINS + 1];
};

__device__ __forceinline__ int pk_bin(float m, const float *t, int Nbin) {
  if (!(m >= t[0]) || m >= t[Nbin]) return -1;
  int lo = 0, hi = Nbin;  // t[lo] <= m < t[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (m >= t[mid])
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Geometry of the visited modes for the table-driven row kernel: entry
// [key(lo, hi)][c] of the modes (a, b, c) with {a, b} = {lo, hi} (lo <= hi <=
// NN/2; key = hi (hi + 1) / 2 + lo) holds P2, P4, P6 and the bin (as int bits,
// -1 outside the bins), computed with the row kernel's own expressions
// (fac a a + fac b b is the same float either way round).
__host__ __device__ inline long pk_key(long lo, long hi) { return hi * (hi + 1) / 2 + lo; }

__global__ void k_pk_table(int NN, int Nbin, float fac, PkEdges edges, float4 *__restrict__ tab) {
  const long N = NN, NH = N / 2 + 1, hi = blockIdx.y;
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (hi + 1) * NH) return;
  const long lo = e / NH, c = e - lo * NH, a = lo, b = hi;
  const float ab = fac * a * a + fac * b * b;
  const float m = __fsqrt_rn(ab + fac * c * c);
  int d = pk_bin(m, edges.t, Nbin);
  float P2 = 0.f, P4 = 0.f, P6 = 0.f;
  if (d >= 0) {
    const float mu = __fdiv_rn((float)c, N * m);
    P2 = (float)(0.5 * (3. * mu * mu - 1.));
    const double m2 = (double)mu * mu;
    const float mu4 = (float)(m2 * m2), mu6 = (float)(m2 * m2 * m2);
    P4 = (float)(0.125 * (35.0 * mu4 - 30.0 * mu * mu + 3));
    P6 = (float)(0.0625 * (231.0 * mu6 - 315.0 * mu4 + 105.0 * mu * mu - 5));
  } else {
    d = -1;
  }
  tab[pk_key(lo, hi) * NH + c] = make_float4(P2, P4, P6, __int_as_float(d));
}

// NV = 9: every sum of a bin from the modes themselves. NV = 4 with TAB: the
// field-dependent sums alone (|Delta|^2 and its P2, P4, P6 copies), the
// Legendre weights and bins read from the geometry table; each sum is formed
// in the same order either way, so both give the same bits.
// 3 CTAs per SM, as many as shared memory allows: at most 85 registers per thread
// (98 unbounded, 2 CTAs per SM; 0.46 -> 0.38 ms at NN=384, bit-identical); the
// table-driven form keeps fewer values and fits 4 CTAs per SM
template <int NV, bool TAB>
__global__ void __launch_bounds__(PK_THREADS, TAB ? 4 : 3) k_pk_rows(const double2 *__restrict__ r2c, int NN, int Nbin, float fac,
                                                        PkEdges edges, const float4 *__restrict__ tab,
                                                        double *__restrict__ part) {
  __shared__ double acc[PK_THREADS / 32][PK_FAST_BINS * NV];
  __shared__ float te[PK_FAST_BINS + 1];
  __shared__ double2 zbuf[PK_THREADS / 32][32 * PK_ROW_LOADS];
  __shared__ float4 tbuf[PK_THREADS / 32][TAB ? 32 * PK_ROW_LOADS : 1];  // the table rows of the same modes
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long N = NN, NH = N / 2 + 1, half = N / 2;
  for (int q = threadIdx.x; q <= Nbin; q += PK_THREADS) te[q] = edges.t[q];
  for (int q = lane; q < Nbin * NV; q += 32) acc[warp][q] = 0.0;
  __syncthreads();
  // per-lane running sums of the warp's current bin D (warp-uniform), added
  // to the warp's accumulators by a fixed shuffle tree when the bin changes
  double r[NV];
#pragma unroll
  for (int t = 0; t < NV; ++t) r[t] = 0.0;
  int D = -1;
  auto flush = [&]() {
    if (D >= 0) {
#pragma unroll
      for (int t = 0; t < NV; ++t) {
        double s = r[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) acc[warp][D * NV + t] += s;
      }
    }
#pragma unroll
    for (int t = 0; t < NV; ++t) r[t] = 0.0;
  };
  for (int rr = 0; rr < PK_ROWS / (PK_THREADS / 32); ++rr) {
    const long row = (long)blockIdx.x * PK_ROWS + warp + (PK_THREADS / 32) * rr;
    if (row >= N * N) break;
    const long i = row / N, j = row - i * N;
    // every mode a row contributes has a = fold(i), b = fold(j) (funcs.c:925-1048)
    const long a = (i > half) ? N - i : i, b = (j > half) ? N - j : j;
    const float ab = fac * a * a + fac * b * b;
    const float4 *trow = TAB ? tab + pk_key(a < b ? a : b, a < b ? b : a) * NH : nullptr;
    const double2 *rowp = r2c + row * NH;
    for (long g0 = 0; g0 < NH; g0 += 32 * PK_ROW_LOADS) {
      // the group's loads first, all in flight at once, into the warp's buffer
      {
        double2 zg[PK_ROW_LOADS];
        float4 tg[TAB ? PK_ROW_LOADS : 1];
#pragma unroll
        for (int q = 0; q < PK_ROW_LOADS; ++q) {
          const long c = g0 + 32 * q + lane;
          zg[q] = c < NH ? rowp[c] : make_double2(0.0, 0.0);
          if (TAB) tg[TAB ? q : 0] = c < NH ? __ldg(trow + c) : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        }
#pragma unroll
        for (int q = 0; q < PK_ROW_LOADS; ++q) {
          zbuf[warp][32 * q + lane] = zg[q];
          if (TAB) tbuf[warp][TAB ? 32 * q + lane : 0] = tg[TAB ? q : 0];
        }
        __syncwarp();
      }
#pragma unroll 1
      for (int q = 0; q < PK_ROW_LOADS; ++q) {
      const long k0 = g0 + 32 * q;
      if (k0 >= NH) break;
      const long c = k0 + lane;
      int d = -1;
      double v[NV];
#pragma unroll
      for (int t = 0; t < NV; ++t) v[t] = 0.0;
      long bb;
      if (TAB) {
        if (c < NH && pk_visit(i, j, c, N, &bb) >= 0) {
          const float4 g = tbuf[warp][TAB ? 32 * q + lane : 0];
          d = __float_as_int(g.w);
          if (d >= 0) {
            const double2 z = zbuf[warp][32 * q + lane];
            const double pw = (z.x * z.x) + (z.y * z.y);
            v[0] = pw, v[1] = pw * g.x, v[2] = pw * g.y, v[3] = pw * g.z;
          }
        }
      } else if (c < NH && pk_visit(i, j, c, N, &bb) >= 0) {
        const float m = __fsqrt_rn(ab + fac * c * c);  // = (float)sqrt((double)...), see pk_mode
        d = pk_bin(m, te, Nbin);
        if (d >= 0) {
          const double2 z = zbuf[warp][32 * q + lane];
          const float mu = __fdiv_rn((float)c, N * m);
          const float P2 = (float)(0.5 * (3. * mu * mu - 1.));
          const double m2 = (double)mu * mu;
          const float mu4 = (float)(m2 * m2), mu6 = (float)(m2 * m2 * m2);
          const float P4 = (float)(0.125 * (35.0 * mu4 - 30.0 * mu * mu + 3));
          const float P6 = (float)(0.0625 * (231.0 * mu6 - 315.0 * mu4 + 105.0 * mu * mu - 5));
          const double pw = (z.x * z.x) + (z.y * z.y);
          v[0] = pw, v[1] = pw * P2, v[2] = pw * P4, v[3] = pw * P6;
          if (NV > 4) {
            v[4 % NV] = (double)m, v[5 % NV] = 1.0;
            v[6 % NV] = (double)(P2 * P2), v[7 % NV] = (double)(P4 * P4), v[8 % NV] = (double)(P6 * P6);
          }
        }
      }
      const int dmax = __reduce_max_sync(0xffffffffu, d);
      if (dmax < 0) continue;  // nothing counted in these 32 modes
      const int dmin = (int)__reduce_min_sync(0xffffffffu, d >= 0 ? (unsigned)d : 0xffffffffu);
      if (dmin == dmax && dmax == D) {
#pragma unroll
        for (int t = 0; t < NV; ++t) r[t] += v[t];
        continue;
      }
      flush();
      if (dmin < dmax) {
        // the bins below dmax: segmented scan over runs of equal bins (the
        // counted bins of a row are non-decreasing in k), run tails add
        const int ds = d < dmax ? d : -1;
#pragma unroll
        for (int t = 0; t < NV; ++t) r[t] = ds >= 0 ? v[t] : 0.0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int db = __shfl_up_sync(0xffffffffu, ds, off);
          const bool same = lane >= off && db == ds;
#pragma unroll
          for (int t = 0; t < NV; ++t) {
            const double y = __shfl_up_sync(0xffffffffu, r[t], off);
            if (same) r[t] += y;
          }
        }
        const int dn = __shfl_down_sync(0xffffffffu, ds, 1);
        if (ds >= 0 && (lane == 31 || dn != ds))
#pragma unroll
          for (int t = 0; t < NV; ++t) acc[warp][ds * NV + t] += r[t];
        __syncwarp();
      }
      D = dmax;
#pragma unroll
      for (int t = 0; t < NV; ++t) r[t] = d == dmax ? v[t] : 0.0;
      }
      __syncwarp();
    }
  }
  flush();
  __syncthreads();
  for (int q = threadIdx.x; q < Nbin * NV; q += PK_THREADS) {
    double s = 0.0;
    for (int w = 0; w < PK_THREADS / 32; ++w) s += acc[w][q];
    part[(size_t)blockIdx.x * Nbin * NV + q] = s;
  }
}

// Sum of nblk partials in a fixed order: one CTA per value, strided thread
// sums, then a fixed shuffle / shared-memory tree.
__global__ void __launch_bounds__(256) k_pk_total(const double *__restrict__ part, int nblk, int Nbin, int nv,
                                                  double *__restrict__ tot) {
  __shared__ double w8[8];
  const int q = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[(size_t)b * Nbin * nv + q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) w8[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += w8[w];
    tot[q] = t;
  }
}

// the bin the reference gives m (funcs.c:941), as a float so that no value is
// out of int range
static float pk_floor_bin(float m, long NN, float scale) { return floorf((float)(log10((double)(m * NN)) / scale)); }

static void pk_edges(long NN, int Nbin, float scale, PkEdges *e) {
  const float top = 2.0f;  // |k| in these units is at most sqrt(3)/2
  uint32_t top_bits;
  memcpy(&top_bits, &top, 4);
  for (int d = 0; d <= Nbin; ++d) {
    if (!(pk_floor_bin(top, NN, scale) >= (float)d)) {
      e->t[d] = INFINITY;
      continue;
    }
    uint32_t lo = 0, hi = top_bits;  // bin(lo) < d <= bin(hi), over non-negative float bit patterns
    while (hi - lo > 1) {
      const uint32_t mid = lo + (hi - lo) / 2;
      float x;
      memcpy(&x, &mid, 4);
      if (pk_floor_bin(x, NN, scale) >= (float)d)
        hi = mid;
      else
        lo = mid;
    }
    memcpy(&e->t[d], &hi, 4);
  }
}

}  // namespace beam

using namespace beam;

extern "C" int beam_gpu_power_multipoles(beam_gpu_ctx *ctx, long NN, double LL, int Nbin, const double *r2c,
                                         int r2c_on_device, double *out) {
  if (!ctx || !r2c || !out || NN < 2 || NN % 2 || NN > 4096 || Nbin < 1 || Nbin > 1024 || !(LL > 0)) {
    set_detail("power multipoles: NN even in [2, 4096], 1 <= Nbin <= 1024, LL > 0, non-null buffers");
    return BEAM_EINVAL;
  }
  if (r2c_on_device && ((uintptr_t)r2c & 15)) {  // read as 16-byte complex values
    set_detail("power multipoles: the device r2c buffer must be 16-byte aligned");
    return BEAM_EINVAL;
  }
  BEAM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t n_r2c = (size_t)NN * NN * (NN + 2);
  size_t bytes = 0;
  double *d_r2c = nullptr, *part = nullptr, *tot = nullptr;
  auto release = [&]() {
    if (!r2c_on_device && d_r2c) cudaFree(d_r2c);
  };
  int rc = BEAM_OK;
  const double *src = r2c;
  if (!r2c_on_device) {
    rc = dev_alloc(&bytes, &d_r2c, n_r2c);
    if (rc == BEAM_OK && cudaMemcpyAsync(d_r2c, r2c, sizeof(double) * n_r2c, cudaMemcpyHostToDevice, st) != cudaSuccess)
      rc = BEAM_ECUDA;
    src = d_r2c;
  }
  const bool fast = Nbin <= PK_FAST_BINS;
  const long nblk = fast ? (NN * NN + PK_ROWS - 1) / PK_ROWS : NN;  // partial sums: per CTA or per plane
  // partial sums and totals in the context's scratch (no allocation per call)
  void *ws = nullptr;
  if (rc == BEAM_OK) rc = ctx_scratch(ctx, sizeof(double) * ((size_t)nblk + 1) * Nbin * PK_VALS, &ws);
  if (rc == BEAM_OK) {
    part = (double *)ws;
    tot = part + (size_t)nblk * Nbin * PK_VALS;
  }
  if (rc != BEAM_OK) {
    release();
    return rc;
  }
  // the reference's float constants (funcs.c:898-900,922)
  const float fac = 1. / (1. * NN * NN);
  const float scale = log10(0.5 * NN) / Nbin;
  std::vector<double> q((size_t)Nbin * PK_VALS);
  cudaError_t e = cudaSuccess;
  if (fast) {
    PkEdges edges;
    pk_edges(NN, Nbin, scale, &edges);
    // The bins' geometric sums (mean |k|, mode count, sums of P_l^2) and each
    // mode's weights and bin depend on NN and Nbin alone: the first call with
    // these sizes forms every sum from the modes and keeps the geometry (a
    // table of at most PK_TAB_MAX bytes); later calls read the table and form
    // only the field's sums, in the same order.
    constexpr size_t PK_TAB_MAX = 256ull << 20;
    const long NH = NN / 2 + 1;
    const size_t tab_bytes = sizeof(float4) * (size_t)pk_key(0, NH) * (size_t)NH;
    const bool cached = ctx->pk_tab && ctx->pk_NN == NN && ctx->pk_Nbin == Nbin;
    if (cached) {
      k_pk_rows<4, true><<<(unsigned)nblk, PK_THREADS, 0, st>>>((const double2 *)src, (int)NN, Nbin, fac, edges,
                                                                 (const float4 *)ctx->pk_tab, part);
      k_pk_total<<<(unsigned)(Nbin * 4), 256, 0, st>>>(part, (int)nblk, Nbin, 4, tot);
      std::vector<double> f((size_t)Nbin * 4);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(f.data(), tot, sizeof(double) * f.size(), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      for (int d = 0; d < Nbin; ++d)
        for (int t = 0; t < PK_VALS; ++t)
          q[(size_t)d * PK_VALS + t] = t < 4 ? f[(size_t)d * 4 + t] : ctx->pk_geo[(size_t)d * PK_VALS + t];
    } else {
      k_pk_rows<PK_VALS, false><<<(unsigned)nblk, PK_THREADS, 0, st>>>((const double2 *)src, (int)NN, Nbin, fac, edges,
                                                                       nullptr, part);
      k_pk_total<<<(unsigned)(Nbin * PK_VALS), 256, 0, st>>>(part, (int)nblk, Nbin, PK_VALS, tot);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(q.data(), tot, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      // keep the geometry for the next call, when the table fits its bound
      if (e == cudaSuccess && tab_bytes <= PK_TAB_MAX) {
        if (ctx->pk_tab_bytes < tab_bytes) {
          if (ctx->pk_tab) cudaFree(ctx->pk_tab);
          ctx->pk_tab = nullptr;
          ctx->pk_tab_bytes = 0;
          if (cudaMalloc(&ctx->pk_tab, tab_bytes) == cudaSuccess)
            ctx->pk_tab_bytes = tab_bytes;
          else
            (void)cudaGetLastError();  // no table: later calls form every sum, as this one
        }
        ctx->pk_NN = 0;
        if (ctx->pk_tab) {
          dim3 grid((unsigned)((NH * NH + 255) / 256), (unsigned)NH);
          k_pk_table<<<grid, 256, 0, st>>>((int)NN, Nbin, fac, edges, (float4 *)ctx->pk_tab);
          if (cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess) {
            ctx->pk_NN = NN;
            ctx->pk_Nbin = Nbin;
            ctx->pk_geo = q;
          }
        }
      }
    }
  } else {
    const size_t smem = sizeof(double) * (size_t)Nbin * PK_VALS;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_pk_planes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_pk_planes<<<(unsigned)NN, PK_THREADS, smem, st>>>((const double2 *)src, (int)NN, Nbin, fac, scale, part);
    k_pk_total<<<(unsigned)(Nbin * PK_VALS), 256, 0, st>>>(part, (int)nblk, Nbin, PK_VALS, tot);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.data(), tot, sizeof(double) * q.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
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
