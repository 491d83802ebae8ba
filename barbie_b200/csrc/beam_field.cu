// Field ingestion on the device: the reference's field generator
// (generate_field.c:78-88 with ngrf_2d_funcs.c:341-584,734-765) and its
// real-space-to-r2c step, producing the r2c buffer double[NN][NN][NN+2] that
// beam_gpu_run reads, without leaving HBM.
//
// 3D transforms. A 3D DFT of the padded r2c layout is three passes of batched
// 1D transforms, one per axis, each reading and writing the buffer once:
//   * rows (last axis, contiguous): r2c / c2r of M rows per CTA, each row's N
//     reals taken as N/2 complex pairs (one half-length complex FFT and a
//     twist);
//   * columns (axes 0 and 1, strided): M adjacent k-columns per CTA, so every
//     global access is M consecutive complex values (128 B at M = 8).
// A CTA stages its M lines in shared memory with 16-byte asynchronous copies
// (the whole tile in flight at once) and runs a Stockham autosort FFT (radix
// 4, 2 and 3 stages, N = 2^a 3^b) between two buffers, one butterfly per
// thread per step, with the twiddle table exp(-2 pi i n / N) in shared memory.
// The transforms are unnormalised, FFTW's convention. HBM-bound: each pass
// moves 2 x 16 N^2 (N/2+1) bytes.
//
// Fused element work (no extra passes):
//   * Make_Image's division by vol on the load of the first backward pass;
//   * the per-row sum of squares for Non_Gauss's variance on the store of the
//     last backward pass (rows), reduced in a fixed order by k_field_var;
//   * Non_Gauss (x += ff (x^2 - var)) and Get_Modes (x *= LL^3) on the load of
//     the first forward pass (rows);
//   * RSD's (1 + beta mu^2) on the store of the last forward pass (axis 0).
//
// Gaussian modes (Fill_Modes). One thread per group of draws of the
// reference's fill order (points, lines, planes, cubes); the index of each
// draw in that order is a closed form of the group, and draw n of the stream
// is a counter-based normal deviate (Philox4x32-10 + Box-Muller), so the
// modes are filled in parallel with the values the sequential order gives.
//
// The file is compiled without FMA contraction, so the amplitude, scaling and
// RSD factors round as the reference's C expressions do.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "beam_internal.h"

namespace beam {

constexpr int FFT_THREADS = 256;
constexpr int FFT_MAX_STAGES = 12;
constexpr long FIELD_MAX_N = 1024;
constexpr long FFT_TILE = 3072;  // complex values of one staging buffer (lines x length), at most

struct FftGeom {
  int N;         // line length
  int M;         // lines per CTA (a power of two)
  int lgM;       // log2 M
  int nst;       // stages
  unsigned rad;  // radix of stage s: 2-bit code (rad >> 2s) & 3, 0 -> 4, 1 -> 2, 2 -> 3
};

// n / d as a multiply-high: exact for n, d < 2^16 (n d < 2^32), d >= 2
struct FastDiv {
  unsigned d, mul;
};
static FastDiv fast_div(unsigned d) { return FastDiv{d, (unsigned)(((1ull << 32) + d - 1) / d)}; }
__device__ __forceinline__ unsigned fdiv(unsigned n, FastDiv f) { return __umulhi(n, f.mul); }

__host__ __device__ __forceinline__ int fft_radix(unsigned rad, int s) {
  const unsigned c = (rad >> (2 * s)) & 3u;
  return c == 0 ? 4 : (c == 1 ? 2 : 3);
}

// N = 2^a 3^b: radix-4 stages, one radix-2 stage for an odd power of two, then
// radix-3; M lines per CTA, the largest power of two <= 16 with M N <= tile
static bool fft_geom(long N, FftGeom *g, long tile = FFT_TILE) {
  if (N < 2 || N > FIELD_MAX_N) return false;
  tile = std::min(std::max(tile, 1L), FFT_TILE);
  g->N = (int)N;
  g->M = 16;
  g->lgM = 4;
  while (g->M > 1 && N * g->M > tile) g->M >>= 1, g->lgM--;
  g->nst = 0;
  g->rad = 0;
  long n = N;
  while (n % 4 == 0 && g->nst < FFT_MAX_STAGES) g->nst++, n /= 4;
  while (n % 2 == 0 && g->nst < FFT_MAX_STAGES) g->rad |= 1u << (2 * g->nst++), n /= 2;
  while (n % 3 == 0 && g->nst < FFT_MAX_STAGES) g->rad |= 2u << (2 * g->nst++), n /= 3;
  return n == 1;
}

// ---------------------------------------------------------------------------
// Counter-based normal deviates: draw n of the stream with seed s is
// Philox4x32-10(counter (n lo, n hi, 0, 0), key (s lo, s hi)) -> (u1, u2) ->
// sqrt(-2 ln u1) cos(2 pi u2), u1 in (0, 1] and u2 in [0, 1) from the two
// 64-bit halves (53 bits each). Philox: Salmon et al., "Parallel random
// numbers: as easy as 1, 2, 3", SC'11.
__device__ __forceinline__ double field_normal(unsigned long long seed, unsigned long long n) {
  unsigned c0 = (unsigned)n, c1 = (unsigned)(n >> 32), c2 = 0u, c3 = 0u;
  unsigned k0 = (unsigned)seed, k1 = (unsigned)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned long long p0 = 0xD2511F53ull * c0, p1 = 0xCD9E8D57ull * c2;
    const unsigned n0 = (unsigned)(p1 >> 32) ^ c1 ^ k0, n1 = (unsigned)p1;
    const unsigned n2 = (unsigned)(p0 >> 32) ^ c3 ^ k1, n3 = (unsigned)p0;
    c0 = n0, c1 = n1, c2 = n2, c3 = n3;
    if (r < 9) k0 += 0x9E3779B9u, k1 += 0xBB67AE85u;
  }
  const unsigned long long a = (((unsigned long long)c1 << 32) | c0) >> 11;
  const unsigned long long b = (((unsigned long long)c3 << 32) | c2) >> 11;
  const double u1 = (double)(a + 1) * 0x1.0p-53, u2 = (double)b * 0x1.0p-53;
  return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

// Pk (ngrf_2d_funcs.c:143-155) with p(k) = 1.0 * k^-2 (ngrf_2d_funcs.c:132-140)
__device__ __forceinline__ double field_pk(double C, long i, long j, long k) {
  const double kx = C * i, ky = C * j, kz = C * k;
  const double kk = sqrt(kx * kx + ky * ky + kz * kz);
  return 1.0 * pow(kk, -2.0);
}

// Fill_Modes (ngrf_2d_funcs.c:341-510). Groups g in the reference's order,
// with hh = N/2 - 1 interior values per half axis:
//   g = 0            the k = 0 mode (zero, no draw)
//   g = 1..7         points (i, j, k) in {0, N/2}^3, one draw each (draw g-1)
//   8 + [0, 12 hh)   lines: (i, j) in {0,1}^2 x 3 axes x hh, two draws each
//   next 12 hh^2     planes: (i, m) in {0,1}^2 x 3 orientations x hh^2, two draws
//   next hh^3        cubes: four modes, eight draws
__global__ void k_field_fill(double2 *__restrict__ A, long N, unsigned long long seed, double volfac, double C) {
  const long h = N / 2, NH = N / 2 + 1, hh = h - 1;
  const long nL = 12 * hh, nP = 12 * hh * hh, nC = hh * hh * hh;
  long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= 8 + nL + nP + nC) return;
  auto at = [&](long i, long j, long k) { return (i * N + j) * NH + k; };
  auto put2 = [&](long x, double amp, unsigned long long n) {
    const double re = amp * field_normal(seed, n), im = amp * field_normal(seed, n + 1);
    A[x] = make_double2(re, im);
    return make_double2(re, im);
  };
  if (g < 8) {
    if (g == 0) {
      A[0] = make_double2(0.0, 0.0);
      return;
    }
    const long i = g >> 2, j = (g >> 1) & 1, k = g & 1;
    const double amp = sqrt(volfac * field_pk(C, i * h, j * h, k * h));
    A[at(i * h, j * h, k * h)] = make_double2(amp * field_normal(seed, g - 1), 0.0);
    return;
  }
  g -= 8;
  if (g < nL) {  // ngrf_2d_funcs.c:387-428
    const long ij = g / (3 * hh), rem = g % (3 * hh), axis = rem / hh, k = rem % hh + 1;
    const long i = ij >> 1, j = ij & 1;
    const unsigned long long n = 7 + 2 * (unsigned long long)g;
    if (axis == 0) {
      const double2 v = put2(at(k, i * h, j * h), sqrt(volfac * field_pk(C, k, i * h, j * h)), n);
      A[at(N - k, i * h, j * h)] = make_double2(v.x, -v.y);
    } else if (axis == 1) {
      const double2 v = put2(at(i * h, k, j * h), sqrt(volfac * field_pk(C, i * h, k, j * h)), n);
      A[at(i * h, N - k, j * h)] = make_double2(v.x, -v.y);
    } else {
      put2(at(i * h, j * h, k), sqrt(volfac * field_pk(C, i * h, j * h, k)), n);
    }
    return;
  }
  g -= nL;
  if (g < nP) {  // ngrf_2d_funcs.c:432-481
    const long im = g / (3 * hh * hh), rem = g % (3 * hh * hh), orient = rem / (hh * hh), q = rem % (hh * hh);
    const long i = im >> 1, m = im & 1, j = q / hh + 1, k = q % hh + 1;
    const unsigned long long n = 7 + 24 * (unsigned long long)hh + 2 * (unsigned long long)g;
    const long jj1 = m ? N - j : j;
    if (orient == 0) {
      put2(at(i * h, jj1, k), sqrt(volfac * field_pk(C, i * h, j, k)), n);
    } else if (orient == 1) {
      put2(at(jj1, i * h, k), sqrt(volfac * field_pk(C, j, i * h, k)), n);
    } else {
      const long jj2 = m ? j : N - j;
      const double2 v = put2(at(jj1, k, i * h), sqrt(volfac * field_pk(C, j, k, i * h)), n);
      A[at(jj2, N - k, i * h)] = make_double2(v.x, -v.y);
    }
    return;
  }
  g -= nP;  // cubes, ngrf_2d_funcs.c:483-505
  const long i = g / (hh * hh) + 1, j = (g / hh) % hh + 1, k = g % hh + 1;
  const unsigned long long n = 7 + 24 * (unsigned long long)hh + 24 * (unsigned long long)(hh * hh) +
                               8 * (unsigned long long)g;
  const double amp = sqrt(volfac * field_pk(C, i, j, k));
  put2(at(i, j, k), amp, n);
  put2(at(N - i, j, k), amp, n + 2);
  put2(at(i, N - j, k), amp, n + 4);
  put2(at(N - i, N - j, k), amp, n + 6);
}

// ---------------------------------------------------------------------------
// Staging: 16-byte asynchronous copies global -> shared (cp.async), so a CTA's
// whole tile is in flight at once.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Stockham FFT of the CTA's M lines of length g.N, from b0 into the returned
// buffer; element p of line m is at m sm + p sp (columns: sm = 1, sp = M;
// rows: sm = an odd pitch, sp = 1). Stage s of radix R (Ns = product of the
// earlier radices): butterfly j reads positions j + r N/R, applies the
// twiddles exp(-+2 pi i r (j mod Ns)/(Ns R)), and writes positions
// (j - j mod Ns) R + j mod Ns + r Ns. Consecutive threads take consecutive
// lines of one butterfly, so a quarter warp touches 8 distinct bank groups.
// tw holds exp(-2 pi i t/(tws N)).
template <bool FWD>
__device__ __forceinline__ double2 twmul(double2 a, double2 w) {
  const double wy = FWD ? w.y : -w.y;
  return make_double2(__fma_rn(a.x, w.x, -(a.y * wy)), __fma_rn(a.x, wy, a.y * w.x));
}

template <bool FWD>
__device__ double2 *fft_lines(double2 *b0, double2 *b1, const double2 *__restrict__ tw, int tws, const FftGeom &g,
                              int sm, int sp) {
  const int N = g.N, M = g.M;
  int Ns = 1;
  for (int s = 0; s < g.nst; ++s) {
    const int R = fft_radix(g.rad, s), NR = N / R, tstr = tws * (N / (Ns * R));
    const bool pow2 = (Ns & (Ns - 1)) == 0;
    for (int b = threadIdx.x; b < M * NR; b += blockDim.x) {
      const int m = b & (M - 1), j = b >> g.lgM;
      const int js = pow2 ? (j & (Ns - 1)) : (j % Ns), o = (j - js) * R + js;
      const double2 *x = b0 + m * sm;
      double2 *y = b1 + m * sm;
      if (R == 4) {
        const double2 a0 = x[j * sp];
        const double2 a1 = twmul<FWD>(x[(j + NR) * sp], tw[js * tstr]);
        const double2 a2 = twmul<FWD>(x[(j + 2 * NR) * sp], tw[2 * js * tstr]);
        const double2 a3 = twmul<FWD>(x[(j + 3 * NR) * sp], tw[3 * js * tstr]);
        const double2 y0 = make_double2(a0.x + a2.x, a0.y + a2.y), y1 = make_double2(a0.x - a2.x, a0.y - a2.y);
        const double2 y2 = make_double2(a1.x + a3.x, a1.y + a3.y), y3 = make_double2(a1.x - a3.x, a1.y - a3.y);
        y[o * sp] = make_double2(y0.x + y2.x, y0.y + y2.y);
        y[(o + 2 * Ns) * sp] = make_double2(y0.x - y2.x, y0.y - y2.y);
        if (FWD) {  // y1 -+ i y3
          y[(o + Ns) * sp] = make_double2(y1.x + y3.y, y1.y - y3.x);
          y[(o + 3 * Ns) * sp] = make_double2(y1.x - y3.y, y1.y + y3.x);
        } else {
          y[(o + Ns) * sp] = make_double2(y1.x - y3.y, y1.y + y3.x);
          y[(o + 3 * Ns) * sp] = make_double2(y1.x + y3.y, y1.y - y3.x);
        }
      } else if (R == 2) {
        const double2 a0 = x[j * sp];
        const double2 a1 = twmul<FWD>(x[(j + NR) * sp], tw[js * tstr]);
        y[o * sp] = make_double2(a0.x + a1.x, a0.y + a1.y);
        y[(o + Ns) * sp] = make_double2(a0.x - a1.x, a0.y - a1.y);
      } else {  // R == 3
        const double c = 0.86602540378443864676;  // sqrt(3)/2
        const double2 a0 = x[j * sp];
        const double2 a1 = twmul<FWD>(x[(j + NR) * sp], tw[js * tstr]);
        const double2 a2 = twmul<FWD>(x[(j + 2 * NR) * sp], tw[2 * js * tstr]);
        const double2 t = make_double2(a1.x + a2.x, a1.y + a2.y), d = make_double2(a1.x - a2.x, a1.y - a2.y);
        const double2 mm = make_double2(__fma_rn(-0.5, t.x, a0.x), __fma_rn(-0.5, t.y, a0.y));
        y[o * sp] = make_double2(a0.x + t.x, a0.y + t.y);
        if (FWD) {  // mm -+ i c d
          y[(o + Ns) * sp] = make_double2(__fma_rn(c, d.y, mm.x), __fma_rn(-c, d.x, mm.y));
          y[(o + 2 * Ns) * sp] = make_double2(__fma_rn(-c, d.y, mm.x), __fma_rn(c, d.x, mm.y));
        } else {
          y[(o + Ns) * sp] = make_double2(__fma_rn(-c, d.y, mm.x), __fma_rn(c, d.x, mm.y));
          y[(o + 2 * Ns) * sp] = make_double2(__fma_rn(c, d.y, mm.x), __fma_rn(-c, d.x, mm.y));
        }
      }
    }
    __syncthreads();
    double2 *t = b0;
    b0 = b1;
    b1 = t;
    Ns *= R;
  }
  return b0;
}

// Column pass over axis 0 or 1 of the half-complex array (complex strides):
// CTA blockIdx.x = outer * ntile + tile covers k-columns [tile M, tile M + M).
struct ColPass {
  double2 *data;
  long outer_stride, elem_stride;
  int NH, ntile;
  double in_div;  // > 0: loaded values are divided by it (Make_Image, ngrf_2d_funcs.c:521-527)
  int rsd;        // axis-0 pass: RSD factor on the store (ngrf_2d_funcs.c:743-762)
  double beta;
};

template <bool FWD>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_cols(ColPass a, FftGeom g, const double2 *__restrict__ twg) {
  extern __shared__ double2 fsm[];
  const int N = g.N, M = g.M;
  double2 *tw = fsm, *b0 = fsm + N, *b1 = b0 + (size_t)N * M;
  const long outer = blockIdx.x / a.ntile;
  const int k0 = (int)(blockIdx.x % a.ntile) * M, mc = min(M, a.NH - k0);
  double2 *base = a.data + outer * a.outer_stride + k0;
  for (int e = threadIdx.x; e < N * M; e += blockDim.x) {
    const int p = e >> g.lgM, m = e & (M - 1);
    if (m < mc)
      cp_async16(b0 + e, base + p * a.elem_stride + m);
    else
      b0[e] = make_double2(0.0, 0.0);
  }
  for (int p = threadIdx.x; p < N; p += blockDim.x) tw[p] = twg[p];
  cp_async_wait_all();
  __syncthreads();
  if (a.in_div > 0) {
    for (int e = threadIdx.x; e < N * M; e += blockDim.x) b0[e] = make_double2(b0[e].x / a.in_div, b0[e].y / a.in_div);
    __syncthreads();
  }
  const double2 *r = fft_lines<FWD>(b0, b1, tw, 1, g, 1, M);
  for (int e = threadIdx.x; e < N * M; e += blockDim.x) {
    const int p = e >> g.lgM, m = e & (M - 1);
    if (m >= mc) continue;
    double2 v = r[e];
    if (a.rsd) {  // element (i, j, k) = (p, outer, k0 + m)
      const long k = k0 + m;
      const double ia = (p > N / 2) ? (N - p) : p, ja = (outer > N / 2) ? (N - outer) : outer;
      const double kk = sqrt(1. * (ia * ia + ja * ja + (double)(k * k)));
      if (p + outer + k != 0) {
        const double myu = k / kk;
        v.x *= (1. + a.beta * myu * myu);
        v.y *= (1. + a.beta * myu * myu);
      }
    }
    base[p * a.elem_stride + m] = v;
  }
}

// Row passes over the last axis of the padded buffer (N+2 doubles per row).
// A real row of N values is read as its L = N/2 complex pairs
// z[n] = x[2n] + i x[2n+1] (its memory layout), so one complex FFT of length L
// per row with a twist on either side does the real transform:
//   r2c: Z = FFT_L(z); X[k] = E + W^k O for k = 0..L, W = exp(-2 pi i/N),
//        E = (Z[k] + conj Z[L-k])/2, O = (Z[k] - conj Z[L-k])/(2i);
//   c2r: Z[k] = E' + i O', E' = X[k] + conj X[L-k], O' = (X[k] - conj X[L-k]) W^-k
//        (the imaginary parts of X[0] and X[L] dropped); z = IFFT_L(Z).
struct RowPass {
  double *data;
  const double *src;  // r2c: rows read from here (data, or a dense real cube)
  long src_pitch;     // doubles
  long nrows;
  const double *var;  // r2c: Non_Gauss with this variance first (nullptr: none)
  double ff, lcube;   // r2c: x += ff (x^2 - var); x *= lcube (ngrf_2d_funcs.c:540-546,580-582)
  double *row_sumsq;  // c2r: per-row sum of x^2 of the output
  FastDiv divL, divNH;  // by L = N/2 and NH = L + 1
};

// shared pitch of a staged row of L complex values: odd, so the lines of one
// butterfly fall in distinct bank groups
__host__ __device__ __forceinline__ int row_pitch(int L) { return L | 1; }

// g: the half-length geometry (g.N = L); tw: the length-N table
__global__ void __launch_bounds__(FFT_THREADS) k_fft_rows_r2c(RowPass a, FftGeom g, const double2 *__restrict__ twg) {
  extern __shared__ double2 fsm[];
  const int L = g.N, M = g.M, N = 2 * L, NH = L + 1, S = row_pitch(L);
  double2 *tw = fsm, *b0 = fsm + N, *b1 = b0 + (size_t)M * NH;
  const long r0 = (long)blockIdx.x * M;
  for (int e = threadIdx.x; e < M * L; e += blockDim.x) {
    const int m = (int)fdiv(e, a.divL), n = e - m * L;
    if (r0 + m < a.nrows)
      cp_async16(b0 + m * S + n, a.src + (r0 + m) * a.src_pitch + 2 * n);
    else
      b0[m * S + n] = make_double2(0.0, 0.0);
  }
  for (int p = threadIdx.x; p < N; p += blockDim.x) tw[p] = twg[p];
  cp_async_wait_all();
  __syncthreads();
  if (a.var || a.lcube != 1.0) {
    const double var = a.var ? *a.var : 0.0;
    for (int e = threadIdx.x; e < M * L; e += blockDim.x) {
      const int m = (int)fdiv(e, a.divL), n = e - m * L;
      double x = b0[m * S + n].x, y = b0[m * S + n].y;
      if (a.var) {
        x += a.ff * (x * x - var);
        y += a.ff * (y * y - var);
      }
      b0[m * S + n] = make_double2(x * a.lcube, y * a.lcube);
    }
    __syncthreads();
  }
  const double2 *Z = fft_lines<true>(b0, b1, tw, 2, g, S, 1);
  double2 *out = (double2 *)a.data;
  for (int e = threadIdx.x; e < M * NH; e += blockDim.x) {
    const int m = (int)fdiv(e, a.divNH), k = e - m * NH;
    if (r0 + m >= a.nrows) continue;
    const double2 zk = Z[m * S + (k == L ? 0 : k)], zc = Z[m * S + (k == 0 ? 0 : L - k)];
    const double2 E = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));
    const double2 O = make_double2(0.5 * (zk.y + zc.y), -0.5 * (zk.x - zc.x));  // (zk - conj zc) / (2i)
    const double2 w = tw[k];
    out[(r0 + m) * NH + k] = make_double2(__fma_rn(w.x, O.x, __fma_rn(-w.y, O.y, E.x)),
                                          __fma_rn(w.x, O.y, __fma_rn(w.y, O.x, E.y)));
  }
}

__global__ void __launch_bounds__(FFT_THREADS) k_fft_rows_c2r(RowPass a, FftGeom g, const double2 *__restrict__ twg) {
  extern __shared__ double2 fsm[];
  const int L = g.N, M = g.M, N = 2 * L, NH = L + 1, S = row_pitch(L);
  double2 *tw = fsm, *b0 = fsm + N, *b1 = b0 + (size_t)M * NH;
  const long r0 = (long)blockIdx.x * M;
  const double2 *in = (const double2 *)a.data;
  for (int e = threadIdx.x; e < M * NH; e += blockDim.x) {  // the rows' spectra into b1 (pitch NH)
    const int m = (int)fdiv(e, a.divNH);
    if (r0 + m < a.nrows)
      cp_async16(b1 + e, in + r0 * NH + e);
    else
      b1[e] = make_double2(0.0, 0.0);
  }
  for (int p = threadIdx.x; p < N; p += blockDim.x) tw[p] = twg[p];
  cp_async_wait_all();
  __syncthreads();
  for (int e = threadIdx.x; e < M * L; e += blockDim.x) {
    const int m = (int)fdiv(e, a.divL), k = e - m * L;
    double2 xk = b1[m * NH + k], xc = b1[m * NH + L - k];
    if (k == 0) xk.y = 0.0, xc.y = 0.0;  // DC and Nyquist are real
    const double2 Ep = make_double2(xk.x + xc.x, xk.y - xc.y);
    const double2 d = make_double2(xk.x - xc.x, xk.y + xc.y);  // xk - conj xc
    const double2 w = tw[k];                                    // O' = d conj(w)
    const double2 Op = make_double2(__fma_rn(d.x, w.x, d.y * w.y), __fma_rn(d.y, w.x, -(d.x * w.y)));
    b0[m * S + k] = make_double2(Ep.x - Op.y, Ep.y + Op.x);
  }
  __syncthreads();
  const double2 *z = fft_lines<false>(b0, b1, tw, 2, g, S, 1);
  for (int e = threadIdx.x; e < M * L; e += blockDim.x) {
    const int m = (int)fdiv(e, a.divL), n = e - m * L;
    if (r0 + m < a.nrows) ((double2 *)(a.data + (r0 + m) * (N + 2)))[n] = z[m * S + n];
  }
  if (a.row_sumsq) {  // one warp per row, lanes in a fixed order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int m = warp; m < M; m += FFT_THREADS / 32) {
      double s = 0.0;
      for (int n = lane; n < L; n += 32) {
        const double2 v = z[m * S + n];
        s += v.x * v.x;
        s += v.y * v.y;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0 && r0 + m < a.nrows) a.row_sumsq[r0 + m] = s;
    }
  }
}

// variance of the image (Non_Gauss, ngrf_2d_funcs.c:563-570): the row sums in
// a fixed order, / (1. * N * N * N)
__global__ void __launch_bounds__(1024) k_field_var(const double *__restrict__ row_sumsq, long nrows, long N,
                                                    double *__restrict__ var) {
  __shared__ double part[32];
  double s = 0.0;
  for (long r = threadIdx.x; r < nrows; r += blockDim.x) s += row_sumsq[r];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = part[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *var = s / (1. * N * N * N);
  }
}

// ---------------------------------------------------------------------------
// host side

static bool field_size_ok(long N) {
  if (N < 4 || N % 2 || N > FIELD_MAX_N) return false;
  long n = N;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

// exp(-2 pi i n / N) rounded from long double
static void twiddles(long N, std::vector<double2> &tw) {
  tw.resize(N);
  const long double pi = acosl(-1.0L);
  for (long n = 0; n < N; ++n) {
    const long double t = 2.0L * pi * (long double)n / (long double)N;
    tw[n] = make_double2((double)cosl(t), (double)-sinl(t));
  }
}

struct FieldRun {
  beam_gpu_ctx *ctx;
  long N;
  FftGeom gc, gr;               // column lines (length N), row lines (length N/2)
  double2 *tw = nullptr;        // device twiddle table, length N
  double *row_sumsq = nullptr;  // [N^2]
  double *var = nullptr;
  int launches = 0;
};

static size_t cols_smem(const FftGeom &g) { return sizeof(double2) * ((size_t)g.N + 2 * (size_t)g.N * g.M); }
static size_t rows_smem(const FftGeom &g) { return sizeof(double2) * (2 * (size_t)g.N + 2 * (size_t)(g.N + 1) * g.M); }

static int field_workspace(FieldRun &f) {
  beam_gpu_ctx *c = f.ctx;
  const size_t need = sizeof(double2) * f.N + sizeof(double) * (f.N * f.N + 2);
  if (c->field_ws_bytes < need) {
    if (c->field_ws) cudaFree(c->field_ws);
    c->field_ws = nullptr;
    c->field_ws_bytes = 0;
    size_t got = 0;
    int rc = dev_alloc(&got, (char **)&c->field_ws, need);
    if (rc != BEAM_OK) return rc;
    c->field_ws_bytes = need;
  }
  f.tw = (double2 *)c->field_ws;
  f.var = (double *)(f.tw + f.N);
  f.row_sumsq = f.var + 2;
  std::vector<double2> tw;
  twiddles(f.N, tw);
  BEAM_CUDA(cudaMemcpyAsync(f.tw, tw.data(), sizeof(double2) * f.N, cudaMemcpyHostToDevice, c->stream));
  // a pageable host array: wait before it goes out of scope
  BEAM_CUDA(cudaStreamSynchronize(c->stream));
  const int sc = (int)cols_smem(f.gc), sr = (int)rows_smem(f.gr);
  BEAM_CUDA(cudaFuncSetAttribute(k_fft_cols<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sc));
  BEAM_CUDA(cudaFuncSetAttribute(k_fft_cols<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sc));
  BEAM_CUDA(cudaFuncSetAttribute(k_fft_rows_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, sr));
  BEAM_CUDA(cudaFuncSetAttribute(k_fft_rows_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, sr));
  return BEAM_OK;
}

// column passes: axis 0 (i; outer index j) or axis 1 (j; outer index i)
template <bool FWD>
static void launch_cols(FieldRun &f, double *buf, int axis, double in_div, int rsd, double beta) {
  const long N = f.N, NH = N / 2 + 1;
  ColPass a{};
  a.data = (double2 *)buf;
  a.outer_stride = axis == 0 ? NH : N * NH;
  a.elem_stride = axis == 0 ? N * NH : NH;
  a.NH = (int)NH;
  a.ntile = (int)((NH + f.gc.M - 1) / f.gc.M);
  a.in_div = in_div;
  a.rsd = rsd;
  a.beta = beta;
  k_fft_cols<FWD><<<(unsigned)(N * a.ntile), FFT_THREADS, cols_smem(f.gc), f.ctx->stream>>>(a, f.gc, f.tw);
  ++f.launches;
}

static void launch_rows_r2c(FieldRun &f, double *buf, const double *src, long src_pitch, bool nongauss, double ff,
                            double lcube) {
  RowPass a{};
  a.data = buf;
  a.src = src;
  a.src_pitch = src_pitch;
  a.nrows = f.N * f.N;
  a.var = nongauss ? f.var : nullptr;
  a.ff = ff;
  a.lcube = lcube;
  a.divL = fast_div((unsigned)(f.N / 2));
  a.divNH = fast_div((unsigned)(f.N / 2 + 1));
  k_fft_rows_r2c<<<(unsigned)((a.nrows + f.gr.M - 1) / f.gr.M), FFT_THREADS, rows_smem(f.gr), f.ctx->stream>>>(
      a, f.gr, f.tw);
  ++f.launches;
}

static void launch_rows_c2r(FieldRun &f, double *buf) {
  RowPass a{};
  a.data = buf;
  a.nrows = f.N * f.N;
  a.row_sumsq = f.row_sumsq;
  a.divL = fast_div((unsigned)(f.N / 2));
  a.divNH = fast_div((unsigned)(f.N / 2 + 1));
  k_fft_rows_c2r<<<(unsigned)((a.nrows + f.gr.M - 1) / f.gr.M), FFT_THREADS, rows_smem(f.gr), f.ctx->stream>>>(
      a, f.gr, f.tw);
  ++f.launches;
}

static int field_begin(beam_gpu_ctx *ctx, long NN, double LL, FieldRun &f) {
  if (!field_size_ok(NN) || !(LL > 0) || !std::isfinite(LL)) {
    set_detail("field: NN must be 2^a 3^b, even, in [4, 1024], and LL > 0");
    return BEAM_EINVAL;
  }
  f.ctx = ctx;
  f.N = NN;
  long tc = FFT_TILE, tr = FFT_TILE;  // staging tiles: beam_gpu_field_autotune's choice, if any
  const auto tuned = ctx->field_tiles.find(NN);
  if (tuned != ctx->field_tiles.end()) tc = tuned->second.first, tr = tuned->second.second;
  if (!fft_geom(NN, &f.gc, tc) || !fft_geom(NN / 2, &f.gr, tr) || cols_smem(f.gc) > ctx->smem_optin ||
      rows_smem(f.gr) > ctx->smem_optin) {
    set_detail("field: no FFT geometry for this NN");
    return BEAM_EINVAL;
  }
  BEAM_CUDA(cudaSetDevice(ctx->device));
  return field_workspace(f);
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// the output buffer: the caller's device buffer, or a temporary one
static int field_out(const FieldRun &f, double *r2c, int r2c_on_device, double **buf) {
  if (r2c_on_device) {
    if (!aligned16(r2c)) {
      set_detail("field: the device r2c buffer must be 16-byte aligned");
      return BEAM_EINVAL;
    }
    *buf = r2c;
    return BEAM_OK;
  }
  size_t got = 0;
  return dev_alloc(&got, buf, (size_t)f.N * f.N * (f.N + 2));
}

static int field_end(FieldRun &f, double *buf, double *r2c, int r2c_on_device, double *var_out) {
  cudaStream_t st = f.ctx->stream;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !r2c_on_device)
    e = cudaMemcpyAsync(r2c, buf, sizeof(double) * f.N * f.N * (f.N + 2), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && var_out) e = cudaMemcpyAsync(var_out, f.var, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (!r2c_on_device) cudaFree(buf);
  if (e != cudaSuccess) {
    set_detail(std::string("field: ") + cudaGetErrorString(e));
    return BEAM_ECUDA;
  }
  f.ctx->field_launches = f.launches;
  return BEAM_OK;
}

}  // namespace beam

using namespace beam;

extern "C" int beam_gpu_field_launches(const beam_gpu_ctx *ctx) { return ctx ? ctx->field_launches : -1; }

extern "C" int beam_gpu_field_generate(beam_gpu_ctx *ctx, long NN, unsigned long long seed, double LL, double ff,
                                       double beta, double *r2c, int r2c_on_device, double *sigma) {
  if (!ctx || !r2c || !std::isfinite(ff) || !std::isfinite(beta)) {
    set_detail("field generate: null context or buffer, or non-finite ff / beta");
    return BEAM_EINVAL;
  }
  FieldRun f;
  int rc = field_begin(ctx, NN, LL, f);
  if (rc != BEAM_OK) return rc;
  double *buf = nullptr;
  if ((rc = field_out(f, r2c, r2c_on_device, &buf)) != BEAM_OK) return rc;
  const long N = NN, h = N / 2, hh = h - 1;
  // generate_field.c:54-56
  const double vol = pow((N * LL), 3), C = 2. * M_PI / (N * LL);
  const long groups = 8 + 12 * hh + 12 * hh * hh + hh * hh * hh;
  k_field_fill<<<(unsigned)((groups + 255) / 256), 256, 0, ctx->stream>>>((double2 *)buf, N, seed, vol / 2., C);
  ++f.launches;
  // Make_Image: / vol, c2r (axis 0, axis 1, rows); the rows keep their sums of squares
  launch_cols<false>(f, buf, 0, vol, 0, 0.0);
  launch_cols<false>(f, buf, 1, 0.0, 0, 0.0);
  launch_rows_c2r(f, buf);
  // Non_Gauss's variance, then Non_Gauss + Get_Modes + r2c (rows, axis 1, axis 0 with RSD)
  k_field_var<<<1, 1024, 0, ctx->stream>>>(f.row_sumsq, N * N, N, f.var);
  ++f.launches;
  launch_rows_r2c(f, buf, buf, N + 2, true, ff, pow(LL, 3.));
  launch_cols<true>(f, buf, 1, 0.0, 0, 0.0);
  launch_cols<true>(f, buf, 0, 0.0, 1, beta);
  double var = 0.0;
  rc = field_end(f, buf, r2c, r2c_on_device, &var);
  if (rc == BEAM_OK && sigma) *sigma = pow(var, 0.5);
  return rc;
}

extern "C" int beam_gpu_field_ingest(beam_gpu_ctx *ctx, long NN, double LL, double beta, const double *cube,
                                     int cube_on_device, double *r2c, int r2c_on_device) {
  if (!ctx || !cube || !r2c || !std::isfinite(beta)) {
    set_detail("field ingest: null context or buffer, or non-finite beta");
    return BEAM_EINVAL;
  }
  if (cube_on_device && !aligned16(cube)) {
    set_detail("field ingest: the device cube must be 16-byte aligned");
    return BEAM_EINVAL;
  }
  if (cube_on_device && r2c_on_device && NN > 0 && NN <= FIELD_MAX_N) {  // the row pass reads one, writes the other
    const uintptr_t c0 = (uintptr_t)cube, c1 = c0 + sizeof(double) * (size_t)NN * NN * NN;
    const uintptr_t r0 = (uintptr_t)r2c, r1 = r0 + sizeof(double) * (size_t)NN * NN * (NN + 2);
    if (c0 < r1 && r0 < c1) {
      set_detail("field ingest: the cube and the r2c buffer overlap");
      return BEAM_EINVAL;
    }
  }
  FieldRun f;
  int rc = field_begin(ctx, NN, LL, f);
  if (rc != BEAM_OK) return rc;
  double *buf = nullptr;
  if ((rc = field_out(f, r2c, r2c_on_device, &buf)) != BEAM_OK) return rc;
  const long N = NN;
  const double *src = cube;
  long pitch = N;
  if (!cube_on_device) {  // host rows into the padded buffer
    cudaError_t e = cudaMemcpy2DAsync(buf, sizeof(double) * (N + 2), cube, sizeof(double) * N, sizeof(double) * N,
                                      (size_t)N * N, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
      if (!r2c_on_device) cudaFree(buf);
      set_detail(std::string("field ingest: ") + cudaGetErrorString(e));
      return BEAM_ECUDA;
    }
    src = buf;
    pitch = N + 2;
  }
  // Get_Modes (x LL^3, r2c: rows, axis 1, axis 0) and RSD on the last store
  launch_rows_r2c(f, buf, src, pitch, false, 0.0, pow(LL, 3.));
  launch_cols<true>(f, buf, 1, 0.0, 0, 0.0);
  launch_cols<true>(f, buf, 0, 0.0, 1, beta);
  return field_end(f, buf, r2c, r2c_on_device, nullptr);
}

// FFT staging tiles per NN: each candidate tile (lines x length per CTA) timed
// on one column pass and one row pass over a scratch buffer holding a fixed
// pattern; the fastest of each is kept for the context's later field calls
// with this NN. The transforms do not depend on the tile (every line is
// transformed alike), so results are unchanged bit for bit.
extern "C" int beam_gpu_field_autotune(beam_gpu_ctx *ctx, long NN, beam_field_tune_report *rep) {
  if (!ctx) return BEAM_EINVAL;
  FieldRun f;
  ctx->field_tiles.erase(NN);
  int rc = field_begin(ctx, NN, 1.0, f);
  if (rc != BEAM_OK) return rc;
  const long N = NN;
  const size_t n = (size_t)N * N * (N + 2);
  double *buf = nullptr;
  size_t got = 0;
  if ((rc = dev_alloc(&got, &buf, n)) != BEAM_OK) return rc;
  static const long tiles[] = {768, 1536, 3072};
  constexpr int NT = (int)(sizeof(tiles) / sizeof(tiles[0]));
  static_assert(NT <= BEAM_FIELD_TUNE_MAX, "report size");
  float ms_c[NT], ms_r[NT];
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = BEAM_ECUDA;
  cudaStream_t st = ctx->stream;
  for (int k = 0; k < NT && rc == BEAM_OK; ++k) {
    for (int pass = 0; pass < 2 && rc == BEAM_OK; ++pass) {
      float best = 1e30f;
      if (pass == 0 ? !fft_geom(N, &f.gc, tiles[k]) : !fft_geom(N / 2, &f.gr, tiles[k])) {
        rc = BEAM_EINVAL;
        break;
      }
      if ((rc = field_workspace(f)) != BEAM_OK || (rc = fill_pattern(buf, n, st, ctx->num_sms)) != BEAM_OK) break;
      for (int r = -1; r < 3; ++r) {  // r = -1: warm-up
        cudaEventRecord(e0, st);
        if (pass == 0)
          launch_cols<true>(f, buf, 0, 0.0, 0, 0.0);
        else
          launch_rows_r2c(f, buf, buf, N + 2, false, 0.0, 1.0);
        cudaEventRecord(e1, st);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
          rc = BEAM_ECUDA;
          break;
        }
        if (r >= 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) best = std::min(best, ms);
      }
      (pass == 0 ? ms_c : ms_r)[k] = best;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  if (rc != BEAM_OK) {
    set_detail("field autotune: a timing launch failed");
    return rc;
  }
  int bc = 0, br = 0;
  for (int k = 1; k < NT; ++k) {
    if (ms_c[k] < ms_c[bc]) bc = k;
    if (ms_r[k] < ms_r[br]) br = k;
  }
  ctx->field_tiles[NN] = std::make_pair((int)tiles[bc], (int)tiles[br]);
  if (rep) {
    rep->n = NT;
    rep->best_cols = bc;
    rep->best_rows = br;
    for (int k = 0; k < NT; ++k) {
      rep->tile[k] = (int)tiles[k];
      rep->cols_ms[k] = ms_c[k];
      rep->rows_ms[k] = ms_r[k];
    }
  }
  return BEAM_OK;
}
