// Triangle sums of the int8 path (BEAM_PREC_INT8) on the int8 tensor cores
// (sm_100a, mma.sync m16n8k32 with s32 accumulation).
//
// The sum is the one of beam_triangle.cu (and of barbie.c:329-337 through the
// closed-triangle identity of beam_plan.cu): for every accepted combo (p1, p3)
// of a ring triplet, over the runs of its in-plane triangle list (consecutive
// triangles sharing the run leg's mode k2),
//   S(p1, p3) = sum_runs Re( y_k2(-p1-p3) W(p1, p3) ),  W = sum_run x_k1(p1) z_k3(p3).
// Here W is formed exactly: x and z are cut into five 8-bit slices against a
// power-of-two scale per (ring, plane) (k_build_slices, beam_run.cu), and
//   W = 2^(ex + ez - 14) sum_{L<=5} 2^(-8L) acc_L,  acc_L = sum_{i+j=L} sum_run z_i x_j,
// each acc_L an int32 sum of exact 8-bit products (19 slice pairs). The dropped
// pairs (i + j > 5) and the slices' truncation leave a relative error near
// 2^-44 of the legs' scales per product; the run's end (y W) and everything
// after it are FP64.
//
// MMA shape: A (16 x 32) = the z leg: rows = 16 planes p3 of the tile's
// window, K = 16 triangles x (Re, Im); B (32 x 8) = the x leg: columns = 8
// planes p1, K in the same order, as (Re x, -Im x) for Re W and (Im x, Re x)
// for Im W. A warp's tile is one window x up to two p1 blocks (TriTile:
// p1_0[0..1], p3_0 the window); a chunk is one run's next 16 triangles.
#include <type_traits>

#include "beam_device.cuh"
#include "beam_internal.h"

namespace beam {

struct I8Args {
  const TriItem *items;
  const TriTile *tiles;
  const int32_t *tile_combo;
  const TriDesc *descs;
  const unsigned char *S;  // realization 0's mode data (FP64 rows, slice rows, scales)
  long long s_stride;      // bytes per realization
  size_t xtab_off, ztab_off, scale_off;  // byte offsets of the slice tables and the scales
  int W, colbase;
  const int32_t *u_cfirst, *u_ncombo;
  const long long *u_part;
  double *part;
  long long part_stride;
  int *status;
  int stage;  // bytes per stage
};

// D += A B on the int8 tensor cores; slice 0 is signed, slices 1-4 unsigned.
template <int I, int J>
__device__ __forceinline__ void mma_i8(int (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
#define BEAM_MMA_I8(TA, TB)                                                                                  \
  asm volatile("mma.sync.aligned.m16n8k32.row.col.s32." TA "." TB ".s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, " \
               "{%0,%1,%2,%3};"                                                                              \
               : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])                                              \
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1))
  if constexpr (I == 0 && J == 0) BEAM_MMA_I8("s8", "s8");
  else if constexpr (I == 0) BEAM_MMA_I8("s8", "u8");
  else if constexpr (J == 0) BEAM_MMA_I8("u8", "s8");
  else BEAM_MMA_I8("u8", "u8");
#undef BEAM_MMA_I8
}

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
  return r;
}

// Producer: the copies of one chunk into stage `st`: per triangle the x leg's
// table segment (ring r1, columns [colx, colx + Lx)) and the z leg's (ring
// r3, [colz, colz + Lz)), per chunk the run leg's FP64 row (ring r2, [coly,
// coly + Ly)). Lane j < nt copies triangle j's segments.
__device__ __forceinline__ void i8_issue(const I8Args &a, const TriItem &it, const unsigned char *S, unsigned char *st,
                                         uint32_t full, int packed, uint32_t xz, int y) {
  const int lane = threadIdx.x & 31;
  const int nt = chunk_nt(packed);
  const int px = i8_pitch(I8_XW * it.Lx), pz = i8_pitch(I8_ZW * it.Lz);
  uint32_t *xs = reinterpret_cast<uint32_t *>(st), *zs = xs + TRI_CHUNK * px;
  double2 *ys = reinterpret_cast<double2 *>(zs + TRI_CHUNK * pz);
  if (lane == 0) mbar_expect_tx(full, (uint32_t)(nt * (I8_XW * it.Lx + I8_ZW * it.Lz) * 4 + it.Ly * 16));
  __syncwarp();
  if (lane < nt) {
    const int mx = it.m1 + (int)(xz & 0xffffu), mz = it.m3 + (int)(xz >> 16);
    const uint32_t *xt = reinterpret_cast<const uint32_t *>(S + a.xtab_off);
    const uint32_t *zt = reinterpret_cast<const uint32_t *>(S + a.ztab_off);
    bulk_g2s(smem_addr(xs + lane * px), xt + ((size_t)mx * a.W + it.colx) * I8_XW, (uint32_t)(it.Lx * I8_XW * 4), full);
    bulk_g2s(smem_addr(zs + lane * pz), zt + ((size_t)mz * a.W + it.colz) * I8_ZW, (uint32_t)(it.Lz * I8_ZW * 4), full);
  }
  if (lane == 0) {
    const double2 *S64 = reinterpret_cast<const double2 *>(S);
    bulk_g2s(smem_addr(ys), S64 + (size_t)(it.m2 + y) * a.W + it.coly, (uint32_t)(it.Ly * 16), full);
  }
}

// v as a double without the conversion unit: the bit pattern 0x43300000 : (v +
// 2^31) is the double 2^52 + 2^31 + v, from which one exact FP64 subtraction
// leaves v.
__device__ __forceinline__ double i2d_exact(int v) {
  return __hiloint2double(0x43300000, v ^ (int)0x80000000) - 4503601774854144.0;
}

// Slice pair (i, j) in a loop the compiler unrolls: the branches fold.
__device__ __forceinline__ void mma_i8_ij(int i, int j, int (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  if (i == 0 && j == 0) mma_i8<0, 0>(d, a, b0, b1);
  else if (i == 0) mma_i8<0, 1>(d, a, b0, b1);
  else if (j == 0) mma_i8<1, 0>(d, a, b0, b1);
  else mma_i8<1, 1>(d, a, b0, b1);
}

// One chunk (16 triangles of one run) of a tile with NB p1 blocks. Lane (g,
// t) = (lane / 4, lane % 4) holds the A rows g and g + 8 (planes p3) and the
// B column g (plane p1) for triangles 2t, 2t+1, 8+2t, 9+2t; its accumulator
// cells are (row g + 8 (c / 2), column 2t + c % 2). Rows of triangles past
// the run's part here are zeroed in A. At the run's end each cell adds
// Re(y W) to its sum and its accumulators restart.
template <int NB>
__device__ __forceinline__ void i8_chunk(const uint32_t *xs, const uint32_t *zs, const double2 *ys, int px, int pz,
                                         int packed, int t, const int (&ox)[I8_NBT], int oz0, int oz1, const int (&oyb)[I8_NBT],
                                         int Ly, int (&acc)[I8_NBT][I8_LEVELS][2][4], double *sum) {
  const int len = chunk_len(packed, 0);
  const int T[4] = {2 * t, 2 * t + 1, 8 + 2 * t, 9 + 2 * t};
  // A: slices (0,1), (2,3), (4) of the four triangles on the two planes
  uint32_t zw[4][2][I8_ZW];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int k = 0; k < I8_ZW; ++k) {
      const bool on = T[q] < len;
      zw[q][0][k] = on ? zs[T[q] * pz + oz0 * I8_ZW + k] : 0u;
      zw[q][1][k] = on ? zs[T[q] * pz + oz1 * I8_ZW + k] : 0u;
    }
  uint32_t av[I8_SLICES][4];
#pragma unroll
  for (int i = 0; i < I8_SLICES; ++i) {
    const uint32_t sel = (i & 1) ? 0x7632u : 0x5410u;
    const int k = i >> 1;
    av[i][0] = prmt(zw[0][0][k], zw[1][0][k], sel);
    av[i][1] = prmt(zw[0][1][k], zw[1][1][k], sel);
    av[i][2] = prmt(zw[2][0][k], zw[3][0][k], sel);
    av[i][3] = prmt(zw[2][1][k], zw[3][1][k], sel);
  }
#pragma unroll
  for (int j = 0; j < I8_SLICES; ++j)
#pragma unroll
    for (int n = 0; n < NB; ++n) {
      uint32_t xw[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) xw[q] = xs[T[q] * px + ox[n] * I8_XW + j];
      const uint32_t br0 = prmt(xw[0], xw[1], 0x5410u), br1 = prmt(xw[2], xw[3], 0x5410u);
      const uint32_t bi0 = prmt(xw[0], xw[1], 0x7632u), bi1 = prmt(xw[2], xw[3], 0x7632u);
#pragma unroll
      for (int i = 0; i < I8_SLICES && i + j < I8_LEVELS; ++i) {
        mma_i8_ij(i, j, acc[n][i + j][0], av[i], br0, br1);
        mma_i8_ij(i, j, acc[n][i + j][1], av[i], bi0, bi1);
      }
    }
  if (chunk_cont_out(packed)) return;  // the run goes on in the next chunk
#pragma unroll
  for (int n = 0; n < NB; ++n)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double wr = i2d_exact(acc[n][I8_LEVELS - 1][0][c]), wi = i2d_exact(acc[n][I8_LEVELS - 1][1][c]);
#pragma unroll
      for (int l = I8_LEVELS - 2; l >= 0; --l) {
        wr = fma(wr, 0.00390625, i2d_exact(acc[n][l][0][c]));
        wi = fma(wi, 0.00390625, i2d_exact(acc[n][l][1][c]));
      }
      int o = oyb[n] - (c & 1) - 8 * (c >> 1);
      o = (unsigned)o < (unsigned)Ly ? o : 0;
      const double2 y = ys[o];
      sum[(n * 4 + c) * 32] += fma(y.x, wr, -y.y * wi);
#pragma unroll
      for (int l = 0; l < I8_LEVELS; ++l) acc[n][l][0][c] = acc[n][l][1][c] = 0;
    }
}

// Consumer warp: tile `warp` of the item over its chunks. Rows of the window
// outside the staged z columns, and y of cells outside the staged p2 range,
// read column 0 (those cells hold no combo and are never stored). At the end
// each cell with a combo stores sum x 2^(ex(p1) + ez(p3) - 14).
__device__ __forceinline__ void i8_consume(const I8Args &a, const TriItem &it, const unsigned char *S,
                                           const unsigned char *stages, uint64_t *full, uint64_t *empty,
                                           volatile int *s_fail, const volatile int *s_packed, int warp, int lane,
                                           int nch, int real, double *sum) {
  const TriTile tl = a.tiles[it.tile0 + warp];
  const int nblk = tl.nblk;
  const int g = lane >> 2, t = lane & 3;
  const int px = i8_pitch(I8_XW * it.Lx), pz = i8_pitch(I8_ZW * it.Lz);
  int ox[I8_NBT], oyb[I8_NBT];
  int oz0 = tl.p3_0[0] + g + a.colbase - it.colz, oz1 = oz0 + 8;
  oz0 = (unsigned)oz0 < (unsigned)it.Lz ? oz0 : 0;
  oz1 = (unsigned)oz1 < (unsigned)it.Lz ? oz1 : 0;
#pragma unroll
  for (int n = 0; n < I8_NBT; ++n) {
    ox[n] = tl.p1_0[n] + g + a.colbase - it.colx;
    // y of cell c: plane -(p1_0 + 2t + c % 2) - (p3_0 + g + 8 (c / 2))
    oyb[n] = -tl.p1_0[n] - 2 * t - tl.p3_0[n] - g + a.colbase - it.coly;
  }
  int acc[I8_NBT][I8_LEVELS][2][4];
#pragma unroll
  for (int n = 0; n < I8_NBT; ++n)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      sum[(n * 4 + c) * 32] = 0.0;
#pragma unroll
      for (int l = 0; l < I8_LEVELS; ++l) acc[n][l][0][c] = acc[n][l][1][c] = 0;
    }
  for (int c = 0; c < nch; ++c) {
    const int s = c % I8_STAGES;
    if (*s_fail || !mbar_wait_bounded(smem_addr(&full[s]), (uint32_t)((c / I8_STAGES) & 1))) {
      *s_fail = 1;
      if (lane == 0) atomicOr(a.status, DEV_TIMEOUT);
      return;
    }
    const int packed = s_packed[s];  // this chunk's layout, written by the producer
    const uint32_t *xs = reinterpret_cast<const uint32_t *>(stages + (size_t)s * a.stage);
    const uint32_t *zs = xs + TRI_CHUNK * px;
    const double2 *ys = reinterpret_cast<const double2 *>(zs + TRI_CHUNK * pz);
    if constexpr (I8_NBT == 2) {
      if (nblk == 2) i8_chunk<2>(xs, zs, ys, px, pz, packed, t, ox, oz0, oz1, oyb, it.Ly, acc, sum);
      else i8_chunk<1>(xs, zs, ys, px, pz, packed, t, ox, oz0, oz1, oyb, it.Ly, acc, sum);
    } else {
      i8_chunk<1>(xs, zs, ys, px, pz, packed, t, ox, oz0, oz1, oyb, it.Ly, acc, sum);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[s]));
  }
  const int nc = a.u_ncombo[it.u];
  double *out = a.part + (long long)real * a.part_stride + a.u_part[it.u] + (long long)it.split * nc - a.u_cfirst[it.u];
  const int32_t *scale = reinterpret_cast<const int32_t *>(S + a.scale_off);
  const int32_t *tc = a.tile_combo + (size_t)(it.tile0 + warp) * (TRI_P1 * 32);
#pragma unroll
  for (int n = 0; n < I8_NBT; ++n)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (n >= nblk) continue;
      const int col = 2 * t + (c & 1), row = g + 8 * (c >> 1);
      const int cidx = tc[col * 32 + n * I8_BW + row];
      if (cidx < 0) continue;
      const int p1 = tl.p1_0[n] + col, p3 = tl.p3_0[n] + row;
      const int e = scale[it.rx * a.W + p1 + a.colbase] + scale[it.rz * a.W + p3 + a.colbase] - 14;
      out[cidx] = ldexp(sum[(n * 4 + c) * 32], e);
    }
}

// One CTA per item of one tile class (blockIdx.x) and realization
// (blockIdx.y): a consumer warp per tile, then the producer warp, streaming
// chunks through I8_STAGES stages of a.stage bytes.
__global__ void __launch_bounds__(32 * (I8_MAX_TILES + 1), I8_MINB) k_triangle_i8(I8Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[I8_STAGES], empty[I8_STAGES];
  __shared__ volatile int s_fail;
  __shared__ volatile int s_packed[I8_STAGES];
  const TriItem it = a.items[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncons = (blockDim.x >> 5) - 1;
  if (tid == 0) {
    for (int s = 0; s < I8_STAGES; ++s) {
      mbar_init(smem_addr(&full[s]), 1);
      mbar_init(smem_addr(&empty[s]), ncons);
    }
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int real = blockIdx.y;
  const unsigned char *S = a.S + (size_t)real * a.s_stride;
  const int nch = it.ch1 - it.ch0;
  if (warp == ncons) {
    int issued = 0;
    bool failed = false;
    // chunk descriptors are read TRI_META_AHEAD chunks ahead of their copies
    struct Meta {
      int packed, y;
      uint32_t xz;
    };
    auto meta = [&](int ch) {
      const TriDesc *d = a.descs + ch;
      return Meta{d->packed, d->y[0], lane < TRI_CHUNK ? *reinterpret_cast<const uint32_t *>(&d->xz[lane][0]) : 0u};
    };
    const Meta none{0, 0, 0u};
    Meta m0 = nch > 0 ? meta(it.ch0) : none, m1 = nch > 1 ? meta(it.ch0 + 1) : none;
    Meta m2 = nch > 2 ? meta(it.ch0 + 2) : none, m3 = nch > 3 ? meta(it.ch0 + 3) : none;
    static_assert(TRI_META_AHEAD == 4, "the descriptor ring below holds four chunks");
    for (int c = 0; c < nch; ++c) {
      const int s = c % I8_STAGES;
      if (c >= I8_STAGES &&
          (s_fail || !mbar_wait_bounded(smem_addr(&empty[s]), (uint32_t)(((c / I8_STAGES) - 1) & 1)))) {
        failed = true;
        break;
      }
      const Meta cur = m0;
      m0 = m1;
      m1 = m2;
      m2 = m3;
      if (c + TRI_META_AHEAD < nch) m3 = meta(it.ch0 + c + TRI_META_AHEAD);
      if (lane == 0) s_packed[s] = cur.packed;  // published by i8_issue's arrive on full[s]
      i8_issue(a, it, S, smem_raw + (size_t)s * a.stage, smem_addr(&full[s]), cur.packed, cur.xz, cur.y);
      issued = c + 1;
    }
    if (failed) {
      s_fail = 1;
      if (lane == 0) atomicOr(a.status, DEV_TIMEOUT);
      // let the copies in flight land before the CTA's shared memory is released
      for (int c = issued - I8_STAGES > 0 ? issued - I8_STAGES : 0; c < issued; ++c)
        mbar_wait_bounded(smem_addr(&full[c % I8_STAGES]), (uint32_t)((c / I8_STAGES) & 1));
    }
    return;
  }
  // each consumer lane's 8 running sums, 32 lanes apart (after the stages)
  double *sums = reinterpret_cast<double *>(smem_raw + (size_t)I8_STAGES * a.stage) + warp * 8 * 32 + lane;
  i8_consume(a, it, S, smem_raw, full, empty, &s_fail, s_packed, warp, lane, nch, real, sums);
}

int triangle_i8_init_attributes(size_t smem_optin) {
  cudaFuncAttributes fa;
  BEAM_CUDA(cudaFuncGetAttributes(&fa, k_triangle_i8));
  const int dyn = (int)(smem_optin > fa.sharedSizeBytes ? smem_optin - fa.sharedSizeBytes : 0);
  BEAM_CUDA(cudaFuncSetAttribute(k_triangle_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  return BEAM_OK;
}

// One launch per tile count n (n consumer warps + the producer) on side
// streams forked from and joined back into the slot's stream; each covers its
// class's items for realizations [0, nreal) (blockIdx.y).
int launch_triangle_i8(beam_gpu_plan *p, RunSlot *s, int nreal) {
  const DevPlan &d = p->d;
  I8Args a;
  a.items = d.items;
  a.tiles = d.tiles;
  a.tile_combo = d.tile_combo;
  a.descs = d.descs;
  a.S = static_cast<const unsigned char *>(s->S);
  a.s_stride = (long long)mode_data_bytes(d);
  a.xtab_off = i8_fp64_bytes(d);
  a.ztab_off = i8_fp64_bytes(d) + i8_xtab_bytes(d);
  a.scale_off = i8_fp64_bytes(d) + i8_slice_bytes(d);
  a.W = d.W;
  a.colbase = d.colbase;
  a.u_cfirst = d.u_cfirst;
  a.u_ncombo = d.u_ncombo;
  a.u_part = d.u_part;
  a.part = s->part;
  a.part_stride = d.n_part;
  a.status = s->status;
  Lane *ln = s->lane;
  BEAM_CUDA(cudaEventRecord(ln->fork, ln->stream));
  for (int n = I8_MAX_TILES; n >= 1; --n) {
    const int first = d.class_first[n], count = d.class_first[n + 1] - first;
    if (count == 0) continue;
    cudaStream_t st = ln->side[n - 1];
    BEAM_CUDA(cudaStreamWaitEvent(st, ln->fork, 0));
    I8Args b = a;
    b.items = d.items + first;
    b.stage = d.class_stage[n];
    const size_t smem = (size_t)I8_STAGES * b.stage + (size_t)n * 8 * 32 * sizeof(double);
    k_triangle_i8<<<dim3((unsigned)count, (unsigned)nreal), 32 * (n + 1), smem, st>>>(b);
    BEAM_CUDA(cudaGetLastError());
    s->launches++;
    BEAM_CUDA(cudaEventRecord(ln->join[n - 1], st));
    BEAM_CUDA(cudaStreamWaitEvent(ln->stream, ln->join[n - 1], 0));
  }
  return BEAM_OK;
}

}  // namespace beam
