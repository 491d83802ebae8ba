// Triangle-sum kernel of libbeam_gpu (sm_100a): for every accepted triangle of
// the reference loop, the in-plane closed-triangle sum
//   B = NN^2 Re sum_{k1+k2+k3=0} x_{k1}(p1) y_{k2}(p2) z_{k3}(p3)
// which equals the pixel sum of barbie.c:329-337 (see beam_plan.cu).
//
// A CTA takes one work item: n tiles of one ring triplet (r1, r2, r3) over a
// range of its in-plane triangle list, with one consumer warp per tile (FP64)
// or per pair of tiles (mixed) and one producer warp. The list is k2-major, cut into pieces (runs of one
// k2) and chunks (<= TRI_CHUNK triangles, <= TRI_PIECES pieces) described by
// TriDesc records. The producer streams chunks into a TRI_STAGES-deep ring of
// shared stages with TMA bulk copies -- per triangle the r1 row of k1 over the
// CTA's planes p1 and the r3 row of k3 over its planes p3, per piece the r2 row
// of k2 over its planes p2 -- completing on full[s] (transaction bytes). Each
// consumer releases a stage on empty[s]; the producer refills it when all have.
//
// A consumer warp accumulates, over each piece (one k2), the complex outer
// product w(p1, p3) += x_{k1}(p1) z_{k3}(p3) of its tile and at the end of the
// piece adds Re(y_{k2}(-p1-p3) w(p1, p3)) to the tile's sums. The FP64 path
// forms the outer products on the FP64 tensor cores (tri_consume_dmma: five
// 128-bit shared loads per warp for 4096 FMA), the mixed path with packed FP32
// FMA on 4 x 4 patches of combos per lane (tri_consume_fma).
#include <type_traits>

#include "beam_device.cuh"
#include "beam_internal.h"

namespace beam {

template <typename C>
struct TriAcc;
template <>
struct TriAcc<double2> {
  typedef double t;
};
template <>
struct TriAcc<float2> {
  typedef float t;
};

struct TriArgs {
  const TriItem *items;  // this launch's items
  const TriTile *tiles;
  const int32_t *tile_combo;
  const TriDesc *descs;
  const void *S;
  int W;
  int colbase;  // column of plane 0 in a signed-plane row
  const int32_t *u_cfirst, *u_ncombo;
  const long long *u_part;
  double *part;
  int *status;
  int stage;              // complex values per stage
  int nreal;              // realizations per launch
  int real;               // realization of the item being summed
  int stage_of[TRI_WARPS + 1];  // stage size of each tile count (the persistent kernel's items)
  long long s_stride;     // complex values of S per realization
  long long part_stride;  // partial sums per realization
};

// What the producer needs to issue one chunk's copies, loaded one chunk ahead
// of the issue with independent loads: the chunk layout, and for this lane the
// mode rows of triangle `lane` (x: ring r1, z: ring r3) and of piece `lane` (y).
struct TriMeta {
  int packed;
  uint32_t xz;  // k1 | k3 << 16
  int y;
};

__device__ __forceinline__ TriMeta tri_meta(const TriArgs &a, int ch) {
  const int lane = threadIdx.x & 31;
  const TriDesc *d = a.descs + ch;
  TriMeta m;
  m.packed = d->packed;
  m.xz = lane < TRI_CHUNK ? *reinterpret_cast<const uint32_t *>(&d->xz[lane][0]) : 0u;
  m.y = lane < TRI_PIECES ? d->y[lane] : 0;
  return m;
}

template <typename C>
__device__ __forceinline__ void tri_issue(const TriArgs &a, const TriItem &it, const C *S, C *st, uint32_t full,
                                          const TriMeta &m) {
  const int lane = threadIdx.x & 31;
  const int nt = chunk_nt(m.packed), npc = chunk_npc(m.packed);
  constexpr bool F64 = std::is_same<C, double2>::value;
  const int px = stage_pitch(it.Lx, F64), pz = stage_pitch(it.Lz, F64);
  C *xs = st, *zs = st + TRI_CHUNK * px, *ys = zs + TRI_CHUNK * pz;
  if (lane == 0) mbar_expect_tx(full, (uint32_t)((nt * (it.Lx + it.Lz) + npc * it.Ly) * sizeof(C)));
  __syncwarp();
  // one copy per row; a mixed row segment starts at a multiple of 4 columns,
  // i.e. on a whole block of its 4-column real/imaginary layout
  if (lane < nt) {
    const int mx = it.m1 + (int)(m.xz & 0xffffu), mz = it.m3 + (int)(m.xz >> 16);
    bulk_g2s(smem_addr(xs + lane * px), S + (size_t)mx * a.W + it.colx, (uint32_t)(it.Lx * sizeof(C)), full);
    bulk_g2s(smem_addr(zs + lane * pz), S + (size_t)mz * a.W + it.colz, (uint32_t)(it.Lz * sizeof(C)), full);
  }
  if (lane < npc)
    bulk_g2s(smem_addr(ys + lane * it.Ly), S + (size_t)(it.m2 + m.y) * a.W + it.coly, (uint32_t)(it.Ly * sizeof(C)),
             full);
}

// Wait until chunk c has landed in its stage; false (status set) when the
// bounded wait gave up or another warp's did.
__device__ __forceinline__ bool tri_wait_chunk(const TriArgs &a, uint64_t *full, volatile int *s_fail, int c,
                                               int lane) {
  if (*s_fail || !mbar_wait_bounded(smem_addr(&full[c % TRI_STAGES]), (uint32_t)((c / TRI_STAGES) & 1))) {
    *s_fail = 1;
    if (lane == 0) atomicOr(a.status, DEV_TIMEOUT);
    return false;
  }
  return true;
}

// Partial-sum slots of this CTA's item (split `it.split`) for realization a.real.
__device__ __forceinline__ double *tri_out(const TriArgs &a, const TriItem &it) {
  const int nc = a.u_ncombo[it.u];
  return a.part + (long long)a.real * a.part_stride + a.u_part[it.u] + (long long)it.split * nc -
         a.u_cfirst[it.u];
}

// Packed FP32 pairs (fma.rn.f32x2: two independent FP32 FMAs in one
// instruction, sm_100).
__device__ __forceinline__ unsigned long long f2pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2unpack(unsigned long long v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ void fma2(unsigned long long &d, unsigned long long a, unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}

// Items whose tiles the packed FP32 consumer takes two to a warp (three tiles
// or more; measured at NN=384, pairing from 4 or 5 tiles was 1.5% and 9%
// slower); the others get one tile per warp.
constexpr int TRI_PAIR_MIN = 3;
__host__ __device__ constexpr bool fma_pairs_tiles(int ntiles) { return ntiles >= TRI_PAIR_MIN; }
// Consumer warps of a mixed-path CTA with n tiles, and the most of any class.
__host__ __device__ constexpr int fma_cons_warps(int n) { return fma_pairs_tiles(n) ? (n + 1) / 2 : n; }
constexpr int fma_max_cons_warps(int n = 1) {
  return n > TRI_WARPS ? 0
                       : (fma_cons_warps(n) > fma_max_cons_warps(n + 1) ? fma_cons_warps(n)
                                                                        : fma_max_cons_warps(n + 1));
}

// Mixed-precision consumer for items of one or two tiles: one tile per warp
// (the pairing of the consumer below would leave such a CTA a single consumer
// warp). Lane l works on block l / TRI_BW of the tile: plane
// p3 = p3_0[l / TRI_BW] + l % TRI_BW and the block's 8 planes p1. A
// triangle's 8 x values are two float4 loads per part (x read warp-wide from
// one address per block) and the accumulators of planes (q, q+1) are packed
// pairs, with the same FP32 operations, in the same order, per combo as below.
template <typename C>
__device__ __forceinline__ void tri_consume_fma_tile(const TriArgs &a, const TriItem &it, const C *stages,
                                                     uint64_t *full, uint64_t *empty, volatile int *s_fail,
                                                     const volatile int *s_packed, int warp, int lane, int nch) {
  static_assert(std::is_same<C, float2>::value && TRI_P1 == 8, "the packed consumer is the FP32 path, 8 planes p1");
  const int32_t *tc = a.tile_combo + (size_t)(it.tile0 + warp) * (TRI_P1 * 32) + lane;
  bool any = false;
#pragma unroll
  for (int q = 0; q < TRI_P1; ++q) any |= (tc[q * 32] >= 0);
  // the lane's block nb: planes p1_0[nb] + q and p3 = p3_0[nb] + lane % TRI_BW
  const int nb = lane / TRI_BW;
  const int p1b = a.tiles[it.tile0 + warp].p1_0[nb], p3 = a.tiles[it.tile0 + warp].p3_0[nb] + lane % TRI_BW;
  const int ox0 = p1b + a.colbase - it.colx;                          // x reads ox0 + q (a multiple of 4)
  const int oz = any ? p3 + a.colbase - it.colz : 0;                  // z read
  const int oy0 = any ? -p1b - p3 + a.colbase - it.coly : TRI_P1 - 1;  // y reads oy0 - q
  double sum[TRI_P1];
  unsigned long long wr[TRI_P1 / 2] = {}, wi[TRI_P1 / 2] = {};  // the run's W, planes (2h, 2h+1), across chunks
#pragma unroll
  for (int q = 0; q < TRI_P1; ++q) sum[q] = 0.0;
  for (int c = 0; c < nch; ++c) {
    const int s = c % TRI_STAGES;
    if (!tri_wait_chunk(a, full, s_fail, c, lane)) return;
    const int packed = s_packed[s];  // piece layout of this chunk, written by the producer
    const float *xs = reinterpret_cast<const float *>(stages + s * a.stage);
    const float *zs = xs + 2 * TRI_CHUNK * it.Lx;
    const float *ys = zs + 2 * TRI_CHUNK * it.Lz;
    const int npc = chunk_npc(packed);
    int tt = 0;
    for (int pc = 0; pc < npc; ++pc) {
      const int len = chunk_len(packed, pc);
      if (pc != 0 || !chunk_cont_in(packed)) {
#pragma unroll
        for (int h = 0; h < TRI_P1 / 2; ++h) wr[h] = wi[h] = 0ull;
      }
      for (int j = 0; j < len; ++j, ++tt) {
        const float *zr = zs + 2 * tt * it.Lz + mixed_re(oz);
        const float z_re = zr[0], z_im = zr[4];
        const unsigned long long ZR = f2pack(z_re, z_re), ZI = f2pack(z_im, z_im), NZI = f2pack(-z_im, -z_im);
        const float *xr = xs + 2 * tt * it.Lx + 2 * ox0;  // ox0 is a multiple of 4: block ox0 / 4
#pragma unroll
        for (int g = 0; g < TRI_P1; g += 4) {
          const float4 re = *reinterpret_cast<const float4 *>(xr + 2 * g);
          const float4 im = *reinterpret_cast<const float4 *>(xr + 2 * g + 4);
          const unsigned long long r0 = f2pack(re.x, re.y), r1 = f2pack(re.z, re.w);
          const unsigned long long i0 = f2pack(im.x, im.y), i1 = f2pack(im.z, im.w);
          fma2(wr[g / 2], i0, NZI);
          fma2(wr[g / 2], r0, ZR);
          fma2(wi[g / 2], i0, ZR);
          fma2(wi[g / 2], r0, ZI);
          fma2(wr[g / 2 + 1], i1, NZI);
          fma2(wr[g / 2 + 1], r1, ZR);
          fma2(wi[g / 2 + 1], i1, ZR);
          fma2(wi[g / 2 + 1], r1, ZI);
        }
      }
      if (pc == npc - 1 && chunk_cont_out(packed)) break;  // the run goes on in the next chunk
      const float *yr = ys + 2 * pc * it.Ly;
#pragma unroll
      for (int h = 0; h < TRI_P1 / 2; ++h) {
        float r0, r1, i0, i1;
        f2unpack(wr[h], r0, r1);
        f2unpack(wi[h], i0, i1);
        const float *y0 = yr + mixed_re(oy0 - 2 * h), *y1 = yr + mixed_re(oy0 - 2 * h - 1);
        sum[2 * h] += (double)fma(y0[0], r0, -y0[4] * i0);
        sum[2 * h + 1] += (double)fma(y1[0], r1, -y1[4] * i1);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[s]));
  }
  double *out = tri_out(a, it);
#pragma unroll
  for (int q = 0; q < TRI_P1; ++q) {
    const int cidx = tc[q * 32];
    if (cidx >= 0) out[cidx] = sum[q];
  }
}

// Mixed-precision consumer: FP32 FMA, two tiles per warp. Lane l works on
// block j = l / 4 of the warp's eight (tile j / 4 of its pair, block j % 4 of
// that tile) and in it on a 4 x 4 patch of combos: planes
// p1 = p1_0 + 4 ph + i and p3 = p3_0 + 4 vh + c (i, c < 4; ph = (l >> 1) & 1,
// vh = l & 1). Staged rows keep the 4-column blocks of the mode rows (4 real
// parts, then their 4 imaginary parts; mixed_re), and p1_0, p3_0 and the
// staged columns are multiples of 4, so a triangle's x of the patch's planes
// p1 is one float4 per part and its z of the planes p3 another. Over a piece
// the lane accumulates, per combo,
//   wr = fma(xr, zr, fma(xi, -zi, wr)),  wi = fma(xr, zi, fma(xi, zr, wi))
// with planes (i, i+1) as packed pairs, and at the end of the piece adds
// Re(y_k2(-p1-p3) w) to the combo's FP64 sum. Per triangle a warp makes four
// 128-bit shared loads for 2048 FMA (16 wavefronts, against 18 for 1024 FMA
// with one plane p3 and 8 planes p1 per lane).
template <typename C>
__device__ __forceinline__ void tri_consume_fma(const TriArgs &a, const TriItem &it, const C *stages, uint64_t *full,
                                                uint64_t *empty, volatile int *s_fail, const volatile int *s_packed,
                                                int warp, int lane, int nch) {
  static_assert(std::is_same<C, float2>::value && TRI_P1 == 8 && TRI_BW == 8,
                "the packed consumer is the FP32 path over 8 x 8 blocks");
  const int j = lane >> 2, ph = (lane >> 1) & 1, vh = lane & 1;
  const int tpair = 2 * warp + (j >> 2);           // the lane's tile within the item
  const bool have = tpair < it.ntiles;             // an odd item's last warp has one tile
  const int tile = it.tile0 + (have ? tpair : 2 * warp), nb = j & 3;
  const int P1 = a.tiles[tile].p1_0[nb] + 4 * ph, P3 = a.tiles[tile].p3_0[nb] + 4 * vh;  // patch origin
  // combo of (i, c): tile_combo[tile][4 ph + i][8 nb + 4 vh + c]
  const int32_t *tc = a.tile_combo + (size_t)tile * (TRI_P1 * 32) + (4 * ph) * 32 + nb * TRI_BW + 4 * vh;
  bool any = false;
  if (have) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) any |= (tc[i * 32 + c] >= 0);
  }
  // x reads [ox, ox+4) (whole blocks: always staged); z and y of a lane
  // without combos read columns that are staged for every item
  const int ox = P1 + a.colbase - it.colx;
  const int oz = any ? P3 + a.colbase - it.colz : 0;
  // y of (i, c): column oy0 - i - c; oy0 is a multiple of 4 (P1, P3, colbase
  // and coly are), and a lane without combos reads columns 2..8
  const int oy0 = any ? -P1 - P3 + a.colbase - it.coly : 8;
  double sum[4][4];
  unsigned long long wr[4][2] = {}, wi[4][2] = {};  // the run's W, [c][planes (2h, 2h+1)], across chunks
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 4; ++c) sum[i][c] = 0.0;
  for (int ch = 0; ch < nch; ++ch) {
    const int s = ch % TRI_STAGES;
    if (!tri_wait_chunk(a, full, s_fail, ch, lane)) return;
    const int packed = s_packed[s];  // piece layout of this chunk, written by the producer
    const float *xs = reinterpret_cast<const float *>(stages + s * a.stage);
    const float *zs = xs + 2 * TRI_CHUNK * it.Lx;
    const float *ys = zs + 2 * TRI_CHUNK * it.Lz;
    const int npc = chunk_npc(packed);
    int tt = 0;
    for (int pc = 0; pc < npc; ++pc) {
      const int len = chunk_len(packed, pc);
      if (pc != 0 || !chunk_cont_in(packed)) {
#pragma unroll
        for (int c = 0; c < 4; ++c) wr[c][0] = wr[c][1] = wi[c][0] = wi[c][1] = 0ull;
      }
      for (int k = 0; k < len; ++k, ++tt) {
        const float *xr = xs + 2 * tt * it.Lx + 2 * ox;  // block ox / 4: 4 real, then 4 imaginary parts
        const float *zr = zs + 2 * tt * it.Lz + 2 * oz;
        const float4 xre = *reinterpret_cast<const float4 *>(xr);
        const float4 xim = *reinterpret_cast<const float4 *>(xr + 4);
        const float4 zre = *reinterpret_cast<const float4 *>(zr);
        const float4 zim = *reinterpret_cast<const float4 *>(zr + 4);
        const unsigned long long r0 = f2pack(xre.x, xre.y), r1 = f2pack(xre.z, xre.w);
        const unsigned long long i0 = f2pack(xim.x, xim.y), i1 = f2pack(xim.z, xim.w);
        const float zrv[4] = {zre.x, zre.y, zre.z, zre.w}, ziv[4] = {zim.x, zim.y, zim.z, zim.w};
        // each accumulator's two FMAs in the order above, the second ones of
        // plane c - 1 after the first ones of plane c (independent work
        // between dependent FMAs)
#pragma unroll
        for (int c = 0; c <= 4; ++c) {
          if (c < 4) {
            const unsigned long long ZR = f2pack(zrv[c], zrv[c]), NZI = f2pack(-ziv[c], -ziv[c]);
            fma2(wr[c][0], i0, NZI);
            fma2(wi[c][0], i0, ZR);
            fma2(wr[c][1], i1, NZI);
            fma2(wi[c][1], i1, ZR);
          }
          if (c > 0) {
            const unsigned long long ZR = f2pack(zrv[c - 1], zrv[c - 1]), ZI = f2pack(ziv[c - 1], ziv[c - 1]);
            fma2(wr[c - 1][0], r0, ZR);
            fma2(wi[c - 1][0], r0, ZI);
            fma2(wr[c - 1][1], r1, ZR);
            fma2(wi[c - 1][1], r1, ZI);
          }
        }
      }
      if (pc == npc - 1 && chunk_cont_out(packed)) break;  // the run goes on in the next chunk
      // y of the 7 planes p2 the patch spans, (i, c) reading y[i + c] =
      // column oy0 - i - c: column oy0 is the first of its 4-column block,
      // oy0 - 4 .. oy0 - 1 the whole block before it, oy0 - 6 and oy0 - 5
      // the last two of the block before that
      const float *yr = ys + 2 * pc * it.Ly;
      float yre[7], yim[7];
      {
        const float4 b1r = *reinterpret_cast<const float4 *>(yr + 2 * (oy0 - 4));
        const float4 b1i = *reinterpret_cast<const float4 *>(yr + 2 * (oy0 - 4) + 4);
        const float2 b0r = *reinterpret_cast<const float2 *>(yr + 2 * (oy0 - 8) + 2);
        const float2 b0i = *reinterpret_cast<const float2 *>(yr + 2 * (oy0 - 8) + 6);
        yre[0] = yr[2 * oy0];
        yim[0] = yr[2 * oy0 + 4];
        yre[1] = b1r.w, yre[2] = b1r.z, yre[3] = b1r.y, yre[4] = b1r.x;
        yim[1] = b1i.w, yim[2] = b1i.z, yim[3] = b1i.y, yim[4] = b1i.x;
        yre[5] = b0r.y, yre[6] = b0r.x;
        yim[5] = b0i.y, yim[6] = b0i.x;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float r0, r1, i0, i1;
          f2unpack(wr[c][h], r0, r1);
          f2unpack(wi[c][h], i0, i1);
          sum[2 * h][c] += (double)fma(yre[2 * h + c], r0, -yim[2 * h + c] * i0);
          sum[2 * h + 1][c] += (double)fma(yre[2 * h + 1 + c], r1, -yim[2 * h + 1 + c] * i1);
        }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[s]));
  }
  if (!any) return;
  double *out = tri_out(a, it);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int cidx = tc[i * 32 + c];
      if (cidx >= 0) out[cidx] = sum[i][c];
    }
}

// D += A * B for one 8x8x4 FP64 tile on the tensor cores (mma.sync m8n8k4,
// the FP64 MMA of sm_80 and later; tcgen05 has no FP64 kind). Lane l holds
// a = A[l/4][l%4], b = B[l%4][l/4] and d0, d1 = D[l/4][2*(l%4)], D[l/4][2*(l%4)+1].
__device__ __forceinline__ void dmma884(double &d0, double &d1, double av, double bv) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(av), "d"(bv));
}

// The pieces of one staged chunk for a tile with NB blocks in use: per group
// of four triangles, x and z loads and four MMAs per block; at each run's
// end, sum += Re(y W) per combo. A run that goes on in the next chunk keeps
// its W (carried in wr/wi) and is multiplied by y there. Blocks NB..3 of a
// tile hold no combos and are skipped.
template <int NB>
__device__ __forceinline__ void dmma_pieces(const double2 *xs, const double2 *zs, const double2 *ys, int px, int pz,
                                            int Ly, int packed, const int (&ox)[4], const int (&oz)[4],
                                            const int (&oyb)[4], int t, double (&wr)[4][2], double (&wi)[4][2],
                                            double (&sum)[4][2]) {
  const int npc = chunk_npc(packed);
  int tt = 0;
  for (int pc = 0; pc < npc; ++pc) {
    const int len = chunk_len(packed, pc);
    if (pc != 0 || !chunk_cont_in(packed)) {
#pragma unroll
      for (int n = 0; n < NB; ++n) wr[n][0] = wr[n][1] = wi[n][0] = wi[n][1] = 0.0;
    }
    // one group of four triangles; only a piece's last group can be partial
    // (CHECK: its rows past the piece's end are zeroed)
    auto group = [&](int k0, auto check) {
      constexpr bool CHECK = decltype(check)::value;
      const bool on = !CHECK || k0 + t < len;
      const int row = tt + (on ? k0 + t : 0);
      double2 xv[NB], zv[NB];
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        xv[n] = xs[row * px + ox[n]];
        zv[n] = zs[row * pz + oz[n]];
        if (CHECK && !on) xv[n] = zv[n] = make_double2(0.0, 0.0);
      }
      // first the products of the real parts of x, then those of the
      // imaginary parts: each accumulator's two MMAs are 2 NB apart
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        dmma884(wr[n][0], wr[n][1], xv[n].x, zv[n].x);
        dmma884(wi[n][0], wi[n][1], xv[n].x, zv[n].y);
      }
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        dmma884(wr[n][0], wr[n][1], -xv[n].y, zv[n].y);
        dmma884(wi[n][0], wi[n][1], xv[n].y, zv[n].x);
      }
    };
    int k0 = 0;
    for (; k0 + 4 <= len; k0 += 4) group(k0, std::false_type{});
    if (k0 < len) group(k0, std::true_type{});
    tt += len;
    if (pc == npc - 1 && chunk_cont_out(packed)) break;  // the run goes on in the next chunk
    const double2 *yr = ys + pc * Ly;
#pragma unroll
    for (int n = 0; n < NB; ++n)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int o = oyb[n] - e;
        o = (unsigned)o < (unsigned)Ly ? o : 0;
        const double2 y = yr[o];
        sum[n][e] += fma(y.x, wr[n][e], -y.y * wi[n][e]);
      }
  }
}

// FP64 consumer on the FP64 tensor cores. The warp's tile is four blocks n of
// 8 planes p1 x 8 planes p3 (TriTile). Per group of four triangles of a
// piece, every block gets W_n += X_n Z_n^T in complex arithmetic as four real
// m8n8k4 MMAs (Wr += Xr Zr^T - Xi Zi^T, Wi += Xr Zi^T + Xi Zr^T). Lane l
// supplies x of plane p1_0[n] + l/4 and z of plane p3_0[n] + l/4 for triangle
// l%4 of the group (zero past the piece's end) and holds the W entries of
// combos (p1_0[n] + l/4, p3_0[n] + 2(l%4) + e), e < 2. At the end of the
// piece each such entry adds Re(y_k2(-p1-p3) * W) to its sum. Per group of
// four triangles a warp makes 8 128-bit shared loads for 4096 FMA.
__device__ __forceinline__ void tri_consume_dmma(const TriArgs &a, const TriItem &it, const double2 *stages,
                                                 uint64_t *full, uint64_t *empty, volatile int *s_fail,
                                                 const volatile int *s_packed, int warp, int lane, int nch) {
  static_assert(TRI_P1 == 8, "the DMMA consumer tiles 8 planes p1");
  const TriTile tl = a.tiles[it.tile0 + warp];
  const int nblk = tl.nblk;
  const int g = lane >> 2, t = lane & 3;
  const int px = stage_pitch(it.Lx, true), pz = stage_pitch(it.Lz, true);  // staged row pitches
  const int32_t *tc = a.tile_combo + (size_t)(it.tile0 + warp) * (TRI_P1 * 32) + g * 32 + 2 * t;
  // block n: x of plane p1_0[n] + g (inside the staged x row for every lane),
  // z of plane p3_0[n] + g; z of planes outside the staged p3 range and y of
  // combos outside the staged p2 range read column 0 instead (those combos'
  // sums are never stored)
  int ox[4], oz[4], oyb[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    ox[n] = tl.p1_0[n] + g + a.colbase - it.colx;
    const int o = tl.p3_0[n] + g + a.colbase - it.colz;
    oz[n] = (unsigned)o < (unsigned)it.Lz ? o : 0;
    oyb[n] = -(tl.p1_0[n] + g) - (tl.p3_0[n] + 2 * t) + a.colbase - it.coly;  // y of (n, e): oyb[n] - e
  }
  double sum[4][2], wr[4][2], wi[4][2];  // wr/wi: the current run's W, carried across chunks
#pragma unroll
  for (int n = 0; n < 4; ++n) sum[n][0] = sum[n][1] = wr[n][0] = wr[n][1] = wi[n][0] = wi[n][1] = 0.0;
  for (int c = 0; c < nch; ++c) {
    const int s = c % TRI_STAGES;
    if (!tri_wait_chunk(a, full, s_fail, c, lane)) return;
    const int packed = s_packed[s];  // piece layout of this chunk, written by the producer
    const double2 *xs = stages + s * a.stage;
    const double2 *zs = xs + TRI_CHUNK * px;
    const double2 *ys = zs + TRI_CHUNK * pz;
    switch (nblk) {  // warp-uniform: the tile's blocks in use
      case 1: dmma_pieces<1>(xs, zs, ys, px, pz, it.Ly, packed, ox, oz, oyb, t, wr, wi, sum); break;
      case 2: dmma_pieces<2>(xs, zs, ys, px, pz, it.Ly, packed, ox, oz, oyb, t, wr, wi, sum); break;
      case 3: dmma_pieces<3>(xs, zs, ys, px, pz, it.Ly, packed, ox, oz, oyb, t, wr, wi, sum); break;
      default: dmma_pieces<4>(xs, zs, ys, px, pz, it.Ly, packed, ox, oz, oyb, t, wr, wi, sum); break;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_addr(&empty[s]));
  }
  double *out = tri_out(a, it);
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int cidx = tc[8 * n + e];
      if (cidx >= 0) out[cidx] = sum[n][e];
    }
}

// Largest CTA of each instantiation (TRI_WARPS tiles plus the producer) and
// the CTAs per SM its register budget is sized for.
template <typename C>
struct TriBounds {
  static constexpr int threads = 32 * (TRI_WARPS + 1), blocks = 2;
};
template <>
struct TriBounds<float2> {
  static constexpr int threads = 32 * (fma_max_cons_warps() + 1), blocks = 3;
};

// Consumer warps of a CTA for an item of n tiles: one per tile on the FP64
// tensor cores and for the FP32 consumer of one or two tiles, one per pair of
// tiles for the packed FP32 consumer of more.
template <typename C>
__host__ __device__ inline int cons_warps(int n) {
  return std::is_same<C, double2>::value ? n : fma_cons_warps(n);
}

// One work item (its tiles over its chunks, realization a.real) on this CTA:
// warp `producer` streams the chunks into the stage ring, warps [0, ncons)
// consume them, any other warp takes no part. The caller has initialised the
// barriers (empty[] counting ncons arrivals).
template <typename C>
__device__ __forceinline__ void tri_run_item(const TriArgs &a, const TriItem &it, unsigned char *smem_raw,
                                             uint64_t *full, uint64_t *empty, volatile int *s_fail,
                                             volatile int *s_packed, int producer, int ncons) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  C *stages = reinterpret_cast<C *>(smem_raw);
  const C *S = static_cast<const C *>(a.S) + (size_t)a.real * a.s_stride;
  const int nch = it.ch1 - it.ch0;

  if (warp == producer) {
    // ------------------------------------------------------------ producer
    int issued = 0;
    bool failed = false;
    // chunk descriptors are read TRI_META_AHEAD chunks ahead of their copies
    // (they stream from DRAM: one chunk of lookahead left the ring waiting on them)
    const TriMeta none{0, 0u, 0};
    TriMeta m0 = nch > 0 ? tri_meta(a, it.ch0) : none, m1 = nch > 1 ? tri_meta(a, it.ch0 + 1) : none;
    TriMeta m2 = nch > 2 ? tri_meta(a, it.ch0 + 2) : none, m3 = nch > 3 ? tri_meta(a, it.ch0 + 3) : none;
    static_assert(TRI_META_AHEAD == 4, "the descriptor ring below holds four chunks");
    for (int c = 0; c < nch; ++c) {
      const int s = c % TRI_STAGES;
      if (c >= TRI_STAGES &&
          (*s_fail || !mbar_wait_bounded(smem_addr(&empty[s]), (uint32_t)(((c / TRI_STAGES) - 1) & 1)))) {
        failed = true;
        break;
      }
      const TriMeta cur = m0;
      m0 = m1;
      m1 = m2;
      m2 = m3;
      if (c + TRI_META_AHEAD < nch) m3 = tri_meta(a, it.ch0 + c + TRI_META_AHEAD);
      if (lane == 0) s_packed[s] = cur.packed;  // published by tri_issue's arrive on full[s]
      tri_issue<C>(a, it, S, stages + s * a.stage, smem_addr(&full[s]), cur);
      issued = c + 1;
    }
    if (failed) {
      *s_fail = 1;
      if (lane == 0) atomicOr(a.status, DEV_TIMEOUT);
      // let the copies in flight (the last TRI_STAGES issued) land before the
      // CTA's shared memory can be released or restaged
      for (int c = issued - TRI_STAGES > 0 ? issued - TRI_STAGES : 0; c < issued; ++c)
        mbar_wait_bounded(smem_addr(&full[c % TRI_STAGES]), (uint32_t)((c / TRI_STAGES) & 1));
    }
    return;
  }
  if (warp >= ncons) return;

  // -------------------------------------------------------------- consumer
  if constexpr (std::is_same<C, double2>::value)
    tri_consume_dmma(a, it, stages, full, empty, s_fail, s_packed, warp, lane, nch);
  else if (!fma_pairs_tiles(it.ntiles))
    tri_consume_fma_tile<C>(a, it, stages, full, empty, s_fail, s_packed, warp, lane, nch);
  else
    tri_consume_fma<C>(a, it, stages, full, empty, s_fail, s_packed, warp, lane, nch);
}

// One CTA per item of one tile class (blockIdx.x) and realization (blockIdx.y);
// the CTA has cons_warps(n) consumer warps and the producer warp last.
template <typename C>
__global__ void __launch_bounds__(TriBounds<C>::threads, TriBounds<C>::blocks) k_triangle(TriArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[TRI_STAGES], empty[TRI_STAGES];
  __shared__ volatile int s_fail;
  __shared__ volatile int s_packed[TRI_STAGES];
  const TriItem it = a.items[blockIdx.x];
  const int tid = threadIdx.x;
  const int ncons = (blockDim.x >> 5) - 1;  // consumer warps (cons_warps); warp ncons produces
  if (tid == 0) {
    for (int s = 0; s < TRI_STAGES; ++s) {
      mbar_init(smem_addr(&full[s]), 1);
      mbar_init(smem_addr(&empty[s]), ncons);
    }
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  TriArgs b = a;
  b.real = blockIdx.y;
  tri_run_item<C>(b, it, smem_raw, full, empty, &s_fail, s_packed, ncons, ncons);
}

// Persistent form: every item of every tile class and every realization in one
// launch. A CTA (the largest class's shape: its consumer warps plus the
// producer warp last) takes work units from a device counter -- unit w is
// item order[w / nreal] (items in decreasing order of work) for realization
// w % nreal -- sets its barriers up for the unit's consumer count, sums it and
// takes the next, until the units run out. The counter must be zero at launch.
template <typename C>
__global__ void __launch_bounds__(TriBounds<C>::threads, TriBounds<C>::blocks)
    k_triangle_q(TriArgs a, const int32_t *__restrict__ order, int n_units, int *counter) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t full[TRI_STAGES], empty[TRI_STAGES];
  __shared__ volatile int s_fail;
  __shared__ volatile int s_packed[TRI_STAGES];
  __shared__ int s_unit;
  const int tid = threadIdx.x;
  const int producer = (blockDim.x >> 5) - 1;
  if (tid == 0) s_fail = 0;
  bool inited = false;
  for (;;) {
    if (tid == 0) s_unit = atomicAdd(counter, 1);
    __syncthreads();  // every warp is done with the previous unit
    const int w = s_unit;
    if (w >= n_units || s_fail) break;
    const TriItem it = a.items[order[w / a.nreal]];
    const int ncons = cons_warps<C>(it.ntiles);
    if (tid == 0) {
      for (int s = 0; s < TRI_STAGES; ++s) {
        if (inited) {
          mbar_inval(smem_addr(&full[s]));
          mbar_inval(smem_addr(&empty[s]));
        }
        mbar_init(smem_addr(&full[s]), 1);
        mbar_init(smem_addr(&empty[s]), ncons);
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    inited = true;
    __syncthreads();  // barriers ready; s_unit read by every thread
    TriArgs b = a;
    b.real = w % a.nreal;
    b.stage = a.stage_of[it.ntiles];
    tri_run_item<C>(b, it, smem_raw, full, empty, &s_fail, s_packed, producer, ncons);
  }
}

// Sum the splits of each combo in split order, scale by NN^2 and store the
// triangle's B at its bin-order position; realization blockIdx.y.
__global__ void k_reduce(long long n_combo, const int32_t *__restrict__ combo_u, const int32_t *__restrict__ u_cfirst,
                         const int32_t *__restrict__ u_ncombo, const int32_t *__restrict__ u_nsplit,
                         const long long *__restrict__ u_part, const int32_t *__restrict__ combo_out,
                         const double *__restrict__ part, long long part_stride, double nn2,
                         double *__restrict__ B, long long b_stride) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_combo) return;
  part += (long long)blockIdx.y * part_stride;
  B += (long long)blockIdx.y * b_stride;
  int u = combo_u[c];
  int nc = u_ncombo[u], ns = u_nsplit[u];
  const double *p = part + u_part[u] + (c - u_cfirst[u]);
  double s = 0.0;
  for (int k = 0; k < ns; ++k) s += p[(long long)k * nc];
  B[combo_out[c]] = nn2 * s;
}

template <typename C>
static size_t tri_smem(int stage, int ntiles) {
  (void)ntiles;
  return (size_t)TRI_STAGES * stage * sizeof(C);
}

// Allow both instantiations the device's opt-in shared memory (less their
// static barriers) once per context; each launch still asks only for its
// class's stages.
template <typename C>
static int allow_optin(size_t smem_optin) {
  cudaFuncAttributes fa;
  BEAM_CUDA(cudaFuncGetAttributes(&fa, k_triangle<C>));
  int dyn = (int)(smem_optin > fa.sharedSizeBytes ? smem_optin - fa.sharedSizeBytes : 0);
  BEAM_CUDA(cudaFuncSetAttribute(k_triangle<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  BEAM_CUDA(cudaFuncGetAttributes(&fa, k_triangle_q<C>));
  dyn = (int)(smem_optin > fa.sharedSizeBytes ? smem_optin - fa.sharedSizeBytes : 0);
  BEAM_CUDA(cudaFuncSetAttribute(k_triangle_q<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  return BEAM_OK;
}

int triangle_init_attributes(size_t smem_optin) {
  BEAM_TRY(allow_optin<double2>(smem_optin));
  BEAM_TRY(allow_optin<float2>(smem_optin));
  BEAM_TRY(triangle_i8_init_attributes(smem_optin));
  return BEAM_OK;
}

// One launch per tile count n (CTAs of cons_warps(n) consumer warps + 1 producer warp), on
// side streams forked from and joined back into the slot's stream, so the
// launches overlap. Each launch covers its class's items for all realizations
// (blockIdx.y).
template <typename C>
static int launch_classes(beam_gpu_plan *p, RunSlot *s, TriArgs a) {
  DevPlan &d = p->d;
  Lane *ln = s->lane;
  BEAM_CUDA(cudaEventRecord(ln->fork, ln->stream));
  for (int n = TRI_WARPS; n >= 1; --n) {
    int first = d.class_first[n], count = d.class_first[n + 1] - first;
    if (count == 0) continue;
    cudaStream_t st = ln->side[n - 1];
    BEAM_CUDA(cudaStreamWaitEvent(st, ln->fork, 0));
    TriArgs b = a;
    b.items = d.items + first;
    b.stage = d.class_stage[n];
    k_triangle<C><<<dim3((unsigned)count, (unsigned)a.nreal), 32 * (cons_warps<C>(n) + 1), tri_smem<C>(b.stage, n),
                    st>>>(b);
    BEAM_CUDA(cudaGetLastError());
    s->launches++;
    BEAM_CUDA(cudaEventRecord(ln->join[n - 1], st));
    BEAM_CUDA(cudaStreamWaitEvent(ln->stream, ln->join[n - 1], 0));
  }
  return BEAM_OK;
}

// All classes and realizations in one launch of the persistent kernel on the
// slot's stream: the work counter is zeroed first (a memset node in a
// captured graph), then as many CTAs as fit the device at once take units.
template <typename C>
static int launch_persistent(beam_gpu_plan *p, RunSlot *s, TriArgs a) {
  DevPlan &d = p->d;
  cudaStream_t st = s->lane->stream;
  int max_stage = 0;
  for (int n = 1; n <= TRI_WARPS; ++n) {
    a.stage_of[n] = d.class_stage[n];
    max_stage = std::max(max_stage, d.class_stage[n]);
  }
  a.stage_of[0] = 0;
  const size_t smem = tri_smem<C>(max_stage, TRI_WARPS);
  const int threads = TriBounds<C>::threads;
  int per_sm = 0;
  BEAM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_triangle_q<C>, threads, smem));
  if (per_sm < 1) {
    set_detail("the persistent triangle kernel does not fit an SM");
    return BEAM_EINVAL;
  }
  const long long units = (long long)d.n_items * a.nreal;
  if (units > 0x7fffffffLL) {
    set_detail("too many triangle-sum work units for one persistent launch");
    return BEAM_EINVAL;
  }
  const int grid = (int)std::min<long long>(units, (long long)per_sm * std::max(1, p->ctx->num_sms));
  int *counter = s->status + 1;
  BEAM_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
  k_triangle_q<C><<<grid, threads, smem, st>>>(a, d.q_order, (int)units, counter);
  BEAM_CUDA(cudaGetLastError());
  s->launches++;
  return BEAM_OK;
}

int run_triangle_sums(beam_gpu_plan *p, RunSlot *s, int n) {
  DevPlan &d = p->d;
  if (d.n_combo == 0) {
    for (int k = 1; k <= 3; ++k) mark(s, k);
    return BEAM_OK;
  }
  TriArgs a;
  a.items = d.items;
  a.tiles = d.tiles;
  a.tile_combo = d.tile_combo;
  a.descs = d.descs;
  a.S = s->S;
  a.W = d.W;
  a.colbase = d.colbase;
  a.u_cfirst = d.u_cfirst;
  a.u_ncombo = d.u_ncombo;
  a.u_part = d.u_part;
  a.part = s->part;
  a.status = s->status;
  a.stage = 0;
  a.nreal = n;
  a.real = 0;
  for (int k = 0; k <= TRI_WARPS; ++k) a.stage_of[k] = 0;
  a.s_stride = (long long)d.n_modes * d.W;
  a.part_stride = d.n_part;
  mark(s, 1);
  const bool persistent = p->tri_launch == BEAM_LAUNCH_PERSISTENT;
  if (d.i8)
    BEAM_TRY(launch_triangle_i8(p, s, n));
  else if (d.elem == sizeof(double2))
    BEAM_TRY(persistent ? launch_persistent<double2>(p, s, a) : launch_classes<double2>(p, s, a));
  else
    BEAM_TRY(persistent ? launch_persistent<float2>(p, s, a) : launch_classes<float2>(p, s, a));
  mark(s, 2);
  double nn2 = (double)p->geom.NN * (double)p->geom.NN;
  dim3 grid((unsigned)((d.n_combo + 255) / 256), (unsigned)n);
  k_reduce<<<grid, 256, 0, s->lane->stream>>>(d.n_combo, d.combo_u, d.u_cfirst, d.u_ncombo, d.u_nsplit, d.u_part,
                                              d.combo_out, s->part, d.n_part, nn2, s->B, d.n_combo);
  BEAM_CUDA(cudaGetLastError());
  s->launches++;
  mark(s, 3);
  return BEAM_OK;
}

}  // namespace beam
