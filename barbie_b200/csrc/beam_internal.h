// Internal declarations shared by the libbeam_gpu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <exception>
#include <map>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "beam_gpu.h"
#include "geometry.h"

namespace beam {

struct PixelPath;  // FFT-path state (beam_fft.cu)

// Thread-local detail text for the last failure (beam_gpu_last_error_detail).
void set_detail(const std::string &s);

// Host-side C++ failures (allocation, thread start) as an error code, so no
// exception leaves a C entry point.
template <typename F>
int host_guard(F &&f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    set_detail("host memory allocation failed");
    return BEAM_ENOMEM;
  } catch (const std::exception &e) {
    set_detail(std::string("host: ") + e.what());
    return BEAM_ENOMEM;
  }
}

// fn(k) for k = 0 .. n-1 on up to n - 1 extra host threads. k = 0, and every k
// whose thread could not be started, run on the calling thread, so a failed
// thread start costs time, not an exception.
template <typename F>
void host_parallel(int n, const F &fn) {
  std::vector<std::thread> th;
  int started = 1;
  try {
    th.reserve(n > 1 ? n - 1 : 0);
    for (; started < n; ++started) th.emplace_back(fn, started);
  } catch (...) {
  }
  fn(0);
  for (int k = started; k < n; ++k) fn(k);
  for (std::thread &t : th) t.join();
}

// Evaluate a CUDA runtime call; on failure record the detail and return BEAM_ECUDA
// (or BEAM_EDEVMEM for allocation failures) from the enclosing function.
#define BEAM_CUDA(call)                                                        \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ::beam::set_detail(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return e_ == cudaErrorMemoryAllocation ? BEAM_EDEVMEM : BEAM_ECUDA;      \
    }                                                                          \
  } while (0)

#define BEAM_TRY(expr)              \
  do {                              \
    int rc_ = (expr);               \
    if (rc_ != BEAM_OK) return rc_; \
  } while (0)

// Device-side status word written by kernels whose waits are bounded.
enum : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_BAD_INDEX = 2 };

// Triangle-sum decomposition. Of each ring triplet's three legs, leg 1 (ring
// r1, plane p1 >= 0) is the "x" leg; of the other two, the plan makes the one
// whose modes repeat most in the in-plane list the run leg "y" (below: ring
// r2, plane p2 = -p1-p3) and the other the tile leg "z" (ring r3, plane p3).
// Each warp owns a tile of TRI_P1 planes p1 x 32 planes p3 (one p3 per lane)
// of one ring triplet's accepted (p1, p2) "combos"; a CTA holds up to
// TRI_WARPS tiles of the same triplet. The triplet's in-plane triangles are
// listed y-major, so consecutive triangles sharing the y mode form a run;
// runs are packed into chunks of at most TRI_CHUNK triangles and TRI_PIECES
// pieces (a run's part within one chunk), one pipeline stage each, a run
// longer than a chunk's room going on in the next chunk.
constexpr int TRI_WARPS = 7;   // most tiles per CTA (one consumer warp each, plus one producer warp)
constexpr int TRI_CLASSES = 12;  // most tiles per CTA on any path (int8: I8_MAX_TILES)
constexpr int TRI_P1 = 8;      // planes p1 per thread
constexpr int TRI_CHUNK = 16;  // in-plane triangles per stage
constexpr int TRI_PIECES = 4;  // pieces per stage
constexpr int TRI_STAGES = 3;  // pipeline depth
constexpr int TRI_META_AHEAD = 4;  // chunks whose descriptors the producer has in flight ahead of their copies
constexpr int TRI_PAD = 8;     // zero columns on each side of a mode row (>= TRI_P1 - 1)

// A warp's tile: TRI_BLOCKS blocks of TRI_P1 planes p1 x TRI_BW planes p3 of
// one ring triplet; tile column TRI_BW * n + c is plane p3_0[n] + c, tile row
// a of block n plane p1_0[n] + a.
constexpr int TRI_BW = 8, TRI_BLOCKS = 32 / TRI_BW;
struct TriTile {
  int p1_0[TRI_BLOCKS], p3_0[TRI_BLOCKS];
  int nblk;  // blocks in use (1..TRI_BLOCKS); the rest repeat block 0 and hold no combos
};

struct TriChunk {
  long long t0;  // first in-plane triangle (global list index)
  int pc0;       // first piece in the global piece table
  int packed;    // nt (bits 0-4), npc (bits 5-7), piece lengths (5 bits each from bit 8)
};
// fields of TriChunk::packed / TriDesc::packed. A run longer than the room
// left in a chunk continues in the next chunk: the chunk's last piece is then
// marked CONT_OUT (its outer product is carried, not yet multiplied by the run
// leg) and the next chunk's first piece CONT_IN (it adds to the carried one).
constexpr int CHUNK_CONT_IN = 1 << 28, CHUNK_CONT_OUT = 1 << 29;
__host__ __device__ inline int chunk_nt(int packed) { return packed & 31; }
__host__ __device__ inline int chunk_npc(int packed) { return (packed >> 5) & 7; }
__host__ __device__ inline int chunk_len(int packed, int piece) { return (packed >> (8 + 5 * piece)) & 31; }
__host__ __device__ inline bool chunk_cont_in(int packed) { return (packed & CHUNK_CONT_IN) != 0; }
__host__ __device__ inline bool chunk_cont_out(int packed) { return (packed & CHUNK_CONT_OUT) != 0; }
__host__ __device__ inline int chunk_pack(int nt, int npc, int lens, int flags = 0) {
  return nt | (npc << 5) | (lens << 8) | flags;
}

// What the kernel reads per chunk: the layout and, for each triangle and
// piece, the row (mode index within its ring) to stage -- one independent
// load per producer lane.
struct TriDesc {
  uint16_t xz[TRI_CHUNK][2];  // triangle j: k1 (ring r1) and k3 (ring r3)
  uint16_t y[TRI_PIECES];     // piece j: k2 (ring r2)
  int packed;                 // as TriChunk::packed
  int pad;
};
static_assert(sizeof(TriDesc) % 16 == 0 && TRI_CHUNK <= 31 && TRI_PIECES <= 4, "TriDesc layout");
constexpr int TRI_TAU_MAX = 512;  // first cap on the in-plane triangles one CTA walks (mixed; FP64 twice)

// The mixed path's mode rows are blocked by 4 columns: block b of a row holds
// the real parts of columns 4b..4b+3, then their imaginary parts (8 floats).
// Float offset of the real part of column col within its row; the imaginary
// part is 4 floats further.
__host__ __device__ inline int mixed_re(int col) { return ((col >> 2) << 3) | (col & 3); }

// Shared-memory pitch (complex values) of a staged x or z row of L values.
// The FP64 consumer reads a quarter-warp's 8 lanes as 2 planes x 4 rows with
// 16-byte loads; rows 2 (mod 8) 16-byte units apart put those 8 lanes on
// distinct banks. The mixed-precision consumer reads rows as staged.
__host__ __device__ inline int stage_pitch(int L, bool fp64) { return fp64 ? L + ((2 - L) & 7) : L; }

// One CTA of triangle-sum work: tiles [tile0, tile0 + ntiles) of ring triplet u
// over chunks [ch0, ch1) (the triplet's split `split`). Rows staged per chunk
// are columns [colx, colx+Lx) of ring r1's mode rows (one per triangle),
// [colz, colz+Lz) of ring r3's (one per triangle) and [coly, coly+Ly) of ring
// r2's (one per piece); the column of plane q is q + Q - 1.
struct TriItem {
  int u, split;
  int ch0, ch1;
  int tile0, ntiles;
  int m1, m2, m3;  // first mode of rings r1, r2, r3 in the mode table
  int colx, Lx, colz, Lz, coly, Ly;
  int rx, rz;      // rings of the x leg (r1) and the tile leg (r3): their slice scales (int8 path)
};

// The int8 path (BEAM_PREC_INT8). Every mode value v of ring r on the plane of
// column c is cut into five 8-bit slices against the scale 2^e(r, c) >
// max |Re|, |Im| over the ring's modes there:
//   v = 2^(e - 7) (a0 + a1 2^-8 + a2 2^-16 + a3 2^-24 + a4 2^-32 + d), 0 <= d < 2^-32,
// a0 = floor(v 2^(7-e)) in [-128, 127] (signed), a1..a4 in [0, 255] (unsigned).
// A run's outer product W(p1, p3) = sum x(p1) z(p3) is then
//   2^(ex + ez - 14) sum_L 2^(-8L) acc_L,  acc_L = sum over slice pairs i + j = L < I8_LEVELS,
// each acc_L an exact int32 sum of 8-bit products on the tensor cores. A
// warp's tile is one window of I8_BW planes p3 (the MMA's 16 rows, z leg) x
// up to two blocks of 8 planes p1 (its 8 columns each, x leg); a CTA's group
// is I8_GROUP_WINDOWS windows x up to TRI_WARPS p1 blocks (at most
// I8_MAX_TILES tiles); a chunk is 16
// triangles of one run (the MMA's K = 32: 16 triangles x real, imaginary).
// Slice rows: per mode, the x table (I8_XW words per column: slice s as the
// bytes (Re, -Im, Im, Re)) and the z table (I8_ZW words per column: slices
// (0,1), (2,3), (4) as (Re, Im) byte pairs), each column-interleaved so a
// row segment is one copy.
#ifndef BEAM_I8_NBT
#define BEAM_I8_NBT 2
#endif
#ifndef BEAM_I8_MAX_TILES
#define BEAM_I8_MAX_TILES 5
#endif
#ifndef BEAM_I8_STAGES
#define BEAM_I8_STAGES 3
#endif
#ifndef BEAM_I8_MINB
#define BEAM_I8_MINB 2
#endif
constexpr int I8_BW = 16;        // planes p3 per tile window
constexpr int I8_NBT = BEAM_I8_NBT;              // p1 blocks per tile
constexpr int I8_MAX_TILES = BEAM_I8_MAX_TILES;  // tiles per CTA (2 CTAs of 6 warps per SM at 168 registers)
#ifndef BEAM_I8_GROUP_WINDOWS
#define BEAM_I8_GROUP_WINDOWS 2
#endif
constexpr int I8_GROUP_WINDOWS = BEAM_I8_GROUP_WINDOWS;  // windows of a CTA's group
constexpr int I8_STAGES = BEAM_I8_STAGES;        // pipeline depth
constexpr int I8_MINB = BEAM_I8_MINB;            // CTAs per SM the register budget is sized for
constexpr int I8_SLICES = 5;
#ifndef BEAM_I8_LEVELS
#define BEAM_I8_LEVELS 6
#endif
constexpr int I8_LEVELS = BEAM_I8_LEVELS;  // slice pairs i + j < I8_LEVELS are summed (6: the 19 pairs up to i + j = 5)
constexpr int I8_XW = 5;         // x table words per column
constexpr int I8_ZW = 3;         // z table words per column
constexpr int I8_RUN_MAX = 2048; // longest run summed in int32 (|acc| < 2048 x 2 x 5 x 255^2 < 2^31)

// int8 path staging. A chunk's stage holds, per triangle, the x leg's table
// segment (Lx columns x I8_XW words) and the z leg's (Lz x I8_ZW), then the
// run leg's FP64 row (Ly columns). Triangle rows are i8_pitch(words) apart:
// rounded up to 4 (mod 8), so the 32 lanes' words (column g, triangle rows 2t)
// fall on 32 distinct banks for both 5- and 3-word columns.
__host__ __device__ inline int i8_pitch(int words) { return words + ((12 - (words & 7)) & 7); }
__host__ __device__ inline int i8_stage_bytes(const TriItem &it) {
  return TRI_CHUNK * (i8_pitch(I8_XW * it.Lx) + i8_pitch(I8_ZW * it.Lz)) * 4 + it.Ly * 16;
}

// Device-side tables of a plan (read-only while it runs; per-run buffers live
// in RunSlot).
struct DevPlan {
  // ring modes on the planes in use
  // A mode's row holds planes q = -(Q-1)..Q-1 at columns colbase + q, with
  // TRI_PAD zero columns on either side (reads of neighbouring planes by
  // threads whose combos are not accepted stay inside the row).
  int n_modes = 0, Q = 0, W = 0, colbase = 0;
  int16_t *mode_ij = nullptr;     // [n_modes][2] grid indices (i, j)
  int32_t *mode_neg = nullptr;    // [n_modes] mode at -k
  int16_t *ringmap = nullptr;     // [NN*NN] ring of each pixel or -1
  int16_t *pixlocal = nullptr;    // [NN*NN] index of the pixel within its ring's mode list
  // in-plane triangle lists of the used ring triplets
  long long n_terms = 0;
  ushort4 *tri_list = nullptr;    // [n_terms] local mode indices (i1, i2, i3) in rings r1, r2, r3
  // accepted triangles grouped by ring triplet ("combos": plane pairs p1, p2)
  int n_used = 0;
  long long n_combo = 0;
  int32_t *combo_u = nullptr;     // [n_combo] used ring triplet
  int32_t *combo_out = nullptr;   // [n_combo] bin-order position of the triangle
  int32_t *u_cfirst = nullptr;    // [n_used] first combo
  int32_t *u_ncombo = nullptr;    // [n_used]
  int32_t *u_nsplit = nullptr;    // [n_used] triangle-range splits
  long long *u_part = nullptr;    // [n_used] first partial-sum slot (split-major)
  int n_tiles = 0;
  TriTile *tiles = nullptr;       // [n_tiles]
  int32_t *tile_combo = nullptr;  // [n_tiles][TRI_P1][32] combo id or -1
  long long n_chunks = 0, n_pieces = 0;
  TriChunk *chunks = nullptr;     // plan construction only
  int2 *pieces = nullptr;         // (triangles, k2 local index of the run's r2 mode)
  TriDesc *descs = nullptr;       // [n_chunks], read by the kernel
  int n_items = 0;
  TriItem *items = nullptr;       // [n_items]: grouped by tile count, largest work first in a group
  int32_t *q_order = nullptr;     // [n_items] items in decreasing order of work (persistent kernel)
  int class_first[TRI_CLASSES + 2] = {};  // items with n tiles: [class_first[n], class_first[n+1])
  int class_stage[TRI_CLASSES + 1] = {};  // stage size (complex values; int8: bytes) of the CTAs with n tiles
  long long n_part = 0;           // partial-sum slots per realization
  size_t elem = 0;                // bytes of one complex mode value (16 FP64, 8 mixed, 48 int8: FP64 + slices)
  int i8 = 0;                     // int8 path: S holds FP64 rows, slice rows, then ring scales
  int n_rings = 0;
  int32_t *ring_first = nullptr;  // [n_rings + 1] first mode of each ring (int8 path)
  // epilogue (bin order)
  int n_bins = 0;
  int32_t *bin_first = nullptr;   // [n_bins+1]
  double *ep_px = nullptr, *ep_pz = nullptr;  // [n_combo]
  double *ep_ana = nullptr;       // [n_combo] analytic bispectrum of the triangle
  int32_t *ep_cnt = nullptr;      // [n_combo] exact in-plane triangle count
  int n_epchunks = 0;             // bins cut into chunks of at most EP_CHUNK triangles
  int32_t *ep_chunk_first = nullptr;  // [n_epchunks+1] triangle ranges (bin order)
  int32_t *bin_chunk = nullptr;   // [n_bins+1] chunk ranges per bin
};
constexpr int EP_CHUNK = 1024;  // most triangles per epilogue CTA

// Bytes of one realization's mode data. The int8 path keeps, after the FP64
// rows (the run leg's values), the x and z slice tables (I8_XW and I8_ZW
// words per mode and column) and the scale exponents e(r, c) (int32 [n_rings][W]).
inline size_t i8_fp64_bytes(const DevPlan &d) { return (size_t)d.n_modes * d.W * 16; }
inline size_t i8_xtab_bytes(const DevPlan &d) { return (size_t)d.n_modes * d.W * I8_XW * 4; }
inline size_t i8_slice_bytes(const DevPlan &d) { return (size_t)d.n_modes * d.W * (I8_XW + I8_ZW) * 4; }
inline size_t mode_data_bytes(const DevPlan &d) {
  if (!d.i8) return d.elem * (size_t)d.n_modes * d.W;
  return i8_fp64_bytes(d) + i8_slice_bytes(d) + (((size_t)d.n_rings * d.W * 4 + 255) & ~(size_t)255);
}
// sections of a realization's bin array: sum B*bs, sum Num*norm, bs/(vol*norm),
// sum Biana*Num*bs (each [n_bins][16])
constexpr int BIN_SECTIONS = 4;

// A stream plus the side streams the per-class triangle-sum launches fork onto.
struct Lane {
  cudaStream_t stream = nullptr;
  cudaStream_t side[TRI_CLASSES] = {};
  cudaEvent_t fork = nullptr, join[TRI_CLASSES] = {};
};
// priority: the streams' CUDA priority (0 = default; lower is more urgent)
int lane_create(Lane *l, int priority = 0);
void lane_destroy(Lane *l);

// Per-run buffers for up to `cap` realizations of one plan, processed together
// (realization r of a launch is its blockIdx.y). The plan's own slot (cap 1)
// serves beam_gpu_run; batches and the job server create more. All device
// buffers are realization-major.
struct RunSlot {
  int cap = 0;
  Lane *lane = nullptr;           // where the slot's work is queued
  Lane own;                       // used when the slot has a lane of its own
  double *staging = nullptr;      // [cap][n_modes][Q] complex128 rows of the r2c buffers
  const double **src = nullptr;   // [2*cap] device: staged rows per realization, then device r2c buffers
  const double **h_src = nullptr; // [2*cap] pinned mirror of src
  void *S = nullptr;              // [cap][n_modes][W] complex mode data (double2 or float2)
  double *part = nullptr;         // [cap][n_part] partial sums (zero where never written)
  double *B = nullptr;            // [cap][n_combo] triangle sums, bin order
  double *bins = nullptr;         // [cap][BIN_SECTIONS][n_bins][16]: bs, norm, out, analytic sum
  long long *bin_count = nullptr; // [cap][n_bins]
  double *ep_part = nullptr;      // [cap][n_epchunks][33] epilogue chunk sums
  int *status = nullptr;          // device status word, then the persistent triangle kernel's work counter
  double *h_staging = nullptr;    // pinned [cap][n_modes][Q]
  double *h_bins = nullptr;       // pinned [cap][BIN_SECTIONS][n_bins][16]
  long long *h_count = nullptr;   // pinned [cap][n_bins]
  int *h_status = nullptr;        // pinned status copy
  cudaEvent_t ev[5] = {};         // stage boundaries (beam_gpu_plan_last_timings)
  cudaEvent_t done = nullptr;     // end of the last queued run
  bool timed = false;
  bool capturing = false;         // inside slot_run_graph's stream capture (no stage marks)
  int launches = 0;               // kernels launched by the last queued run
  cudaGraphExec_t graph = nullptr;  // captured host-input run of graph_n realizations
  int graph_n = 0;
  size_t bytes = 0;               // device bytes of the slot
};

}  // namespace beam

struct beam_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;  // == lane.stream
  int num_sms = 0;
  size_t smem_optin = 0;
  beam::Lane lane;
  // field generator / ingestion workspace (twiddles, row sums, variance), kept
  // between calls; launches of the last field call
  void *field_ws = nullptr;
  size_t field_ws_bytes = 0;
  int field_launches = 0;
  // FFT staging tiles (complex values) chosen by beam_gpu_field_autotune per
  // NN: {column passes, row passes}
  std::map<long, std::pair<int, int>> field_tiles;
  // small per-context scratch (power-multipole partial sums), kept between calls
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  // power multipoles: the geometry of the last (NN, Nbin) -- per visited mode
  // class its Legendre weights and bin (beam_pk.cu) and the per-bin sums that
  // do not depend on the field -- kept for the next call with the same sizes
  void *pk_tab = nullptr;
  size_t pk_tab_bytes = 0;
  long pk_NN = 0;
  int pk_Nbin = 0;
  std::vector<double> pk_geo;
};

struct beam_gpu_plan {
  beam_gpu_ctx *ctx = nullptr;
  beam_cfg cfg{};
  beam_geom geom{};
  beam::DevPlan d;
  // host mirrors
  std::vector<int> used_rp;              // used ring triplet -> rp
  std::vector<long long> tri_first;      // [n_used+1] triangle-list ranges
  std::vector<int32_t> ring_first;       // [Nr+1] mode ranges per ring (empty for unused rings)
  std::vector<int16_t> mode_ij;          // [n_modes][2]
  std::vector<int32_t> bin_pos;          // [ntri] loop order -> bin order
  std::vector<int32_t> loop_of_bin;      // [ntri] bin order -> loop order
  std::vector<int> u_owner;              // [n_used] shard that sums each used ring triplet
  size_t device_bytes = 0;               // tables (slots count separately)
  beam::PixelPath *pix = nullptr;        // plane-ring transform tables / pixel method
  beam::RunSlot *main = nullptr;         // slot of beam_gpu_run and friends (ctx->lane)
  beam::RunSlot *batch[2] = {};          // double-buffered slots of beam_gpu_run_batch
  // triangle-sum work decomposition (build_work): first cap on the in-plane
  // triangles one CTA walks (split-K over the triangle list), and the number
  // of items' worth of work per SM the load balance aims at; set by
  // beam_gpu_plan_autotune
  long long tau0 = beam::TRI_TAU_MAX;
  double balance = 8.0;
  long long n_run_combos = 0;  // sum over owned triplets of runs x combos (beam_plan_info.n_run_combos)
  float build_ms[5] = {};      // creation phases (beam_plan_info.build_ms)
  int tri_launch = BEAM_LAUNCH_CLASSES;  // how the triangle sums are launched (BEAM_LAUNCH_*)
};

namespace beam {
// stage boundary k of the slot's current run, on its stream
inline void mark(RunSlot *s, int k) {
  if (s->ev[k] && !s->capturing) cudaEventRecord(s->ev[k], s->lane->stream);
}
// plan construction (beam_plan.cu)
int build_plan_tables(beam_gpu_plan *p);
void free_plan_tables(beam_gpu_plan *p);
int count_closed_triangles(beam_gpu_plan *p, std::vector<long long> &counts);
// run slots (beam_run.cu); lane == nullptr gives the slot a lane of its own
size_t slot_bytes(const beam_gpu_plan *p, int cap);
int slot_create(beam_gpu_plan *p, int cap, Lane *lane, RunSlot **out, int priority = 0);
void slot_destroy(RunSlot *s);
// per-realization steps on a slot, for realizations [0, n) (beam_run.cu)
void gather_host(const beam_gpu_plan *p, RunSlot *s, int r, const double *r2c, int m0 = 0, int m1 = -1);
int upload_modes(beam_gpu_plan *p, RunSlot *s, int n, bool staged, bool staged_on_device = false);
int gather_mapped(beam_gpu_plan *p, RunSlot *s, const double *r2c_mapped);
int run_triangle_sums(beam_gpu_plan *p, RunSlot *s, int n);
// int8 path: slice tables of realizations [0, n) from their FP64 rows (beam_run.cu); the
// triangle sums (beam_tri_i8.cu)
int build_slices(beam_gpu_plan *p, RunSlot *s, int n);
int launch_triangle_i8(beam_gpu_plan *p, RunSlot *s, int nreal);
int triangle_i8_init_attributes(size_t smem_optin);
int run_epilogue(beam_gpu_plan *p, RunSlot *s, int n);
int fetch_results(beam_gpu_plan *p, RunSlot *s, int n);
int check_status(RunSlot *s);
// the context's scratch buffer, grown to at least bytes (contents undefined)
int ctx_scratch(beam_gpu_ctx *ctx, size_t bytes, void **out);
// a fixed pseudo-random pattern in [-1, 1) over n doubles (autotuning inputs)
int fill_pattern(double *v, size_t n, cudaStream_t st, int num_sms);
int slot_run_graph(beam_gpu_plan *p, RunSlot *s, int n);
int copy_result(const beam_gpu_plan *p, const RunSlot *s, int r, beam_result *res);
template <typename T>
int dev_alloc(size_t *total, T **ptr, size_t count) {
  size_t bytes = sizeof(T) * (count ? count : 1);
  cudaError_t e = cudaMalloc((void **)ptr, bytes);
  if (e != cudaSuccess) {
    set_detail(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    return BEAM_EDEVMEM;
  }
  *total += bytes;
  return BEAM_OK;
}
template <typename T>
int dev_alloc(beam_gpu_plan *p, T **ptr, size_t count) {
  return dev_alloc(&p->device_bytes, ptr, count);
}
}  // namespace beam
