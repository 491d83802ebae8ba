// Internal declarations shared by the libbeam_gpu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "beam_gpu.h"
#include "geometry.h"

namespace beam {

struct PixelPath;  // FFT-path state (beam_fft.cu)

// Thread-local detail text for the last failure (beam_gpu_last_error_detail).
void set_detail(const std::string &s);

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

// Threads per triangle-sum CTA and in-plane triangles staged per pipeline stage.
// Triangle-sum decomposition. Each warp owns a tile of TRI_P1 planes p1 x 32
// planes p3 (one p3 per lane, p2 = -p1-p3) of one ring triplet's accepted
// (p1, p2) "combos"; a CTA holds up to TRI_WARPS tiles of the same triplet.
// The triplet's in-plane triangles are listed k2-major, so consecutive
// triangles sharing k2 form a run; runs are cut into pieces of at most
// TRI_CHUNK triangles and whole pieces are packed into chunks of at most
// TRI_CHUNK triangles, one pipeline stage each.
constexpr int TRI_WARPS = 7;   // most tiles per CTA (one consumer warp each, plus one producer warp)
constexpr int TRI_P1 = 8;      // planes p1 per thread
constexpr int TRI_CHUNK = 16;  // in-plane triangles per stage
constexpr int TRI_PIECES = 4;  // pieces per stage
constexpr int TRI_STAGES = 3;  // pipeline depth
constexpr int TRI_PAD = 8;     // zero columns on each side of a mode row (>= TRI_P1 - 1)

struct TriTile {
  int p1_0, p3_0;  // planes p1_0 + a (a < TRI_P1) and p3_0 + lane
};

struct TriChunk {
  long long t0;  // first in-plane triangle (global list index)
  int pc0;       // first piece in the global piece table
  int packed;    // nt (bits 0-4), npc (bits 5-7), piece lengths (5 bits each from bit 8)
};
// fields of TriChunk::packed / TriDesc::packed
__host__ __device__ inline int chunk_nt(int packed) { return packed & 31; }
__host__ __device__ inline int chunk_npc(int packed) { return (packed >> 5) & 7; }
__host__ __device__ inline int chunk_len(int packed, int piece) { return (packed >> (8 + 5 * piece)) & 31; }
__host__ __device__ inline int chunk_pack(int nt, int npc, int lens) { return nt | (npc << 5) | (lens << 8); }

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
constexpr int TRI_TAU_MAX = 512;  // most in-plane triangles walked by one CTA

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
};

// Device-side tables and buffers of a plan.
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
  int class_first[TRI_WARPS + 2] = {};  // items with n tiles: [class_first[n], class_first[n+1])
  int class_stage[TRI_WARPS + 1] = {};  // stage size (complex values) of the CTAs with n tiles
  long long n_part = 0;
  double *part = nullptr;         // [n_part] partial sums
  // per-realization buffers
  double *staging = nullptr;      // [n_modes][Q] complex128 rows of the r2c buffer
  double *S64 = nullptr;          // [n_modes][W] complex128 signed-plane mode data
  float *S32 = nullptr;           // [n_modes][W] complex64 (mixed precision)
  double *B = nullptr;            // [n_combo] triangle sums, bin order
  // epilogue (bin order)
  int n_bins = 0;
  int32_t *bin_first = nullptr;   // [n_bins+1]
  double *ep_px = nullptr, *ep_pz = nullptr;  // [n_combo]
  int32_t *ep_cnt = nullptr;      // [n_combo] exact in-plane triangle count
  double *bins = nullptr;         // [3][n_bins][16]: bs, norm, out
  long long *bin_count = nullptr; // [n_bins]
  int *status = nullptr;          // device status word
};

}  // namespace beam

struct beam_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  size_t smem_optin = 0;
  // side streams forked from `stream` for the per-class triangle-sum launches
  cudaStream_t side[beam::TRI_WARPS] = {};
  cudaEvent_t fork = nullptr, join[beam::TRI_WARPS] = {};
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
  double *h_staging = nullptr;           // pinned [n_modes][Q] complex128
  double *h_bins = nullptr;              // pinned [3][n_bins][16]
  long long *h_count = nullptr;          // pinned [n_bins]
  size_t device_bytes = 0;
  beam::PixelPath *pix = nullptr;        // plane-ring transform tables / pixel method
  cudaEvent_t ev[5] = {};                // stage boundaries of the last run (beam_gpu_plan_last_timings)
  bool timed = false;
};

namespace beam {
// stage boundary k of the current run, on the context's stream
inline void mark(beam_gpu_plan *p, int k) {
  if (p->ev[k]) cudaEventRecord(p->ev[k], p->ctx->stream);
}
// plan construction (beam_plan.cu)
int build_plan_tables(beam_gpu_plan *p);
void free_plan_tables(beam_gpu_plan *p);
int count_closed_triangles(beam_gpu_plan *p, std::vector<long long> &counts);
// per-realization steps (beam_run.cu)
int upload_modes_host(beam_gpu_plan *p, const double *r2c);
int upload_modes_device(beam_gpu_plan *p, const double *r2c_dev);
int run_triangle_sums(beam_gpu_plan *p);
int run_epilogue(beam_gpu_plan *p);
int check_status(beam_gpu_plan *p);
template <typename T>
int dev_alloc(beam_gpu_plan *p, T **ptr, size_t count) {
  size_t bytes = sizeof(T) * (count ? count : 1);
  cudaError_t e = cudaMalloc((void **)ptr, bytes);
  if (e != cudaSuccess) {
    set_detail(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    return BEAM_EDEVMEM;
  }
  p->device_bytes += bytes;
  return BEAM_OK;
}
}  // namespace beam
