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
constexpr int TRI_THREADS = 256;
constexpr int TRI_CHUNK = 16;  // upper bound; the launch may stage fewer
constexpr int TRI_MAX_SLOTS = 16;  // combos per thread

// One unit of triangle-sum work: combos [c0, c1) of one used ring triplet over
// its in-plane triangles [t0, t1). Rows staged per triangle are the columns
// [p1lo, p1lo+L1), [p2lo, p2lo+L2), [p3lo, p3lo+L3) of the signed-plane mode
// rows of rings r1, r2, r3 (column of plane q is q + Q - 1).
struct TriItem {
  int u;               // used ring triplet
  int split;           // index of this triangle range among the triplet's splits
  int c0, c1;          // combos (global combo indices)
  long long t0, t1;    // in-plane triangles (global triangle-list indices)
  int m1, m2, m3;      // first mode of rings r1, r2, r3 in the mode table
  int p1lo, L1, p2lo, L2, p3lo, L3;
};

// Device-side tables and buffers of a plan.
struct DevPlan {
  // ring modes on the planes in use
  int n_modes = 0, Q = 0, W = 0;  // modes, planes |p| < Q in use, signed-plane row width 2Q-1
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
  int32_t *combo_p1 = nullptr, *combo_p2 = nullptr;  // [n_combo]
  int32_t *combo_u = nullptr;     // [n_combo] used ring triplet
  int32_t *combo_out = nullptr;   // [n_combo] bin-order position of the triangle
  int32_t *u_cfirst = nullptr;    // [n_used] first combo
  int32_t *u_ncombo = nullptr;    // [n_used]
  int32_t *u_nsplit = nullptr;    // [n_used] triangle-range splits
  long long *u_part = nullptr;    // [n_used] first partial-sum slot (split-major)
  int n_items = 0;
  TriItem *items = nullptr;       // [n_items], largest work first
  long long n_part = 0;
  double *part = nullptr;         // [n_part] partial sums
  int max_row = 0;                // max L1+L2+L3 over items
  int chunk = TRI_CHUNK;          // in-plane triangles per stage (fits shared memory)
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
