/* libbeam_gpu: B200 (sm_100a) implementation of the BEAM redshift-space
 * bispectrum estimator hot path of sukhdeepsinghgill/BARBIE, behind a plain C ABI.
 *
 * The reference has no plugin or FFI layer: its boundary is the program
 * `barbie NN NRi UL_k1 LL_k1 BW_k1` (barbie.c:26-399) and its files. The C host
 * drop-in (barbie_b200/host/barbie_main.c) keeps that command line and those
 * files and calls the entry points below, each of which replaces one stage of
 * the reference (cited per function).
 *
 * Conventions: every call returns BEAM_OK (0) or a negative BEAM_E* code and
 * never exits the process; the caller owns host buffers, the library owns
 * device state; a plan is not re-entrant (one host thread per plan at a time);
 * device waits are bounded and report BEAM_ETIMEDOUT. Device buffers the
 * kernels read or write as complex values (r2c buffers, real cubes, plane-ring
 * outputs) must start on a 16-byte boundary, as cudaMalloc'd and torch
 * buffers do; a call given one that does not returns BEAM_EINVAL (a
 * page-locked host r2c buffer off that boundary is gathered on the host
 * instead of being read in place).
 *
 * Array layouts (all row-major, native-endian):
 *   r2c    double[NN][NN][NN+2]: the FFTW in-place r2c buffer of Delta(k),
 *          i.e. complex128[NN][NN][NN/2+1] with the last axis the line of sight
 *          (barbie.c:176-185, field_N<NN>_R<NRi>.txt).
 *   bins   double[n_k1bin][n_mtbin][n_mtbin][16] (barbie.c:87), with
 *          n_k1bin = (UL_k1-LL_k1)/BW_k1 (barbie.c:84).
 */
#ifndef BEAM_GPU_H
#define BEAM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BEAM_API __attribute__((visibility("default")))
#else
#define BEAM_API
#endif

#define BEAM_NPOLES 16

/* error codes */
#define BEAM_OK 0
#define BEAM_EINVAL (-1)     /* invalid configuration or argument */
#define BEAM_ENOMEM (-2)     /* host allocation failed */
#define BEAM_EDEVMEM (-3)    /* device allocation failed or footprint refused */
#define BEAM_ECUDA (-4)      /* a CUDA runtime call failed */
#define BEAM_ETIMEDOUT (-5)  /* a bounded device wait gave up */
#define BEAM_EBUSY (-6)      /* queue full / slot not available */
#define BEAM_EBOUNDS (-7)    /* a triangle's bin index falls outside the bin arrays */
#define BEAM_ENODEV (-8)     /* no usable CUDA device */
#define BEAM_ENOTFOUND (-9)  /* unknown job id */

/* precision of the triple-product sums */
#define BEAM_PREC_FP64 0  /* FP64 throughout (parity path, 1e-10 of the reference) */
#define BEAM_PREC_MIXED 1 /* FP32 mode data and products, FP32 chunk sums, FP64 across chunks */
#define BEAM_PREC_INT8 2  /* FP64 mode data cut into five 8-bit slices per (ring, plane) scale; the
                             slice products and each run's sums exact in int32 on the int8 tensor
                             cores; FP64 from the run's end on (error ~1e-7 of a bin, far below 1e-5).
                             Mode values must be finite: a NaN or infinity is not carried through the
                             slices as the FP64 path carries it */

/* how the per-triangle sums B = sum_x Re(F1 F2 F3) are formed */
#define BEAM_METHOD_TRIANGLE 0 /* over closed in-plane Fourier triangles (default) */
#define BEAM_METHOD_PIXEL 1    /* over the NN^2 pixels of the per-(plane,ring) IFFTs, as the reference */

typedef struct beam_gpu_ctx beam_gpu_ctx;
typedef struct beam_gpu_plan beam_gpu_plan;

/* Estimator configuration. The reference hard-codes all but the first three
 * command-line values in barbie.c:67-84: Nmax=100, Nr=40, n_mtbin=5, LL=1. */
typedef struct beam_cfg {
  long NN;        /* grid size (even) */
  long Nmax;      /* number of line-of-sight planes (barbie.c:71) */
  long Nr;        /* number of rings, a multiple of 10 (barbie.c:72,111-114) */
  int UL_k1;      /* upper k1 limit, grid units (argv[3]) */
  int LL_k1;      /* lower k1 limit (argv[4]) */
  int BW_k1;      /* k1 bin width (argv[5]) */
  int n_mtbin;    /* mu and t bins on [0.5,1] (barbie.c:84) */
  double LL;      /* cell size for vol=(NN*LL)^3 (barbie.c:67,76) */
  int precision;  /* BEAM_PREC_* */
  int method;     /* BEAM_METHOD_* */
  /* One bispectrum split over several GPUs (the analogue of the reference's
   * MPI estimator splitting its loop over ranks, zBS_fast_mpi.c:149,294-296):
   * the plan sums only the ring triplets beam_shard_assign gives shard_index
   * of shard_count, and its bs/norm/count are partial sums that add up across
   * the shards (out is then bs/(vol*norm) of the sums). shard_count 0 or 1:
   * the whole estimator. Triangle method only. */
  int shard_index;
  int shard_count;
} beam_cfg;

/* Fill cfg with the reference's defaults for the given command-line values. */
BEAM_API void beam_cfg_default(beam_cfg *cfg, long NN, int UL_k1, int LL_k1, int BW_k1);

/* Longest-processing-time assignment of n work units (ring triplets, in
 * increasing calCR order) to shard_count shards: units in order of decreasing
 * work (ties: lower index first) each go to the shard with the least work so
 * far (ties: lower shard). Host-only and deterministic, so every rank computes
 * the same owner[] from the same work[]. No counterpart in the reference,
 * whose MPI variants split planes round-robin. */
BEAM_API int beam_shard_assign(const double *work, int n, int shard_count, int *owner);

/* Estimator output; any pointer may be NULL. */
typedef struct beam_result {
  double *bs;     /* bins: sum of B*bs[ii]           (bin_BS_real, barbie.c:360) */
  double *norm;   /* bins: sum of Num*norm[ii]       (bin_normalization, barbie.c:362) */
  double *out;    /* bins: bs/(vol*norm)             (the value barbie.c:390-393 prints) */
  int64_t *count; /* [n_k1bin][n_mtbin][n_mtbin]: exact number of closed triangles summed
                     into the bin (those with B != 0); norm[..][0] = NN^2 * count */
  double *ana_sum; /* bins: sum of Biana*Num*bs[ii], the analytic redshift-space bispectrum of
                      P(k) = k^-2 over the bin's triangles (bin_Biana, barbie.c:300-305,361) */
  double *ana;     /* bins: ana_sum/norm (column 5 of the output files, barbie.c:391-393) */
} beam_result;

typedef struct beam_plan_info {
  int n_k1bin;            /* bins along k1 */
  long n_bins;            /* n_k1bin * n_mtbin^2 */
  long n_closed_triplets; /* ring triplets passing the closure test (calCR's rcount) */
  long n_triples;         /* accepted (p1, ring triplet, p2) triangles of the loop */
  long n_used_triplets;   /* distinct ring triplets among them */
  long n_fourier_terms;   /* sum over accepted triangles of their in-plane triangle counts */
  long n_modes;           /* ring modes on the planes in use */
  int n_planes;           /* planes |p| in use (0..n_planes-1) */
  size_t device_bytes;    /* device memory held by the plan (tables + per-run buffers) */
  double vol;             /* (NN*LL)^3 */
  long n_shard_terms;     /* in-plane triangles this plan's shard sums (n_fourier_terms unsharded) */
  int launches_last_run;  /* kernels the plan's last beam_gpu_run / triangle_sums call launched */
  size_t run_bytes;       /* device bytes of the buffers of one more concurrent realization */
  long n_run_combos;      /* sum over accepted triangles of the runs of their triplet's in-plane list
                             (triangles sharing the mode of the leg whose plane is -p1 - p(tile), whose
                             product with the run's accumulated outer product is formed once per run) */
  float build_ms[5];      /* host wall time of the plan's creation, ms: [0] geometry (rings, triplets,
                             accepted triangles), [1] mode tables and in-plane triangle lists (GPU),
                             [2] work decomposition, [3] remaining device tables, [4] run buffers */
} beam_plan_info;

/* Library / device setup. Replaces the fftw_init_threads / plan_with_nthreads
 * set-up of barbie.c:151-153. */
BEAM_API int beam_gpu_init(int device, beam_gpu_ctx **out);
BEAM_API void beam_gpu_destroy(beam_gpu_ctx *ctx);

/* Geometry plan: ring edges and masks (barbie.c:110-148), closed ring triplets
 * with exact triangle counts (calCR, funcs.c:328-424, in place of the
 * closed_rings_<NN> disk cache, barbie.c:161-164), and the accepted triangles of
 * the loop with their K1/T/MU/px/pz and bins (barbie.c:247-298,343-345). The
 * plan is independent of the field and is reused for every realization. */
BEAM_API int beam_gpu_plan_create(beam_gpu_ctx *ctx, const beam_cfg *cfg, beam_gpu_plan **out);
BEAM_API void beam_gpu_plan_destroy(beam_gpu_plan *plan);
BEAM_API int beam_gpu_plan_get_info(const beam_gpu_plan *plan, beam_plan_info *info);

/* One bispectrum: plane-ring transforms (wrapid_fast/Df, funcs.c:537-566,88-109,
 * held on the device instead of the disk cache), the triple products of the loop
 * (barbie.c:315-337), binning and cal_coeff weights (barbie.c:343-363,
 * funcs.c:708-745) and the normalisation (barbie.c:383-392).
 * r2c: double[NN][NN][NN+2], in host memory (r2c_on_device=0, pageable or
 * pinned) or device memory (r2c_on_device=1). Results go to host memory.
 * Only the ring modes of the planes in use are read (6.6 MB of the 455 MB
 * buffer at NN=384): from pageable memory the host gathers them and copies
 * them over; from page-locked memory (cudaHostAlloc, cudaHostRegister) the
 * device reads them in place. */
BEAM_API int beam_gpu_run(beam_gpu_plan *plan, const double *r2c, int r2c_on_device, beam_result *res);

/* Several realizations of one plan in one call (no counterpart in the
 * reference, which runs one realization per process). Realizations go to the
 * device in batches: each kernel of a batch (mode build, the per-class
 * triangle sums, split reduction, epilogue) is one launch over all of the
 * batch's realizations, and the batch's sequence -- H2D of the gathered mode
 * rows, kernels, D2H of the bins -- is captured once into a CUDA graph and
 * replayed. Two batch buffers alternate, so the host gathers batch i+1 while
 * the device runs batch i. Results equal beam_gpu_run's bit for bit.
 * r2c[i] are host buffers; res[i] receives realization i (res may be NULL).
 * batch: realizations per batch, 0 = chosen from free device memory (<= n). */
BEAM_API int beam_gpu_run_batch(beam_gpu_plan *plan, const double *const *r2c, int n, beam_result *res);
BEAM_API int beam_gpu_run_batch_ex(beam_gpu_plan *plan, const double *const *r2c, int n, beam_result *res,
                                   int batch);

/* How the plan launches its triangle sums (no counterpart in the reference,
 * whose triangle loop is one serial loop, barbie.c:247-365):
 *   BEAM_LAUNCH_CLASSES     one launch per tile class (CTA shape), on side
 *                           streams that overlap (the default);
 *   BEAM_LAUNCH_PERSISTENT  one persistent launch over every item of every
 *                           class and every realization of the run or batch:
 *                           CTAs of the largest class's shape take work units
 *                           from a device counter, largest first.
 * Results are bit-identical either way (every unit sums the same triangles in
 * the same order). Changing the mode drops the plan's captured batch graphs. */
#define BEAM_LAUNCH_CLASSES 0
#define BEAM_LAUNCH_PERSISTENT 1
BEAM_API int beam_gpu_plan_set_triangle_launch(beam_gpu_plan *plan, int mode);

/* calCR (funcs.c:328-424): closed ring triplets in the reference's order as
 * records {r1, r2, r3, Num} with Num = NN^2 * (exact triangle count) -- the
 * quantity the reference computes by FFT with round-off. Writes up to cap
 * records; *rcount receives the total. */
BEAM_API int beam_gpu_closed_rings(beam_gpu_plan *plan, double *rings4, long cap, long *rcount);

/* Df / wrapid_fast (funcs.c:88-109,537-566): for each of n (plane, ring) pairs
 * (0 <= plane < Nmax, 0 <= ring < Nr) the unnormalised backward 2D DFT of the
 * ring-masked plane, k_perp=0 zeroed on plane 0, as complex128[NN][NN] written
 * to out + k*2*NN*NN (host memory unless out_on_device). Runs on the GPU with
 * the library's FFT kernels in FP64. */
BEAM_API int beam_gpu_plane_rings(beam_gpu_plan *plan, const double *r2c, int r2c_on_device,
                         const int *planes, const int *rings, int n, double *out, int out_on_device);

/* Plane-ring transforms without any device allocation. It has no counterpart
 * in the reference; it serves callers that must not call cudaMalloc: code that
 * runs inside an application whose own allocator has already claimed the
 * device memory, processes under a hard device-memory quota, and latency-
 * sensitive loops where cudaMalloc's implicit device synchronisation is not
 * acceptable.
 * Same result as beam_gpu_plane_rings for the same inputs, but all buffers are
 * the caller's: r2c_dev is the r2c buffer double[NN][NN][NN+2] in device
 * memory, out_dev receives n arrays complex128[NN][NN] in device memory, and
 * planes/rings are host arrays of n entries (0 <= plane < Nmax <= NN/2,
 * 0 <= ring < Nr, Nr a multiple of 10). Work is queued on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) of the current device and
 * the call returns without waiting for the transform. The tables are staged
 * from pageable host memory, so the call may first wait for the work already
 * queued on `stream`.
 * The ring tables, twiddles and job list go to a fixed scratch array of
 * BEAM_NOALLOC_SCRATCH_BYTES in the library's device image; each GPU that
 * loads the library holds that array until the process exits. A call whose
 * tables need more (many rings or large NN), whose widest ring needs more
 * shared memory than the device allows, or with n > BEAM_NOALLOC_MAX_JOBS,
 * returns BEAM_EINVAL before queuing anything and explains in
 * beam_gpu_last_error_detail(). The call cannot be captured into a CUDA graph:
 * given a capturing stream it returns BEAM_EINVAL. Every call rewrites the
 * array, so calls whose work overlaps on the GPU race on it: order them on one
 * stream. */
#define BEAM_NOALLOC_SCRATCH_BYTES (2u * 1024u * 1024u)
#define BEAM_NOALLOC_MAX_JOBS 4096
BEAM_API int beam_gpu_plane_rings_noalloc(long NN, long Nmax, long Nr, const double *r2c_dev, const int *planes,
                                          const int *rings, int n, double *out_dev, void *stream);

/* Per-triangle sums B (barbie.c:326-337, the value added at :360 before the bs
 * weight) for all accepted triangles in loop order, written to B (host, n_triples
 * doubles). The plan's method and precision apply. */
BEAM_API int beam_gpu_triangle_sums(beam_gpu_plan *plan, const double *r2c, int r2c_on_device, double *B);

/* The cudaStream_t (as void*) the context launches all its work on, for
 * callers that order their own work after it or record events on it. */
BEAM_API void *beam_gpu_stream(beam_gpu_ctx *ctx);

/* Device time of the stages of the plan's last run/triangle_sums call, in
 * milliseconds, measured with CUDA events on the context's stream:
 * [0] mode upload + gather, [1] triangle sums (the dominant kernel),
 * [2] split reduction, [3] bins epilogue. Writes min(n, 4) values. */
BEAM_API int beam_gpu_plan_last_timings(const beam_gpu_plan *plan, float *ms, int n);

/* ------------------------------------------------------------------ serving
 * A job server on one context (no counterpart in the reference, which runs
 * one realization per process): estimator jobs -- one realization each, any
 * NN / rings / bins / precision -- are submitted as they arrive and run
 * concurrently on the device. A dispatcher thread keeps a cache of plans
 * (geometry tables) keyed by configuration, and admits queued jobs in arrival
 * order as soon as a job slot is free and the device memory the job needs --
 * its plan if not cached, plus one realization's run buffers
 * (beam_plan_info.run_bytes) -- fits the budget, evicting idle cached plans
 * when it must; a job that does not fit lets smaller later jobs go first.
 * Each running job has its own streams and buffers, so jobs admitted while
 * others run overlap with them on the GPU; results do not depend on what else
 * runs (every reduction has a fixed order). While a server runs, it alone
 * uses its context. Jobs need the triangle method and shard_count <= 1. */
typedef struct beam_gpu_server beam_gpu_server;

typedef struct beam_server_cfg {
  size_t mem_budget; /* device bytes for cached plans and running jobs; 0 = 80% of the free memory at creation */
  int max_active;    /* jobs on the device at once; 0 = 4 */
  int max_plans;     /* plans kept for reuse; 0 = 16 */
} beam_server_cfg;

#define BEAM_JOB_QUEUED 0
#define BEAM_JOB_RUNNING 1
#define BEAM_JOB_DONE 2
#define BEAM_JOB_FAILED 3

typedef struct beam_job_info {
  int state;        /* BEAM_JOB_* */
  int error;        /* BEAM_* code of a failed job */
  int n_k1bin;      /* result shape: [n_k1bin][n_mtbin][n_mtbin][16] (known once started) */
  int n_mtbin;
  long n_bins;
  double queue_ms;  /* submission to start of its device work (host clock) */
  double run_ms;    /* start of its device work to results on the host */
  double total_ms;  /* submission to results on the host */
} beam_job_info;

BEAM_API void beam_server_cfg_default(beam_server_cfg *cfg);
BEAM_API int beam_gpu_server_create(beam_gpu_ctx *ctx, const beam_server_cfg *cfg, beam_gpu_server **out);
/* Waits for queued and running jobs, then frees everything the server holds. */
BEAM_API void beam_gpu_server_destroy(beam_gpu_server *srv);
/* Queue one realization: r2c is a host double[NN][NN][NN+2] that must stay
 * valid and unchanged until the job is DONE or FAILED. *job receives its id. */
BEAM_API int beam_gpu_server_submit(beam_gpu_server *srv, const beam_cfg *cfg, const double *r2c, int64_t *job);
/* Wait up to timeout_ms (0: poll, < 0: forever) for the job to finish.
 * BEAM_OK when it is DONE or FAILED (info->state tells which), BEAM_EBUSY
 * when still queued or running, BEAM_ENOTFOUND for an unknown job. */
BEAM_API int beam_gpu_server_wait(beam_gpu_server *srv, int64_t job, int timeout_ms, beam_job_info *info);
/* Copy a DONE job's bins into res (any pointer may be NULL) and forget the
 * job; a FAILED job returns its error and is forgotten too. */
BEAM_API int beam_gpu_server_take(beam_gpu_server *srv, int64_t job, beam_result *res);
/* Device bytes the server holds now (cached plans + job buffers) and at most so far. */
BEAM_API int beam_gpu_server_memory(const beam_gpu_server *srv, size_t *now, size_t *peak);

/* Power spectrum multipoles of an r2c buffer: the reference's calpow_mom
 * (funcs.c:860-1074, driven by calpow_mom.c). Every independent Fourier mode
 * is binned in Nbin logarithmic bins of |k| (bin d holds log10(|k| NN) in
 * [d, d+1) x log10(NN/2)/Nbin); out receives [6][Nbin] doubles: mean |k|
 * (2 pi/(NN LL) units as the reference), P0, P2, P4, P6 and the mode count,
 * normalised as funcs.c:1050-1066 with cell size LL (calpow_mom.c uses 0.56,
 * Nbin 10). r2c in host (r2c_on_device=0) or device memory. Reads the whole
 * buffer once on the context's stream. */
BEAM_API int beam_gpu_power_multipoles(beam_gpu_ctx *ctx, long NN, double LL, int Nbin, const double *r2c,
                                       int r2c_on_device, double *out);

/* Field ingestion on the device. Both calls write the r2c buffer
 * double[NN][NN][NN+2] that beam_gpu_run reads (the reference's on-disk field
 * format, generate_field.c:100-109), into device memory when r2c_on_device is
 * set (the buffer can go straight to beam_gpu_run with r2c_on_device) or
 * host memory otherwise. NN = 2^a 3^b, even, in [4, 1024]. Both run on the
 * context's stream and return when the buffer is complete. */

/* The reference's field generator `field NN NRi` (generate_field.c:78-88;
 * replaces Fill_Modes, Make_Image, Non_Gauss, Get_Modes and RSD of
 * ngrf_2d_funcs.c:341-584,734-765): Gaussian modes of amplitude
 * sqrt((NN LL)^3/2 k^-2), the real image, x += ff (x^2 - var), x LL^3, the r2c
 * transform and the (1 + beta mu^2) redshift-space factor. The reference
 * program uses LL = 0.56, ff = 0.5, beta = 1 and seed = 100020 + 146 NRi
 * (generate_field.c:45-50). The reference draws its modes from GSL's
 * MT19937 + ziggurat; here draw n of the fill order is a counter-based normal
 * deviate (Philox4x32-10 with key = seed, then Box-Muller), so a seed gives
 * the same field on every device but not the GSL field. sigma (may be NULL)
 * receives the Gaussian image's rms, which the reference prints. */
BEAM_API int beam_gpu_field_generate(beam_gpu_ctx *ctx, long NN, unsigned long long seed, double LL, double ff,
                                     double beta, double *r2c, int r2c_on_device, double *sigma);

/* A real-space density cube double[NN][NN][NN] (host or device memory; it
 * must not overlap r2c) to the r2c buffer: Get_Modes (x LL^3, the 3D r2c
 * transform, ngrf_2d_funcs.c:534-550) and RSD with beta (ngrf_2d_funcs.c:734-765;
 * beta = 0 leaves the modes as transformed). */
BEAM_API int beam_gpu_field_ingest(beam_gpu_ctx *ctx, long NN, double LL, double beta, const double *cube,
                                   int cube_on_device, double *r2c, int r2c_on_device);

/* Autotuning. No counterpart in the reference (FFTW's planner is the nearest:
 * FFTW_ESTIMATE, funcs.c:349,546).
 *
 * beam_gpu_plan_autotune: the triangle sums' work decomposition -- tau0, the
 * first cap on the in-plane triangles one CTA walks (the split-K factor of
 * each ring triplet's triangle list), and balance, the items' worth of work
 * per SM the load balance aims at -- chosen by timing each candidate's
 * triangle phase on this device (the plan's tables are rebuilt per candidate,
 * mode data a fixed pattern, reps timed runs each, best kept). The plan keeps
 * the fastest; bins agree with the untuned plan to round-off (only the order
 * of partial sums changes). Takes about (candidates x (rebuild + (reps+1)
 * runs)); reps <= 0 means 3. Triangle method only. */
#define BEAM_TUNE_MAX 16
typedef struct beam_tune_report {
  int n;                          /* candidates tried */
  int best;                       /* the one the plan keeps */
  long long tau0[BEAM_TUNE_MAX];  /* first cap on in-plane triangles per CTA */
  double balance[BEAM_TUNE_MAX];  /* items of work per SM aimed at */
  float ms[BEAM_TUNE_MAX];        /* triangle phase (sums + split reduction), best of reps */
  int items[BEAM_TUNE_MAX];       /* CTA work items of the candidate */
} beam_tune_report;
BEAM_API int beam_gpu_plan_autotune(beam_gpu_plan *plan, int reps, beam_tune_report *rep);

/* beam_gpu_field_autotune: the FFT staging tile (lines x length per CTA) of
 * the field calls' column and row passes for this NN, each candidate timed on
 * one pass over a scratch buffer (NN^2 (NN+2) doubles, freed on return); the
 * context's later field calls with this NN use the fastest. Results do not
 * depend on the tile. */
#define BEAM_FIELD_TUNE_MAX 4
typedef struct beam_field_tune_report {
  int n, best_cols, best_rows;
  int tile[BEAM_FIELD_TUNE_MAX];       /* complex values staged per CTA */
  float cols_ms[BEAM_FIELD_TUNE_MAX];  /* one column pass, best of 3 */
  float rows_ms[BEAM_FIELD_TUNE_MAX];  /* one row pass, best of 3 */
} beam_field_tune_report;
BEAM_API int beam_gpu_field_autotune(beam_gpu_ctx *ctx, long NN, beam_field_tune_report *rep);

/* Kernels the last successful field call on this context launched (0 before
 * any): generate 8 (mode fill, 3 backward passes, variance, 3 forward passes),
 * ingest 3; -1 for a NULL context. */
BEAM_API int beam_gpu_field_launches(const beam_gpu_ctx *ctx);

/* Human-readable text for an error code. */
BEAM_API const char *beam_gpu_strerror(int code);

/* Details of the last error on this thread (CUDA error string etc.). */
BEAM_API const char *beam_gpu_last_error_detail(void);

#ifdef __cplusplus
}
#endif
#endif
