/*
 * mqp.h - C ABI of the B200-native cross-correlation PIV hot path.
 *
 * Drop-in boundary for multi_quickPIV (Julia).  The reference runs the whole
 * PIV hot path in Julia and calls native code only through FFTW's @ccall
 * (src/utils/fft_ops.jl:18-80).  Its user API is
 *   PIV(img1, img2[, mask[, mask_IA]], pivparams; precision)
 *   (src/multi_quickPIV.jl:17-29)
 * built on setPIVParameters (src/piv_parameters.jl:67-81).  This library
 * replaces the per-interrogation-area loop behind that API
 * (src/multi_quickPIV.jl:57-93, i.e. allocate_tmp_data / prepare_inputs! /
 * crosscorrelation! / gaussian_displacement / compute_SN per IA) with one
 * call per image pair, so a Julia method
 *   PIV(img1, img2, pivparams; backend=:b200)
 * can ccall mqp_piv with the arrays it already holds.
 *
 * Conventions
 *  - Arrays are column-major (Julia order).  dims[0] is Julia dimension 1.
 *  - VF has shape (N, vf_1, ..., vf_N), component fastest, Float64, as
 *    allocate_outputs (src/utils/piv_ops.jl:25-31) lays it out; SN has shape
 *    (vf_1, ..., vf_N).  The caller owns every buffer it passes in.
 *  - Every function returns MQP_OK (0) or a negative MQP_ERR_* code; the
 *    message of the last failure on a context is mqp_last_error(ctx).
 *    Nothing aborts the process.
 *  - A context is bound to one CUDA device and owns its device buffers and
 *    stream.  Calls on one context are serialised; use one context per host
 *    thread for concurrency.
 */
#ifndef MQP_H
#define MQP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MQP_ABI_VERSION 1

#if defined(_WIN32)
#define MQP_API __declspec(dllexport)
#else
#define MQP_API __attribute__((visibility("default")))
#endif

/* status codes */
#define MQP_OK 0
#define MQP_ERR_INVALID (-1)     /* bad argument, shape or parameter */
#define MQP_ERR_UNSUPPORTED (-2) /* valid in the reference but not on this path */
#define MQP_ERR_CUDA (-3)        /* CUDA runtime failure */
#define MQP_ERR_OOM (-4)         /* device allocation failed */
#define MQP_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define MQP_ERR_BUSY (-6)        /* admission refused (serving) */
#define MQP_ERR_NOT_FOUND (-7)   /* unknown request / stream id */

/* correlation algorithms: the CORRTYPES of src/piv_parameters.jl:1-6 */
#define MQP_FFTCC 0
#define MQP_ZNCC 1
#define MQP_NSQECC 2
#define MQP_MASK_NSQECC 3

/* element types of the images (and mask) */
#define MQP_F32 0
#define MQP_F64 1

/*
 * PIVParameters (src/piv_parameters.jl:28-45) as a POD.  Fields hold the
 * STORED values of the Julia struct, i.e. after setPIVParameters' positional
 * constructor has swapped unpadded/good_pad (src/piv_parameters.jl:57-59).
 * filtFun / mask_filtFun are fixed to maxval (Julia closures cannot cross
 * the ABI).
 */
typedef struct mqp_params {
  int32_t corr_alg;        /* MQP_FFTCC | MQP_ZNCC | MQP_NSQECC (mask given => masked NSQECC) */
  int32_t interSize[3];    /* per Julia dimension */
  int32_t searchMargin[3];
  int32_t overlap[3];
  int32_t step[3];         /* used when has_step != 0 */
  int32_t has_step;        /* 0: step = interSize - overlap (src/piv_parameters.jl:87) */
  int32_t multipass;       /* >= 1 */
  int32_t computeSN;
  int32_t unpadded;        /* stored value; must be 1 (src/utils/piv_ops.jl:257-268) */
  int32_t good_pad;        /* stored value */
  int32_t odd_pad;
  double threshold;        /* skip IA when threshold >= 0 and maxval(IA) < threshold */
  double mask_threshold;   /* masked PIV: skip when > 0 and maxval(mask IA) < it */
  double ovp_th;           /* carried for completeness; unused by the reference kernels */
  int32_t refine;          /* 0: multipass re-runs scale 1 (the reference); 1: whole-pixel predictor
                              refinement; 2: refinement with window deformation (no masks) */
  int32_t reserved[7];
} mqp_params;

typedef struct mqp_ctx mqp_ctx;

/* ABI version of the loaded library (MQP_ABI_VERSION). */
MQP_API int mqp_abi_version(void);

/* Create a context on CUDA device `device`.  Fails with MQP_ERR_CUDA when no
 * such device exists. */
MQP_API int mqp_create(mqp_ctx** out, int device);

/* Release a context and its device memory. */
MQP_API int mqp_destroy(mqp_ctx* ctx);

/* Message of the last failing call on ctx (or of the last failing
 * mqp_create when ctx is NULL).  Valid until the next call on ctx. */
MQP_API const char* mqp_last_error(const mqp_ctx* ctx);

/* get_vectorfield_size (src/utils/piv_ops.jl:6-14): vf_dims_out[d] for
 * d < ndims (the rest set to 1). */
MQP_API int mqp_vf_dims(const mqp_params* p, int ndims, const int64_t dims[3], int64_t vf_dims_out[3]);

/* PIV on HOST arrays (src/multi_quickPIV.jl:17-29).  img1, img2 (and mask,
 * nullable) are column-major arrays of `dtype` with extents dims[0..ndims).
 * mask != NULL selects masked NSQECC; mask_skip (nullable) is the separate
 * skip mask of the double-masked method (src/multi_quickPIV.jl:27-29).  VF
 * receives N*prod(vf) doubles, SN (nullable; used when computeSN) prod(vf).
 * Blocks until the result is in VF/SN.
 * Window limits (the reference takes any size; beyond these the call
 * returns MQP_ERR_UNSUPPORTED): 2D search windows interSize + 2 searchMargin
 * up to 256 per axis, above 128 only unmasked with interrogation windows up
 * to 128; 3D up to 128 per axis, above 64 with interrogation windows up to
 * 64.  Refinement passes run at scaled windows and must fit as well. */
MQP_API int mqp_piv(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask,
            const void* mask_skip, int dtype, int ndims, const int64_t dims[3],
            const mqp_params* p, double* VF, double* SN, int64_t vf_dims_out[3]);

/* The same on DEVICE arrays already resident in HBM, enqueued on `stream`
 * (a cudaStream_t; NULL = the legacy default stream, as in the CUDA
 * runtime).  Returns once the work is enqueued; synchronise the stream
 * before reading d_VF / d_SN. */
MQP_API int mqp_piv_device(mqp_ctx* ctx, const void* d_img1, const void* d_img2, const void* d_mask,
                   const void* d_mask_skip, int dtype, int ndims, const int64_t dims[3],
                   const mqp_params* p, double* d_VF, double* d_SN, void* stream);

/* Debug/test entry: the fully-overlapping similarity planes (the block
 * tmp_data[1][1:2SM+1, ...] the reference searches, src/utils/piv_ops.jl:257-260)
 * for the IAs [ia_begin, ia_end) of the vector field, written to the host
 * buffer `planes` as (2SM1+1, 2SM2+1[, 2SM3+1], n) doubles. */
MQP_API int mqp_correlation_planes(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask,
                           int dtype, int ndims, const int64_t dims[3], const mqp_params* p,
                           int64_t ia_begin, int64_t ia_end, double* planes);

/* Kernel timing (tracing).  While enabled, every kernel class is bracketed
 * by CUDA events on the stream it is launched on; mqp_profile_read waits
 * for the recorded work and returns the accumulated device times. */
typedef struct mqp_profile {
  int64_t launches_integral; /* integral-image scan kernels */
  int64_t launches_piv;      /* fused correlation kernels */
  int64_t launches_other;    /* predictor / post-processing kernels */
  double ms_integral;
  double ms_piv;
  double ms_other;
  int64_t ia_count;          /* interrogation areas processed by the fused kernels */
} mqp_profile;

MQP_API int mqp_profile_enable(mqp_ctx* ctx, int enable); /* also resets the counters */
MQP_API int mqp_profile_read(mqp_ctx* ctx, mqp_profile* out);

/* Launch tuning of a context (no counterpart in the reference, whose FFTW
 * plans take no such knobs).  Results never depend on these values.
 *   MQP_TUNE_CHUNK3D         IAs per chunk of the 3D path (0 = from the budget)
 *   MQP_TUNE_CHUNK3D_BUDGET  device bytes of 3D chunk scratch (default 1 GiB)
 *   MQP_TUNE_HOST_PIECES     column pieces of the pipelined host-array 2D path
 *                            (single pass, images >= 1024 columns; default 3,
 *                            1 = copy everything first; at most 16)
 * Returns MQP_ERR_INVALID for an unknown key or a negative value. */
#define MQP_TUNE_CHUNK3D 1
#define MQP_TUNE_CHUNK3D_BUDGET 2
#define MQP_TUNE_HOST_PIECES 3
MQP_API int mqp_set_tuning(mqp_ctx* ctx, int key, int64_t value);

/*
 * Batched PIV plans.  No counterpart in the reference (whose PIV takes one
 * pair): many image pairs of mixed size, dimensionality (2D/3D), algorithm,
 * mask and pass count on DEVICE arrays, computed by one pre-allocated
 * schedule captured into a CUDA graph.  Every pair's VF/SN equal what
 * mqp_piv_device returns for it alone.
 *
 * The plan keeps the device pointers of the items (and owns all scratch):
 * run it as often as wanted while they stay valid; results are written to
 * the items' VF/SN.  Creating a plan allocates and synchronises; running
 * it enqueues one graph launch on `stream` and returns.
 */
typedef struct mqp_batch_item {
  const void* img1;       /* device images, column-major, dims[0] fastest */
  const void* img2;
  const void* mask;       /* masked NSQECC mask (device) or NULL */
  const void* mask_skip;  /* double-masked skip mask (device) or NULL */
  int32_t dtype;          /* MQP_F32 / MQP_F64 */
  int32_t ndims;          /* 2 or 3 */
  int64_t dims[3];
  mqp_params params;      /* refine + multipass > 1 gives a multi-pass pair */
  double* VF;             /* device (ndims, vf...) */
  double* SN;             /* device (vf...) or NULL */
} mqp_batch_item;

typedef struct mqp_batch_options {
  int32_t use_graph;       /* capture the schedule into one CUDA graph (default 1) */
  int32_t grab;            /* 2D work-queue entries a warp takes at once (default 2) */
  int64_t chunk3d;         /* IAs per 3D chunk (0 = from chunk3d_budget) */
  int64_t chunk3d_budget;  /* device bytes of 3D chunk scratch (0 = 1 GiB) */
  int32_t reserved[8];
} mqp_batch_options;

typedef struct mqp_plan mqp_plan;

MQP_API int mqp_batch_plan_create(mqp_ctx* ctx, const mqp_batch_item* items, int32_t n_items,
                                  const mqp_batch_options* opt /* NULL = defaults */, mqp_plan** out);
MQP_API int mqp_batch_plan_run(mqp_plan* plan, void* stream);
/* IAs of all passes, kernel launches and scratch bytes of one run */
MQP_API int mqp_batch_plan_info(const mqp_plan* plan, int64_t* total_ia, int64_t* launches, int64_t* scratch_bytes);
MQP_API int mqp_batch_plan_destroy(mqp_plan* plan);

/*
 * Serving.  No counterpart in the reference (a serial per-call PIV): a
 * request loop for time-lapse streams.  Each stream (fixed frame size, dtype
 * and single-pass PIV parameters) keeps its last frames and their integral
 * images resident on the device; every submitted frame t+1 becomes one
 * request PIV(frame t, frame t+1), admitted continuously by a worker thread
 * as execution slots and the device-memory budget free up, its work
 * overlapping on the device with the other slots'.  Results are identical to
 * mqp_piv on the same pair.  Frames are host arrays (copied at submit).
 */
typedef struct mqp_server mqp_server;

typedef struct mqp_server_options {
  int32_t slots;              /* concurrent requests on the device (default 4) */
  int32_t reserved0;
  int64_t hbm_budget_bytes;   /* transient device bytes requests may hold (0 = free memory - reserve) */
  int64_t hbm_reserve_bytes;  /* kept free when the budget is derived (default 4 GiB) */
  int64_t chunk3d_budget;     /* 3D chunk scratch per request (default 512 MiB) */
  int32_t reserved[8];
} mqp_server_options;

typedef struct mqp_server_stats {
  int64_t completed, failed, queued, running;
  int64_t admitted_while_busy;  /* requests admitted while other slots were running */
  double p50_ms, p99_ms, max_ms; /* submit -> result latency of completed requests */
  int64_t ia_done;
  double ia_per_s;              /* completed IAs / (last completion - first submit) */
  int64_t budget_bytes, in_use_bytes;
  double wait_p50_ms, wait_p99_ms; /* submit -> issue to a slot (queued) */
  double run_p50_ms, run_p99_ms;   /* issue -> finished (on the device) */
} mqp_server_stats;

MQP_API int mqp_server_create(int device, const mqp_server_options* opt /* NULL = defaults */, mqp_server** out);
/* A stream: its first frame (host, column-major) and the parameters of every request. */
MQP_API int mqp_server_open_stream(mqp_server* srv, const void* first_frame, int dtype, int ndims, const int64_t dims[3],
                                   const mqp_params* p, int32_t* stream_id);
/* Queue PIV(previous frame, frame) of a stream; returns immediately. */
MQP_API int mqp_server_submit(mqp_server* srv, int32_t stream_id, const void* frame, uint64_t* request_id);
/* Collect a request's VF/SN (host, shapes as mqp_piv) and its latency: wait_ms = 0 polls
 * (MQP_ERR_BUSY while running), < 0 waits, > 0 waits at most that long (MQP_ERR_TIMEOUT). */
MQP_API int mqp_server_result(mqp_server* srv, uint64_t request_id, int32_t wait_ms, double* VF, double* SN,
                              double* latency_ms);
MQP_API int mqp_server_get_stats(mqp_server* srv, mqp_server_stats* out);
MQP_API int mqp_server_reset_stats(mqp_server* srv);
MQP_API const char* mqp_server_last_error(const mqp_server* srv);
MQP_API int mqp_server_destroy(mqp_server* srv);

/*
 * Vector-field post-processing: the local-window operations of
 * src/postprocessing/postprocessing.jl on a Float64 field of `ncomp`
 * components over an `ndims`-D grid (column-major, component fastest: the
 * VF array PIV returns; a scalar map has ncomp = 1).  Windows of half-size
 * `radius` are clamped at the field border as localOp does
 * (postprocessing.jl:62-72).  Which input/outputs each op uses:
 *
 *   op                         replaces (postprocessing.jl)          in      out
 *   MQP_POST_MAGNITUDES        magnitudes(VF)             :184-192   VF      d_out (dims)
 *   MQP_POST_AVERAGE           average(radius, VF)        :364-381   VF      d_out (ncomp, dims)
 *   MQP_POST_SIMILARITY_AVG    similarityAveraging        :475-523   VF      d_out (ncomp, dims)
 *   MQP_POST_COLLECTIVENESS    collectiveness(radius, VF) :291-331   VF      d_outf (dims, Float32)
 *   MQP_POST_TH_MASK           TH_masking(th, map; cmp)   :660-670   map     d_mask_out
 *   MQP_POST_STD_MASK          STD_masking(n, map)        :598-609   map     d_mask_out
 *   MQP_POST_REPLACE           the replacement step of STD_filtering / TH_filtering /
 *                              remove_low_SN (:630-643, :692-706, :723-732)
 *                                                                    VF,mask d_out (ncomp, dims)
 *   MQP_POST_LOCAL_MAGNITUDE   local_magnitude_mask       :202-218   VF      d_out, d_mask_out (removed)
 *   MQP_POST_MATLAB_DIVERGENCE matlab_divergence(VF)      :918-941   VF      d_outf (dims, Float32)
 *   MQP_POST_DIVERGENCE        divergence(radii, VF; ...) :853-903   VF      d_out (dims)
 *
 * TH_filtering, remove_low_SN, divergence and the default replaceFun of
 * STD_filtering cannot run in the reference (see each op's notes in the
 * library source); these entries compute what they were written to compute.
 */
#define MQP_POST_MAGNITUDES 0
#define MQP_POST_AVERAGE 1
#define MQP_POST_SIMILARITY_AVG 2
#define MQP_POST_COLLECTIVENESS 3
#define MQP_POST_TH_MASK 4
#define MQP_POST_STD_MASK 5
#define MQP_POST_REPLACE 6
#define MQP_POST_LOCAL_MAGNITUDE 7
#define MQP_POST_MATLAB_DIVERGENCE 8
#define MQP_POST_DIVERGENCE 9

#define MQP_REPLACE_ZERO 0   /* zeroReplace */
#define MQP_REPLACE_MEDIAN 1 /* medianReplace */
#define MQP_REPLACE_MEAN 2   /* meanReplace: the window mean its docstring describes */

#define MQP_DIVIDE_NONE 0
#define MQP_DIVIDE_N 1       /* divide_by = "N" */
#define MQP_DIVIDE_MAGS 2    /* divide_by = "mags" */

typedef struct mqp_field {
  int32_t ncomp;    /* components per vector (1 = scalar map) */
  int32_t ndims;    /* grid dimensions, 1..4 */
  int64_t dims[4];  /* grid size (unused entries ignored) */
} mqp_field;

typedef struct mqp_post_params {
  int32_t op;                   /* MQP_POST_* */
  int32_t radius[4];            /* window half-size per grid axis (divergence: the sink radii) */
  double max_angle;             /* degrees: collectiveness (default 40), similarityAveraging (20) */
  int32_t normalize;            /* similarityAveraging (default 1), divergence (default 0) */
  int32_t scale_by_similarity;  /* similarityAveraging (default 1) */
  double similarity_exponent;   /* similarityAveraging (default 2) */
  double threshold;             /* TH_MASK: th; STD_MASK: n; LOCAL_MAGNITUDE: ratio */
  int32_t cmp;                  /* TH_MASK: 0 = (x > th), 1 = (x < th) */
  int32_t replace;              /* REPLACE: MQP_REPLACE_* */
  double min_speed;             /* divergence (default 0) */
  int32_t divide_by;            /* divergence: MQP_DIVIDE_* (default N) */
  int32_t circle;               /* divergence (default 0) */
  int32_t reserved[8];
} mqp_post_params;

/* On device arrays, enqueued on `stream` (NULL = legacy default stream). */
MQP_API int mqp_postprocess_device(mqp_ctx* ctx, const mqp_post_params* p, const mqp_field* f, const double* d_in,
                                   const uint8_t* d_mask, double* d_out, float* d_outf, uint8_t* d_mask_out,
                                   void* stream);
/* The same on host arrays (copied through the context's device buffers; blocks). */
MQP_API int mqp_postprocess(mqp_ctx* ctx, const mqp_post_params* p, const mqp_field* f, const double* in,
                            const uint8_t* mask, double* out, float* outf, uint8_t* mask_out);

/*
 * Pseudo-trajectories over a vector-field time series: PIVtrajectories and
 * PIVtrajectories_grid (src/postprocessing/postprocessing.jl:988-1120).  The
 * field components U, V (and W in 3D) are column-major arrays of `dtype`
 * with extents (dims[0], dims[1][, dims[2]], frames), as the reference's 4-D
 * U, V, W (a 2-D field over time, U and V only, is this build's extension).
 * Each particle starts at an integer position of the sampling region, moves
 * by the displacement sampled at its rounded position (Float32 positions,
 * round to nearest with ties to even, the reference's round(Int64, x)) and
 * stops, its remaining positions frozen, when the rounded position leaves
 * the field.  Positions are 1-based like the reference's.  Outputs TY, TX
 * (TZ) are Float32 (numT, numpoints) column-major, numT = T1 - T0.
 *
 *  - T0, T1: 1-based frames; frames T0 .. T1-1 must exist (the last step
 *    samples frame T1-1, as the reference does).
 *  - sub_lo[d] > sub_hi[d] selects the reference's default 2 : dims[d]-1;
 *    otherwise the 1-based inclusive range sub_lo[d] : sub_hi[d] (grid: with
 *    step[d]).
 *  - grid = 0: numpoints random starting positions.  Julia's `rand` stream is
 *    not reproducible outside Julia, so a counter-based generator replaces
 *    it: start along axis d = lo + step * (splitmix64(seed + (3p+d+1) *
 *    0x9E3779B97F4A7C15) mod len).  grid = 1: every point of the sampling
 *    grid, y fastest (the reference's loop order); numpoints is ignored and
 *    mqp_traj_count gives the count.
 *  - scale[d] multiplies component d (in FP64, then rounded to Float32, as
 *    Julia's Float32(scale * U[...]) with a Float64 field).
 *  - A non-finite rounded position counts as leaving the field (the reference
 *    throws InexactError there).
 */
typedef struct mqp_traj_params {
  int32_t ndims;      /* 2 or 3 */
  int64_t dims[3];    /* grid extents of one frame */
  int64_t frames;     /* frames in the arrays */
  int32_t T0, T1;
  int64_t sub_lo[3], sub_hi[3], step[3];
  double scale[3];
  int32_t grid;
  int64_t numpoints;
  uint64_t seed;
  int32_t reserved[8];
} mqp_traj_params;

/* Particles a request follows (numpoints, or the grid's point count). */
MQP_API int mqp_traj_count(const mqp_traj_params* p, int64_t* numpoints_out);
/* On device arrays, enqueued on `stream` (NULL = legacy default stream). */
MQP_API int mqp_trajectories_device(mqp_ctx* ctx, const mqp_traj_params* p, int dtype, const void* d_U,
                                    const void* d_V, const void* d_W, float* d_TY, float* d_TX, float* d_TZ,
                                    void* stream);
/* The same on host arrays (only frames T0 .. T1-1 are copied; blocks). */
MQP_API int mqp_trajectories(mqp_ctx* ctx, const mqp_traj_params* p, int dtype, const void* U, const void* V,
                             const void* W, float* TY, float* TX, float* TZ);

/*
 * Time-lapse ingest.  A multi-page TIFF reader (the reference reads its 2D+t
 * and 3D+t stacks with LIBTIFF, README.md:55-68): classic TIFF in either byte
 * order, one sample per pixel, strips or tiles, no compression or PackBits,
 * 8/16/32-bit unsigned or signed integers and 32/64-bit floats.  Pages come
 * back in Julia's array order: page k of height H and width W is the
 * column-major H x W array at dst + k*H*W (dimension 1 = image rows).
 */
typedef struct mqp_tiff mqp_tiff;
typedef struct mqp_tiff_info {
  int64_t width, height, pages;   /* of page 0; pages in the file */
  int32_t bits, sample_format;    /* BitsPerSample; SampleFormat 1 uint, 2 int, 3 float */
  int32_t compression, tiled;     /* 1 none, 32773 PackBits; strips (0) or tiles (1) */
  int32_t uniform;                /* 1 when every page has page 0's size */
} mqp_tiff_info;

/* Opens (maps) a file; on failure *out may still hold a handle whose
 * mqp_tiff_last_error says why (close it). */
MQP_API int mqp_tiff_open(const char* path, mqp_tiff** out);
MQP_API int mqp_tiff_get_info(const mqp_tiff* t, mqp_tiff_info* info);
/* Pages [first_page, first_page + npages), all of one size, converted to
 * dtype (MQP_F32 / MQP_F64) into dst (H*W*npages elements). */
MQP_API int mqp_tiff_read(mqp_tiff* t, int64_t first_page, int64_t npages, int dtype, void* dst);
MQP_API const char* mqp_tiff_last_error(const mqp_tiff* t);
MQP_API int mqp_tiff_close(mqp_tiff* t);

/* A time-lapse frame source over a TIFF stack: frames of pages_per_frame
 * consecutive pages (1 for 2D+t, the depth for 3D+t), read ahead by a thread
 * into a ring of `ring` host buffers, pinned when a CUDA device is present
 * (so their copies to the device run at full speed).  mqp_frame_source_next
 * blocks until the next frame is read and returns it; the pointer stays
 * valid until the following call.  MQP_ERR_NOT_FOUND after the last frame
 * (trailing pages that do not fill a frame are ignored). */
typedef struct mqp_frame_source mqp_frame_source;
MQP_API int mqp_frame_source_create(const char* path, int64_t pages_per_frame, int dtype, int ring,
                                    mqp_frame_source** out);
/* frames in the stack, a frame's dims (H, W, pages_per_frame), pinned or not */
MQP_API int mqp_frame_source_info(const mqp_frame_source* s, int64_t* frames, int64_t dims[3], int32_t* pinned);
MQP_API int mqp_frame_source_next(mqp_frame_source* s, const void** frame, int64_t* index);
MQP_API const char* mqp_frame_source_last_error(const mqp_frame_source* s);
MQP_API int mqp_frame_source_destroy(mqp_frame_source* s);

/*
 * Allocation-free 2D PIV.  No counterpart in the reference: it exists for
 * callers that cannot allocate GPU memory when they compute a vector field
 * (code running under a framework that owns all device memory through its
 * own pool, real-time loops that must not meet cudaMalloc's implicit
 * synchronisation or failure mid-run, hosts that budget every device byte
 * up front).  It computes what mqp_piv_device computes for 2D images
 * (FFTCC, ZNCC, NSQECC; no mask) on caller-owned device arrays, without a
 * context and without allocating: its only scratch is a fixed array of
 * MQP_NOALLOC_SCRATCH_BYTES built into the library, which every GPU that
 * loads the library holds until the process exits.
 *
 *  - Scratch needed: NSQECC one, ZNCC three FP64 integral images of
 *    (dims[0]+1) x (dims[1]+1) doubles plus about 1/8 of one for scan totals;
 *    FFTCC none.  48 MiB covers NSQECC up to about 2400 x 2400 and ZNCC up to
 *    about 1400 x 1400.  Larger images are rejected with MQP_ERR_INVALID and
 *    a message; use mqp_piv_device for them.
 *  - The first call on a device looks up the scratch array's device address
 *    (with that device current); later calls look it up again unless their
 *    stream is capturing, in which case the address cached by an earlier
 *    call is used: make the first call on a device before any stream capture.
 *  - One pass only: refine with multipass > 1 (the coarse-to-fine passes of
 *    mqp_piv_device, which keep predictors between passes) returns
 *    MQP_ERR_UNSUPPORTED; multipass < 1 returns MQP_ERR_INVALID.  An empty
 *    vector field returns MQP_OK without touching d_VF (which may be NULL).
 *  - All calls share the one scratch array and it keeps the last call's
 *    contents (every element is rewritten before it is read, so nothing needs
 *    clearing).  Calls whose GPU work overlaps (different streams, or
 *    different host threads on one device) race on it: serialise them.
 *  - Work is enqueued on `stream` (NULL = the legacy default stream); errors
 *    are written to err (errlen bytes, may be NULL) and returned as MQP_ERR_*.
 */
#define MQP_NOALLOC_SCRATCH_BYTES (48u * 1024u * 1024u)

MQP_API int mqp_piv2d_noalloc(const void* d_img1, const void* d_img2, int dtype, const int64_t dims[2],
                              const mqp_params* p, double* d_VF, double* d_SN, void* stream, char* err,
                              int errlen);

#ifdef __cplusplus
}
#endif

#endif /* MQP_H */
