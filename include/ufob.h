/*
 * ufob.h -- C ABI of the B200 filtered-backprojection engine.
 *
 * The engine replaces the GPU work of three ufo-filters tasks on the FBP path:
 *   fft ! filter ! ifft   (the ramp-filter stage, fused into one kernel)
 *   backproject           (parallel beam)
 *   general-backproject   (parallel, cone and laminography)
 * Each task keeps the reference's property names, types, ranges and defaults;
 * the *_props structs below mirror the GObject properties field by field and
 * ufob_*_set_property() accepts the reference's property names as strings, so
 * a GObject plugin adapter can forward g_object_set() calls unchanged.
 *
 * Conventions
 *  - Every function returns ufob_status; on failure ufob_last_error() returns a
 *    thread-local message (the analogue of the reference's GError text).
 *  - Pointers named d_* are device pointers owned by the caller; the engine
 *    owns its plans, tables and workspaces and frees them in ufob_*_destroy().
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Work is enqueued asynchronously on it, like a task's in-order queue.
 *  - A handle may be used from one host thread at a time.
 *  - There is no CPU fallback: without a usable sm_100 device every run
 *    function fails with UFOB_ERR_CUDA.
 */
#ifndef UFOB_H
#define UFOB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UFOB_VERSION_MAJOR 0
#define UFOB_VERSION_MINOR 1

typedef enum {
    UFOB_OK = 0,
    UFOB_ERR_INVALID = 1,     /* bad argument or property value */
    UFOB_ERR_SETUP = 2,       /* UFO_TASK_ERROR_SETUP in the reference */
    UFOB_ERR_REQUISITION = 3, /* UFO_TASK_ERROR_GET_REQUISITION in the reference */
    UFOB_ERR_CUDA = 4,        /* CUDA runtime / launch failure, or no device */
    UFOB_ERR_NOMEM = 5,       /* device allocation failed */
    UFOB_ERR_TIMEOUT = 6,     /* a bounded device-side wait ran out */
    UFOB_ERR_UNSUPPORTED = 7  /* valid in the reference, not implemented here */
} ufob_status;

typedef enum {
    UFOB_F32 = 0,
    UFOB_F16 = 1,
    UFOB_BF16 = 2,
    UFOB_F64 = 3,
    UFOB_U8 = 4,
    UFOB_U16 = 5,
    UFOB_U32 = 6
} ufob_dtype;

const char *ufob_last_error(void);
const char *ufob_status_string(ufob_status status);
/* Returns UFOB_OK when a CUDA device of compute capability 10.x is usable. */
ufob_status ufob_device_check(int *cc_major, int *cc_minor, int *num_sms);
/* Synchronises the current device and reports (then clears) the device error
 * word that kernels with bounded waits set instead of trapping:
 * UFOB_ERR_TIMEOUT if a wait gave up since the last call. */
ufob_status ufob_device_status(void);

/* ------------------------------------------------------------------ filter
 * Fused `fft dimensions=1 [size-x] ! filter ! ifft dimensions=1 [crop-width]`.
 * Replaces: src/ufo-fft-task.c:123-336 (spread, forward FFT),
 *           src/ufo-filter-task.c:117-144,278-336 (coefficients, multiply),
 *           src/ufo-ifft-task.c:111-177,287-311 (backward FFT, crop, 1/N).
 */
typedef enum {
    UFOB_FILTER_RAMP = 0,          /* "ramp" */
    UFOB_FILTER_RAMP_FROMREAL = 1, /* "ramp-fromreal" (default) */
    UFOB_FILTER_BUTTERWORTH = 2,   /* "butterworth" */
    UFOB_FILTER_FARIS_BYER = 3,    /* "faris-byer" */
    UFOB_FILTER_HAMMING = 4,       /* "hamming" */
    UFOB_FILTER_BH3 = 5            /* "bh3" */
} ufob_filter_type;

/* Layout of filtered output rows (engine extension, not a reference property). */
typedef enum {
    UFOB_LAYOUT_ROWS = 0,  /* [rows][crop_width] of the output dtype */
    UFOB_LAYOUT_PAIRS = 1, /* [rows][pair_stride] 32-bit pairs (s[j-1], s[j]), F16/BF16 only;
                              pair_stride = round_up(crop_width + 1, 4) */
    UFOB_LAYOUT_QUADS = 2  /* F16 only, for a stack of sinograms: [ceil(nslices/4)][height][cells]
                              16-byte cells, cell j of group g holding the taps s[j-1], s[j] of
                              slices 4g..4g+3 as halves (s0[j-1], s1[j-1], s2[j-1], s3[j-1],
                              s0[j], s1[j], s2[j], s3[j]); cells >= crop_width + 1 */
} ufob_layout;

typedef struct {
    int filter;         /* ufob_filter_type, property "filter"; default ramp-fromreal */
    float cutoff;       /* "cutoff" [0,1], default 0.5 */
    float order;        /* "order" [2,32], default 4 (Butterworth) */
    float tau;          /* "tau", default 0.1 (Faris-Byer) */
    float theta;        /* "theta", default 1.0 (Faris-Byer) */
    float scale;        /* "scale", default 1.0 */
    uint32_t size_x;    /* fft "size-x" [0,32768], 0 = input width */
    uint32_t crop_width;/* ifft "crop-width" [0,32768], 0 = FFT width */
} ufob_filter_props;

typedef struct ufob_filter ufob_filter;

void ufob_filter_props_init(ufob_filter_props *props);
ufob_status ufob_filter_create(const ufob_filter_props *props, ufob_filter **out);
ufob_status ufob_filter_set_property(ufob_filter *f, const char *name, double value);
ufob_status ufob_filter_set_property_string(ufob_filter *f, const char *name, const char *value);
/* Output size for an input of `width` x `height` (get_requisition). */
ufob_status ufob_filter_get_requisition(ufob_filter *f, uint32_t width, uint32_t height,
                                        uint32_t *out_width, uint32_t *out_height);
/* Filter `rows` rows of `width` floats (row pitch in_pitch floats, 0 = width).
 * out_dtype F32/F16/BF16, out_layout per ufob_layout, out_pitch in elements
 * (0 = packed).  The interleaved coefficient vector the reference would upload
 * is available through ufob_filter_coefficients(). */
ufob_status ufob_filter_run(ufob_filter *f, const float *d_in, uint32_t width, uint32_t rows,
                            uint32_t in_pitch, void *d_out, ufob_dtype out_dtype, ufob_layout out_layout,
                            uint32_t out_pitch, void *stream);
/* Filter a stack [nslices][height][in_pitch] into the F16 QUADS layout
 * (cells per row out_pitch, 0 = crop_width + 1), the input of the fastest
 * half-precision backprojection. */
ufob_status ufob_filter_run_quads(ufob_filter *f, const float *d_in, uint32_t width, uint32_t height,
                                  uint32_t nslices, uint32_t in_pitch, void *d_out, uint32_t out_pitch,
                                  void *stream);
/* Host copy of the 2*nfft interleaved coefficients for an input of `width`. */
ufob_status ufob_filter_coefficients(ufob_filter *f, uint32_t width, float *host_out, uint32_t n);
/* The reference `filter` task alone: multiply complex-interleaved rows
 * [rows][2*nfft] element-wise by the coefficient vector (filter.cl:20-29). */
ufob_status ufob_filter_apply_spectrum(ufob_filter *f, const float *d_in, float *d_out, uint32_t width2,
                                       uint32_t rows, void *stream);
void ufob_filter_destroy(ufob_filter *f);

/* -------------------------------------------------------------- backproject
 * Parallel-beam backprojection.  Replaces src/ufo-backproject-task.c:96-267
 * and src/kernels/backproject.cl:24-94.
 */
typedef enum { UFOB_BP_NEAREST = 0, UFOB_BP_TEXTURE = 1 } ufob_bp_mode;

typedef struct {
    uint32_t num_projections; /* "num-projections", 0 = sinogram height */
    uint32_t offset;          /* "offset": first LUT entry used */
    double axis_pos;          /* "axis-pos", <= 0 means width / 2; default -1 */
    double angle_step;        /* "angle-step", <= 0 means pi / num-projections */
    double angle_offset;      /* "angle-offset" [rad] */
    int mode;                 /* "mode": ufob_bp_mode, default texture (linear) */
    uint32_t roi_x, roi_y;    /* "roi-x", "roi-y" */
    uint32_t roi_width;       /* "roi-width", 0 = sinogram width */
    uint32_t roi_height;      /* "roi-height", 0 = sinogram width */
    /* engine extensions */
    int compensated;          /* blocked Kahan over angle blocks: 1 on; 0 or -1 (default) off, since
                                 16-bit storage rounding outweighs the FP32 block sums' error */
    int tile;                 /* kernel shape id from the autotuner, -1 = automatic */
    int half_sums;            /* F16 QUADS sinograms only: 0 (default) every product accumulated in
                                 FP32; 1 interpolation and sums over blocks of 8 angles in packed
                                 FP16, block sums accumulated in FP32 (faster, larger error) */
    int angle_groups;         /* one F32/pair sinogram: 0 (default) automatic, 1 one launch, 2/4/8
                                 equal angle groups backprojected as slices of one launch whose
                                 partial images are summed in group order */
} ufob_bp_props;

typedef struct ufob_backproject ufob_backproject;

void ufob_bp_props_init(ufob_bp_props *props);
ufob_status ufob_backproject_create(const ufob_bp_props *props, ufob_backproject **out);
ufob_status ufob_backproject_set_property(ufob_backproject *bp, const char *name, double value);
ufob_status ufob_backproject_set_property_string(ufob_backproject *bp, const char *name, const char *value);
ufob_status ufob_backproject_get_requisition(ufob_backproject *bp, uint32_t width, uint32_t height,
                                             uint32_t *out_width, uint32_t *out_height);
/* Backproject `nslices` sinograms of `height` rows x `width` bins.
 * sino_dtype F32 with sino_layout ROWS (row pitch in floats, 0 = width), or
 * F16/BF16 with layout PAIRS as written by ufob_filter_run (pitch in pairs), or
 * F16 with layout QUADS as written by ufob_filter_run_quads (pitch in cells,
 * slice_pitch = cells per group of four slices).
 * Sinogram z starts at d_sino + z * slice_pitch elements (0 = height * pitch).
 * Output slice z is [roi_height][roi_width] floats at d_out + z * roi_w * roi_h. */
ufob_status ufob_backproject_run(ufob_backproject *bp, const void *d_sino, ufob_dtype sino_dtype,
                                 ufob_layout sino_layout, uint32_t width, uint32_t height, uint32_t nslices,
                                 uint32_t pitch, uint64_t slice_pitch, float *d_out, void *stream);
void ufob_backproject_destroy(ufob_backproject *bp);

/* Allocation-free backprojection (engine addition; it has no counterpart in
 * the reference).  For callers that cannot allocate device memory: hosts that
 * manage every byte of device memory in their own pool, and acquisition
 * pipelines that must not risk the device-wide synchronisation an allocation
 * can imply.  Same result as ufob_backproject_run() with the same properties
 * within round-off (a single sinogram is not split into angle groups here, so
 * its partial sums are added in another order), but stateless and without
 * any cudaMalloc/cudaFree: the only scratch, the per-angle sin/cos table,
 * lives in a fixed device array of UFOB_STATIC_MAX_ANGLES entries (256 KiB,
 * held by every GPU that loads the library until the process exits).
 *  - height (sinogram rows) must not exceed UFOB_STATIC_MAX_ANGLES;
 *  - sinogram rows must be 16-byte aligned (no restaging);
 *  - the first call on a device looks up the table's device address (set-up):
 *    make it before any stream capture;
 *  - all calls share the table and each rewrites it, so calls whose work
 *    overlaps on the GPU (unordered streams) race. */
#define UFOB_STATIC_MAX_ANGLES 32768
ufob_status ufob_backproject_run_static(const ufob_bp_props *props, const void *d_sino, ufob_dtype sino_dtype,
                                        ufob_layout sino_layout, uint32_t width, uint32_t height, uint32_t nslices,
                                        uint32_t pitch, uint64_t slice_pitch, float *d_out, void *stream);

/* ------------------------------------------------------- stacked-backproject
 * Replaces src/ufo-stacked-backproject-task.c (get_requisition :200-250,
 * process :302-430, properties :600-690) and src/kernels/stacked-backproject.cl.
 * Properties: "num-projections", "offset", "axis-pos", "angle-step",
 * "angle-offset", "roi-x", "roi-y", "roi-width", "roi-height" (as backproject)
 * and "precision-mode" (0 = int8, 1 = half, 2 = single; default single; nicks
 * "int8", "half", "single").  Input: a stack of sinograms [nslices][height]
 * [width] float32; output [nslices][roi_height][roi_width] float32.  The image
 * orientation is the stacked task's: h = bx cos - by sin + axis.  Unlike the
 * reference, slices past the last full group of 2 (single) or 4 (half, int8)
 * are reconstructed too (the reference leaves them unwritten).
 */
typedef struct ufob_stacked_bp ufob_stacked_bp;
ufob_status ufob_stacked_bp_create(ufob_stacked_bp **out);
ufob_status ufob_stacked_bp_set_property(ufob_stacked_bp *sb, const char *name, double value);
ufob_status ufob_stacked_bp_set_property_string(ufob_stacked_bp *sb, const char *name, const char *value);
ufob_status ufob_stacked_bp_get_requisition(ufob_stacked_bp *sb, uint32_t width, uint32_t height,
                                            uint32_t *out_width, uint32_t *out_height);
ufob_status ufob_stacked_bp_run(ufob_stacked_bp *sb, const float *d_sino, uint32_t width, uint32_t height,
                                uint32_t nslices, float *d_out, void *stream);
void ufob_stacked_bp_destroy(ufob_stacked_bp *sb);

/* ------------------------------------------------------------------- fbp
 * Whole `fft ! filter ! ifft ! backproject` chain for a stack of sinograms
 * [nslices][height][width] float32 -> [nslices][roi_h][roi_w] float32.
 * `storage` is the filtered-sinogram storage type (F32, F16 or BF16).  The
 * engine streams slice groups through its own workspace.  Host-pointer
 * variant: inputs/outputs in host memory (pinned or pageable), copies are
 * overlapped with compute on internal streams, in chunks of slices_per_chunk
 * slices (0 = 32); from 32 up, the first and the last chunk are 16 slices, so
 * the first compute waits for a short upload and little download trails the
 * last one.
 */
typedef struct ufob_fbp ufob_fbp;
ufob_status ufob_fbp_create(const ufob_filter_props *fprops, const ufob_bp_props *bprops, ufob_dtype storage,
                            ufob_fbp **out);
ufob_status ufob_fbp_run(ufob_fbp *fbp, const float *d_sino, uint32_t width, uint32_t height, uint32_t nslices,
                         float *d_out, void *stream);
ufob_status ufob_fbp_run_host(ufob_fbp *fbp, const float *h_sino, uint32_t width, uint32_t height,
                              uint32_t nslices, float *h_out, uint32_t slices_per_chunk);
ufob_status ufob_fbp_get_requisition(ufob_fbp *fbp, uint32_t width, uint32_t height, uint32_t *out_width,
                                     uint32_t *out_height);
/* Per-kernel timing: with timing enabled every filter and backprojection
 * launch of later runs is bracketed by CUDA events on its stream;
 * ufob_fbp_kernel_times() synchronises on them and returns the summed
 * durations and launch counts since timing was (re)enabled. */
ufob_status ufob_fbp_set_timing(ufob_fbp *fbp, int enable);
ufob_status ufob_fbp_kernel_times(ufob_fbp *fbp, double *filter_ms, uint32_t *filter_launches, double *bp_ms,
                                  uint32_t *bp_launches);
void ufob_fbp_destroy(ufob_fbp *fbp);

/* ------------------------------------------------------ general-backproject
 * Replaces src/ufo-general-backproject-task.c (setup :1411-1462,
 * get_requisition :1464-1587, process :1610-1706, generate :1708-1764).
 * Array-valued properties (the geometry, regions) are set with
 * ufob_gbp_set_array(); a single value broadcasts to all projections.
 */
typedef struct ufob_gbp ufob_gbp;
ufob_status ufob_gbp_create(ufob_gbp **out);
ufob_status ufob_gbp_set_property(ufob_gbp *g, const char *name, double value);
/* String properties as the reference's enums (parameter, compute-type, result-type, store-type,
 * addressing-mode), plus the engine property "interpolation": "exact" (default, FP32 weights)
 * or "texture" (the texture unit's linear filter with 8-bit weights, as the reference samples
 * on a GPU; FP32 compute type).  compute-type "half" rounds the projection samples to FP16
 * and keeps coordinates, weights and sums in FP32 (staged from a rounded FP32 copy where staging
 * applies, else through texture gathers of 16-bit texels); the reference's half type also
 * computes those in half precision.  The engine property "staging": "auto" (default) stages
 * each projection's detector window in shared memory by TMA where the geometry lets a z-column
 * of voxels share its detector column (float or half compute, float result/store types, exact
 * weights, parameter z, clamp addressing, width a multiple of 4), else samples through texture
 * gathers; "texture" always uses the gathers.
 * Both give the same values to FP32 rounding. */
ufob_status ufob_gbp_set_property_string(ufob_gbp *g, const char *name, const char *value);
ufob_status ufob_gbp_set_array(ufob_gbp *g, const char *name, const double *values, uint32_t n);
/* setup(): validates num-projections, gray mapping; builds angle tables. */
ufob_status ufob_gbp_setup(ufob_gbp *g);
/* Slice size and slice count for projections of width x height. */
ufob_status ufob_gbp_get_requisition(ufob_gbp *g, uint32_t width, uint32_t height, uint32_t *out_width,
                                     uint32_t *out_height, uint32_t *num_slices);
/* Reconstruct from all num-projections projections at once:
 * d_proj = [n][height][width] float32 (row pitch = width).  d_volume receives
 * [num_slices][out_h][out_w] of the store-type.  Equivalent to process() for
 * every projection followed by generate() for every slice. */
ufob_status ufob_gbp_run(ufob_gbp *g, const float *d_proj, uint32_t width, uint32_t height, void *d_volume,
                         void *stream);
/* Streaming form of the reductor: push one projection (process()), then read
 * slices out (generate()).  generate fails with UFOB_ERR_INVALID until all
 * num-projections projections were pushed, as the reference refuses output. */
ufob_status ufob_gbp_process(ufob_gbp *g, const float *d_projection, uint32_t width, uint32_t height,
                             void *stream);
ufob_status ufob_gbp_generate(ufob_gbp *g, void *d_slice, uint32_t index, void *stream);
void ufob_gbp_destroy(ufob_gbp *g);

/* ------------------------------------------------------- lamino-backproject
 * Replaces src/ufo-lamino-backproject-task.c (setup :164-237, get_requisition
 * :239-256, process :280-500, generate :502-517, properties :690-811) and the
 * kernels generated from src/kernels/templates/{z,center,lamino,roll}_template.in.
 * Numeric properties: "z", "num-projections", "overall-angle" (default pi),
 * "tomo-angle" (default unset: overall-angle * i / num-projections for
 * projection i), "lamino-angle", "roll-angle", "parameter" (0 z, 1 x-center,
 * 2 lamino-angle, 3 roll-angle; nicks "z", "x-center", "lamino-angle",
 * "roll-angle").  Array properties (ufob_lamino_set_array): "x-region",
 * "y-region" (3 integers from, to, step), "region" (3 floats: the swept
 * parameter), "projection-offset" (2 integers), "center" (2 floats).  String
 * property "addressing-mode" ("clamp" default, "clamp_to_edge", "none").
 * Output: [nz][ny][nx] float32, nx = (to - from - 1) / step + 1 of x-region
 * (likewise ny), nz = ceil((region.to - region.from) / region.step).
 */
typedef struct ufob_lamino ufob_lamino;
ufob_status ufob_lamino_create(ufob_lamino **out);
ufob_status ufob_lamino_set_property(ufob_lamino *l, const char *name, double value);
ufob_status ufob_lamino_set_property_string(ufob_lamino *l, const char *name, const char *value);
ufob_status ufob_lamino_set_array(ufob_lamino *l, const char *name, const double *values, uint32_t n);
ufob_status ufob_lamino_setup(ufob_lamino *l);
ufob_status ufob_lamino_get_requisition(ufob_lamino *l, uint32_t *nx, uint32_t *ny, uint32_t *nz);
/* All num-projections projections [n][height][width] at once (projection i is
 * the task's i-th process() call) -> the volume. */
ufob_status ufob_lamino_run(ufob_lamino *l, const float *d_proj, uint32_t width, uint32_t height, float *d_volume,
                            void *stream);
/* Streaming form of the reductor: process() per projection, then one
 * generate() of the whole volume (fails before all projections arrived). */
ufob_status ufob_lamino_process(ufob_lamino *l, const float *d_projection, uint32_t width, uint32_t height,
                                void *stream);
ufob_status ufob_lamino_generate(ufob_lamino *l, float *d_volume, void *stream);
void ufob_lamino_destroy(ufob_lamino *l);

/* ------------------------------------------------------------ batched jobs
 * Uneven batch of parallel-beam reconstructions run by one persistent kernel
 * over a device work queue (captured in a CUDA graph on first use).
 */
typedef struct {
    const float *d_sino;  /* [height][width] float32 */
    float *d_out;         /* [roi_height][roi_width] float32 */
    uint32_t width, height;
    double axis_pos;      /* <= 0: width / 2 */
    double angle_step;    /* <= 0: pi / height */
    double angle_offset;
} ufob_job;

/* Each job runs `fft size-x=N ! filter ! ifft crop-width=width ! backproject`
 * with N = fprops->size_x if set, else the next power of two >= width (the
 * filter needs a power-of-two spectrum), and a width x width output.  Rows
 * must be 16-byte aligned (width a multiple of 4).  The first run of a batch
 * autotunes the backprojection tile shape (cached on disk under
 * $UFOB_TUNE_CACHE or $HOME/.cache/ufob/tune.txt; UFOB_TUNE=0 skips tuning)
 * and captures the batch into a CUDA graph, replayed while the jobs' pointers,
 * sizes and geometry stay the same.  Engine addition: the reference runs one
 * task graph per item. */
typedef struct ufob_batch ufob_batch;
ufob_status ufob_batch_create(const ufob_filter_props *fprops, ufob_dtype storage, ufob_batch **out);
ufob_status ufob_batch_run(ufob_batch *b, const ufob_job *jobs, uint32_t n, void *stream);
/* Tile-shape variant the autotuner chose for the current batch (-1 before the first run). */
int ufob_batch_variant(ufob_batch *b);
/* Number of tile-shape variants, and pinning one of them (0 .. count-1) in place of the
 * autotuner (-1, the default, restores autotuning); takes effect at the next run. */
int ufob_batch_variants(void);
ufob_status ufob_batch_set_variant(ufob_batch *b, int variant);
void ufob_batch_destroy(ufob_batch *b);

/* ---------------------------------------------------------- preprocessing
 * The tasks in front of `fft` in a reconstruction graph, each on its own and
 * fused into the filter stage's row loads (ufob_filter_run_projections,
 * ufob_fbp_run_projections), so raw projections go to filtered sinograms in
 * one pass over HBM.
 *
 * flat-field-correct: replaces src/ufo-flat-field-correct-task.c:120-170 and
 * src/kernels/ffc.cl:20-50.  Properties (names, defaults as the reference): */
typedef struct {
    int fix_nan_and_inf;    /* "fix-nan-and-inf", default 0: NaN/Inf results become 0 */
    int absorption_correct; /* "absorption-correct", default 0: log(flat' / data') instead of data' / flat' */
    int sinogram_input;     /* "sinogram-input", default 0: dark and flat are one row of `width` */
    float dark_scale;       /* "dark-scale", default 1.0 */
    float flat_scale;       /* "flat-scale", default 1.0 */
} ufob_ffc_props;
void ufob_ffc_props_init(ufob_ffc_props *props);
/* Set one property by its reference name (booleans as 0/1). */
ufob_status ufob_ffc_set_property(ufob_ffc_props *props, const char *name, double value);
/* n_frames frames [n_frames][height][width] (or sinograms with sinogram_input)
 * corrected with one dark and one flat frame [height][width] (one row [width]
 * with sinogram_input): out = (data - dark * dark_scale) / (flat * flat_scale -
 * dark * dark_scale), or the log of the inverse ratio with absorption_correct. */
ufob_status ufob_flat_field_correct(const ufob_ffc_props *props, const float *d_data, const float *d_dark,
                                    const float *d_flat, uint32_t width, uint32_t height, uint32_t n_frames,
                                    float *d_out, void *stream);

/* cone-beam-projection-weight: replaces
 * src/ufo-cone-beam-projection-weight-task.c:113-151 and
 * src/kernels/conebeam.cl:20-36.  Array properties "center-position-x",
 * "center-position-z", "source-distance", "detector-distance" (no default: they
 * must be set) and "axis-angle-x" (default 0); a single value broadcasts, else
 * projection i uses value i.  The handle counts the projections it has weighted,
 * as the task's process() counter does. */
typedef struct ufob_cone_weight ufob_cone_weight;
ufob_status ufob_cone_weight_create(ufob_cone_weight **out);
ufob_status ufob_cone_weight_set_array(ufob_cone_weight *w, const char *name, const double *values, uint32_t n);
ufob_status ufob_cone_weight_set_property(ufob_cone_weight *w, const char *name, double value);
/* Weight projections [n][height][width] (projection indices count .. count+n-1;
 * count advances by n).  d_out may equal d_in. */
ufob_status ufob_cone_weight_run(ufob_cone_weight *w, const float *d_in, uint32_t width, uint32_t height,
                                 uint32_t n, float *d_out, void *stream);
/* Projection index the next run starts at (0 after create). */
ufob_status ufob_cone_weight_set_count(ufob_cone_weight *w, uint32_t count);
uint32_t ufob_cone_weight_get_count(const ufob_cone_weight *w);
void ufob_cone_weight_destroy(ufob_cone_weight *w);

/* transpose-projections: replaces src/ufo-transpose-projections-task.c:60-120
 * (an OpenMP row copy on the host there).  Projections [n][height][width] become
 * projections first .. first+n-1 of `height` sinograms [height][n_total][width]. */
ufob_status ufob_transpose_projections(const float *d_proj, uint32_t width, uint32_t height, uint32_t n,
                                       float *d_sinos, uint32_t n_total, uint32_t first, void *stream);

/* Preprocessing fused into a filter run.  NULL members switch a step off. */
typedef struct {
    const ufob_ffc_props *ffc;  /* flat-field correction with d_dark, d_flat */
    const float *d_dark;        /* [height][width], or [width] with ffc->sinogram_input */
    const float *d_flat;
    ufob_cone_weight *cone;     /* cone-beam weight; its count advances by n_projections */
} ufob_preprocess;

/* Filter projections [n_projections][height][width] (row pitch `pitch`, 0 =
 * width) after the steps of `pre` (NULL = none), for detector rows first_row ..
 * first_row + n_rows - 1 (n_rows 0 = the rest).
 *   sinograms = 0: output rows in projection order [n_projections][n_rows][..]
 *     (the FDK order: cone-beam-projection-weight ! fft ! filter ! ifft);
 *   sinograms = 1: output sinograms [n_rows][n_projections][..], i.e. the
 *     transpose-projections step fused into the loads; out_layout QUADS gives
 *     the slice-quad cells of that sinogram stack.
 * Output layouts and pitches as ufob_filter_run / ufob_filter_run_quads. */
ufob_status ufob_filter_run_projections(ufob_filter *f, const ufob_preprocess *pre, const float *d_proj,
                                        uint32_t width, uint32_t height, uint32_t n_projections, uint32_t pitch,
                                        int sinograms, uint32_t first_row, uint32_t n_rows, void *d_out,
                                        ufob_dtype out_dtype, ufob_layout out_layout, uint32_t out_pitch,
                                        void *stream);
/* `flat-field-correct ! transpose-projections ! fft ! filter ! ifft !
 * backproject` for detector rows first_row .. first_row + n_rows - 1 (n_rows 0 =
 * all) of projections [n_projections][height][width] on the device: one
 * reconstructed slice per detector row, [n_rows][roi_h][roi_w]. */
ufob_status ufob_fbp_run_projections(ufob_fbp *fbp, const ufob_preprocess *pre, const float *d_proj,
                                     uint32_t width, uint32_t height, uint32_t n_projections, uint32_t first_row,
                                     uint32_t n_rows, float *d_out, void *stream);

/* ------------------------------------------------------------- utilities */
/* Analytic parallel-beam projection of ellipses (rows cx, cy, a, b, phi, rho
 * in units where the reconstruction circle has radius 1) into [P][W] float
 * sinograms in pixel-length units: used to synthesise inputs on the device. */
ufob_status ufob_phantom_sinogram(const double *h_ellipses, uint32_t n_ellipses, uint32_t width,
                                  uint32_t n_angles, double angle_step, double axis, double scale, float *d_sino,
                                  void *stream);

/* Stack [nz][n_angles][width] of sinograms of an ellipsoid phantom (rows cx,
 * cy, cz, a, b, c, phi, rho; at most 64), slice z cutting the phantom at height
 * (z + 0.5 - nz/2) / scale. */
ufob_status ufob_phantom_stack(const double *h_ellipsoids, uint32_t n, uint32_t width, uint32_t n_angles,
                               uint32_t nslices, double angle_step, double axis, double scale, float *d_sino,
                               void *stream);
/* Parallel-beam forward projection of a width x width slice into
 * [n_angles][width] by unit-step ray marching with linear sampling; replaces
 * src/kernels/forwardproject.cl:24-58 (src/ufo-forwardproject-task.c). */
ufob_status ufob_forwardproject(const float *d_slice, uint32_t width, uint32_t n_angles, double axis_pos,
                                double angle_step, float *d_sino, void *stream);
/* Rasterise ellipse phantoms into [n_images][N][N]: image i uses rows
 * h_offsets[i] .. h_offsets[i+1]-1 of h_ellipses (cx, cy, a, b, phi, rho), pixel
 * centres mapped to ((x + 0.5 - axis) / scale, (y + 0.5 - axis) / scale),
 * supersample^2 samples per pixel. */
ufob_status ufob_phantom_images(const double *h_ellipses, const uint32_t *h_offsets, uint32_t n_images, uint32_t N,
                                double axis, double scale, int supersample, float *d_out, void *stream);
/* ------------------------------------------------------------------- sparse-view CNN
 * Engine addition with no counterpart in the reference: a 4-level U-Net
 * (32/64/128/256 channels, 3x3 convolutions, BF16 weights and activations,
 * FP32 accumulation on tcgen05 tensor cores) that corrects a 90-angle FBP slice
 * toward the dense (1800-angle) reconstruction.  Images are [B][H][W] FP32 on
 * the device, H and W multiples of 32 (4x space-to-depth, then 3 poolings).  Parameters/gradients/Adam moments are
 * exchanged as one FP32 vector: per layer (16->32, 32->64, 64->128, 128->256,
 * 256->128, 128->64, 64->32, 32->16) weights [Cout][9][Cin] then bias [Cout]. */
typedef struct ufob_cnn ufob_cnn;
ufob_status ufob_cnn_create(uint64_t seed, float scale, ufob_cnn **out);
void ufob_cnn_destroy(ufob_cnn *net);
/* out = fbp + scale * net(fbp / scale) */
ufob_status ufob_cnn_forward(ufob_cnn *net, const float *d_fbp, float *d_out, int batch, int height, int width,
                             void *stream);
/* The same network through the training kernels (NHWC activations); the
 * inference path above must agree with it to BF16 rounding. */
ufob_status ufob_cnn_forward_nhwc(ufob_cnn *net, const float *d_fbp, float *d_out, int batch, int height, int width,
                                  void *stream);
/* One Adam step (beta 0.9/0.999) on the mean squared error against d_target;
 * *loss_out (host, may be NULL) receives the loss before the step. */
ufob_status ufob_cnn_train_step(ufob_cnn *net, const float *d_fbp, const float *d_target, int batch, int height,
                                int width, float lr, double *loss_out, void *stream);
uint64_t ufob_cnn_num_params(void);
/* which: 0 parameters, 1 gradients of the last step (get only), 2 Adam m, 3 Adam v */
ufob_status ufob_cnn_get_state(ufob_cnn *net, int which, float *h_values, uint64_t n);
ufob_status ufob_cnn_set_state(ufob_cnn *net, int which, const float *h_values, uint64_t n);
int64_t ufob_cnn_get_step(const ufob_cnn *net);
ufob_status ufob_cnn_set_step(ufob_cnn *net, int64_t step);
/* The network's convolution primitives (NHWC BF16 activations, weights
 * [Cout][9][Cin] BF16, zero padding, tap t = 3*(dy+1) + (dx+1)).
 * forward: out = relu?(conv(in, w) + bias + residual), written as BF16 (d_out)
 * and/or FP32 (d_out_f32); channels multiples of 16 in [16, 256], Cin > 64 a
 * multiple of 64.  wgrad: d_dw[Cout][9][Cin] += sum over pixels of dz x in (FP32). */
ufob_status ufob_conv3x3_forward(const void *d_in, const void *d_w, const float *d_bias, const void *d_residual,
                                 void *d_out, float *d_out_f32, int nb, int h, int w, int cin, int cout, int relu,
                                 void *stream);
ufob_status ufob_conv3x3_wgrad(const void *d_in, const void *d_dz, float *d_dw, int nb, int h, int w, int cin,
                               int cout, void *stream);
/* Number of engine kernels launched by this process so far. */
uint64_t ufob_launch_count(void);
/* Number of device allocations (cudaMalloc) the engine has made in this
 * process so far; its workspaces grow on demand and are reused. */
uint64_t ufob_device_alloc_count(void);
/* Sustained shared-memory load bandwidth (GB/s, 32-bit conflict-free loads)
 * and FP32 FMA throughput (TFLOP/s) of the current device, measured by two
 * short micro-kernels: the on-chip ceilings of voxel-driven backprojection. */
ufob_status ufob_measure_peaks(double *smem_gbs, double *fp32_tflops);

#ifdef __cplusplus
}
#endif
#endif /* UFOB_H */
