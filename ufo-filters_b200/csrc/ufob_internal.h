// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/ufob.h"

namespace ufob {

// Thread-local error text returned by ufob_last_error().
void set_error(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
ufob_status fail(ufob_status st, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
ufob_status cuda_fail(cudaError_t e, const char *what);
ufob_status ensure_device();  // UFOB_ERR_CUDA unless an sm_100 device is current
int num_sms();
void note_launch(uint64_t n = 1);  // count kernels launched (ufob_launch_count)

#define UFOB_CUDA_TRY(expr)                                       \
    do {                                                          \
        cudaError_t _e = (expr);                                  \
        if (_e != cudaSuccess) return ::ufob::cuda_fail(_e, #expr); \
    } while (0)

// Raises a kernel's dynamic shared-memory limit on the current device, once per device: the
// attribute belongs to the device's context, so a process that drives several GPUs sets it on
// each of them.  `done` is the calling launcher's own record, one bit per device ordinal < 64
// (higher ordinals set the attribute on every call).
template <typename K>
inline cudaError_t smem_limit_per_device(K kern, int bytes, std::atomic<uint64_t> &done)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

#define UFOB_TRY(expr)                        \
    do {                                      \
        ufob_status _s = (expr);              \
        if (_s != UFOB_OK) return _s;         \
    } while (0)

// Device buffer owned by an engine object.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    ufob_status ensure(size_t n);  // grow to at least n bytes (contents not kept)
    template <typename T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

// Device error word: kernels with bounded waits record a code here instead of
// trapping.  0 = no error.
int *device_error_word();
ufob_status check_device_error_word(cudaStream_t stream);

inline uint32_t round_up(uint32_t v, uint32_t m) { return (v + m - 1) / m * m; }
inline bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }
inline int ilog2(uint64_t v) {
    int l = 0;
    while ((1ull << l) < v) l++;
    return l;
}

// ---------------------------------------------------------------- filter stage
struct FilterPlan {
    uint32_t nfft = 0;
    std::vector<float> coeff;  // 2*nfft interleaved coefficients, as the reference uploads
    DevBuf d_coeff;            // same on the device (float)
    DevBuf d_gains;            // float2 [nfft/2 + 1]: symmetrised per-bin gains
    DevBuf d_twiddle;          // float2 [nfft]: exp(-2 pi i m / nfft), FP64-computed
    DevBuf d_pass_tw;          // float2: per-pass twiddles of the register-radix kernel (256 <= nfft <= 4096)
};

// Host restatement of the reference's coefficient builders (before the
// ramp-fromreal transform).  Returns false and sets the error on bad width.
bool build_filter_coefficients(const ufob_filter_props &p, uint32_t nfft, std::vector<float> &coeff);
ufob_status filter_plan_build(const ufob_filter_props &p, uint32_t nfft, FilterPlan &plan, cudaStream_t stream);
ufob_status filter_rows_launch(const FilterPlan &plan, const float *d_in, uint32_t width, uint32_t rows,
                               uint32_t in_pitch, void *d_out, ufob_dtype out_dtype, ufob_layout out_layout,
                               uint32_t out_w, uint32_t out_pitch, cudaStream_t stream);
ufob_status filter_spectrum_launch(const float *d_coeff, const float *d_in, float *d_out, uint32_t width2,
                                   uint32_t rows, cudaStream_t stream);

// ---------------------------------------------------------------- preprocessing
// Per-projection constants of the cone-beam projection weight, computed in FP32
// on the host the way src/ufo-cone-beam-projection-weight-task.c:128-139 does.
struct ConeParams {
    float cx, cz;  // center-position-x/z
    float mr;      // source / (source + detector distance)
    float sd;      // source distance
    float od;      // source + detector distance (source distance when cos(axis-angle-x) ~ 1)
    float cs;      // cos(axis-angle-x)
    float pad0, pad1;
};

// Where logical row r of a row-wise stage comes from.  r = outer * n_inner +
// inner; the row starts at base + outer * outer_stride + inner * inner_stride
// floats.  Its (detector row, projection) is (outer, inner) when proj_inner is
// set (projections read as sinograms) and (inner, outer) otherwise.  Optional
// per-element steps, applied in the reference's graph order: flat-field
// correction (src/kernels/ffc.cl:20-50; dark/flat rows of corr_pitch floats
// indexed by the detector row, or one row for every detector row when
// corr_pitch is 0) and the cone-beam weight (src/kernels/conebeam.cl:20-36;
// detector row y0 + y, per-projection constants cone[projection]).
struct RowSource {
    const float *base = nullptr;
    uint64_t outer_stride = 0, inner_stride = 0;
    uint32_t n_inner = 1, proj_inner = 0;
    uint32_t y0 = 0;
    const float *dark = nullptr, *flat = nullptr;
    uint32_t corr_pitch = 0;
    float dark_scale = 1.f, flat_scale = 1.f;
    int absorption = 0, fix_abnormal = 0;
    const ConeParams *cone = nullptr;
    bool has_pre() const { return dark != nullptr || cone != nullptr; }
#ifdef __CUDACC__
    __host__ __device__
#endif
    RowSource cone_only() const  // the same source without its flat-field step
    {
        RowSource r = *this;
        r.dark = r.flat = nullptr;
        return r;
    }
};

#ifdef __CUDACC__
#define UFOB_HD __host__ __device__
#else
#define UFOB_HD
#endif

// Rows of `pitch` floats, one after another.
UFOB_HD inline RowSource plain_rows(const float *base, uint32_t pitch)
{
    RowSource s;
    s.base = base;
    s.outer_stride = pitch;
    return s;
}

#ifdef __CUDACC__
// Detector row `y` (relative to the dark/flat base) and projection `p` of one
// row; x = detector column.  FP32 with the reference's operation order, IEEE
// division and square root.
// Flat-field correction of value v with its dark and flat values (ffc.cl:31-45).
__device__ __forceinline__ float ffc_value(const RowSource &s, float v, float dark, float flat)
{
    const float cd = __fmul_rn(dark, s.dark_scale);
    const float cf = __fmul_rn(flat, s.flat_scale);
    v = s.absorption ? logf(__fdiv_rn(__fsub_rn(cf, cd), __fsub_rn(v, cd)))
                     : __fdiv_rn(__fsub_rn(v, cd), __fsub_rn(cf, cd));
    if (s.fix_abnormal && !isfinite(v)) v = 0.f;
    return v;
}

__device__ __forceinline__ float preprocess_value(const RowSource &s, float v, uint32_t x, uint32_t y, uint32_t p)
{
    if (s.dark) {
        const size_t i = (size_t)y * s.corr_pitch + x;
        v = ffc_value(s, v, __ldg(s.dark + i), __ldg(s.flat + i));
    }
    if (s.cone) {  // conebeam.cl:29-35
        const ConeParams c = s.cone[p];
        const float fx = __fmul_rn(__fadd_rn(__fsub_rn((float)x, c.cx), 0.5f), c.mr);
        const float fy = __fmul_rn(__fadd_rn(__fsub_rn((float)(s.y0 + y), c.cz), 0.5f), c.mr);
        const float den = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.od, c.od), __fmul_rn(fx, fx)), __fmul_rn(fy, fy)));
        v = __fdiv_rn(__fmul_rn(__fmul_rn(v, c.sd), c.cs), den);
    }
    return v;
}

// Start of logical row r and its (detector row, projection).
__device__ __forceinline__ const float *row_start(const RowSource &s, uint32_t r, uint32_t &y, uint32_t &p)
{
    const uint32_t o = r / s.n_inner, i = r - o * s.n_inner;
    y = s.proj_inner ? o : i;
    p = s.proj_inner ? i : o;
    return s.base + o * s.outer_stride + i * s.inner_stride;
}
#endif

// Filter stage over a general row source (see RowSource); rows = logical rows.
ufob_status filter_rows_launch_src(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t rows,
                                   void *d_out, ufob_dtype out_dtype, ufob_layout out_layout, uint32_t out_w,
                                   uint32_t out_pitch, cudaStream_t stream);
// Slice-quad output of `nz` sinograms of P rows, logical row = slice * P + angle.
ufob_status filter_quads_launch_src(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t P,
                                    uint32_t nz, void *d_out, uint32_t out_w, uint32_t out_pitch,
                                    cudaStream_t stream);
// RowSource for projections [n][height][pitch]: detector rows first_row ..
// first_row + n_rows - 1 in projection order (sinograms = false, r = projection
// * n_rows + row) or as sinograms (true, r = row * n + projection), with the
// steps of `pre` (its cone weight's count advances by n).
ufob_status projection_source(const ufob_preprocess *pre, const float *d_proj, uint32_t width, uint32_t height,
                              uint32_t n, uint32_t pitch, bool sinograms, uint32_t first_row, uint32_t n_rows,
                              RowSource &src, cudaStream_t s);
struct BPGeometry;
// stacked-backproject helpers: FP32 stack [Z][P][W] -> slice-quad cells
// [ceil(Z/4)][P][W+1]; the whole int8 path (d_work >= ceil(Z/4)*P*W words,
// d_keys = 2 words of device scratch).
ufob_status pack_quads_launch(const float *d_in, uint32_t W, uint32_t P, uint32_t Z, void *d_out, cudaStream_t s);
ufob_status stacked_u8_launch(const BPGeometry &g, const float *d_sino, void *d_work, uint32_t *d_keys, float *d_out,
                              cudaStream_t s);
// Row-wise preprocessing alone: logical row r of `src` (width floats) to
// out + outer * out_outer + inner * out_inner, with the same (outer, inner) split.
ufob_status rows_pre_launch(const RowSource &src, uint32_t width, uint64_t rows, float *out, uint64_t out_outer,
                            uint64_t out_inner, cudaStream_t stream);

// ------------------------------------------------------- parallel backprojection
struct BPGeometry {
    uint32_t W = 0, P = 0, nz = 0;  // sinogram width, rows used, slices
    uint32_t roi_x = 0, roi_y = 0, roi_w = 0, roi_h = 0;
    float axis = 0.f;
    float norm = 0.f;              // pi / P
    const float2 *d_sincos = nullptr;  // [P] (sin, cos) of the angles actually used
};

// sin/cos of angle_offset + (lut_offset + p) * step for p < P, in FP64 on the device.
ufob_status sincos_table_launch(double angle_offset, double step, uint32_t lut_offset, uint32_t P, float2 *d_out,
                                cudaStream_t stream, bool mirror = false);

enum SinoKind { SINO_F32 = 0, SINO_F16_PAIRS = 1, SINO_BF16_PAIRS = 2 };

ufob_status bp_linear_launch(const BPGeometry &g, const void *d_sino, SinoKind kind, uint32_t pitch,
                             uint64_t slice_pitch, float *d_out, bool kahan, int tile, cudaStream_t stream);
// One sinogram split into `groups` angle groups of height / groups rows (tile 8, slice z = group
// z), partial images summed into d_out; d_part holds groups x roi_h x roi_w floats.
ufob_status bp_linear_split_launch(const BPGeometry &g, const void *d_sino, SinoKind kind, uint32_t pitch,
                                   uint32_t groups, int tile, float *d_part, float *d_out, bool kahan,
                                   cudaStream_t stream);

// Slice-quad FP16 form (four slices' tap pairs per 16-byte cell): filter stage
// and backprojection.  acc: 0 FP32 accumulation of every product, 1 FP16 lerp
// + FP32 accumulation, 2 FP16 sums over 8-angle blocks + FP32 accumulation.
ufob_status filter_quads_launch(const FilterPlan &plan, const float *d_in, uint32_t width, uint32_t P, uint32_t nz,
                                uint32_t in_pitch, void *d_out, uint32_t out_w, uint32_t out_pitch,
                                cudaStream_t stream);
ufob_status bp_quads_launch(const BPGeometry &g, const void *d_sino, uint32_t pitch, uint64_t group_pitch,
                            float *d_out, bool kahan, int acc, int tile, cudaStream_t stream);
int bp_quad_tiles();

// Kernel arguments of one backprojection (one stack or one batch job).
struct BPArgs {
    uint32_t P, nz;
    uint32_t roi_x, roi_y, roi_w, roi_h;
    float axis, norm;
    const float2 *sincos;
    float *out;
    int *err;
    // angle-table entries between consecutive slices: 0 for a stack (all slices share the
    // angles); the group length when the slices are angle groups of one sinogram
    uint32_t sincos_zstride = 0;
};

// ------------------------------------------------------- uneven batches (persistent kernels)
// One job of the filter stage: its rows, FFT width and tables.
struct BatchFilter {
    const float *in;
    void *out;
    const float2 *tw, *gains;
    uint32_t width, rows, in_pitch, out_w, out_pitch, N;
    int log2N;
};
// One job of the backprojection stage: tensor map (64-byte aligned, in global
// memory), arguments and tile grid.
struct alignas(64) BatchBP {
    CUtensorMap map;
    BPArgs args;
    uint32_t tiles_x, tiles_y;
};
// filter stage over (job, row pair) items; out_kind: 0 F32 rows, 3 F16 pairs, 4 BF16 pairs
ufob_status filter_batch_launch(const BatchFilter *d_jobs, const uint2 *d_items, uint32_t n_items, uint32_t maxN,
                                uint32_t *d_counter, int out_kind, cudaStream_t s);
// backprojection stage over (job, tile) items with tile-shape variant `variant`
int bp_batch_variants();
void bp_batch_tile(int variant, int *tx, int *ty, int *window);
ufob_status bp_batch_launch(const BatchBP *d_jobs, const uint2 *d_items, uint32_t n_items, uint32_t *d_counter,
                            SinoKind kind, bool kahan, int variant, cudaStream_t s);
ufob_status make_sino_map(CUtensorMap *map, const void *base, uint32_t elems, uint32_t P, uint32_t nz,
                          uint32_t pitch, uint64_t slice_pitch, uint32_t box_x, uint32_t box_z);
ufob_status make_image_map(CUtensorMap *map, const void *base, uint32_t W, uint32_t H, uint32_t n, uint64_t pitch,
                           uint64_t plane, uint32_t box_w, uint32_t box_h);
ufob_status bp_nearest_launch(const BPGeometry &g, const float *d_sino, uint32_t pitch, uint64_t slice_pitch,
                              float *d_out, cudaStream_t stream);

}  // namespace ufob
