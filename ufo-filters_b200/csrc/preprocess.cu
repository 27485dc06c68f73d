// The tasks in front of `fft` in a reconstruction graph: flat-field
// correction, projection -> sinogram transposition and the cone-beam
// projection weight.
//
// Reference behaviour restated here:
//  * src/kernels/ffc.cl:20-50, src/ufo-flat-field-correct-task.c:120-170 --
//    per element (data - dark*ds) / (flat*fs - dark*ds), or with
//    absorption-correct log((flat*fs - dark*ds) / (data - dark*ds)); NaN/Inf
//    optionally replaced by 0; with sinogram-input the dark/flat are one row.
//  * src/ufo-transpose-projections-task.c:60-120 -- row y of projection p
//    becomes row p of sinogram y (a host-side OpenMP memcpy there).
//  * src/ufo-cone-beam-projection-weight-task.c:113-151,
//    src/kernels/conebeam.cl:20-36 -- per projection (FP32 constants from the
//    double properties of index `count`, a single value broadcasting), element
//    (x, y) is multiplied by sd * cos(axis-angle-x) / sqrt(od^2 + u^2 + v^2)
//    with u = (x - cx + 1/2) * sd / (sd + dd), v likewise with cz, and od =
//    sd + dd, or sd when cos(axis-angle-x) > 0.9999999.
//
// B200 formulation.  All three are one row-wise, HBM-bound pass described by a
// RowSource (where logical row r starts and which per-element steps apply).
// The same description drives the filter stage's loads, so in a graph the
// steps cost no pass of their own: raw projections are read once, corrected,
// weighted, transposed and filtered in one kernel.  On their own (drop-in for
// each task) they run through k_rows_pre: 16-byte vector loads and stores when
// rows and pointers allow, two vectors per thread in flight.
#include <math.h>

#include <algorithm>
#include <cmath>

#include "ufob_internal.h"

namespace ufob {

static constexpr int kPreThreads = 256;
static constexpr int kPreItems = 2;  // vectors per thread

// Logical row r of `src` to out + outer * out_outer + inner * out_inner.
// blockIdx.x = row * segs + segment; a segment is kPreThreads * kPreItems vectors.
template <int VEC, bool PRE>
__global__ void __launch_bounds__(kPreThreads) k_rows_pre(const RowSource src, uint32_t width, uint64_t rows,
                                                          uint32_t segs, float *__restrict__ out, uint64_t out_outer,
                                                          uint64_t out_inner)
{
    const uint64_t b = blockIdx.x + (uint64_t)blockIdx.y * gridDim.x;
    const uint64_t r = b / segs;
    if (r >= rows) return;
    const uint32_t seg = (uint32_t)(b - r * segs);
    uint32_t y, p;
    const float *in = row_start(src, (uint32_t)r, y, p);
    const uint32_t o = (uint32_t)r / src.n_inner, i = (uint32_t)r - o * src.n_inner;
    float *dst = out + o * out_outer + i * out_inner;
    const uint32_t x0 = (seg * kPreThreads * kPreItems + threadIdx.x) * VEC;
    if (VEC == 4) {
        float4 v[kPreItems];
#pragma unroll
        for (int k = 0; k < kPreItems; k++) {
            const uint32_t x = x0 + k * kPreThreads * 4;
            if (x < width) v[k] = __ldg(reinterpret_cast<const float4 *>(in + x));
        }
#pragma unroll
        for (int k = 0; k < kPreItems; k++) {
            const uint32_t x = x0 + k * kPreThreads * 4;
            if (x >= width) continue;
            if (PRE) {
                v[k].x = preprocess_value(src, v[k].x, x, y, p);
                v[k].y = preprocess_value(src, v[k].y, x + 1, y, p);
                v[k].z = preprocess_value(src, v[k].z, x + 2, y, p);
                v[k].w = preprocess_value(src, v[k].w, x + 3, y, p);
            }
            *reinterpret_cast<float4 *>(dst + x) = v[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPreItems; k++) {
            const uint32_t x = x0 + k * kPreThreads;
            if (x >= width) continue;
            float v = __ldg(in + x);
            if (PRE) v = preprocess_value(src, v, x, y, p);
            dst[x] = v;
        }
    }
}

template <int VEC, bool PRE>
static ufob_status launch_pre(const RowSource &src, uint32_t width, uint64_t rows, float *out, uint64_t out_outer,
                              uint64_t out_inner, cudaStream_t s)
{
    const uint32_t per_block = kPreThreads * kPreItems * VEC;
    const uint32_t segs = (width + per_block - 1) / per_block;
    const uint64_t blocks = rows * segs;
    // 2-D grid: x up to 2^31 - 1 blocks, y covers the rest
    const uint32_t gx = (uint32_t)std::min<uint64_t>(blocks, 1u << 30);
    const uint64_t gy = (blocks + gx - 1) / gx;
    if (gy > 65535) return fail(UFOB_ERR_UNSUPPORTED, "preprocess: %llu rows are too many for one launch",
                                (unsigned long long)rows);
    k_rows_pre<VEC, PRE><<<dim3(gx, (uint32_t)gy), kPreThreads, 0, s>>>(src, width, rows, segs, out, out_outer,
                                                                        out_inner);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

ufob_status rows_pre_launch(const RowSource &src, uint32_t width, uint64_t rows, float *out, uint64_t out_outer,
                            uint64_t out_inner, cudaStream_t s)
{
    if (!width || !rows) return UFOB_OK;
    if (rows > 0xffffffffull) return fail(UFOB_ERR_UNSUPPORTED, "preprocess: more than 2^32 rows");
    // vector path: every row start and the dark/flat rows 16-byte aligned, width a multiple of 4
    const bool vec = (width % 4 == 0) && ((uintptr_t)src.base % 16 == 0) && ((uintptr_t)out % 16 == 0) &&
                     (src.outer_stride % 4 == 0) && (src.inner_stride % 4 == 0) && (out_outer % 4 == 0) &&
                     (out_inner % 4 == 0);
    const bool pre = src.has_pre();
    if (vec) return pre ? launch_pre<4, true>(src, width, rows, out, out_outer, out_inner, s)
                        : launch_pre<4, false>(src, width, rows, out, out_outer, out_inner, s);
    return pre ? launch_pre<1, true>(src, width, rows, out, out_outer, out_inner, s)
               : launch_pre<1, false>(src, width, rows, out, out_outer, out_inner, s);
}

}  // namespace ufob

using namespace ufob;

// ------------------------------------------------------------ cone-beam weight handle

namespace {
const char *const kConeNames[5] = {"center-position-x", "center-position-z", "source-distance", "detector-distance",
                                   "axis-angle-x"};
bool name_eq(const char *a, const char *b)
{
    if (!a) return false;
    for (; *a && *b; a++, b++)
        if (!(*a == *b || (*a == '_' && *b == '-'))) return false;
    return *a == *b;
}
int cone_col(const char *name)
{
    for (int i = 0; i < 5; i++)
        if (name_eq(name, kConeNames[i])) return i;
    return -1;
}
}  // namespace

struct ufob_cone_weight {
    // src/ufo-cone-beam-projection-weight-task.c:302-309: four arrays start empty, axis-angle-x = {0}
    std::vector<double> v[5] = {{}, {}, {}, {}, {0.0}};
    uint32_t count = 0;
    std::vector<ConeParams> host;
    DevBuf d_params;
};

namespace ufob {

// FP32 constants of projections first .. first+n-1 (task.c:128-139), uploaded
// into the handle's device table.
ufob_status cone_params_upload(ufob_cone_weight *w, uint32_t first, uint32_t n, const ConeParams **d_out,
                               cudaStream_t s)
{
    for (int c = 0; c < 5; c++) {
        const size_t k = w->v[c].size();
        if (k == 0) return fail(UFOB_ERR_SETUP, "cone-beam-projection-weight: %s is not set", kConeNames[c]);
        if (k != 1 && k < (size_t)first + n)
            return fail(UFOB_ERR_INVALID, "cone-beam-projection-weight: %s has %zu values, projection %u needs more",
                        kConeNames[c], k, first + n - 1);
    }
    w->host.resize(n);
    for (uint32_t i = 0; i < n; i++) {
        auto at = [&](int c) { return w->v[c].size() == 1 ? w->v[c][0] : w->v[c][first + i]; };
        ConeParams &q = w->host[i];
        q.cs = (float)cos(at(4));
        q.cx = (float)at(0);
        q.cz = (float)at(1);
        q.sd = (float)at(2);
        const float dd = (float)at(3);
        float od = q.sd + dd;
        q.mr = q.sd / od;
        if (q.cs > 0.9999999f) od = q.sd;
        q.od = od;
        q.pad0 = q.pad1 = 0.f;
    }
    UFOB_TRY(w->d_params.ensure(sizeof(ConeParams) * std::max<uint32_t>(n, 1)));
    UFOB_CUDA_TRY(cudaMemcpyAsync(w->d_params.ptr, w->host.data(), sizeof(ConeParams) * n, cudaMemcpyHostToDevice, s));
    *d_out = w->d_params.as<ConeParams>();
    return UFOB_OK;
}

// Flat-field part of a RowSource from the task properties.
static ufob_status set_ffc(RowSource &src, const ufob_ffc_props *p, const float *dark, const float *flat,
                          uint32_t width)
{
    if (!dark || !flat) return fail(UFOB_ERR_INVALID, "flat-field-correct: dark and flat are required");
    src.dark = dark;
    src.flat = flat;
    src.corr_pitch = p->sinogram_input ? 0 : width;
    src.dark_scale = p->dark_scale;
    src.flat_scale = p->flat_scale;
    src.absorption = p->absorption_correct != 0;
    src.fix_abnormal = p->fix_nan_and_inf != 0;
    return UFOB_OK;
}

// RowSource for projections [n][height][pitch]: detector rows first_row ..
// first_row + n_rows - 1, in projection order (sinograms = false) or as
// sinograms (true), with the steps of `pre`.
ufob_status projection_source(const ufob_preprocess *pre, const float *d_proj, uint32_t width, uint32_t height,
                              uint32_t n, uint32_t pitch, bool sinograms, uint32_t first_row, uint32_t n_rows,
                              RowSource &src, cudaStream_t s)
{
    if (first_row + (uint64_t)n_rows > height)
        return fail(UFOB_ERR_INVALID, "projections: rows %u..%u outside the height %u", first_row,
                    first_row + n_rows - 1, height);
    src = RowSource();
    src.base = d_proj + (size_t)first_row * pitch;
    if (sinograms) {  // r = row * n + projection
        src.n_inner = n;
        src.proj_inner = 1;
        src.outer_stride = pitch;
        src.inner_stride = (uint64_t)height * pitch;
    } else {  // r = projection * n_rows + row
        src.n_inner = n_rows;
        src.proj_inner = 0;
        src.outer_stride = (uint64_t)height * pitch;
        src.inner_stride = pitch;
    }
    src.y0 = first_row;
    if (pre && pre->ffc) {
        const size_t off = pre->ffc->sinogram_input ? 0 : (size_t)first_row * width;
        if (!pre->d_dark || !pre->d_flat) return fail(UFOB_ERR_INVALID, "flat-field-correct: dark and flat are required");
        UFOB_TRY(set_ffc(src, pre->ffc, pre->d_dark + off, pre->d_flat + off, width));
    }
    if (pre && pre->cone) {
        UFOB_TRY(cone_params_upload(pre->cone, pre->cone->count, n, &src.cone, s));
        pre->cone->count += n;
    }
    return UFOB_OK;
}

}  // namespace ufob

extern "C" {

void ufob_ffc_props_init(ufob_ffc_props *p)
{
    if (!p) return;
    // src/ufo-flat-field-correct-task.c:303-314
    p->fix_nan_and_inf = 0;
    p->absorption_correct = 0;
    p->sinogram_input = 0;
    p->dark_scale = 1.0f;
    p->flat_scale = 1.0f;
}

ufob_status ufob_ffc_set_property(ufob_ffc_props *p, const char *name, double value)
{
    if (!p) return fail(UFOB_ERR_INVALID, "ffc props are NULL");
    if (name_eq(name, "fix-nan-and-inf")) p->fix_nan_and_inf = value != 0.0;
    else if (name_eq(name, "absorption-correct")) p->absorption_correct = value != 0.0;
    else if (name_eq(name, "sinogram-input")) p->sinogram_input = value != 0.0;
    else if (name_eq(name, "dark-scale")) p->dark_scale = (float)value;
    else if (name_eq(name, "flat-scale")) p->flat_scale = (float)value;
    else return fail(UFOB_ERR_INVALID, "flat-field-correct: no property named '%s'", name ? name : "(null)");
    return UFOB_OK;
}

ufob_status ufob_flat_field_correct(const ufob_ffc_props *props, const float *d_data, const float *d_dark,
                                    const float *d_flat, uint32_t width, uint32_t height, uint32_t n_frames,
                                    float *d_out, void *stream)
{
    if (!props || !d_data || !d_out) return fail(UFOB_ERR_INVALID, "flat_field_correct: NULL argument");
    UFOB_TRY(ensure_device());
    RowSource src = plain_rows(d_data, width);
    UFOB_TRY(set_ffc(src, props, d_dark, d_flat, width));
    // row r of the stack is detector row r % height of its frame
    src.n_inner = height;
    src.outer_stride = (uint64_t)height * width;
    src.inner_stride = width;
    return rows_pre_launch(src, width, (uint64_t)height * n_frames, d_out, (uint64_t)height * width, width,
                           (cudaStream_t)stream);
}

ufob_status ufob_cone_weight_create(ufob_cone_weight **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "cone_weight_create: out is NULL");
    *out = new ufob_cone_weight;
    return UFOB_OK;
}

ufob_status ufob_cone_weight_set_array(ufob_cone_weight *w, const char *name, const double *values, uint32_t n)
{
    if (!w || (!values && n)) return fail(UFOB_ERR_INVALID, "cone_weight_set_array: NULL argument");
    const int c = cone_col(name);
    if (c < 0) return fail(UFOB_ERR_INVALID, "cone-beam-projection-weight: no property named '%s'", name ? name : "(null)");
    w->v[c].assign(values, values + n);
    return UFOB_OK;
}

ufob_status ufob_cone_weight_set_property(ufob_cone_weight *w, const char *name, double value)
{
    return ufob_cone_weight_set_array(w, name, &value, 1);
}

ufob_status ufob_cone_weight_run(ufob_cone_weight *w, const float *d_in, uint32_t width, uint32_t height, uint32_t n,
                                 float *d_out, void *stream)
{
    if (!w || !d_in || !d_out) return fail(UFOB_ERR_INVALID, "cone_weight_run: NULL argument");
    UFOB_TRY(ensure_device());
    if (!n || !width || !height) return UFOB_OK;
    ufob_preprocess pre = {nullptr, nullptr, nullptr, w};
    RowSource src;
    UFOB_TRY(projection_source(&pre, d_in, width, height, n, width, false, 0, height, src, (cudaStream_t)stream));
    return rows_pre_launch(src, width, (uint64_t)height * n, d_out, (uint64_t)height * width, width,
                           (cudaStream_t)stream);
}

ufob_status ufob_cone_weight_set_count(ufob_cone_weight *w, uint32_t count)
{
    if (!w) return fail(UFOB_ERR_INVALID, "cone weight handle is NULL");
    w->count = count;
    return UFOB_OK;
}

uint32_t ufob_cone_weight_get_count(const ufob_cone_weight *w) { return w ? w->count : 0; }

void ufob_cone_weight_destroy(ufob_cone_weight *w) { delete w; }

ufob_status ufob_transpose_projections(const float *d_proj, uint32_t width, uint32_t height, uint32_t n,
                                       float *d_sinos, uint32_t n_total, uint32_t first, void *stream)
{
    if (!d_proj || !d_sinos) return fail(UFOB_ERR_INVALID, "transpose_projections: NULL argument");
    if ((uint64_t)first + n > n_total)
        return fail(UFOB_ERR_INVALID, "transpose-projections: projections %u..%u exceed num-projections %u", first,
                    first + n - 1, n_total);
    UFOB_TRY(ensure_device());
    if (!n || !width || !height) return UFOB_OK;
    RowSource src;
    UFOB_TRY(projection_source(nullptr, d_proj, width, height, n, width, true, 0, height, src, (cudaStream_t)stream));
    // logical row (y, i) -> sinogram y, row first + i
    return rows_pre_launch(src, width, (uint64_t)height * n, d_sinos + (size_t)first * width,
                           (uint64_t)n_total * width, width, (cudaStream_t)stream);
}

}  // extern "C"
