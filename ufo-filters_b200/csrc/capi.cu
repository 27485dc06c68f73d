// C ABI: task objects mirroring the reference's `filter` (with its fft/ifft
// neighbours), `backproject` and the fused FBP chain.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <strings.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <string>

#include "ufob_internal.h"

namespace ufob {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

ufob_status fail(ufob_status st, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

ufob_status cuda_fail(cudaError_t e, const char *what)
{
    cudaGetLastError();  // clear a sticky launch error so the caller can retry with other sizes
    return fail(e == cudaErrorMemoryAllocation ? UFOB_ERR_NOMEM : UFOB_ERR_CUDA, "%s: %s (%s)", what,
                cudaGetErrorString(e), cudaGetErrorName(e));
}

static std::atomic<uint64_t> g_device_allocs{0};

ufob_status DevBuf::ensure(size_t n)
{
    if (n <= bytes && ptr) return UFOB_OK;
    release();
    if (!n) return UFOB_OK;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return cuda_fail(e, "cudaMalloc");
    }
    g_device_allocs.fetch_add(1, std::memory_order_relaxed);
    bytes = n;
    return UFOB_OK;
}

static int g_num_sms = 0;
static std::atomic<uint64_t> g_launches{0};

void note_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Checked once per device ordinal (cheap attribute queries; cudaGetDeviceProperties
// costs milliseconds and must stay off the per-call path).
static std::atomic<int> g_device_ok[64];

ufob_status ensure_device()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice (no usable CUDA device)");
    if (dev >= 0 && dev < 64 && g_device_ok[dev].load(std::memory_order_acquire)) return UFOB_OK;
    int major = 0, minor = 0, sms = 0;
    e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    if (major != 10)
        return fail(UFOB_ERR_CUDA, "device %d is sm_%d%d; this engine is built for sm_100a only", dev, major, minor);
    g_num_sms = sms;
    if (dev >= 0 && dev < 64) g_device_ok[dev].store(1, std::memory_order_release);
    return UFOB_OK;
}

int num_sms()
{
    if (!g_num_sms) ensure_device();
    return g_num_sms ? g_num_sms : 148;
}

__device__ int g_device_error = 0;

int *device_error_word()
{
    static std::atomic<int *> cached[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64) {
        int *c = cached[dev].load(std::memory_order_acquire);
        if (c) return c;
    }
    void *p = nullptr;
    cudaGetSymbolAddress(&p, g_device_error);
    if (dev >= 0 && dev < 64 && p) cached[dev].store(reinterpret_cast<int *>(p), std::memory_order_release);
    return reinterpret_cast<int *>(p);
}

ufob_status check_device_error_word(cudaStream_t stream)
{
    int v = 0, zero = 0;
    UFOB_CUDA_TRY(cudaMemcpyFromSymbolAsync(&v, g_device_error, sizeof v, 0, cudaMemcpyDeviceToHost, stream));
    UFOB_CUDA_TRY(cudaStreamSynchronize(stream));
    if (v) {
        UFOB_CUDA_TRY(cudaMemcpyToSymbol(g_device_error, &zero, sizeof zero));
        return fail(UFOB_ERR_TIMEOUT, "a device-side bounded wait gave up (code 0x%x)", v);
    }
    return UFOB_OK;
}

static bool streq(const char *a, const char *b) { return a && b && strcasecmp(a, b) == 0; }

// property names may use '-' or '_' (GObject canonicalises both)
static bool prop_is(const char *name, const char *canon)
{
    if (!name) return false;
    for (; *name && *canon; name++, canon++) {
        char a = *name == '_' ? '-' : *name;
        if (a != *canon) return false;
    }
    return *name == 0 && *canon == 0;
}

}  // namespace ufob

using namespace ufob;

// =================================================================== filter

struct ufob_filter {
    ufob_filter_props props;
    FilterPlan plan;
};

static const char *kFilterNames[] = {"ramp", "ramp-fromreal", "butterworth", "faris-byer", "hamming", "bh3"};

extern "C" {

const char *ufob_last_error(void) { return g_last_error.c_str(); }

const char *ufob_status_string(ufob_status s)
{
    switch (s) {
    case UFOB_OK: return "ok";
    case UFOB_ERR_INVALID: return "invalid argument";
    case UFOB_ERR_SETUP: return "setup error";
    case UFOB_ERR_REQUISITION: return "get_requisition error";
    case UFOB_ERR_CUDA: return "CUDA error";
    case UFOB_ERR_NOMEM: return "out of device memory";
    case UFOB_ERR_TIMEOUT: return "device wait timed out";
    case UFOB_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

ufob_status ufob_device_check(int *cc_major, int *cc_minor, int *nsm)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    if (cc_major) *cc_major = prop.major;
    if (cc_minor) *cc_minor = prop.minor;
    if (nsm) *nsm = prop.multiProcessorCount;
    return ensure_device();
}

void ufob_filter_props_init(ufob_filter_props *p)
{
    // src/ufo-filter-task.c:531-545, src/ufo-fft-task.c:541-568, src/ufo-ifft-task.c:496-515
    p->filter = UFOB_FILTER_RAMP_FROMREAL;
    p->cutoff = 0.5f;
    p->order = 4.0f;
    p->tau = 0.1f;
    p->theta = 1.0f;
    p->scale = 1.0f;
    p->size_x = 0;
    p->crop_width = 0;
}

static ufob_status validate_filter_props(const ufob_filter_props *p)
{
    if (p->filter < 0 || p->filter > UFOB_FILTER_BH3) return fail(UFOB_ERR_INVALID, "filter: unknown filter %d", p->filter);
    if (!(p->cutoff >= 0.f && p->cutoff <= 1.f)) return fail(UFOB_ERR_INVALID, "filter: cutoff %g outside [0, 1]", p->cutoff);
    if (!(p->order >= 2.f && p->order <= 32.f)) return fail(UFOB_ERR_INVALID, "filter: order %g outside [2, 32]", p->order);
    if (p->size_x > 32768) return fail(UFOB_ERR_INVALID, "fft: size-x %u outside [0, 32768]", p->size_x);
    if (p->crop_width > 32768) return fail(UFOB_ERR_INVALID, "ifft: crop-width %u outside [0, 32768]", p->crop_width);
    return UFOB_OK;
}

ufob_status ufob_filter_create(const ufob_filter_props *props, ufob_filter **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "filter_create: out is NULL");
    ufob_filter_props p;
    ufob_filter_props_init(&p);
    if (props) p = *props;
    UFOB_TRY(validate_filter_props(&p));
    ufob_filter *f = new ufob_filter;
    f->props = p;
    *out = f;
    return UFOB_OK;
}

ufob_status ufob_filter_set_property(ufob_filter *f, const char *name, double v)
{
    if (!f) return fail(UFOB_ERR_INVALID, "filter handle is NULL");
    ufob_filter_props p = f->props;
    if (prop_is(name, "filter")) p.filter = (int)v;
    else if (prop_is(name, "cutoff")) p.cutoff = (float)v;
    else if (prop_is(name, "order")) p.order = (float)v;
    else if (prop_is(name, "tau")) p.tau = (float)v;
    else if (prop_is(name, "theta")) p.theta = (float)v;
    else if (prop_is(name, "scale")) p.scale = (float)v;
    else if (prop_is(name, "size-x")) { if (v < 0 || v > 32768) return fail(UFOB_ERR_INVALID, "size-x out of range"); p.size_x = (uint32_t)v; }
    else if (prop_is(name, "crop-width")) { if (v < 0 || v > 32768) return fail(UFOB_ERR_INVALID, "crop-width out of range"); p.crop_width = (uint32_t)v; }
    else return fail(UFOB_ERR_INVALID, "filter: no property named '%s'", name ? name : "(null)");
    UFOB_TRY(validate_filter_props(&p));
    f->props = p;
    f->plan.nfft = 0;  // coefficients depend on every property
    f->plan.coeff.clear();
    return UFOB_OK;
}

ufob_status ufob_filter_set_property_string(ufob_filter *f, const char *name, const char *value)
{
    if (!f) return fail(UFOB_ERR_INVALID, "filter handle is NULL");
    if (prop_is(name, "filter")) {
        for (int i = 0; i < 6; i++)
            if (streq(value, kFilterNames[i])) return ufob_filter_set_property(f, name, i);
        return fail(UFOB_ERR_INVALID, "filter: unknown filter '%s'", value ? value : "(null)");
    }
    char *end = nullptr;
    double v = value ? strtod(value, &end) : 0.0;
    if (!value || end == value) return fail(UFOB_ERR_INVALID, "filter: '%s' is not a number", value ? value : "(null)");
    return ufob_filter_set_property(f, name, v);
}

static ufob_status filter_sizes(const ufob_filter_props &p, uint32_t width, uint32_t *nfft, uint32_t *out_w)
{
    if (!width) return fail(UFOB_ERR_REQUISITION, "fft: input width is 0");
    if (p.size_x && p.size_x < width)
        return fail(UFOB_ERR_REQUISITION, "Specified size must be greater than or equal to input size");
    uint32_t n = p.size_x ? p.size_x : width;
    if (!is_pow2(2ull * n))
        return fail(UFOB_ERR_REQUISITION, "Invalid filter input width %u, must be a power of two", 2 * n);
    if (p.crop_width > n) return fail(UFOB_ERR_REQUISITION, "Cropped size must be less than or equal to input size");
    *nfft = n;
    *out_w = p.crop_width ? p.crop_width : n;
    return UFOB_OK;
}

ufob_status ufob_filter_get_requisition(ufob_filter *f, uint32_t width, uint32_t height, uint32_t *ow, uint32_t *oh)
{
    if (!f) return fail(UFOB_ERR_INVALID, "filter handle is NULL");
    uint32_t n, w;
    UFOB_TRY(filter_sizes(f->props, width, &n, &w));
    if (ow) *ow = w;
    if (oh) *oh = height;
    return UFOB_OK;
}

ufob_status ufob_filter_run(ufob_filter *f, const float *d_in, uint32_t width, uint32_t rows, uint32_t in_pitch,
                            void *d_out, ufob_dtype out_dtype, ufob_layout out_layout, uint32_t out_pitch,
                            void *stream)
{
    if (!f || !d_in || !d_out) return fail(UFOB_ERR_INVALID, "filter_run: NULL argument");
    UFOB_TRY(ensure_device());
    uint32_t n, w;
    UFOB_TRY(filter_sizes(f->props, width, &n, &w));
    cudaStream_t s = (cudaStream_t)stream;
    UFOB_TRY(filter_plan_build(f->props, n, f->plan, s));
    if (!in_pitch) in_pitch = width;
    if (!out_pitch) out_pitch = out_layout == UFOB_LAYOUT_PAIRS ? round_up(w + 1, 4) : w;
    if (out_layout == UFOB_LAYOUT_QUADS)
        return fail(UFOB_ERR_INVALID, "filter: the QUADS layout needs the stack shape: use ufob_filter_run_quads");
    return filter_rows_launch(f->plan, d_in, width, rows, in_pitch, d_out, out_dtype, out_layout, w, out_pitch, s);
}

ufob_status ufob_filter_run_quads(ufob_filter *f, const float *d_in, uint32_t width, uint32_t height,
                                  uint32_t nslices, uint32_t in_pitch, void *d_out, uint32_t out_pitch, void *stream)
{
    if (!f || !d_in || !d_out) return fail(UFOB_ERR_INVALID, "filter_run_quads: NULL argument");
    UFOB_TRY(ensure_device());
    uint32_t n, w;
    UFOB_TRY(filter_sizes(f->props, width, &n, &w));
    cudaStream_t s = (cudaStream_t)stream;
    UFOB_TRY(filter_plan_build(f->props, n, f->plan, s));
    if (!in_pitch) in_pitch = width;
    if (!out_pitch) out_pitch = w + 1;
    if (!height || !nslices) return UFOB_OK;
    return filter_quads_launch(f->plan, d_in, width, height, nslices, in_pitch, d_out, w, out_pitch, s);
}

ufob_status ufob_filter_run_projections(ufob_filter *f, const ufob_preprocess *pre, const float *d_proj,
                                        uint32_t width, uint32_t height, uint32_t n_projections, uint32_t pitch,
                                        int sinograms, uint32_t first_row, uint32_t n_rows, void *d_out,
                                        ufob_dtype out_dtype, ufob_layout out_layout, uint32_t out_pitch,
                                        void *stream)
{
    if (!f || !d_proj || !d_out) return fail(UFOB_ERR_INVALID, "filter_run_projections: NULL argument");
    UFOB_TRY(ensure_device());
    uint32_t n, w;
    UFOB_TRY(filter_sizes(f->props, width, &n, &w));
    cudaStream_t s = (cudaStream_t)stream;
    UFOB_TRY(filter_plan_build(f->props, n, f->plan, s));
    if (!pitch) pitch = width;
    if (pitch < width) return fail(UFOB_ERR_INVALID, "filter: input pitch %u < width %u", pitch, width);
    if (first_row > height) return fail(UFOB_ERR_INVALID, "filter: first row %u beyond height %u", first_row, height);
    if (!n_rows) n_rows = height - first_row;
    if (out_layout == UFOB_LAYOUT_QUADS && !sinograms)
        return fail(UFOB_ERR_INVALID, "filter: the QUADS layout holds sinograms (sinograms = 1)");
    if (!n_projections || !n_rows) return UFOB_OK;
    RowSource src;
    UFOB_TRY(projection_source(pre, d_proj, width, height, n_projections, pitch, sinograms != 0, first_row, n_rows,
                               src, s));
    if (out_layout == UFOB_LAYOUT_QUADS) {
        if (out_dtype != UFOB_F16) return fail(UFOB_ERR_INVALID, "filter: the QUADS layout is F16 only");
        if (!out_pitch) out_pitch = w + 1;
        return filter_quads_launch_src(f->plan, src, width, n_projections, n_rows, d_out, w, out_pitch, s);
    }
    if (!out_pitch) out_pitch = out_layout == UFOB_LAYOUT_PAIRS ? round_up(w + 1, 4) : w;
    return filter_rows_launch_src(f->plan, src, width, n_projections * n_rows, d_out, out_dtype, out_layout, w,
                                  out_pitch, s);
}

ufob_status ufob_filter_coefficients(ufob_filter *f, uint32_t width, float *host_out, uint32_t count)
{
    if (!f || !host_out) return fail(UFOB_ERR_INVALID, "filter_coefficients: NULL argument");
    UFOB_TRY(ensure_device());
    uint32_t n, w;
    UFOB_TRY(filter_sizes(f->props, width, &n, &w));
    UFOB_TRY(filter_plan_build(f->props, n, f->plan, 0));
    if (count < 2 * n) return fail(UFOB_ERR_INVALID, "filter_coefficients: need room for %u floats", 2 * n);
    memcpy(host_out, f->plan.coeff.data(), sizeof(float) * 2 * n);
    return UFOB_OK;
}

ufob_status ufob_filter_apply_spectrum(ufob_filter *f, const float *d_in, float *d_out, uint32_t width2,
                                       uint32_t rows, void *stream)
{
    if (!f || !d_in || !d_out) return fail(UFOB_ERR_INVALID, "filter_apply_spectrum: NULL argument");
    UFOB_TRY(ensure_device());
    if (!is_pow2(width2))
        return fail(UFOB_ERR_REQUISITION, "Invalid filter input width %u, must be a power of two", width2);
    UFOB_TRY(filter_plan_build(f->props, width2 / 2, f->plan, (cudaStream_t)stream));
    return filter_spectrum_launch(f->plan.d_coeff.as<float>(), d_in, d_out, width2, rows, (cudaStream_t)stream);
}

void ufob_filter_destroy(ufob_filter *f) { delete f; }

}  // extern "C"

// =================================================================== backproject

struct ufob_backproject {
    ufob_bp_props props;
    DevBuf sincos;
    DevBuf aligned;  // copy of a sinogram whose pitch is not TMA-compatible
    DevBuf partial;  // per-angle-group images of one small sinogram (split_plan)
    // cache key of the sin/cos table
    uint32_t key_P = 0, key_nproj = 0, key_offset = 0;
    double key_step = 0, key_aoff = 0;
    bool mirror = false;  // stacked-backproject orientation (-sin table)
};

extern "C" {

void ufob_bp_props_init(ufob_bp_props *p)
{
    // src/ufo-backproject-task.c:520-541
    p->num_projections = 0;
    p->offset = 0;
    p->axis_pos = -1.0;
    p->angle_step = -1.0;
    p->angle_offset = 0.0;
    p->mode = UFOB_BP_TEXTURE;
    p->roi_x = p->roi_y = 0;
    p->roi_width = p->roi_height = 0;
    p->compensated = -1;
    p->tile = -1;
    p->half_sums = 0;
    p->angle_groups = 0;
}

static ufob_status validate_bp_props(const ufob_bp_props *p)
{
    if (p->num_projections > 32768) return fail(UFOB_ERR_INVALID, "num-projections outside [0, 32768]");
    if (p->offset > 32768) return fail(UFOB_ERR_INVALID, "offset outside [0, 32768]");
    if (!(p->axis_pos >= -1.0 && p->axis_pos <= 32768.0)) return fail(UFOB_ERR_INVALID, "axis-pos outside [-1, 32768]");
    if (!(p->angle_offset >= 0.0)) return fail(UFOB_ERR_INVALID, "angle-offset must be >= 0");
    if (p->mode != UFOB_BP_NEAREST && p->mode != UFOB_BP_TEXTURE) return fail(UFOB_ERR_INVALID, "unknown mode %d", p->mode);
    return UFOB_OK;
}

ufob_status ufob_backproject_create(const ufob_bp_props *props, ufob_backproject **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "backproject_create: out is NULL");
    ufob_bp_props p;
    ufob_bp_props_init(&p);
    if (props) p = *props;
    UFOB_TRY(validate_bp_props(&p));
    ufob_backproject *bp = new ufob_backproject;
    bp->props = p;
    *out = bp;
    return UFOB_OK;
}

ufob_status ufob_backproject_set_property(ufob_backproject *bp, const char *name, double v)
{
    if (!bp) return fail(UFOB_ERR_INVALID, "backproject handle is NULL");
    ufob_bp_props p = bp->props;
    if (prop_is(name, "num-projections")) p.num_projections = (uint32_t)std::max(0.0, v);
    else if (prop_is(name, "offset")) p.offset = (uint32_t)std::max(0.0, v);
    else if (prop_is(name, "axis-pos")) p.axis_pos = v;
    else if (prop_is(name, "angle-step")) p.angle_step = v;
    else if (prop_is(name, "angle-offset")) p.angle_offset = v;
    else if (prop_is(name, "mode")) p.mode = (int)v;
    else if (prop_is(name, "roi-x")) p.roi_x = (uint32_t)std::max(0.0, v);
    else if (prop_is(name, "roi-y")) p.roi_y = (uint32_t)std::max(0.0, v);
    else if (prop_is(name, "roi-width")) p.roi_width = (uint32_t)std::max(0.0, v);
    else if (prop_is(name, "roi-height")) p.roi_height = (uint32_t)std::max(0.0, v);
    else if (prop_is(name, "compensated")) p.compensated = (int)v;
    else if (prop_is(name, "tile")) p.tile = (int)v;
    else if (prop_is(name, "half-sums")) p.half_sums = (int)v;
    else if (prop_is(name, "angle-groups")) {
        const int k = (int)v;
        if (!(k == 0 || k == 1 || k == 2 || k == 4 || k == 8) || (double)k != v)
            return fail(UFOB_ERR_INVALID, "angle-groups must be 0 (automatic), 1, 2, 4 or 8");
        p.angle_groups = k;
    }
    else return fail(UFOB_ERR_INVALID, "backproject: no property named '%s'", name ? name : "(null)");
    if ((prop_is(name, "num-projections") || prop_is(name, "offset") || prop_is(name, "roi-x") ||
         prop_is(name, "roi-y") || prop_is(name, "roi-width") || prop_is(name, "roi-height")) && v < 0)
        return fail(UFOB_ERR_INVALID, "backproject: '%s' must be >= 0", name);
    UFOB_TRY(validate_bp_props(&p));
    bp->props = p;
    return UFOB_OK;
}

ufob_status ufob_backproject_set_property_string(ufob_backproject *bp, const char *name, const char *value)
{
    if (!bp) return fail(UFOB_ERR_INVALID, "backproject handle is NULL");
    if (prop_is(name, "mode")) {
        if (streq(value, "nearest")) return ufob_backproject_set_property(bp, name, UFOB_BP_NEAREST);
        if (streq(value, "texture")) return ufob_backproject_set_property(bp, name, UFOB_BP_TEXTURE);
        return fail(UFOB_ERR_INVALID, "backproject: unknown mode '%s'", value ? value : "(null)");
    }
    char *end = nullptr;
    double v = value ? strtod(value, &end) : 0.0;
    if (!value || end == value) return fail(UFOB_ERR_INVALID, "backproject: '%s' is not a number", value ? value : "(null)");
    return ufob_backproject_set_property(bp, name, v);
}

static ufob_status bp_sizes(const ufob_bp_props &p, uint32_t width, uint32_t height, uint32_t *nproj, uint32_t *ow,
                            uint32_t *oh)
{
    if (!width || !height) return fail(UFOB_ERR_REQUISITION, "backproject: empty sinogram %ux%u", width, height);
    uint32_t n = p.num_projections ? p.num_projections : height;
    if (height > n)
        return fail(UFOB_ERR_REQUISITION,
                    "Total number of projections (%u) must be greater than or equal to sinogram height (%u)", n, height);
    if ((uint64_t)p.offset + height > n)
        return fail(UFOB_ERR_REQUISITION, "offset (%u) + sinogram height (%u) exceeds the %u angle table entries",
                    p.offset, height, n);
    *nproj = n;
    *ow = p.roi_width ? p.roi_width : width;
    *oh = p.roi_height ? p.roi_height : width;  // src/ufo-backproject-task.c:239-244
    return UFOB_OK;
}

ufob_status ufob_backproject_get_requisition(ufob_backproject *bp, uint32_t width, uint32_t height, uint32_t *ow,
                                             uint32_t *oh)
{
    if (!bp) return fail(UFOB_ERR_INVALID, "backproject handle is NULL");
    uint32_t n, w, h;
    UFOB_TRY(bp_sizes(bp->props, width, height, &n, &w, &h));
    if (ow) *ow = w;
    if (oh) *oh = h;
    return UFOB_OK;
}

}  // extern "C"

// Prepare the geometry (sin/cos table on the device) for one run.
static ufob_status bp_prepare(ufob_backproject *bp, uint32_t width, uint32_t height, uint32_t nslices, BPGeometry &g,
                              cudaStream_t s)
{
    uint32_t nproj, ow, oh;
    UFOB_TRY(bp_sizes(bp->props, width, height, &nproj, &ow, &oh));
    const ufob_bp_props &p = bp->props;
    const double step = p.angle_step > 0.0 ? p.angle_step : M_PI / (double)nproj;
    if (bp->key_P != height || bp->key_nproj != nproj || bp->key_offset != p.offset || bp->key_step != step ||
        bp->key_aoff != p.angle_offset || !bp->sincos.ptr) {
        UFOB_TRY(bp->sincos.ensure(sizeof(float2) * height));
        UFOB_TRY(sincos_table_launch(p.angle_offset, step, p.offset, height, bp->sincos.as<float2>(), s, bp->mirror));
        bp->key_P = height;
        bp->key_nproj = nproj;
        bp->key_offset = p.offset;
        bp->key_step = step;
        bp->key_aoff = p.angle_offset;
    }
    g.W = width;
    g.P = height;
    g.nz = nslices;
    g.roi_x = p.roi_x;
    g.roi_y = p.roi_y;
    g.roi_w = ow;
    g.roi_h = oh;
    // axis-pos <= 0: width / 2 in float (src/ufo-backproject-task.c:125-134)
    g.axis = p.axis_pos <= 0.0 ? (float)width / 2.0f : (float)p.axis_pos;
    g.norm = (float)M_PI / (float)height;  // M_PI_F / n_projections with n = sinogram height (backproject.cl:93)
    g.d_sincos = bp->sincos.as<float2>();
    return UFOB_OK;
}

// Compensated block sums only on request: with 16-bit sinogram storage the storage rounding
// (2^-11 relative for FP16) bounds the error, and FP32 sums over 32-angle blocks add orders of
// magnitude less (2048^2 x 1500 with FP16 cells: the same relative L2 against FP64 to seven
// digits, with the compensated kernel 2% slower).
static bool want_kahan(const ufob_bp_props &p, SinoKind, uint32_t)
{
    return p.compensated > 0;
}

// A single sinogram is split into 2, 4 or 8 equal angle groups (at least 32 angles each) whose
// partial images are summed, when that spreads its 32x96 tiles more evenly over the SMs: the
// busiest SM's share of tiles over the average one drops by more than 5%; 1 = no split.
// Launch plan of one sinogram (nz == 1): tile shape (single-slice ids: 32 x 16, 32, 64, 96, 128
// pixels) and angle groups (1, 2, 4, 8; each group >= 32 rows).  A plan is scored by the time of
// its busiest SM: CTAs (tiles x groups, a partial tile costing a full one) spread evenly, each SM
// running its share at the tile's measured update rate (half of it with a single CTA per SM,
// whose 8 warps do not fill the SM), plus the ordered sum of the partial images at HBM speed.
// Ties keep the earlier candidate.  A caller's tile or group count pins that part of the plan.
struct SplitPlan {
    int tile;
    uint32_t groups;
};

static SplitPlan split_plan(const BPGeometry &g, int fixed_tile, int fixed_groups)
{
    // per-SM update rate of each single-slice tile relative to 32 x 96, measured on B200 from one
    // 2048^2 sinogram of 1500 angles (32 x 96: 14.0 G updates/s per SM)
    struct Cand {
        int tile;
        uint32_t rows;
        double rate;
    };
    static const Cand kCands[] = {{8, 96, 1.0}, {11, 128, 0.979}, {10, 64, 0.942}, {9, 32, 0.780}, {0, 16, 0.609}};
    const double sms = (double)num_sms(), sm_rate = 14.01e9;
    SplitPlan best{fixed_tile, 1};
    if (g.nz != 1) return best;
    double best_t = 1e300;
    for (const Cand &c : kCands) {
        if (fixed_tile >= 0 && c.tile != fixed_tile) continue;
        for (uint32_t k = 1; k <= 8; k *= 2) {
            if (fixed_groups > 0 && k != (uint32_t)fixed_groups) continue;
            if (k > 1 && (g.P % k || g.P / k < 32)) continue;
            const double ctas = (double)((g.roi_w + 31) / 32) * (double)((g.roi_h + c.rows - 1) / c.rows) * k;
            const double per_sm = std::ceil(ctas / sms);
            double t = per_sm * 32.0 * c.rows * (double)(g.P / k) / (sm_rate * c.rate * std::min(1.0, per_sm / 2.0));
            if (k > 1) t += (k + 1) * 4.0 * g.roi_w * g.roi_h / 6.0e12 + 3.0e-6;
            if (t < best_t * (1.0 - 1e-9)) {
                best_t = t;
                best = SplitPlan{c.tile, k};
            }
        }
    }
    return best;
}

extern "C" ufob_status ufob_backproject_run(ufob_backproject *bp, const void *d_sino, ufob_dtype dtype,
                                            ufob_layout layout, uint32_t width, uint32_t height, uint32_t nslices,
                                            uint32_t pitch, uint64_t slice_pitch, float *d_out, void *stream)
{
    if (!bp || !d_sino || !d_out) return fail(UFOB_ERR_INVALID, "backproject_run: NULL argument");
    UFOB_TRY(ensure_device());
    cudaStream_t s = (cudaStream_t)stream;
    BPGeometry g;
    UFOB_TRY(bp_prepare(bp, width, height, nslices, g, s));
    if (layout == UFOB_LAYOUT_QUADS) {
        if (dtype != UFOB_F16) return fail(UFOB_ERR_INVALID, "backproject: the QUADS layout is F16 only");
        if (bp->props.mode == UFOB_BP_NEAREST)
            return fail(UFOB_ERR_INVALID, "backproject: mode=nearest needs an F32 sinogram");
        if (!pitch) pitch = width + 1;
        if (!slice_pitch) slice_pitch = (uint64_t)pitch * height;
        // tile ids 16 and up: the same shapes with the FP16-lerp accumulation (measurement aid)
        int tile = bp->props.tile, acc = bp->props.half_sums ? 2 : 0;
        if (tile >= 16) {
            acc = 1;
            tile -= 16;
        }
        return bp_quads_launch(g, d_sino, pitch, slice_pitch, d_out, want_kahan(bp->props, SINO_F16_PAIRS, height),
                               acc, tile, s);
    }
    SinoKind kind;
    if (dtype == UFOB_F32 && layout == UFOB_LAYOUT_ROWS) kind = SINO_F32;
    else if (dtype == UFOB_F16 && layout == UFOB_LAYOUT_PAIRS) kind = SINO_F16_PAIRS;
    else if (dtype == UFOB_BF16 && layout == UFOB_LAYOUT_PAIRS) kind = SINO_BF16_PAIRS;
    else return fail(UFOB_ERR_INVALID, "backproject: sinogram must be F32 rows or F16/BF16 pairs");
    const uint32_t elems = kind == SINO_F32 ? width : width + 1;
    if (!pitch) pitch = kind == SINO_F32 ? width : round_up(width + 1, 4);
    if (pitch < elems) return fail(UFOB_ERR_INVALID, "backproject: pitch %u < row length %u", pitch, elems);
    if (!slice_pitch) slice_pitch = (uint64_t)pitch * height;
    if (bp->props.mode == UFOB_BP_NEAREST) {
        if (kind != SINO_F32) return fail(UFOB_ERR_INVALID, "backproject: mode=nearest needs an F32 sinogram");
        return bp_nearest_launch(g, (const float *)d_sino, pitch, slice_pitch, d_out, s);
    }
    const void *src = d_sino;
    if (((uintptr_t)d_sino & 15) || (pitch & 3) || (slice_pitch & 3)) {
        // TMA needs 16-byte aligned rows: restage into an aligned copy
        const uint32_t ap = round_up(elems, 4);
        UFOB_TRY(bp->aligned.ensure((size_t)ap * 4 * height * nslices));
        for (uint32_t z = 0; z < nslices; z++)
            UFOB_CUDA_TRY(cudaMemcpy2DAsync(bp->aligned.as<char>() + (size_t)z * ap * 4 * height, (size_t)ap * 4,
                                            (const char *)d_sino + (size_t)z * slice_pitch * 4, (size_t)pitch * 4,
                                            (size_t)elems * 4, height, cudaMemcpyDeviceToDevice, s));
        src = bp->aligned.ptr;
        pitch = ap;
        slice_pitch = (uint64_t)ap * height;
    }
    const bool kahan = want_kahan(bp->props, kind, height);
    const SplitPlan plan = split_plan(g, bp->props.tile, bp->props.angle_groups);
    if (bp->props.angle_groups > 1 && plan.groups != (uint32_t)bp->props.angle_groups)
        return fail(UFOB_ERR_INVALID,
                    "backproject: angle-groups %d needs one sinogram whose %u rows split into groups of >= 32 and a "
                    "single-slice tile (0, 8, 9, 10, 11)",
                    bp->props.angle_groups, height);
    if (plan.groups > 1) {
        UFOB_TRY(bp->partial.ensure((size_t)plan.groups * g.roi_w * g.roi_h * sizeof(float)));
        return bp_linear_split_launch(g, src, kind, pitch, plan.groups, plan.tile, bp->partial.as<float>(), d_out,
                                      kahan, s);
    }
    return bp_linear_launch(g, src, kind, pitch, slice_pitch, d_out, kahan, plan.tile, s);
}

extern "C" void ufob_backproject_destroy(ufob_backproject *bp) { delete bp; }

// =================================================================== fused FBP

struct ufob_fbp {
    ufob_filter *f = nullptr;
    ufob_backproject *bp = nullptr;
    ufob_dtype storage = UFOB_F32;
    DevBuf work;        // filtered sinograms of one slice group
    DevBuf hin[2];      // device staging of host input chunks
    DevBuf hout[2];     // device staging of host output chunks
    cudaStream_t s_copy = nullptr, s_comp = nullptr, s_d2h = nullptr;  // uploads, compute, downloads
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
    // optional per-kernel timing: event pairs around every filter / backprojection launch
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> t_filter, t_bp;
    size_t ev_used = 0;
    cudaEvent_t next_event()
    {
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }
    ~ufob_fbp()
    {
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        ufob_filter_destroy(f);
        ufob_backproject_destroy(bp);
        for (int i = 0; i < 2; i++) {
            if (ev_in[i]) cudaEventDestroy(ev_in[i]);
            if (ev_done[i]) cudaEventDestroy(ev_done[i]);
            if (ev_out[i]) cudaEventDestroy(ev_out[i]);
        }
        if (s_copy) cudaStreamDestroy(s_copy);
        if (s_d2h) cudaStreamDestroy(s_d2h);
        if (s_comp) cudaStreamDestroy(s_comp);
    }
};

extern "C" ufob_status ufob_fbp_create(const ufob_filter_props *fp, const ufob_bp_props *bpp, ufob_dtype storage,
                                       ufob_fbp **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "fbp_create: out is NULL");
    if (storage != UFOB_F32 && storage != UFOB_F16 && storage != UFOB_BF16)
        return fail(UFOB_ERR_INVALID, "fbp: storage must be F32, F16 or BF16");
    ufob_fbp *x = new ufob_fbp;
    ufob_status st = ufob_filter_create(fp, &x->f);
    if (st == UFOB_OK) st = ufob_backproject_create(bpp, &x->bp);
    if (st != UFOB_OK) {
        delete x;
        return st;
    }
    x->storage = storage;
    *out = x;
    return UFOB_OK;
}

extern "C" ufob_status ufob_fbp_get_requisition(ufob_fbp *x, uint32_t width, uint32_t height, uint32_t *ow,
                                                uint32_t *oh)
{
    if (!x) return fail(UFOB_ERR_INVALID, "fbp handle is NULL");
    uint32_t fw, fh;
    UFOB_TRY(ufob_filter_get_requisition(x->f, width, height, &fw, &fh));
    return ufob_backproject_get_requisition(x->bp, fw, fh, ow, oh);
}

// ------------------------------------------------------------------ stacked-backproject

struct ufob_stacked_bp {
    ufob_backproject *bp = nullptr;  // mirrored sine table
    int precision = 2;               // 0 int8, 1 half, 2 single (src/ufo-stacked-backproject-task.c:705-716)
    DevBuf work, keys;
};

extern "C" ufob_status ufob_stacked_bp_create(ufob_stacked_bp **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "stacked_bp_create: out is NULL");
    ufob_stacked_bp *sb = new ufob_stacked_bp;
    ufob_status st = ufob_backproject_create(nullptr, &sb->bp);
    if (st != UFOB_OK) {
        delete sb;
        return st;
    }
    sb->bp->mirror = true;
    *out = sb;
    return UFOB_OK;
}

extern "C" ufob_status ufob_stacked_bp_set_property(ufob_stacked_bp *sb, const char *name, double v)
{
    if (!sb) return fail(UFOB_ERR_INVALID, "stacked-backproject handle is NULL");
    if (prop_is(name, "precision-mode")) {
        if (!(v == 0 || v == 1 || v == 2)) return fail(UFOB_ERR_INVALID, "stacked-backproject: precision-mode %g", v);
        sb->precision = (int)v;
        return UFOB_OK;
    }
    if (prop_is(name, "mode") || prop_is(name, "tile") || prop_is(name, "half-sums") || prop_is(name, "angle-groups"))
        return fail(UFOB_ERR_INVALID, "stacked-backproject: no property named '%s'", name);
    return ufob_backproject_set_property(sb->bp, name, v);
}

extern "C" ufob_status ufob_stacked_bp_set_property_string(ufob_stacked_bp *sb, const char *name, const char *value)
{
    if (!sb) return fail(UFOB_ERR_INVALID, "stacked-backproject handle is NULL");
    if (prop_is(name, "precision-mode")) {
        static const char *nicks[3] = {"int8", "half", "single"};
        for (int i = 0; i < 3; i++)
            if (streq(value, nicks[i])) return ufob_stacked_bp_set_property(sb, name, i);
        return fail(UFOB_ERR_INVALID, "stacked-backproject: unknown precision-mode '%s'", value ? value : "(null)");
    }
    char *end = nullptr;
    double v = value ? strtod(value, &end) : 0.0;
    if (!value || end == value) return fail(UFOB_ERR_INVALID, "stacked-backproject: '%s' is not a number", value ? value : "(null)");
    return ufob_stacked_bp_set_property(sb, name, v);
}

extern "C" ufob_status ufob_stacked_bp_get_requisition(ufob_stacked_bp *sb, uint32_t width, uint32_t height,
                                                       uint32_t *ow, uint32_t *oh)
{
    if (!sb) return fail(UFOB_ERR_INVALID, "stacked-backproject handle is NULL");
    return ufob_backproject_get_requisition(sb->bp, width, height, ow, oh);
}

extern "C" ufob_status ufob_stacked_bp_run(ufob_stacked_bp *sb, const float *d_sino, uint32_t width, uint32_t height,
                                           uint32_t nslices, float *d_out, void *stream)
{
    if (!sb || !d_sino || !d_out) return fail(UFOB_ERR_INVALID, "stacked_bp_run: NULL argument");
    UFOB_TRY(ensure_device());
    cudaStream_t s = (cudaStream_t)stream;
    if (!nslices) return UFOB_OK;
    if (sb->precision == 2)  // single: FP32 rows, linear interpolation
        return ufob_backproject_run(sb->bp, d_sino, UFOB_F32, UFOB_LAYOUT_ROWS, width, height, nslices, 0, 0, d_out,
                                    stream);
    if (sb->precision == 1) {  // half: FP16 slice-quad cells, FP32 sums
        const uint32_t cells = width + 1;
        UFOB_TRY(sb->work.ensure((size_t)((nslices + 3) / 4) * height * cells * 16));
        UFOB_TRY(pack_quads_launch(d_sino, width, height, nslices, sb->work.ptr, s));
        return ufob_backproject_run(sb->bp, sb->work.ptr, UFOB_F16, UFOB_LAYOUT_QUADS, width, height, nslices, cells,
                                    (uint64_t)cells * height, d_out, stream);
    }
    BPGeometry g;  // int8
    UFOB_TRY(bp_prepare(sb->bp, width, height, nslices, g, s));
    UFOB_TRY(sb->work.ensure((size_t)((nslices + 3) / 4) * height * width * 4));
    UFOB_TRY(sb->keys.ensure(8));
    return stacked_u8_launch(g, d_sino, sb->work.ptr, sb->keys.as<uint32_t>(), d_out, s);
}

extern "C" void ufob_stacked_bp_destroy(ufob_stacked_bp *sb)
{
    if (!sb) return;
    ufob_backproject_destroy(sb->bp);
    delete sb;
}

// Filter + backproject `nz` slices already on the device; logical row
// slice * height + angle of `src` is sinogram row `angle` of slice `slice`.
static ufob_status fbp_group(ufob_fbp *x, const RowSource &src, uint32_t width, uint32_t height, uint32_t nz,
                             float *d_out, cudaStream_t s)
{
    uint32_t nfft, fw;
    UFOB_TRY(filter_sizes(x->f->props, width, &nfft, &fw));
    UFOB_TRY(filter_plan_build(x->f->props, nfft, x->f->plan, s));
    // F16: slice-quad cells (16 B per detector position and four slices), or pairs for a single
    // slice (a quad cell would carry three empty slices); BF16: pairs; F32: rows
    const bool quads = x->storage == UFOB_F16 && nz > 1;
    const bool pairs = x->storage == UFOB_BF16 || (x->storage == UFOB_F16 && nz == 1);
    const uint32_t pitch = quads ? fw + 1 : pairs ? round_up(fw + 1, 4) : round_up(fw, 4);
    const size_t work_bytes = quads ? (size_t)pitch * 16 * height * ((nz + 3) / 4) : (size_t)pitch * 4 * height * nz;
    UFOB_TRY(x->work.ensure(work_bytes));
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    if (x->timing) {
        e0 = x->next_event();
        e1 = x->next_event();
        e2 = x->next_event();
        if (!e0 || !e1 || !e2) return fail(UFOB_ERR_CUDA, "fbp: cannot create timing events");
        UFOB_CUDA_TRY(cudaEventRecord(e0, s));
    }
    const ufob_layout layout = quads ? UFOB_LAYOUT_QUADS : pairs ? UFOB_LAYOUT_PAIRS : UFOB_LAYOUT_ROWS;
    if (quads)
        UFOB_TRY(filter_quads_launch_src(x->f->plan, src, width, height, nz, x->work.ptr, fw, pitch, s));
    else
        UFOB_TRY(filter_rows_launch_src(x->f->plan, src, width, height * nz, x->work.ptr, x->storage, layout, fw,
                                        pitch, s));
    if (x->timing) UFOB_CUDA_TRY(cudaEventRecord(e1, s));
    UFOB_TRY(ufob_backproject_run(x->bp, x->work.ptr, x->storage, layout, fw, height, nz, pitch,
                                  (uint64_t)pitch * height, d_out, s));
    if (x->timing) {
        UFOB_CUDA_TRY(cudaEventRecord(e2, s));
        x->t_filter.emplace_back(e0, e1);
        x->t_bp.emplace_back(e1, e2);
    }
    return UFOB_OK;
}

extern "C" ufob_status ufob_fbp_set_timing(ufob_fbp *x, int enable)
{
    if (!x) return fail(UFOB_ERR_INVALID, "fbp handle is NULL");
    x->timing = enable != 0;
    x->t_filter.clear();
    x->t_bp.clear();
    x->ev_used = 0;
    return UFOB_OK;
}

extern "C" ufob_status ufob_fbp_kernel_times(ufob_fbp *x, double *filter_ms, uint32_t *filter_launches, double *bp_ms,
                                             uint32_t *bp_launches)
{
    if (!x) return fail(UFOB_ERR_INVALID, "fbp handle is NULL");
    double f = 0.0, b = 0.0;
    for (auto &p : x->t_filter) {
        float ms = 0.f;
        UFOB_CUDA_TRY(cudaEventSynchronize(p.second));
        UFOB_CUDA_TRY(cudaEventElapsedTime(&ms, p.first, p.second));
        f += ms;
    }
    for (auto &p : x->t_bp) {
        float ms = 0.f;
        UFOB_CUDA_TRY(cudaEventSynchronize(p.second));
        UFOB_CUDA_TRY(cudaEventElapsedTime(&ms, p.first, p.second));
        b += ms;
    }
    if (filter_ms) *filter_ms = f;
    if (filter_launches) *filter_launches = (uint32_t)x->t_filter.size();
    if (bp_ms) *bp_ms = b;
    if (bp_launches) *bp_launches = (uint32_t)x->t_bp.size();
    return UFOB_OK;
}

static uint32_t group_slices(uint32_t width, uint32_t height, uint32_t nslices)
{
    // bound the filtered workspace to ~2 GiB, in multiples of 32 slices (whole slice tiles of
    // the backprojectors, which run 4 to 32 slices per CTA) or, for very large slices, of 8
    const uint64_t per_slice = (uint64_t)(width + 4) * 4 * height;
    uint64_t g = (2ull << 30) / std::max<uint64_t>(per_slice, 1);
    g = g >= 32 ? g / 32 * 32 : std::max<uint64_t>(8, g / 8 * 8);
    return (uint32_t)std::min<uint64_t>(g, nslices);
}

extern "C" ufob_status ufob_fbp_run(ufob_fbp *x, const float *d_sino, uint32_t width, uint32_t height,
                                    uint32_t nslices, float *d_out, void *stream)
{
    if (!x || !d_sino || !d_out) return fail(UFOB_ERR_INVALID, "fbp_run: NULL argument");
    UFOB_TRY(ensure_device());
    uint32_t ow, oh;
    UFOB_TRY(ufob_fbp_get_requisition(x, width, height, &ow, &oh));
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t G = group_slices(width, height, nslices);
    for (uint32_t z = 0; z < nslices; z += G) {
        const uint32_t nz = std::min(G, nslices - z);
        UFOB_TRY(fbp_group(x, plain_rows(d_sino + (size_t)z * width * height, width), width, height, nz,
                           d_out + (size_t)z * ow * oh, s));
    }
    return UFOB_OK;
}

extern "C" ufob_status ufob_fbp_run_projections(ufob_fbp *x, const ufob_preprocess *pre, const float *d_proj,
                                                uint32_t width, uint32_t height, uint32_t n_projections,
                                                uint32_t first_row, uint32_t n_rows, float *d_out, void *stream)
{
    if (!x || !d_proj || !d_out) return fail(UFOB_ERR_INVALID, "fbp_run_projections: NULL argument");
    UFOB_TRY(ensure_device());
    if (first_row > height) return fail(UFOB_ERR_INVALID, "fbp: first row %u beyond height %u", first_row, height);
    if (!n_rows) n_rows = height - first_row;
    uint32_t ow, oh;
    UFOB_TRY(ufob_fbp_get_requisition(x, width, n_projections, &ow, &oh));
    cudaStream_t s = (cudaStream_t)stream;
    // every slice group reads the same projections: a cone weight restarts at its count each time
    const uint32_t count0 = pre && pre->cone ? ufob_cone_weight_get_count(pre->cone) : 0;
    const uint32_t G = group_slices(width, n_projections, n_rows);
    for (uint32_t z = 0; z < n_rows; z += G) {
        const uint32_t nz = std::min(G, n_rows - z);
        if (pre && pre->cone) UFOB_TRY(ufob_cone_weight_set_count(pre->cone, count0));
        RowSource src;
        UFOB_TRY(projection_source(pre, d_proj, width, height, n_projections, width, true, first_row + z, nz, src, s));
        UFOB_TRY(fbp_group(x, src, width, n_projections, nz, d_out + (size_t)z * ow * oh, s));
    }
    if (pre && pre->cone) UFOB_TRY(ufob_cone_weight_set_count(pre->cone, count0 + n_projections));
    return UFOB_OK;
}

extern "C" ufob_status ufob_fbp_run_host(ufob_fbp *x, const float *h_sino, uint32_t width, uint32_t height,
                                         uint32_t nslices, float *h_out, uint32_t chunk)
{
    if (!x || !h_sino || !h_out) return fail(UFOB_ERR_INVALID, "fbp_run_host: NULL argument");
    UFOB_TRY(ensure_device());
    uint32_t ow, oh;
    UFOB_TRY(ufob_fbp_get_requisition(x, width, height, &ow, &oh));
    if (!chunk) chunk = 32;
    chunk = std::min(chunk, nslices);
    if (!x->s_copy) {
        UFOB_CUDA_TRY(cudaStreamCreateWithFlags(&x->s_copy, cudaStreamNonBlocking));
        UFOB_CUDA_TRY(cudaStreamCreateWithFlags(&x->s_d2h, cudaStreamNonBlocking));
        UFOB_CUDA_TRY(cudaStreamCreateWithFlags(&x->s_comp, cudaStreamNonBlocking));
        for (int i = 0; i < 2; i++) {
            UFOB_CUDA_TRY(cudaEventCreateWithFlags(&x->ev_in[i], cudaEventDisableTiming));
            UFOB_CUDA_TRY(cudaEventCreateWithFlags(&x->ev_done[i], cudaEventDisableTiming));
            UFOB_CUDA_TRY(cudaEventCreateWithFlags(&x->ev_out[i], cudaEventDisableTiming));
        }
    }
    const size_t in_bytes = (size_t)chunk * width * height * 4, out_bytes = (size_t)chunk * ow * oh * 4;
    for (int i = 0; i < 2; i++) {
        UFOB_TRY(x->hin[i].ensure(in_bytes));
        UFOB_TRY(x->hout[i].ensure(out_bytes));
    }
    // Pipeline: H2D(c) on the upload stream -> filter+BP(c) on the compute stream -> D2H(c) on the download
    // stream, double-buffered so chunk c+1's upload and chunk c-1's download overlap chunk c's compute.
    // Chunk sizes: a short first chunk (compute starts after a small upload) and a short last one
    // (little download left after the last compute), `chunk` slices in between.
    const uint32_t edge = chunk >= 32 ? 16 : 0;
    auto chunk_at = [&](uint32_t z) -> uint32_t {
        const uint32_t rest = nslices - z;
        if (edge && z == 0 && nslices >= chunk + 2 * edge) return edge;
        if (rest > chunk + edge) return chunk;
        if (edge && rest >= 2 * edge) return rest - edge;
        return rest;
    };
    uint32_t c = 0;
    for (uint32_t z = 0, nz = 0; z < nslices; z += nz, c++) {
        const int b = c & 1;
        nz = chunk_at(z);
        if (c >= 2) UFOB_CUDA_TRY(cudaStreamWaitEvent(x->s_copy, x->ev_done[b], 0));  // hin[b] free again
        UFOB_CUDA_TRY(cudaMemcpyAsync(x->hin[b].ptr, h_sino + (size_t)z * width * height, (size_t)nz * width * height * 4,
                                      cudaMemcpyHostToDevice, x->s_copy));
        UFOB_CUDA_TRY(cudaEventRecord(x->ev_in[b], x->s_copy));
        UFOB_CUDA_TRY(cudaStreamWaitEvent(x->s_comp, x->ev_in[b], 0));
        if (c >= 2) UFOB_CUDA_TRY(cudaStreamWaitEvent(x->s_comp, x->ev_out[b], 0));  // hout[b] downloaded
        UFOB_TRY(fbp_group(x, plain_rows(x->hin[b].as<float>(), width), width, height, nz, x->hout[b].as<float>(),
                           x->s_comp));
        UFOB_CUDA_TRY(cudaEventRecord(x->ev_done[b], x->s_comp));
        UFOB_CUDA_TRY(cudaStreamWaitEvent(x->s_d2h, x->ev_done[b], 0));
        UFOB_CUDA_TRY(cudaMemcpyAsync(h_out + (size_t)z * ow * oh, x->hout[b].ptr, (size_t)nz * ow * oh * 4,
                                      cudaMemcpyDeviceToHost, x->s_d2h));
        UFOB_CUDA_TRY(cudaEventRecord(x->ev_out[b], x->s_d2h));
    }
    UFOB_CUDA_TRY(cudaStreamSynchronize(x->s_copy));
    UFOB_CUDA_TRY(cudaStreamSynchronize(x->s_comp));
    UFOB_CUDA_TRY(cudaStreamSynchronize(x->s_d2h));
    return check_device_error_word(x->s_comp);
}

extern "C" void ufob_fbp_destroy(ufob_fbp *x) { delete x; }

extern "C" uint64_t ufob_launch_count(void) { return g_launches.load(); }
extern "C" uint64_t ufob_device_alloc_count(void) { return g_device_allocs.load(); }

extern "C" ufob_status ufob_device_status(void)
{
    UFOB_TRY(ensure_device());
    return check_device_error_word(0);
}
