// CPU runtime behind the reference shims: buffers, kernel arguments, an
// NDRange driver (OpenMP over work-items) that runs the reference's OpenCL
// kernels compiled as C++, the OpenCL linear sampler, and an FP64 FFT standing
// in for the vendored OpenCL FFT library.  Test infrastructure only: the CUDA
// engine never links this.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <complex>
#include <vector>

#include "clc_types.hpp"
#include "refshim_internal.h"
extern "C" {
#include "common/ufo-fft.h"
}

thread_local size_t clshim_gid[3], clshim_gsz[3];

// ------------------------------------------------------------------ kernels compiled from the reference
extern "C" {
void backproject_tex(image2d_t, float *, const float *, const float *, unsigned, unsigned, unsigned, unsigned, float);
void backproject_nearest(float *, float *, const float *, const float *, unsigned, unsigned, unsigned, unsigned,
                         float);
void filter(float *, float *, float *);
void fft_spread(float *, float *, int, int, int);
void fft_pack(float *, float *, int, int, float, int);
void forwardproject(image2d_t, float *, float, float);
void flat_correct(float *, float *, const float *, const float *, const int, const int, const int, const float,
                  const float);
void weight_projection(float *, float *, const float2, const float, const float, const float, const float);
}

template <typename T> static T arg(refshim_kernel *k, int i) { return *reinterpret_cast<T *>(k->args[i]); }
static float *mem_ptr(refshim_kernel *k, int i) { return (float *)arg<cl_mem>(k, i)->host; }
static image2d_t img_arg(refshim_kernel *k, int i)
{
    cl_mem m = arg<cl_mem>(k, i);
    return image2d_t{(const float *)m->host, m->width, m->height};
}

template <typename F> static void ndrange(guint ndims, const gsize *g, F body)
{
    const size_t g0 = g[0], g1 = ndims > 1 ? g[1] : 1, g2 = ndims > 2 ? g[2] : 1;
    const long long total = (long long)(g0 * g1 * g2);
#pragma omp parallel for schedule(static)
    for (long long t = 0; t < total; t++) {
        clshim_gid[0] = (size_t)t % g0;
        clshim_gid[1] = ((size_t)t / g0) % g1;
        clshim_gid[2] = (size_t)t / (g0 * g1);
        clshim_gsz[0] = g0;
        clshim_gsz[1] = g1;
        clshim_gsz[2] = g2;
        body();
    }
}

extern "C" void refshim_dispatch(refshim_kernel *k, guint ndims, const gsize *g)
{
    const char *n = k->name;
    if (k->jit) {
        refshim_jit_dispatch(k, ndims, g, NULL);
    } else if (!strcmp(n, "backproject_tex")) {
        image2d_t img = img_arg(k, 0);
        float *out = mem_ptr(k, 1);
        const float *s = mem_ptr(k, 2), *c = mem_ptr(k, 3);
        unsigned x = arg<unsigned>(k, 4), y = arg<unsigned>(k, 5), o = arg<unsigned>(k, 6), p = arg<unsigned>(k, 7);
        float axis = arg<float>(k, 8);
        ndrange(ndims, g, [&] { backproject_tex(img, out, s, c, x, y, o, p, axis); });
    } else if (!strcmp(n, "backproject_nearest")) {
        float *in = mem_ptr(k, 0), *out = mem_ptr(k, 1);
        const float *s = mem_ptr(k, 2), *c = mem_ptr(k, 3);
        unsigned x = arg<unsigned>(k, 4), y = arg<unsigned>(k, 5), o = arg<unsigned>(k, 6), p = arg<unsigned>(k, 7);
        float axis = arg<float>(k, 8);
        ndrange(ndims, g, [&] { backproject_nearest(in, out, s, c, x, y, o, p, axis); });
    } else if (!strcmp(n, "filter")) {
        float *in = mem_ptr(k, 0), *out = mem_ptr(k, 1), *f = mem_ptr(k, 2);
        ndrange(ndims, g, [&] { filter(in, out, f); });
    } else if (!strcmp(n, "fft_spread")) {
        float *out = mem_ptr(k, 0), *in = mem_ptr(k, 1);
        int w = arg<int>(k, 2), h = arg<int>(k, 3), d = arg<int>(k, 4);
        ndrange(ndims, g, [&] { fft_spread(out, in, w, h, d); });
    } else if (!strcmp(n, "fft_pack")) {
        float *in = mem_ptr(k, 0), *out = mem_ptr(k, 1);
        int w = arg<int>(k, 2), h = arg<int>(k, 3), c = arg<int>(k, 5);
        float sc = arg<float>(k, 4);
        ndrange(ndims, g, [&] { fft_pack(in, out, w, h, sc, c); });
    } else if (!strcmp(n, "forwardproject")) {
        image2d_t img = img_arg(k, 0);
        float *out = mem_ptr(k, 1);
        float axis = arg<float>(k, 2), step = arg<float>(k, 3);
        ndrange(ndims, g, [&] { forwardproject(img, out, axis, step); });
    } else {
        fprintf(stderr, "refshim: no CPU build of kernel '%s'\n", n);
        abort();
    }
}

// ------------------------------------------------------------------ FP64 FFT

// In-place complex FFT of `batch` rows of n interleaved floats (forward e^{-i},
// backward e^{+i}, unscaled), computed in FP64: radix-2 for powers of two,
// direct summation otherwise.
extern "C" void refshim_fft(float *data, size_t n, size_t batch, int forward)
{
    const double sgn = forward ? -1.0 : 1.0;
#pragma omp parallel for schedule(static)
    for (long long b = 0; b < (long long)batch; b++) {
        std::vector<std::complex<double>> x(n), y(n);
        float *row = data + (size_t)b * 2 * n;
        for (size_t i = 0; i < n; i++) x[i] = {row[2 * i], row[2 * i + 1]};
        if (n && !(n & (n - 1))) {
            for (size_t i = 1, j = 0; i < n; i++) {  // bit reversal
                size_t bit = n >> 1;
                for (; j & bit; bit >>= 1) j ^= bit;
                j ^= bit;
                if (i < j) std::swap(x[i], x[j]);
            }
            for (size_t len = 2; len <= n; len <<= 1) {
                const double ang = sgn * 2.0 * M_PI / (double)len;
                for (size_t i = 0; i < n; i += len)
                    for (size_t k = 0; k < len / 2; k++) {
                        std::complex<double> w(cos(ang * k), sin(ang * k));
                        std::complex<double> u = x[i + k], v = x[i + k + len / 2] * w;
                        x[i + k] = u + v;
                        x[i + k + len / 2] = u - v;
                    }
            }
            y = x;
        } else {
            for (size_t k = 0; k < n; k++) {
                std::complex<double> acc = 0;
                for (size_t j = 0; j < n; j++) {
                    const double a = sgn * 2.0 * M_PI * (double)((j * k) % n) / (double)n;
                    acc += x[j] * std::complex<double>(cos(a), sin(a));
                }
                y[k] = acc;
            }
        }
        for (size_t i = 0; i < n; i++) {
            row[2 * i] = (float)y[i].real();
            row[2 * i + 1] = (float)y[i].imag();
        }
    }
}

struct _UfoFft {
    UfoFftParameter param;
};

extern "C" {

UfoFft *ufo_fft_new(void) { return (UfoFft *)calloc(1, sizeof(UfoFft)); }
cl_int ufo_fft_update(UfoFft *fft, cl_context, cl_command_queue, UfoFftParameter *param)
{
    fft->param = *param;
    return CL_SUCCESS;
}
cl_int ufo_fft_execute(UfoFft *fft, cl_command_queue, UfoProfiler *, cl_mem in, cl_mem out, UfoFftDirection dir,
                       cl_uint, cl_event *, cl_event *)
{
    const size_t n = fft->param.size[0], batch = fft->param.batch;
    if (in != out) memcpy(out->host, in->host, 2 * n * batch * sizeof(float));
    refshim_fft((float *)out->host, n, batch, dir == UFO_FFT_FORWARD);
    return CL_SUCCESS;
}
void ufo_fft_destroy(UfoFft *fft) { free(fft); }

// ------------------------------------------------------------------ GLib / OpenCL / ufo-core stand-ins

static GParamSpec g_dummy_pspec;
GParamSpec *refshim_pspec(void) { return &g_dummy_pspec; }

void g_set_error(GError **err, int domain, int code, const char *fmt, ...)
{
    if (!err) return;
    GError *e = (GError *)calloc(1, sizeof(GError));
    e->domain = domain;
    e->code = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(e->message, sizeof e->message, fmt, ap);
    va_end(ap);
    *err = e;
}

void *g_object_new(GType, ...) { return NULL; }

cl_mem clCreateBuffer(cl_context, cl_mem_flags flags, size_t size, void *host_ptr, cl_int *err)
{
    cl_mem m = (cl_mem)calloc(1, sizeof(refshim_mem));
    m->size = size;
    m->host = calloc(1, size ? size : 1);
    m->owned = 1;
    if ((flags & CL_MEM_COPY_HOST_PTR) && host_ptr) memcpy(m->host, host_ptr, size);
    if (err) *err = CL_SUCCESS;
    return m;
}
cl_int clSetKernelArg(cl_kernel k, cl_uint i, size_t size, const void *value)
{
    if (i >= REFSHIM_MAX_ARGS || size > 64) return -51;
    memcpy(k->args[i], value, size);
    k->arg_size[i] = size;
    return CL_SUCCESS;
}
cl_int clRetainKernel(cl_kernel) { return CL_SUCCESS; }
cl_int clReleaseKernel(cl_kernel) { return CL_SUCCESS; }
cl_int clRetainContext(cl_context) { return CL_SUCCESS; }
cl_int clReleaseContext(cl_context) { return CL_SUCCESS; }
cl_int clReleaseMemObject(cl_mem m)
{
    if (m && m->owned) {
        free(m->host);
        free(m);
    }
    return CL_SUCCESS;
}

UfoGpuNode *ufo_task_node_get_proc_node(UfoTaskNode *) { return NULL; }
UfoProfiler *ufo_task_node_get_profiler(UfoTaskNode *) { return NULL; }
cl_command_queue ufo_gpu_node_get_cmd_queue(UfoGpuNode *) { return NULL; }
cl_context ufo_resources_get_context(UfoResources *) { return NULL; }

cl_kernel ufo_resources_get_kernel(UfoResources *, const char *file, const char *name, const char *, GError **err)
{
    // kernels compiled into this library (ref_kernels.cpp); any other file is
    // compiled for the CPU when asked for (ref_clc_jit.cpp)
    static const char *builtin[] = {"backproject.cl", "filter.cl", "fft.cl", "forwardproject.cl", NULL};
    bool is_builtin = false;
    for (const char **b = builtin; *b; b++) is_builtin |= file && !strcmp(file, *b);
    if (!is_builtin) return refshim_jit_from_file(file, name, err);
    cl_kernel k = (cl_kernel)calloc(1, sizeof(refshim_kernel));
    snprintf(k->name, sizeof k->name, "%s", name);
    return k;
}

void refshim_buffer_init(UfoBuffer *b, float *data, guint n_dims, gsize d0, gsize d1, gsize d2)
{
    refshim_buffer_init_bytes(b, data, d0 * d1 * d2 * sizeof(float), n_dims, d0, d1, d2);
}
void refshim_buffer_init_bytes(UfoBuffer *b, void *data, size_t bytes, guint n_dims, gsize d0, gsize d1, gsize d2)
{
    memset(b, 0, sizeof *b);
    b->req.n_dims = n_dims;
    b->req.dims[0] = d0;
    b->req.dims[1] = d1;
    b->req.dims[2] = d2;
    b->data = (float *)data;
    b->mem.host = data;
    b->mem.size = bytes;
}

void ufo_buffer_get_requisition(UfoBuffer *b, UfoRequisition *r) { *r = b->req; }
static size_t buffer_floats(UfoBuffer *b)
{
    size_t n = 1;
    for (guint d = 0; d < b->req.n_dims; d++) n *= b->req.dims[d];
    return n;
}
float *ufo_buffer_get_host_array(UfoBuffer *b, cl_command_queue) { return b->data; }
float ufo_buffer_min(UfoBuffer *b, cl_command_queue)
{
    float m = b->data[0];
    for (size_t i = 1, n = buffer_floats(b); i < n; i++) m = b->data[i] < m ? b->data[i] : m;
    return m;
}
float ufo_buffer_max(UfoBuffer *b, cl_command_queue)
{
    float m = b->data[0];
    for (size_t i = 1, n = buffer_floats(b); i < n; i++) m = b->data[i] > m ? b->data[i] : m;
    return m;
}
cl_mem ufo_buffer_get_device_array(UfoBuffer *b, cl_command_queue)
{
    b->mem.is_image = 0;
    return &b->mem;
}
cl_mem ufo_buffer_get_device_image(UfoBuffer *b, cl_command_queue)
{
    b->mem.is_image = 1;
    b->mem.width = (int)b->req.dims[0];
    b->mem.height = (int)b->req.dims[1];
    return &b->mem;
}
void ufo_profiler_call(UfoProfiler *, cl_command_queue, cl_kernel k, guint ndims, const gsize *global,
                       const gsize *local)
{
    if (k->jit)
        refshim_jit_dispatch(k, ndims, global, local);
    else
        refshim_dispatch(k, ndims, global);
}
void ufo_profiler_call_blocking(UfoProfiler *p, cl_command_queue q, cl_kernel k, guint ndims, const gsize *global,
                                const gsize *local)
{
    ufo_profiler_call(p, q, k, ndims, global, local);
}

// The two element-wise kernels of the fft / ifft tasks, launched with the
// arguments and work sizes those tasks use for a 1-D power-of-two transform
// (src/ufo-fft-task.c:239-244, src/ufo-ifft-task.c:297-310).
static refshim_mem wrap(void *p, size_t bytes)
{
    refshim_mem m;
    memset(&m, 0, sizeof m);
    m.host = p;
    m.size = bytes;
    return m;
}

void ref_fft_spread(float *out, float *in, int width, int height, int nfft)
{
    refshim_kernel k;
    memset(&k, 0, sizeof k);
    snprintf(k.name, sizeof k.name, "fft_spread");
    refshim_mem mo = wrap(out, (size_t)2 * nfft * height * 4), mi = wrap(in, (size_t)width * height * 4);
    cl_mem po = &mo, pi = &mi;
    int depth = 1;
    clSetKernelArg(&k, 0, sizeof(cl_mem), &po);
    clSetKernelArg(&k, 1, sizeof(cl_mem), &pi);
    clSetKernelArg(&k, 2, sizeof(int), &width);
    clSetKernelArg(&k, 3, sizeof(int), &height);
    clSetKernelArg(&k, 4, sizeof(int), &depth);
    gsize g[3] = {(gsize)nfft, (gsize)height, 1};
    refshim_dispatch(&k, 3, g);
}

void ref_fft_pack(float *in, float *out, int out_width, int height, int nfft, float scale)
{
    refshim_kernel k;
    memset(&k, 0, sizeof k);
    snprintf(k.name, sizeof k.name, "fft_pack");
    refshim_mem mi = wrap(in, (size_t)2 * nfft * height * 4), mo = wrap(out, (size_t)out_width * height * 4);
    cl_mem pi = &mi, po = &mo;
    int is_complex = 0;
    clSetKernelArg(&k, 0, sizeof(cl_mem), &pi);
    clSetKernelArg(&k, 1, sizeof(cl_mem), &po);
    clSetKernelArg(&k, 2, sizeof(int), &out_width);
    clSetKernelArg(&k, 3, sizeof(int), &height);
    clSetKernelArg(&k, 4, sizeof(float), &scale);
    clSetKernelArg(&k, 5, sizeof(int), &is_complex);
    gsize g[3] = {(gsize)nfft, (gsize)height, 1};
    refshim_dispatch(&k, 3, g);
}

// ffc.cl over one frame of width x height (src/ufo-flat-field-correct-task.c:150-166 launches
// it on the frame's requisition).
void ref_flat_correct(float *out, float *data, const float *dark, const float *flat, int width, int height,
                      int sinogram_input, int absorptivity, int fix_abnormal, float dark_scale, float flat_scale)
{
    gsize g[2] = {(gsize)width, (gsize)height};
    ndrange(2, g, [&] {
        flat_correct(out, data, dark, flat, sinogram_input, absorptivity, fix_abnormal, dark_scale, flat_scale);
    });
}

// conebeam.cl over one projection with the kernel arguments the task computes
// (src/ufo-cone-beam-projection-weight-task.c:128-146).
void ref_weight_projection(float *proj, float *out, int width, int height, float cx, float cz, float sd, float od,
                           float mr, float cs)
{
    gsize g[2] = {(gsize)width, (gsize)height};
    const float2 c = make_float2(cx, cz);
    ndrange(2, g, [&] { weight_projection(proj, out, c, sd, od, mr, cs); });
}

// forwardproject.cl over a slice image (src/ufo-forwardproject-task.c launches
// it on (width, n_angles) work-items).
void ref_forwardproject(float *slice, int width, int n_angles, float axis, float angle_step, float *sino)
{
    refshim_kernel k;
    memset(&k, 0, sizeof k);
    snprintf(k.name, sizeof k.name, "forwardproject");
    refshim_mem mi = wrap(slice, (size_t)width * width * 4), mo = wrap(sino, (size_t)width * n_angles * 4);
    mi.is_image = 1;
    mi.width = width;
    mi.height = width;
    cl_mem pi = &mi, po = &mo;
    clSetKernelArg(&k, 0, sizeof(cl_mem), &pi);
    clSetKernelArg(&k, 1, sizeof(cl_mem), &po);
    clSetKernelArg(&k, 2, sizeof(float), &axis);
    clSetKernelArg(&k, 3, sizeof(float), &angle_step);
    gsize g[2] = {(gsize)width, (gsize)n_angles};
    refshim_dispatch(&k, 2, g);
}

}  // extern "C"
