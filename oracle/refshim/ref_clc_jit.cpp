// Kernels the reference generates at run time (general-backproject's
// make_kernel output) or at build time (the lamino kernels written by
// src/kernels/tools/make_burst_kernels.py), compiled for the CPU when the task
// asks for them: the OpenCL C source is rewritten mechanically (vector literals
// "(float3)(a, b, c)" -> make_float3(a, b, c), the ".xz" swizzle -> .xz(),
// element access "v.s3" -> clgen_elem(v, 0x3)),
// prefixed with the kernel-language prelude clc_gen.hpp, given a wrapper that
// unpacks the argument list the task set with clSetKernelArg, and built with
// g++ into a cached shared object that is loaded with dlopen.  Also the OpenCL
// image, sampler and copy calls and the ufo-core resource/device queries those
// tasks make.  Test infrastructure only: the CUDA engine never links this.
#include <dlfcn.h>
#include <stdarg.h>
#include <sys/stat.h>
#include <unistd.h>

#include <functional>
#include <fstream>
#include <map>
#include <mutex>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

#include "clc_types.hpp"
#include "refshim_internal.h"

namespace {

std::string g_kernels_dir, g_shim_dir, g_cache_dir;
unsigned long g_global_mem = 64ul << 30, g_max_alloc = 4ul << 30, g_max_work_group = 256;

struct Param {
    char kind;         // 'v' value, 'p' pointer, 'i' image, 's' sampler
    std::string type;  // C++ type of the value or of the pointee
};

std::string trim(const std::string &s)
{
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// Parse "kernel void NAME (params)" into argument kinds and types.
bool parse_signature(const std::string &src, const std::string &name, std::vector<Param> &params)
{
    std::smatch m;
    std::regex head("void\\s+" + name + "\\s*\\(");
    if (!std::regex_search(src, m, head)) return false;
    size_t open = (size_t)(m.position(0) + m.length(0)), close = src.find(')', open);
    if (close == std::string::npos) return false;
    std::stringstream ss(src.substr(open, close - open));
    std::string p;
    static const char *quals[] = {"const", "global", "__global", "constant", "__constant", "local", "__local",
                                  "read_only", "write_only", "__read_only", "__write_only", "restrict", nullptr};
    while (std::getline(ss, p, ',')) {
        p = trim(p);
        if (p.empty()) continue;
        Param q;
        const bool ptr = p.find('*') != std::string::npos;
        for (char &c : p)
            if (c == '*') c = ' ';
        std::stringstream ts(p);
        std::vector<std::string> toks;
        for (std::string t; ts >> t;) {
            bool qual = false;
            for (const char **qq = quals; *qq; qq++) qual |= t == *qq;
            if (!qual) toks.push_back(t);
        }
        if (toks.size() < 2) return false;
        toks.pop_back();  // the parameter's name
        for (size_t i = 0; i < toks.size(); i++) q.type += (i ? " " : "") + toks[i];
        if (q.type == "sampler_t")
            q.kind = 's';
        else if (q.type.find("image2d") != std::string::npos)
            q.kind = 'i';
        else
            q.kind = ptr ? 'p' : 'v';
        params.push_back(q);
    }
    return true;
}

bool uses_barriers(const std::string &src) { return src.find("barrier") != std::string::npos; }

std::string rewrite(const std::string &src)
{
    std::string s = std::regex_replace(src, std::regex("\\((float|double|int|uint)([2348])\\)\\s*\\("), "make_$1$2(");
    s = std::regex_replace(s, std::regex("\\.(xz|xy)\\b"), ".$1()");
    if (uses_barriers(s)) {
        // work-group kernels: __local arrays shared by the team, barrier() = the team's barrier
        s = std::regex_replace(s, std::regex("\\b(__local|local)\\b"), "static");
        s = std::regex_replace(s, std::regex("\\bbarrier\\s*\\([^)]*\\)"), "clgen_barrier()");
    }
    s = std::regex_replace(s, std::regex("(\\w+)\\.s([0-9a-f])\\b"), "clgen_elem($1, 0x$2)");
    s = std::regex_replace(s, std::regex("#pragma OPENCL[^\\n]*"), "");
    return s;
}

struct Compiled {
    void *handle = nullptr;
    void (*run)(void **, const size_t *, const size_t *) = nullptr;
    void (*run_groups)(void **, const size_t *, const size_t *) = nullptr; /* kernels with barriers */
};
std::map<std::string, Compiled> g_cache;
std::mutex g_mutex;

bool file_exists(const std::string &p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

}  // namespace

struct refshim_jit {
    std::vector<Param> params;
    Compiled prog;
};

extern "C" {

void refshim_set_device_limits(unsigned long global_mem, unsigned long max_alloc, unsigned long max_work_group)
{
    g_global_mem = global_mem;
    g_max_alloc = max_alloc;
    g_max_work_group = max_work_group;
}

void refshim_set_dirs(const char *kernels_dir, const char *shim_dir, const char *cache_dir)
{
    g_kernels_dir = kernels_dir ? kernels_dir : "";
    g_shim_dir = shim_dir ? shim_dir : "";
    g_cache_dir = cache_dir ? cache_dir : "";
}

GValue *ufo_gpu_node_get_info(UfoGpuNode *, UfoGpuNodeInfo info)
{
    GValue *v = (GValue *)calloc(1, sizeof(GValue));
    switch (info) {
        case UFO_GPU_NODE_INFO_NAME:
            v->g_type = G_TYPE_STRING;
            v->data.s = "GENERIC"; /* no entry of the reference's node table: default burst */
            break;
        case UFO_GPU_NODE_INFO_GLOBAL_MEM_SIZE:
            v->g_type = G_TYPE_ULONG;
            v->data.ul = g_global_mem;
            break;
        case UFO_GPU_NODE_INFO_MAX_MEM_ALLOC_SIZE:
            v->g_type = G_TYPE_ULONG;
            v->data.ul = g_max_alloc;
            break;
        case UFO_GPU_NODE_INFO_LOCAL_MEM_SIZE:
            v->g_type = G_TYPE_ULONG;
            v->data.ul = 48ul << 10;
            break;
        case UFO_GPU_NODE_INFO_MAX_WORK_GROUP_SIZE:
            v->g_type = G_TYPE_ULONG;
            v->data.ul = g_max_work_group;
            break;
    }
    return v;
}

// A kernel file of the reference (src/kernels, src/kernels/templates) or one
// written before the run into the cache folder (the generated lamino kernels).
static bool read_kernel_file(const std::string &filename, std::string &out)
{
    for (const std::string &dir : {g_kernels_dir, g_kernels_dir + "/templates", g_cache_dir}) {
        std::ifstream f(dir + "/" + filename);
        if (f) {
            std::stringstream ss;
            ss << f.rdbuf();
            out = ss.str();
            return true;
        }
    }
    return false;
}

gchar *ufo_resources_get_kernel_source(UfoResources *, const gchar *filename, GError **err)
{
    std::string src;
    if (!read_kernel_file(filename, src)) {
        g_set_error(err, 0, 0, "kernel source %s not found under %s", filename, g_kernels_dir.c_str());
        return NULL;
    }
    return g_strdup(src.c_str());
}

cl_kernel ufo_resources_get_kernel_from_source(UfoResources *, const gchar *source, const gchar *name, const gchar *,
                                               GError **err)
{
    std::vector<Param> params;
    const std::string body = rewrite(source);
    if (!parse_signature(body, name, params)) {
        g_set_error(err, 0, 0, "kernel %s: signature not understood", name);
        return NULL;
    }
    std::ostringstream call, w;
    call << name << "(";
    for (size_t i = 0; i < params.size(); i++) {
        const Param &p = params[i];
        if (i) call << ", ";
        if (p.kind == 'p')
            call << "(" << p.type << " *)a[" << i << "]";
        else if (p.kind == 's')
            call << "*(sampler_t *)a[" << i << "]";
        else
            call << "*(" << p.type << " *)a[" << i << "]";
    }
    call << ")";
    const bool groups = uses_barriers(body);
    w << "#include \"clc_gen.hpp\"\n" << body
      << "\n\nextern \"C\" __attribute__((visibility(\"default\"))) void refshim_gen_run(void **a, const size_t *g, "
      << "const size_t *l)\n{\n    (void)l;\n    CLGEN_NDRANGE(g, " << call.str() << ");\n}\n";
    if (groups)
        w << "extern \"C\" __attribute__((visibility(\"default\"))) void refshim_gen_run_groups(void **a, "
          << "const size_t *g, const size_t *l)\n{\n    CLGEN_WORKGROUPS(g, l, " << call.str() << ");\n}\n";
    const std::string code = w.str();
    const std::string key = std::to_string(std::hash<std::string>()(code));

    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = g_cache.find(key);
    if (it == g_cache.end()) {
        mkdir(g_cache_dir.c_str(), 0755);
        const std::string base = g_cache_dir + "/k" + key, so = base + ".so";
        if (!file_exists(so)) {
            std::ofstream(base + ".cpp") << code;
            const std::string tmp = base + "." + std::to_string(getpid()) + ".so";
            const std::string cmd = "g++ -O2 -std=c++17 -fPIC -shared -fopenmp -w -Wno-psabi -Wno-narrowing -mfma -ffp-contract=fast "
                                    "-fvisibility=hidden -I'" + g_shim_dir + "' -o '" + tmp + "' '" + base +
                                    ".cpp' > '" + base + ".log' 2>&1 && mv -f '" + tmp + "' '" + so + "'";
            if (system(cmd.c_str()) != 0) {
                g_set_error(err, 0, 0, "kernel %s: CPU compilation failed (%s.log)", name, base.c_str());
                return NULL;
            }
        }
        Compiled c;
        c.handle = dlopen(so.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!c.handle) {
            g_set_error(err, 0, 0, "kernel %s: %s", name, dlerror());
            return NULL;
        }
        c.run = (void (*)(void **, const size_t *, const size_t *))dlsym(c.handle, "refshim_gen_run");
        c.run_groups = (void (*)(void **, const size_t *, const size_t *))dlsym(c.handle, "refshim_gen_run_groups");
        it = g_cache.emplace(key, c).first;
    }
    cl_kernel k = (cl_kernel)calloc(1, sizeof(refshim_kernel));
    snprintf(k->name, sizeof k->name, "%s", name);
    k->jit = new refshim_jit{params, it->second};
    return k;
}

cl_kernel refshim_jit_from_file(const char *file, const char *name, GError **err)
{
    std::string src;
    if (!read_kernel_file(file, src)) {
        g_set_error(err, 0, 0, "kernel file %s not found", file);
        return NULL;
    }
    return ufo_resources_get_kernel_from_source(NULL, src.c_str(), name, NULL, err);
}

void refshim_jit_dispatch(refshim_kernel *k, guint ndims, const gsize *global, const gsize *local)
{
    const std::vector<Param> &params = k->jit->params;
    std::vector<void *> a(params.size());
    std::vector<image2d_t> images(params.size());
    std::vector<image2d_array_t> arrays(params.size());
    std::vector<sampler_t> samplers(params.size());
    // value arguments are copied to 64-byte aligned slots: OpenCL vector types
    // (double3, float8, float16) are over-aligned and AVX loads need it
    struct alignas(64) Slot {
        unsigned char b[64];
    };
    std::vector<Slot> values(params.size());
    for (size_t i = 0; i < params.size(); i++) {
        memcpy(values[i].b, k->args[i], sizeof values[i].b);
        void *slot = values[i].b;
        switch (params[i].kind) {
            case 'p':
                a[i] = (*(cl_mem *)slot)->host;
                break;
            case 'i': {
                cl_mem m = *(cl_mem *)slot;
                if (params[i].type == "image2d_array_t") {
                    const int type = m->channel_type == CL_HALF_FLOAT ? 1 : (m->channel_type == CL_UNSIGNED_INT8 ? 2 : 0);
                    arrays[i] = image2d_array_t{m->host, m->width, m->height, m->layers, m->channels, type};
                    a[i] = &arrays[i];
                } else {
                    images[i] = image2d_t{(const float *)m->host, m->width, m->height};
                    a[i] = &images[i];
                }
                break;
            }
            case 's':
                samplers[i] = (*(cl_sampler *)slot)->bits;
                a[i] = &samplers[i];
                break;
            default:
                a[i] = slot;
        }
    }
    size_t g[3] = {global[0], ndims > 1 ? global[1] : 1, ndims > 2 ? global[2] : 1};
    size_t l[3] = {1, 1, 1};
    if (local)
        for (guint d = 0; d < ndims; d++) l[d] = local[d];
    if (local && k->jit->prog.run_groups)
        k->jit->prog.run_groups(a.data(), g, l);
    else
        k->jit->prog.run(a.data(), g, l);
}

// ------------------------------------------------------------------ images, samplers, copies

static cl_mem new_image(size_t width, size_t height, size_t layers, const cl_image_format *fmt)
{
    cl_mem m = (cl_mem)calloc(1, sizeof(refshim_mem));
    m->is_image = 1;
    m->owned = 1;
    m->width = (int)width;
    m->height = (int)height;
    m->layers = (int)(layers ? layers : 1);
    switch (fmt->image_channel_order) {
        case CL_RGBA: m->channels = 4; break;
        case CL_RG: m->channels = 2; break;
        default: m->channels = 1; break;
    }
    m->channel_type = fmt->image_channel_data_type;
    m->elem_bytes = fmt->image_channel_data_type == CL_FLOAT ? 4 : (fmt->image_channel_data_type == CL_HALF_FLOAT ? 2 : 1);
    m->size = width * height * m->layers * m->channels * m->elem_bytes;
    m->host = calloc(1, m->size ? m->size : 1);
    return m;
}

cl_mem clCreateImage2D(cl_context, cl_mem_flags, const cl_image_format *fmt, size_t width, size_t height, size_t,
                       void *host_ptr, cl_int *err)
{
    cl_mem m = new_image(width, height, 1, fmt);
    if (host_ptr) memcpy(m->host, host_ptr, m->size);
    if (err) *err = CL_SUCCESS;
    return m;
}

cl_mem clCreateImage(cl_context, cl_mem_flags, const cl_image_format *fmt, const cl_image_desc *desc, void *host_ptr,
                     cl_int *err)
{
    const size_t layers = desc->image_type == CL_MEM_OBJECT_IMAGE2D_ARRAY ? desc->image_array_size : 1;
    cl_mem m = new_image(desc->image_width, desc->image_height, layers, fmt);
    if (host_ptr) memcpy(m->host, host_ptr, m->size);
    if (err) *err = CL_SUCCESS;
    return m;
}

cl_sampler clCreateSampler(cl_context, cl_bool normalized, cl_addressing_mode addressing, cl_filter_mode filter,
                           cl_int *err)
{
    cl_sampler s = (cl_sampler)calloc(1, sizeof(refshim_sampler));
    int bits = normalized ? CLK_NORMALIZED_COORDS_TRUE : CLK_NORMALIZED_COORDS_FALSE;
    switch (addressing) {
        case CL_ADDRESS_CLAMP_TO_EDGE: bits |= CLK_ADDRESS_CLAMP_TO_EDGE; break;
        case CL_ADDRESS_CLAMP: bits |= CLK_ADDRESS_CLAMP; break;
        case CL_ADDRESS_REPEAT: bits |= CLK_ADDRESS_REPEAT; break;
        case CL_ADDRESS_MIRRORED_REPEAT: bits |= CLK_ADDRESS_MIRRORED_REPEAT; break;
        default: bits |= CLK_ADDRESS_NONE; break;
    }
    bits |= filter == CL_FILTER_LINEAR ? CLK_FILTER_LINEAR : CLK_FILTER_NEAREST;
    s->bits = bits;
    if (err) *err = CL_SUCCESS;
    return s;
}

cl_int clReleaseSampler(cl_sampler s)
{
    free(s);
    return CL_SUCCESS;
}

cl_int clWaitForEvents(cl_uint, const cl_event *) { return CL_SUCCESS; }
cl_int clReleaseEvent(cl_event) { return CL_SUCCESS; }

static size_t texel_bytes(cl_mem m) { return (size_t)m->channels * m->elem_bytes; }

cl_int clEnqueueCopyBufferToImage(cl_command_queue, cl_mem src, cl_mem dst, size_t src_offset, const size_t *origin,
                                  const size_t *region, cl_uint, const cl_event *, cl_event *event)
{
    const size_t tb = texel_bytes(dst), row = region[0] * tb;
    const char *s = (const char *)src->host + src_offset;
    for (size_t z = 0; z < region[2]; z++)
        for (size_t y = 0; y < region[1]; y++) {
            char *d = (char *)dst->host + (((origin[2] + z) * dst->height + origin[1] + y) * dst->width + origin[0]) * tb;
            memcpy(d, s, row);
            s += row;
        }
    if (event) *event = NULL;
    return CL_SUCCESS;
}

cl_int clEnqueueCopyImage(cl_command_queue, cl_mem src, cl_mem dst, const size_t *so, const size_t *dorg,
                          const size_t *region, cl_uint, const cl_event *, cl_event *event)
{
    const size_t tb = texel_bytes(dst), row = region[0] * tb;
    for (size_t z = 0; z < region[2]; z++)
        for (size_t y = 0; y < region[1]; y++) {
            const char *s = (const char *)src->host + (((so[2] + z) * src->height + so[1] + y) * src->width + so[0]) * tb;
            char *d = (char *)dst->host + (((dorg[2] + z) * dst->height + dorg[1] + y) * dst->width + dorg[0]) * tb;
            memcpy(d, s, row);
        }
    if (event) *event = NULL;
    return CL_SUCCESS;
}

cl_int clEnqueueCopyBufferRect(cl_command_queue, cl_mem src, cl_mem dst, const size_t *so, const size_t *dorg,
                               const size_t *region, size_t src_row_pitch, size_t src_slice_pitch,
                               size_t dst_row_pitch, size_t dst_slice_pitch, cl_uint, const cl_event *,
                               cl_event *event)
{
    if (!src_row_pitch) src_row_pitch = region[0];
    if (!src_slice_pitch) src_slice_pitch = region[1] * src_row_pitch;
    if (!dst_row_pitch) dst_row_pitch = region[0];
    if (!dst_slice_pitch) dst_slice_pitch = region[1] * dst_row_pitch;
    for (size_t z = 0; z < region[2]; z++)
        for (size_t y = 0; y < region[1]; y++) {
            const char *s = (const char *)src->host + (so[2] + z) * src_slice_pitch + (so[1] + y) * src_row_pitch + so[0];
            char *d = (char *)dst->host + (dorg[2] + z) * dst_slice_pitch + (dorg[1] + y) * dst_row_pitch + dorg[0];
            memcpy(d, s, region[0]);
        }
    if (event) *event = NULL;
    return CL_SUCCESS;
}

}  // extern "C"
