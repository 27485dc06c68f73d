// Kernel-language prelude for the OpenCL C sources that ref_clc_jit.cpp
// compiles for the CPU at run time (the reference's generated general- and
// laminographic backprojection kernels).  Address-space qualifiers vanish,
// OpenCL vectors are plain structs (3-vectors padded to the size of 4-vectors,
// as in OpenCL), and the built-ins those kernels call are spelled out: mad as a
// fused multiply-add, native_divide as a division, dot, clamp, conversions.
// The rewrite in ref_clc_jit.cpp turns vector literals into make_<type>()
// calls, ".xz" into .xz() and ".sN" element access into clgen_elem(v, N).
// Test infrastructure only.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>

#include <omp.h>

#include "clc_types.hpp"

#define kernel
#define __kernel
#define global
#define __global
#define local
#define __local
#define constant const
#define __constant const
#define read_only
#define write_only
#define __read_only
#define __write_only

typedef _Float16 half;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;

struct double2 {
    double x, y;
};
struct alignas(16) float3 {
    float x, y, z, pad_;
    float2 xz() const { return {x, z}; }
};
struct alignas(32) double3 {
    double x, y, z, pad_;
    double2 xz() const { return {x, z}; }
};
struct alignas(16) int3 {
    int x, y, z, pad_;
};
struct int2 {
    int x, y;
};
struct int4 {
    int x, y, z, w;
};
struct uint4 {
    unsigned x, y, z, w;
};
struct alignas(32) float8 {
    float s[8];
};
struct alignas(64) float16 {
    float s[16];
};

inline double2 make_double2(double a, double b) { return {a, b}; }
inline float3 make_float3(float a, float b, float c) { return {a, b, c, 0.f}; }
inline double3 make_double3(double a, double b, double c) { return {a, b, c, 0.0}; }
inline int3 make_int3(int a, int b, int c) { return {a, b, c, 0}; }
inline int2 make_int2(int a, int b) { return {a, b}; }
inline int4 make_int4(int a, int b, int c, int d) { return {a, b, c, d}; }
inline float4 make_float4(float a, float b, float c, float d) { return {a, b, c, d}; }
inline float4 make_float4(float4 v) { return v; }
inline uint4 make_uint4(uint4 v) { return v; }

inline float4 operator+(float4 a, float4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline float4 &operator+=(float4 &a, float4 b) { a = a + b; return a; }
inline float4 operator*(float4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline float4 operator/(float4 a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
inline float2 operator/(float2 a, float s) { return {a.x / s, a.y / s}; }
inline uint4 operator+(uint4 a, uint4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline uint4 &operator+=(uint4 &a, uint4 b) { a = a + b; return a; }

template <typename V> inline float clgen_elem(const V &v, int i) { return reinterpret_cast<const float *>(&v)[i]; }

inline double2 operator+(double2 a, double2 b) { return {a.x + b.x, a.y + b.y}; }
inline double2 operator-(double2 a, double2 b) { return {a.x - b.x, a.y - b.y}; }

#define CLGEN_VEC3_OPS(V, S)                                                                         \
    inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z, 0}; }                     \
    inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z, 0}; }                     \
    inline V operator-(V a) { return {-a.x, -a.y, -a.z, 0}; }                                         \
    inline V operator*(V a, V b) { return {a.x * b.x, a.y * b.y, a.z * b.z, 0}; }                     \
    inline V operator*(S s, V a) { return {s * a.x, s * a.y, s * a.z, 0}; }                           \
    inline V operator*(V a, S s) { return {a.x * s, a.y * s, a.z * s, 0}; }                           \
    inline V &operator+=(V &a, V b) { a = a + b; return a; }                                          \
    inline V &operator-=(V &a, V b) { a = a - b; return a; }                                          \
    inline V &operator*=(V &a, S s) { a = a * s; return a; }                                          \
    inline S dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }                              \
    inline V mad(S s, V b, V c) { return {std::fma(s, b.x, c.x), std::fma(s, b.y, c.y), std::fma(s, b.z, c.z), 0}; } \
    inline V mad(V a, V b, V c) { return {std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y), std::fma(a.z, b.z, c.z), 0}; }
CLGEN_VEC3_OPS(float3, float)
CLGEN_VEC3_OPS(double3, double)

inline float mad(float a, float b, float c) { return std::fma(a, b, c); }
inline double mad(double a, double b, double c) { return std::fma(a, b, c); }
inline float native_divide(float a, float b) { return a / b; }
inline double native_divide(double a, double b) { return a / b; }
inline float clamp(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline double clamp(double x, double lo, double hi) { return std::fmin(std::fmax(x, lo), hi); }
inline float sincos(float x, float *c)
{
    *c = std::cos(x);
    return std::sin(x);
}
inline float2 convert_float2(float2 v) { return v; }
inline float2 convert_float2(double2 v) { return {(float)v.x, (float)v.y}; }

#define M_PI_F 3.14159265358979323846f
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

static thread_local size_t clgen_gid[3], clgen_gsz[3], clgen_lid[3], clgen_lsz[3], clgen_grp[3];
inline size_t get_global_id(int d) { return clgen_gid[d]; }
inline size_t get_global_size(int d) { return clgen_gsz[d]; }
inline size_t get_local_id(int d) { return clgen_lid[d]; }
inline size_t get_local_size(int d) { return clgen_lsz[d]; }
inline size_t get_group_id(int d) { return clgen_grp[d]; }
// barrier() of a work-group that runs as one OpenMP team (CLGEN_WORKGROUPS)
inline void clgen_barrier() { _Pragma("omp barrier") }

// --- 2-D image arrays (texel (i, j) of layer l; exact linear weights as read_imagef on 2-D images)
inline float clgen_channel(const image2d_array_t &im, size_t texel, int c)
{
    const size_t k = texel * im.channels + c;
    switch (im.type) {
        case 1: return (float)((const _Float16 *)im.data)[k];
        case 2: return (float)((const unsigned char *)im.data)[k];
        default: return ((const float *)im.data)[k];
    }
}
inline float4 clgen_texel(const image2d_array_t &im, int i, int j, int l, int addr)
{
    if (i < 0 || j < 0 || i >= im.width || j >= im.height) {
        if (addr == CLK_ADDRESS_CLAMP) return float4{0.f, 0.f, 0.f, im.channels == 4 ? 0.f : 1.f};
        i = i < 0 ? 0 : (i >= im.width ? im.width - 1 : i);
        j = j < 0 ? 0 : (j >= im.height ? im.height - 1 : j);
    }
    const size_t t = ((size_t)l * im.height + j) * im.width + i;
    float v[4] = {0.f, 0.f, 0.f, 1.f};
    for (int c = 0; c < im.channels; c++) v[c] = clgen_channel(im, t, c);
    return float4{v[0], v[1], v[2], v[3]};
}
inline int clgen_layer(const image2d_array_t &im, float z)
{
    int l = (int)std::rint(z);
    return l < 0 ? 0 : (l >= im.layers ? im.layers - 1 : l);
}
inline float4 read_imagef(image2d_array_t im, sampler_t s, float4 c)
{
    const int addr = s & 0xe, l = clgen_layer(im, c.z);
    if (!(s & CLK_FILTER_LINEAR)) return clgen_texel(im, (int)std::floor(c.x), (int)std::floor(c.y), l, addr);
    const float u = c.x - 0.5f, w = c.y - 0.5f;
    const float fu = std::floor(u), fw = std::floor(w);
    const float a = u - fu, b = w - fw;
    const int i = (int)fu, j = (int)fw;
    const float4 t00 = clgen_texel(im, i, j, l, addr), t10 = clgen_texel(im, i + 1, j, l, addr);
    const float4 t01 = clgen_texel(im, i, j + 1, l, addr), t11 = clgen_texel(im, i + 1, j + 1, l, addr);
    const float w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
    return float4{w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
                  w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
                  w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z,
                  w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w};
}
inline uint4 read_imageui(image2d_array_t im, sampler_t s, float4 c)
{
    const float4 t = clgen_texel(im, (int)std::floor(c.x), (int)std::floor(c.y), clgen_layer(im, c.z), s & 0xe);
    return uint4{(unsigned)t.x, (unsigned)t.y, (unsigned)t.z, (unsigned)t.w};
}
inline void clgen_store(image2d_array_t &im, int4 c, const float *v)
{
    const size_t t = ((size_t)c.z * im.height + c.y) * im.width + c.x;
    for (int k = 0; k < im.channels; k++) {
        const size_t e = t * im.channels + k;
        if (im.type == 1)
            ((_Float16 *)im.data)[e] = (_Float16)v[k];
        else if (im.type == 2)
            ((unsigned char *)im.data)[e] = (unsigned char)(v[k] < 0.f ? 0.f : (v[k] > 255.f ? 255.f : v[k]));
        else
            ((float *)im.data)[e] = v[k];
    }
}
inline void write_imagef(image2d_array_t im, int4 c, float4 v)
{
    const float a[4] = {v.x, v.y, v.z, v.w};
    clgen_store(im, c, a);
}
inline void write_imageui(image2d_array_t im, int4 c, uint4 v)
{
    const float a[4] = {(float)(v.x > 255u ? 255u : v.x), (float)(v.y > 255u ? 255u : v.y),
                        (float)(v.z > 255u ? 255u : v.z), (float)(v.w > 255u ? 255u : v.w)};
    clgen_store(im, c, a);
}

// Runs CALL once per work-item of the global range g, for kernels whose
// work-items are independent (each writes its own voxel).
#define CLGEN_NDRANGE(g, CALL)                                                       \
    do {                                                                             \
        const size_t g0 = (g)[0], g1 = (g)[1], g2 = (g)[2];                          \
        const long long total = (long long)(g0 * g1 * g2);                           \
        _Pragma("omp parallel for schedule(static)")                                 \
        for (long long t = 0; t < total; t++) {                                      \
            clgen_gid[0] = (size_t)t % g0;                                           \
            clgen_gid[1] = ((size_t)t / g0) % g1;                                    \
            clgen_gid[2] = (size_t)t / (g0 * g1);                                    \
            clgen_gsz[0] = g0;                                                       \
            clgen_gsz[1] = g1;                                                       \
            clgen_gsz[2] = g2;                                                       \
            CALL;                                                                    \
        }                                                                            \
    } while (0)

// Runs CALL once per work-item with work-groups of size l: the groups one after
// another, the work-items of a group as one OpenMP team, so that barrier() is
// the team's barrier and __local arrays (made static by the rewrite) are shared
// by the group.
#define CLGEN_WORKGROUPS(g, l, CALL)                                                 \
    do {                                                                             \
        const size_t n0 = (g)[0] / (l)[0], n1 = (g)[1] / (l)[1], n2 = (g)[2] / (l)[2]; \
        const int team = (int)((l)[0] * (l)[1] * (l)[2]);                            \
        for (size_t b2 = 0; b2 < n2; b2++)                                           \
            for (size_t b1 = 0; b1 < n1; b1++)                                       \
                for (size_t b0 = 0; b0 < n0; b0++) {                                 \
                    _Pragma("omp parallel num_threads(team)")                        \
                    {                                                                \
                        if (omp_get_num_threads() != team) abort();                  \
                        const size_t t = (size_t)omp_get_thread_num();               \
                        clgen_lid[0] = t % (l)[0];                                   \
                        clgen_lid[1] = (t / (l)[0]) % (l)[1];                        \
                        clgen_lid[2] = t / ((l)[0] * (l)[1]);                        \
                        const size_t bb[3] = {b0, b1, b2};                           \
                        for (int d = 0; d < 3; d++) {                                \
                            clgen_grp[d] = bb[d];                                    \
                            clgen_lsz[d] = (l)[d];                                   \
                            clgen_gsz[d] = (g)[d];                                   \
                            clgen_gid[d] = bb[d] * (l)[d] + clgen_lid[d];            \
                        }                                                            \
                        CALL;                                                        \
                    }                                                                \
                }                                                                    \
    } while (0)
