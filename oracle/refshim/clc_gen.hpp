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

static thread_local size_t clgen_gid[3], clgen_gsz[3];
inline size_t get_global_id(int d) { return clgen_gid[d]; }
inline size_t get_global_size(int d) { return clgen_gsz[d]; }

// Runs CALL once per work-item of the global range g (work-items of these
// kernels are independent: each writes its own voxel).
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
