// Compile OpenCL C kernel sources as C++: address-space qualifiers vanish,
// `kernel` functions get C linkage, and work-item ids come from the CPU
// NDRange driver in ref_runtime.cpp.  Vector literals such as (float2)(a, b)
// are rewritten to make_float2(a, b) by the build recipe (ref.mk) before
// compilation.  Test infrastructure only.
#pragma once
#include "clc_types.hpp"
#define kernel extern "C"
#define __kernel extern "C"
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
typedef unsigned int uint;
#define M_PI_F 3.14159265358979323846f
extern thread_local size_t clshim_gid[3], clshim_gsz[3];
inline size_t get_global_id(int d) { return clshim_gid[d]; }
inline size_t get_global_size(int d) { return clshim_gsz[d]; }
inline float sincos(float x, float *c)
{
    *c = std::cos(x);
    return std::sin(x);
}
inline float2 normalize(float2 v)
{
    float n = std::sqrt(v.x * v.x + v.y * v.y);
    return {v.x / n, v.y / n};
}
