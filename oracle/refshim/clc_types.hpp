// Types of the OpenCL C kernel-language shim (see clc_shim.hpp).  Test infrastructure only.
#pragma once
#include <cmath>
#include <cstddef>

struct float2 {
    float x, y;
};
inline float2 make_float2(float a, float b) { return float2{a, b}; }
inline float2 operator+(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
inline float2 operator-(float2 a, float2 b) { return {a.x - b.x, a.y - b.y}; }
inline float2 operator*(float s, float2 a) { return {s * a.x, s * a.y}; }
inline float2 operator*(float2 a, float s) { return {s * a.x, s * a.y}; }
inline float2 &operator+=(float2 &a, float2 b) { a.x += b.x; a.y += b.y; return a; }
struct float4 {
    float x, y, z, w;
};
typedef int sampler_t;
// OpenCL 1.2 sampler bits
#define CLK_NORMALIZED_COORDS_FALSE 0x0
#define CLK_NORMALIZED_COORDS_TRUE 0x1
#define CLK_ADDRESS_NONE 0x0
#define CLK_ADDRESS_CLAMP_TO_EDGE 0x2
#define CLK_ADDRESS_CLAMP 0x4
#define CLK_ADDRESS_REPEAT 0x6
#define CLK_ADDRESS_MIRRORED_REPEAT 0x8
#define CLK_FILTER_NEAREST 0x10
#define CLK_FILTER_LINEAR 0x20

struct image2d_t {
    const float *data;
    int width, height;
};

// Linear/nearest sampling with unnormalised coordinates: texel (i, j) is
// centred at (i + 0.5, j + 0.5); CLK_ADDRESS_CLAMP returns the border value 0
// outside the image, CLK_ADDRESS_CLAMP_TO_EDGE (and NONE) clamp the index.
float4 read_imagef(image2d_t img, sampler_t s, float2 coord);

extern thread_local size_t clshim_gid[3], clshim_gsz[3];
inline size_t get_global_id(int d) { return clshim_gid[d]; }
inline size_t get_global_size(int d) { return clshim_gsz[d]; }
