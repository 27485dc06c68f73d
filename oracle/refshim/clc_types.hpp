// Types of the OpenCL C kernel-language shim (see clc_shim.hpp, clc_gen.hpp).
// Test infrastructure only.
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
    float2 xy() const { return {x, y}; }
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

// A single-channel FP32 image (CL_INTENSITY / CL_R with CL_FLOAT).
struct image2d_t {
    const float *data;
    int width, height;
};

// A 2-D image array with 1, 2 or 4 channels per texel of FP32, FP16 or
// unsigned 8-bit values (type 0, 1, 2), layers stacked after each other.
struct image2d_array_t {
    void *data;
    int width, height, layers, channels, type;
};

inline float clshim_texel(const image2d_t &img, int i, int j, int addr)
{
    if (i < 0 || j < 0 || i >= img.width || j >= img.height) {
        if (addr == CLK_ADDRESS_CLAMP) return 0.f;
        i = i < 0 ? 0 : (i >= img.width ? img.width - 1 : i);
        j = j < 0 ? 0 : (j >= img.height ? img.height - 1 : j);
    }
    return img.data[(size_t)j * img.width + i];
}

// Linear/nearest sampling with unnormalised coordinates: texel (i, j) is
// centred at (i + 0.5, j + 0.5) and the linear weights are exact (the CPU
// OpenCL semantics); CLK_ADDRESS_CLAMP returns the border value 0 outside the
// image, CLK_ADDRESS_CLAMP_TO_EDGE (and NONE) clamp the index.
inline float4 read_imagef(image2d_t img, sampler_t s, float2 c)
{
    const int addr = s & 0xe;
    float v;
    if (s & CLK_FILTER_LINEAR) {
        const float u = c.x - 0.5f, w = c.y - 0.5f;
        const float fu = std::floor(u), fw = std::floor(w);
        const float a = u - fu, b = w - fw;
        const int i = (int)fu, j = (int)fw;
        v = (1.f - a) * (1.f - b) * clshim_texel(img, i, j, addr) + a * (1.f - b) * clshim_texel(img, i + 1, j, addr) +
            (1.f - a) * b * clshim_texel(img, i, j + 1, addr) + a * b * clshim_texel(img, i + 1, j + 1, addr);
    } else {
        v = clshim_texel(img, (int)std::floor(c.x), (int)std::floor(c.y), addr);
    }
    return float4{v, 0.f, 0.f, 1.f};
}
