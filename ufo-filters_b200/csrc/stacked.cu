// stacked-backproject: the reference's multi-slice backprojection with three
// storage precisions (src/ufo-stacked-backproject-task.c:302-430,
// src/kernels/stacked-backproject.cl).
//
// Reference behaviour restated here:
//  * geometry: h = bx cos - by sin + axis (the sine enters with the opposite
//    sign to `backproject`), bx/by = pixel - axis + roi offset + 1/2, sum over
//    the sinogram's rows p of sample(h, p) using LUT entries offset + p, times
//    pi / rows;
//  * "single": FP32 sinogram, linear interpolation, zero outside;
//  * "half": the sinogram stored in FP16 (four slices per texel), linear
//    interpolation, FP32 sums;
//  * "int8": the whole input quantised to 8 bits, q = (uint)((v - min) *
//    (255 / (max - min))) with min/max over every value; nearest sample at
//    floor(h) clamped to the edge; integer sums; result ((sum * (max - min) /
//    255) + min) * pi / rows (the min is added once, as the reference does).
//
// B200 formulation.  "single" and "half" are the engine's own backprojectors
// (TMA-staged windows; FP16 slice-quad cells for "half") run with a mirrored
// sine table; this file adds the FP32 -> slice-quad packing for "half" and the
// whole int8 path: a min/max reduction, a packing kernel (four slices' bytes
// per 32-bit word) and a backprojector that sums byte pairs in 16-bit lanes of
// 32-bit registers (two adds per four slices, flushed every 256 angles).
#include <cuda_fp16.h>

#include <algorithm>

#include "ufob_internal.h"

namespace ufob {

// ------------------------------------------------------------ FP32 stack -> slice-quad cells

// cell (g, p, j), j <= W: halves (s0[j-1], s1[j-1], s2[j-1], s3[j-1], s0[j], .., s3[j]) of slices 4g..4g+3
__global__ void k_pack_quads(const float *__restrict__ in, uint32_t W, uint32_t P, uint32_t Z, uint32_t groups,
                             uint4 *__restrict__ out)
{
    const uint64_t cells = (uint64_t)groups * P * (W + 1);
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < cells; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(c % (W + 1));
        const uint64_t gp = c / (W + 1);
        const uint32_t p = (uint32_t)(gp % P), g = (uint32_t)(gp / P);
        float lo[4], hi[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t z = 4 * g + k;
            const float *row = in + ((uint64_t)z * P + p) * W;
            lo[k] = (z < Z && j >= 1) ? __ldg(row + j - 1) : 0.f;
            hi[k] = (z < Z && j < W) ? __ldg(row + j) : 0.f;
        }
        __half2 w0 = __floats2half2_rn(lo[0], lo[1]), w1 = __floats2half2_rn(lo[2], lo[3]);
        __half2 w2 = __floats2half2_rn(hi[0], hi[1]), w3 = __floats2half2_rn(hi[2], hi[3]);
        out[c] = make_uint4(*reinterpret_cast<uint32_t *>(&w0), *reinterpret_cast<uint32_t *>(&w1),
                            *reinterpret_cast<uint32_t *>(&w2), *reinterpret_cast<uint32_t *>(&w3));
    }
}

ufob_status pack_quads_launch(const float *d_in, uint32_t W, uint32_t P, uint32_t Z, void *d_out, cudaStream_t s)
{
    const uint32_t groups = (Z + 3) / 4;
    const uint64_t cells = (uint64_t)groups * P * (W + 1);
    if (!cells) return UFOB_OK;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((cells + 255) / 256, (uint64_t)num_sms() * 16);
    k_pack_quads<<<grid, 256, 0, s>>>(d_in, W, P, Z, groups, reinterpret_cast<uint4 *>(d_out));
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

// ------------------------------------------------------------ int8 path

// Order-preserving map of finite floats onto unsigned integers.
__device__ __forceinline__ uint32_t float_key(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float key_float(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// keys[0] = min key, keys[1] = max key (initialised to UINT_MAX / 0 by the host)
__global__ void k_minmax(const float *__restrict__ in, uint64_t n, uint32_t *__restrict__ keys)
{
    uint32_t kmin = 0xffffffffu, kmax = 0u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = float_key(__ldg(in + i));
        kmin = min(kmin, k);
        kmax = max(kmax, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(keys, kmin);
        atomicMax(keys + 1, kmax);
    }
}

// word (g, p, j): bytes of slices 4g..4g+3 (slices past Z are 0);
// interleave_uint, stacked-backproject.cl:236-253
__global__ void k_pack_u8(const float *__restrict__ in, uint32_t W, uint32_t P, uint32_t Z, uint32_t groups,
                          const uint32_t *__restrict__ keys, uint32_t *__restrict__ out)
{
    const float mn = key_float(keys[0]), mx = key_float(keys[1]);
    const float scale = __fdiv_rn(255.0f, __fsub_rn(mx, mn));
    const uint64_t words = (uint64_t)groups * P * W;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < words; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(c % W);
        const uint64_t gp = c / W;
        const uint32_t p = (uint32_t)(gp % P), g = (uint32_t)(gp / P);
        uint32_t w = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t z = 4 * g + k;
            if (z >= Z) break;
            const float v = __ldg(in + ((uint64_t)z * P + p) * W + j);
            const uint32_t q = min(__float2uint_rz(__fmul_rn(__fsub_rn(v, mn), scale)), 255u);
            w |= q << (8 * k);
        }
        out[c] = w;
    }
}

// One thread = one pixel of four slices; texture_uint + uninterleave_uint,
// stacked-backproject.cl:256-380.
__global__ void __launch_bounds__(256) k_bp_u8(const uint32_t *__restrict__ words, uint32_t W, uint32_t P, uint32_t Z,
                                               const float2 *__restrict__ sincos, uint32_t roi_x, uint32_t roi_y,
                                               uint32_t roi_w, uint32_t roi_h, float axis,
                                               const uint32_t *__restrict__ keys, float *__restrict__ out)
{
    const uint32_t x = blockIdx.x * 32 + threadIdx.x % 32, y = blockIdx.y * 8 + threadIdx.x / 32;
    const uint32_t g = blockIdx.z;
    if (x >= roi_w || y >= roi_h) return;
    const float bx = (float)(roi_x + x) - axis + 0.5f;
    const float by = (float)(roi_y + y) - axis + 0.5f;
    const uint32_t *base = words + (uint64_t)g * P * W;
    uint32_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (uint32_t p0 = 0; p0 < P; p0 += 256) {
        // byte pairs summed in 16-bit lanes: at most 256 * 255 < 65536 per lane
        uint32_t even = 0, odd = 0;
        const uint32_t p1 = min(P, p0 + 256);
        for (uint32_t p = p0; p < p1; p++) {
            const float2 sc = __ldg(&sincos[p]);  // (-sin, cos)
            const float h = fmaf(by, sc.x, fmaf(bx, sc.y, axis));
            const int i = min(max(__float2int_rd(h), 0), (int)W - 1);  // nearest, clamp to edge
            const uint32_t w = __ldg(base + (uint64_t)p * W + i);
            even += w & 0x00ff00ffu;
            odd += (w >> 8) & 0x00ff00ffu;
        }
        s0 += even & 0xffffu;
        s2 += even >> 16;
        s1 += odd & 0xffffu;
        s3 += odd >> 16;
    }
    const float mn = key_float(keys[0]), mx = key_float(keys[1]);
    const float scale = __fdiv_rn(__fsub_rn(mx, mn), 255.0f);
    const float pi_f = 3.14159265358979323846f;
    const uint32_t sums[4] = {s0, s1, s2, s3};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t z = 4 * g + k;
        if (z >= Z) break;
        const float v = __fadd_rn(__fmul_rn((float)sums[k], scale), mn);
        out[((uint64_t)z * roi_h + y) * roi_w + x] = __fdiv_rn(__fmul_rn(v, pi_f), (float)P);
    }
}

ufob_status stacked_u8_launch(const BPGeometry &g, const float *d_sino, void *d_work, uint32_t *d_keys, float *d_out,
                              cudaStream_t s)
{
    const uint32_t W = g.W, P = g.P, Z = g.nz, groups = (Z + 3) / 4;
    const uint64_t n = (uint64_t)W * P * Z;
    if (!n || !g.roi_w || !g.roi_h) return UFOB_OK;
    const uint32_t init[2] = {0xffffffffu, 0u};
    UFOB_CUDA_TRY(cudaMemcpyAsync(d_keys, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const uint32_t grid_r = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)num_sms() * 8);
    k_minmax<<<grid_r, 256, 0, s>>>(d_sino, n, d_keys);
    UFOB_CUDA_TRY(cudaGetLastError());
    const uint64_t words = (uint64_t)groups * P * W;
    const uint32_t grid_p = (uint32_t)std::min<uint64_t>((words + 255) / 256, (uint64_t)num_sms() * 16);
    k_pack_u8<<<grid_p, 256, 0, s>>>(d_sino, W, P, Z, groups, d_keys, reinterpret_cast<uint32_t *>(d_work));
    UFOB_CUDA_TRY(cudaGetLastError());
    dim3 grid((g.roi_w + 31) / 32, (g.roi_h + 7) / 8, groups);
    k_bp_u8<<<grid, 256, 0, s>>>(reinterpret_cast<const uint32_t *>(d_work), W, P, Z, g.d_sincos, g.roi_x, g.roi_y,
                                 g.roi_w, g.roi_h, g.axis, d_keys, d_out);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch(3);
    return UFOB_OK;
}

}  // namespace ufob
