// Parallel-beam backprojection (the `backproject` task).
//
// Reference behaviour (src/kernels/backproject.cl:50-94, src/ufo-backproject-task.c:96-267):
//   bx = x - axis + roi_x + 0.5,  by = y - axis + roi_y + 0.5
//   h_p = by * sin(theta_p) + bx * cos(theta_p) + axis
//   slice[y][x] = pi / P * sum_p lerp(sino[p], h_p)
// with the OpenCL linear sampler: texel i centred at i + 0.5, weights from
// frac(h - 0.5), and 0 outside the sinogram (CLK_ADDRESS_CLAMP).
//
// B200 design.  One CTA owns a TX x TY tile of output pixels for ZT slices of a
// stack that share the geometry (every slice of a parallel-beam stack uses the
// same angles), so the coordinate math of a pixel is done once per angle and
// reused across ZT slices.  For each angle only the detector window that the
// tile can reach (about sqrt(TX^2 + TY^2) bins) is needed; a producer thread
// issues one TMA copy (cp.async.bulk.tensor.3d, box = window x 1 angle x ZT
// slices) per angle into an S-stage shared-memory ring guarded by mbarriers, and
// TMA's zero fill for out-of-range coordinates reproduces CLK_ADDRESS_CLAMP.
// Consumers interpolate in software with full FP32 weights (the CPU-OpenCL
// semantics; GPU texture units quantise the weight to 1/256).  Two storage
// forms are handled:
//   SINO_F32         rows of FP32 bins: two 4-byte shared loads per update;
//   SINO_F16/BF16_PAIRS  32-bit pairs (s[j-1], s[j]) written by the filter
//                    stage: one 4-byte shared load per update (half the
//                    shared-memory gather bytes), FP32 accumulation.
// With `kahan` the sum over each angle block is formed in FP32 and added to the
// running total with Kahan compensation (cost amortised over the block).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>

#include "f32x2.cuh"
#include "tma.cuh"
#include "ufob_internal.h"

namespace ufob {

// ------------------------------------------------------------------ tensor maps

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D map over [nz][P][elems] 4-byte elements; box = (box_x, 1, box_z).
ufob_status make_sino_map(CUtensorMap *map, const void *base, uint32_t elems, uint32_t P, uint32_t nz,
                                 uint32_t pitch, uint64_t slice_pitch, uint32_t box_x, uint32_t box_z)
{
    auto fn = encode_fn();
    if (!fn) return fail(UFOB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[3] = {elems, P, nz};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)slice_pitch * 4};
    cuuint32_t box[3] = {box_x, 1, box_z};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(UFOB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): elems=%u P=%u nz=%u pitch=%u box=%u,%u",
                    (int)r, elems, P, nz, pitch, box_x, box_z);
    return UFOB_OK;
}

// 3-D map over [n][H][W] 4-byte elements (rows `pitch` elements apart, planes `plane` elements
// apart); box = (box_w, box_h, 1).  Coordinates outside the array read 0.
ufob_status make_image_map(CUtensorMap *map, const void *base, uint32_t W, uint32_t H, uint32_t n, uint64_t pitch,
                           uint64_t plane, uint32_t box_w, uint32_t box_h)
{
    auto fn = encode_fn();
    if (!fn) return fail(UFOB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[3] = {W, H, n};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)plane * 4};
    cuuint32_t box[3] = {box_w, box_h, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(UFOB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): image %ux%ux%u pitch=%llu box=%ux%u", (int)r,
                    W, H, n, (unsigned long long)pitch, box_w, box_h);
    return UFOB_OK;
}

// ------------------------------------------------------------------ sin/cos table

// mirror: store -sin, i.e. h = bx cos - by sin + axis (the stacked-backproject orientation,
// src/kernels/stacked-backproject.cl:77)
__global__ void k_sincos(double angle_offset, double step, uint32_t lut_offset, uint32_t P, int mirror, float2 *out)
{
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double s, c;
    sincos(angle_offset + (double)(lut_offset + p) * step, &s, &c);  // FP64, cast to FP32 as the reference LUTs
    const float fs = (float)s;
    out[p] = make_float2(mirror ? -fs : fs, (float)c);
}

ufob_status sincos_table_launch(double angle_offset, double step, uint32_t lut_offset, uint32_t P, float2 *d_out,
                                cudaStream_t stream, bool mirror)
{
    if (!P) return UFOB_OK;
    k_sincos<<<(P + 255) / 256, 256, 0, stream>>>(angle_offset, step, lut_offset, P, mirror ? 1 : 0, d_out);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

// ------------------------------------------------------------------ linear kernel

// Shared-memory stride (32-bit words) between the staged boxes of consecutive angles of the
// row kernel: 128-byte aligned for the TMA destination, and never a multiple of 512 bytes
// (measured on B200: a 512-byte stride made the 32 x 96 single-slice kernel 10% slower; the
// slice-quad kernel measured no such effect and keeps its plain 128-byte rounding).
constexpr int box_stride(int words)
{
    return ((words + 31) / 32 * 32) % 128 == 0 ? (words + 31) / 32 * 32 + 32 : (words + 31) / 32 * 32;
}

// Smallest s with s * s >= v.
constexpr int isqrt_ceil(int v)
{
    int r = 0;
    while (r * r < v) ++r;
    return r;
}

// Detector bins a TX x TY pixel tile reaches at any angle: its projected extent is at most the
// diagonal sqrt((TX-1)^2 + (TY-1)^2), plus one for the floor of the lower end.
template <int TX, int TY>
constexpr int tile_span()
{
    return 1 + isqrt_ceil((TX - 1) * (TX - 1) + (TY - 1) * (TY - 1)) < (int)(1.0 + 1.4143 * (TX > TY ? TX - 1 : TY - 1))
               ? 1 + isqrt_ceil((TX - 1) * (TX - 1) + (TY - 1) * (TY - 1))
               : (int)(1.0 + 1.4143 * (TX > TY ? TX - 1 : TY - 1));
}

template <int TX, int TY, int ZT, int A, int S>
struct BPShape {
    static constexpr int kThreads = 256;
    static constexpr int kRY = TY / (kThreads / TX);  // output rows per thread
    static_assert(TX == 32, "one warp spans the tile width");
    static_assert(kRY >= 1 && kRY * (kThreads / TX) == TY, "tile height");
    // window of detector elements reachable by the tile, plus interpolation tap,
    // one guard element on each side and 3 for the 16-byte TMA alignment
    static constexpr int kSpan = tile_span<TX, TY>();
    static constexpr int kWin = ((kSpan + 2 + 2 + 3) + 3) / 4 * 4;
    // each angle's box lands at a 128-byte aligned shared address (TMA destination rule)
    static constexpr int kAngleStride = box_stride(ZT * kWin);
    static constexpr int kStageElems = A * kAngleStride;
    static constexpr size_t kDataBytes = (size_t)S * kStageElems * 4;
    static constexpr size_t kWinOffset = kDataBytes;
    static constexpr size_t kBarOffset = (kWinOffset + (size_t)S * A * 4 + 7) / 8 * 8;
    static constexpr size_t kSmem = kBarOffset + (size_t)S * 8 + 128;  // +128: manual base alignment
};

// Interpolation weights (1 - w, w) with w = d + 0.5 as a packed 16-bit pair
// (lower half = weight of the lower tap): one pack and one packed FMA,
// (d, d) * (-1, 1) + (0.5, 0.5).
template <int KIND>
__device__ __forceinline__ uint32_t pair_weights(float d)
{
    uint32_t r;
    if (KIND == SINO_F16_PAIRS)
        asm("{\n\t.reg .b32 dd;\n\tcvt.rn.f16x2.f32 dd, %1, %1;\n\tfma.rn.f16x2 %0, dd, %2, %3;\n\t}"
            : "=r"(r)
            : "f"(d), "r"(0x3C00BC00u), "r"(0x38003800u));
    else
        asm("{\n\t.reg .b32 dd;\n\tcvt.rn.bf16x2.f32 dd, %1, %1;\n\tfma.rn.bf16x2 %0, dd, %2, %3;\n\t}"
            : "=r"(r)
            : "f"(d), "r"(0x3F80BF80u), "r"(0x3F003F00u));
    return r;
}

// (a0, a1) += k * (x0, x1) as one packed FP32 FMA (sm_100 fma.rn.f32x2).
__device__ __forceinline__ void fma2(float &a0, float &a1, float k, float x0, float x1)
{
    asm("{\n\t.reg .b64 a, x, kk;\n\tmov.b64 a, {%0, %1};\n\tmov.b64 x, {%2, %3};\n\tmov.b64 kk, {%4, %4};\n\t"
        "fma.rn.f32x2 a, kk, x, a;\n\tmov.b64 {%0, %1}, a;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "f"(x0), "f"(x1), "f"(k));
}

// acc += w_lo * s_lo + w_hi * s_hi with 16-bit operands and FP32 accumulation
// (sm_100 mixed-precision fma.rn.f32.{f16,bf16}; the products are exact in FP32).
template <int KIND>
__device__ __forceinline__ float pair_fma(uint32_t pair, uint32_t wts, float acc)
{
    if (KIND == SINO_F16_PAIRS)
        asm("{\n\t.reg .b16 l, h, wl, wh;\n\tmov.b32 {l, h}, %1;\n\tmov.b32 {wl, wh}, %2;\n\t"
            "fma.rn.f32.f16 %0, wl, l, %0;\n\tfma.rn.f32.f16 %0, wh, h, %0;\n\t}"
            : "+f"(acc)
            : "r"(pair), "r"(wts));
    else
        asm("{\n\t.reg .b16 l, h, wl, wh;\n\tmov.b32 {l, h}, %1;\n\tmov.b32 {wl, wh}, %2;\n\t"
            "fma.rn.f32.bf16 %0, wl, l, %0;\n\tfma.rn.f32.bf16 %0, wh, h, %0;\n\t}"
            : "+f"(acc)
            : "r"(pair), "r"(wts));
    return acc;
}

// Weights of two pixels at once: wlo = (1 - w0, 1 - w1), whi = (w0, w1) with
// w = d + 0.5, each lane rounded once as in pair_weights.
template <int KIND>
__device__ __forceinline__ void pair_weights2(float d0, float d1, uint32_t &wlo, uint32_t &whi)
{
    if (KIND == SINO_F16_PAIRS)
        asm("{\n\t.reg .b32 dd;\n\tcvt.rn.f16x2.f32 dd, %3, %2;\n\t"
            "fma.rn.f16x2 %0, dd, %4, %6;\n\tfma.rn.f16x2 %1, dd, %5, %6;\n\t}"
            : "=r"(wlo), "=r"(whi)
            : "f"(d0), "f"(d1), "r"(0xBC00BC00u), "r"(0x3C003C00u), "r"(0x38003800u));
    else
        asm("{\n\t.reg .b32 dd;\n\tcvt.rn.bf16x2.f32 dd, %3, %2;\n\t"
            "fma.rn.bf16x2 %0, dd, %4, %6;\n\tfma.rn.bf16x2 %1, dd, %5, %6;\n\t}"
            : "=r"(wlo), "=r"(whi)
            : "f"(d0), "f"(d1), "r"(0xBF80BF80u), "r"(0x3F803F80u), "r"(0x3F003F00u));
}

// acc += wlo[L] * s_lo + whi[L] * s_hi (lane L of the two weight pairs); same
// products and order as pair_fma.
template <int KIND, int L>
__device__ __forceinline__ void pair_fma_lanes(uint32_t pair, uint32_t wlo, uint32_t whi, float &acc)
{
    if (KIND == SINO_F16_PAIRS) {
        if (L == 0)
            asm("{\n\t.reg .b16 l, h, a, b, x;\n\tmov.b32 {l, h}, %1;\n\tmov.b32 {a, x}, %2;\n\tmov.b32 {b, x}, %3;\n\t"
                "fma.rn.f32.f16 %0, a, l, %0;\n\tfma.rn.f32.f16 %0, b, h, %0;\n\t}"
                : "+f"(acc)
                : "r"(pair), "r"(wlo), "r"(whi));
        else
            asm("{\n\t.reg .b16 l, h, a, b, x;\n\tmov.b32 {l, h}, %1;\n\tmov.b32 {x, a}, %2;\n\tmov.b32 {x, b}, %3;\n\t"
                "fma.rn.f32.f16 %0, a, l, %0;\n\tfma.rn.f32.f16 %0, b, h, %0;\n\t}"
                : "+f"(acc)
                : "r"(pair), "r"(wlo), "r"(whi));
    } else {
        if (L == 0)
            asm("{\n\t.reg .b16 l, h, a, b, x;\n\tmov.b32 {l, h}, %1;\n\tmov.b32 {a, x}, %2;\n\tmov.b32 {b, x}, %3;\n\t"
                "fma.rn.f32.bf16 %0, a, l, %0;\n\tfma.rn.f32.bf16 %0, b, h, %0;\n\t}"
                : "+f"(acc)
                : "r"(pair), "r"(wlo), "r"(whi));
        else
            asm("{\n\t.reg .b16 l, h, a, b, x;\n\tmov.b32 {l, h}, %1;\n\tmov.b32 {x, a}, %2;\n\tmov.b32 {x, b}, %3;\n\t"
                "fma.rn.f32.bf16 %0, a, l, %0;\n\tfma.rn.f32.bf16 %0, b, h, %0;\n\t}"
                : "+f"(acc)
                : "r"(pair), "r"(wlo), "r"(whi));
    }
}

// Shared-memory carve-up of one backprojection CTA.
template <typename Sh>
struct BPSmem {
    uint32_t *data;  // [S][A][ASTR], angle box = [ZT][WIN]
    int *win;        // [S][A] TMA x origin of each staged window
    uint64_t *full;  // [S] mbarriers
    __device__ __forceinline__ explicit BPSmem(unsigned char *smem_dyn)
    {
        unsigned char *raw =
            reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~(uintptr_t)127);
        data = reinterpret_cast<uint32_t *>(raw);
        win = reinterpret_cast<int *>(raw + Sh::kWinOffset);
        full = reinterpret_cast<uint64_t *>(raw + Sh::kBarOffset);
    }
};

// One output tile (TX x TY pixels x ZT slices) over all angles.  `g` counts
// the angle blocks this CTA has already staged through the S-slot ring, so
// one CTA can run many tiles back to back (slot = running block % S, barrier
// parity = (running block / S) & 1).  Returns false if a bounded wait gave up.
template <int TX, int TY, int ZT, int A, int S, int KIND, bool KAHAN, int FOLD = 1>
__device__ __forceinline__ bool bp_tile(const CUtensorMap *map, const BPArgs &args, int x0, int y0, int z0,
                                        const BPSmem<BPShape<TX, TY, ZT, A, S>> &sm, uint32_t &g)
{
    using Sh = BPShape<TX, TY, ZT, A, S>;
    constexpr int WIN = Sh::kWin;
    constexpr int RY = Sh::kRY;
    constexpr int YSTEP = 256 / TX;
    constexpr bool PAIRS = KIND != SINO_F32;
    constexpr int ASTR = Sh::kAngleStride;
    uint32_t *data = sm.data;
    int *win = sm.win;
    uint64_t *full = sm.full;

    const int tid = threadIdx.x;
    const uint32_t P = args.P;
    const int nblk = (int)((P + A - 1) / A);
    const float axis = args.axis;
    const uint32_t g0 = g;
    const float2 *sincos = args.sincos + (size_t)z0 * args.sincos_zstride;

    // Producer: stage block `blk` of this tile into slot (g0 + blk) % S.
    auto issue = [&](int blk) {
        const int slot = (int)((g0 + (uint32_t)blk) % S);
        const int p0 = blk * A;
        const int nval = min(A, (int)P - p0);
        mbar_arrive_expect_tx(&full[slot], (uint32_t)(nval * ZT * WIN * 4));
        const float cx0 = (float)(args.roi_x + x0) - axis + 0.5f, cx1 = cx0 + (float)(TX - 1);
        const float cy0 = (float)(args.roi_y + y0) - axis + 0.5f, cy1 = cy0 + (float)(TY - 1);
        for (int a = 0; a < nval; a++) {
            const float2 sc = sincos[p0 + a];
            float h0 = fmaf(cy0, sc.x, fmaf(cx0, sc.y, axis));
            float h1 = fmaf(cy0, sc.x, fmaf(cx1, sc.y, axis));
            float h2 = fmaf(cy1, sc.x, fmaf(cx0, sc.y, axis));
            float h3 = fmaf(cy1, sc.x, fmaf(cx1, sc.y, axis));
            float hmin = fminf(fminf(h0, h1), fminf(h2, h3));
            // first element needed: floor(hmin - 0.5) (+1 for pairs), minus one guard element
            int e = (int)floorf(hmin - 0.5f) + (PAIRS ? 1 : 0) - 1;
            e = max(min(e, 1 << 24), -(1 << 24));
            const int xs = e & ~3;  // 16-byte aligned TMA x coordinate (floor for negatives)
            win[slot * A + a] = xs;
            tma_load_3d(data + (size_t)(slot * A + a) * ASTR, map, &full[slot], xs, p0 + a, z0);
        }
    };

    if (tid == 0)
        for (int b = 0; b < S - 1 && b < nblk; b++) issue(b);

    const int lx = tid % TX, ly = tid / TX;
    const float bx = (float)(args.roi_x + x0 + lx) - axis + 0.5f;
    float by[RY];
#pragma unroll
    for (int j = 0; j < RY; j++) by[j] = (float)(args.roi_y + y0 + ly + j * YSTEP) - axis + 0.5f;
    constexpr bool PACK = ZT == 1 && RY % 2 == 0;
    uint64_t by2[RY / 2 > 0 ? RY / 2 : 1];
#pragma unroll
    for (int j = 0; j + 1 < RY; j += 2) by2[j / 2] = f2pack(by[j], by[j + 1]);

    float acc[RY][ZT], comp[RY][ZT];
#pragma unroll
    for (int j = 0; j < RY; j++)
#pragma unroll
        for (int z = 0; z < ZT; z++) acc[j][z] = comp[j][z] = 0.f;

    const float kMagic = 12582912.0f;  // 1.5 * 2^23: adding it rounds to an integer in the mantissa
    const int kMagicBits = __float_as_int(kMagic);
    const float eoff = axis - 1.0f + (PAIRS ? 1.0f : 0.0f);  // h - 0.5 - 0.5 (+1 for pairs)
    bool aborted = false;
    // partial sums run over FOLD angle blocks before they are added (compensated) into the totals
    float part[RY][ZT];
#pragma unroll
    for (int j = 0; j < RY; j++)
#pragma unroll
        for (int z = 0; z < ZT; z++) part[j][z] = 0.f;

    for (int blk = 0; blk < nblk; blk++) {
        if (tid == 0 && blk + S - 1 < nblk) issue(blk + S - 1);
        const int slot = (int)((g0 + (uint32_t)blk) % S);
        const uint32_t parity = ((g0 + (uint32_t)blk) / S) & 1u;
        const bool ok = mbar_wait_bounded(&full[slot], parity, kWaitLimitNs);
        const int p0 = blk * A;
        const int nval = min(A, (int)P - p0);
        const uint32_t *sdata = data + (size_t)slot * A * ASTR;

        if (ok && PACK) {
            // single slice: the coordinate chain of two output rows runs as packed
            // FP32 pairs, halving the per-update arithmetic that a slice stack
            // would otherwise share
            const uint64_t magic2 = f2pack(kMagic, kMagic), half2 = f2pack(0.5f, 0.5f);
#pragma unroll 2
            for (int a = 0; a < nval; a++) {
                const float2 sc = __ldg(&sincos[p0 + a]);
                const int xs = win[slot * A + a];
                const float t = fmaf(bx, sc.y, eoff - (float)xs);
                const uint64_t s2 = f2pack(sc.x, sc.x), t2 = f2pack(t, t);
                const uint32_t *row = sdata + a * ASTR;
#pragma unroll
                for (int j = 0; j < RY; j += 2) {
                    const uint64_t vv = f2fma(by2[j / 2], s2, t2);
                    const uint64_t r = f2add(vv, magic2);
                    const uint64_t d = f2sub(vv, f2sub(r, magic2));
                    float r0, r1;
                    f2unpack(r, r0, r1);
                    uint32_t e0 = (uint32_t)(__float_as_int(r0) - kMagicBits);
                    uint32_t e1 = (uint32_t)(__float_as_int(r1) - kMagicBits);
                    if (PAIRS) {
                        float d0, d1;
                        f2unpack(d, d0, d1);
                        e0 = min(e0, (uint32_t)(WIN - 1));
                        e1 = min(e1, (uint32_t)(WIN - 1));
                        uint32_t wlo, whi;
                        pair_weights2<KIND>(d0, d1, wlo, whi);
                        pair_fma_lanes<KIND, 0>(row[e0], wlo, whi, part[j][0]);
                        pair_fma_lanes<KIND, 1>(row[e1], wlo, whi, part[j + 1][0]);
                    } else {
                        const uint64_t w = f2add(d, half2), omw = f2sub(half2, d);
                        e0 = min(e0, (uint32_t)(WIN - 2));
                        e1 = min(e1, (uint32_t)(WIN - 2));
                        uint64_t pp = f2pack(part[j][0], part[j + 1][0]);
                        pp = f2fma(omw, f2pack(__uint_as_float(row[e0]), __uint_as_float(row[e1])), pp);
                        pp = f2fma(w, f2pack(__uint_as_float(row[e0 + 1]), __uint_as_float(row[e1 + 1])), pp);
                        f2unpack(pp, part[j][0], part[j + 1][0]);
                    }
                }
            }
        } else if (ok) {
#pragma unroll 2
            for (int a = 0; a < nval; a++) {
                const float2 sc = __ldg(&sincos[p0 + a]);
                const int xs = win[slot * A + a];
                const float t = fmaf(bx, sc.y, eoff - (float)xs);
                const uint32_t *row = sdata + a * ASTR;
#pragma unroll
                for (int j = 0; j < RY; j++) {
                    const float vv = fmaf(by[j], sc.x, t);  // element coordinate - 0.5
                    const float r = vv + kMagic;
                    const float fe = r - kMagic;            // rint(vv) == floor(vv + 0.5)
                    const float d = vv - fe;                // weight of the upper tap is d + 0.5
                    uint32_t e = (uint32_t)(__float_as_int(r) - kMagicBits);
                    if (PAIRS) {
                        // one 32-bit pair (s[j-1], s[j]) per update, FP32 accumulation of
                        // half-precision products: no conversions in the slice loop
                        const uint32_t wts = pair_weights<KIND>(d);
                        e = min(e, (uint32_t)(WIN - 1));  // guard: never leaves the angle's window
#pragma unroll
                        for (int z = 0; z < ZT; z++) part[j][z] = pair_fma<KIND>(row[z * WIN + e], wts, part[j][z]);
                    } else {
                        const float w = d + 0.5f, omw = 0.5f - d;
                        e = min(e, (uint32_t)(WIN - 2));
                        if (ZT % 2 == 0) {
                            // two slices per packed FP32 FMA (bit-identical to two fmaf)
#pragma unroll
                            for (int z = 0; z < ZT; z += 2) {
                                const float lo0 = __uint_as_float(row[z * WIN + e]);
                                const float hi0 = __uint_as_float(row[z * WIN + e + 1]);
                                const float lo1 = __uint_as_float(row[(z + 1) * WIN + e]);
                                const float hi1 = __uint_as_float(row[(z + 1) * WIN + e + 1]);
                                fma2(part[j][z], part[j][z + 1], omw, lo0, lo1);
                                fma2(part[j][z], part[j][z + 1], w, hi0, hi1);
                            }
                        } else {
#pragma unroll
                            for (int z = 0; z < ZT; z++) {
                                const float lo = __uint_as_float(row[z * WIN + e]);
                                const float hi = __uint_as_float(row[z * WIN + e + 1]);
                                part[j][z] = fmaf(omw, lo, part[j][z]);
                                part[j][z] = fmaf(w, hi, part[j][z]);
                            }
                        }
                    }
                }
            }
        }
        if ((blk + 1) % FOLD == 0 || blk + 1 == nblk) {
#pragma unroll
            for (int j = 0; j < RY; j++)
#pragma unroll
                for (int z = 0; z < ZT; z++) {
                    if (KAHAN) {
                        const float yk = part[j][z] - comp[j][z];
                        const float tk = acc[j][z] + yk;
                        comp[j][z] = (tk - acc[j][z]) - yk;
                        acc[j][z] = tk;
                    } else {
                        acc[j][z] += part[j][z];
                    }
                    part[j][z] = 0.f;
                }
        }
        if (__syncthreads_or(!ok)) {
            aborted = true;
            break;
        }
    }

    if (aborted) {
        if (tid == 0) {
            atomicExch(args.err, kErrTmaTimeout);
            // let every copy that may still be in flight land before the CTA exits
            for (int s = 0; s < S; s++) {
                for (int k = 0; k < 2; k++) mbar_wait_bounded(&full[s], (uint32_t)k, kWaitLimitNs / 8);
            }
        }
        return false;
    }
    g = g0 + (uint32_t)nblk;

    const float norm = args.norm;
#pragma unroll
    for (int j = 0; j < RY; j++) {
        const int y = y0 + ly + j * YSTEP;
        const int x = x0 + lx;
        if (y >= (int)args.roi_h || x >= (int)args.roi_w) continue;
#pragma unroll
        for (int z = 0; z < ZT; z++) {
            if (z0 + z >= (int)args.nz) break;
            args.out[((size_t)(z0 + z) * args.roi_h + y) * args.roi_w + x] = acc[j][z] * norm;
        }
    }
    return true;
}

template <int S>
__device__ __forceinline__ void init_ring(uint64_t *full)
{
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
}

template <int TX, int TY, int ZT, int A, int S, int KIND, bool KAHAN>
__global__ void __launch_bounds__(256) k_bp_linear(const __grid_constant__ CUtensorMap map, const BPArgs args)
{
    using Sh = BPShape<TX, TY, ZT, A, S>;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const BPSmem<Sh> sm(smem_dyn);
    init_ring<S>(sm.full);
    uint32_t g = 0;
    bp_tile<TX, TY, ZT, A, S, KIND, KAHAN>(&map, args, blockIdx.x * TX, blockIdx.y * TY, blockIdx.z * ZT, sm, g);
}

// ------------------------------------------------------------------ persistent batch kernel

// Work item = (job, tile); items are ordered by decreasing cost (largest
// angle count first) and taken dynamically from a device counter, so the
// CTAs of one persistent launch balance jobs of very different sizes.
template <int TX, int TY, int A, int S, int KIND, bool KAHAN>
__global__ void __launch_bounds__(256) k_bp_batch(const BatchBP *__restrict__ jobs, const uint2 *__restrict__ items,
                                                  uint32_t n_items, uint32_t *__restrict__ counter)
{
    using Sh = BPShape<TX, TY, 1, A, S>;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const BPSmem<Sh> sm(smem_dyn);
    __shared__ uint32_t s_item;
    init_ring<S>(sm.full);
    uint32_t g = 0;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        __syncthreads();
        if (it >= n_items) break;
        const uint2 w = items[it];  // (job, tile index)
        const BatchBP *j = jobs + w.x;
        const int tx = (int)(w.y % j->tiles_x), ty = (int)(w.y / j->tiles_x);
        if (threadIdx.x == 0)
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&j->map) : "memory");
        if (!bp_tile<TX, TY, 1, A, S, KIND, KAHAN, 2>(&j->map, j->args, tx * TX, ty * TY, 0, sm, g)) break;
    }
}

// ------------------------------------------------------------------ slice-quad FP16 kernel
//
// Storage form SINO_F16_QUADS, written by the filter stage for a stack: cell
// (g, p, j) of 16 bytes carries both interpolation taps of the four slices
// 4g..4g+3 at angle p,
//   word 0 = (s0[j-1], s1[j-1])   word 1 = (s2[j-1], s3[j-1])
//   word 2 = (s0[j],   s1[j])     word 3 = (s2[j],   s3[j])
// for j = 0..W (taps outside the row are 0).  One 128-bit shared load then
// feeds four updates, so the per-update instruction count is dominated by the
// FMAs themselves.  The TMA box is (4 words, window, 1 angle, ZT/4 groups);
// the window coordinate is not the innermost one and needs no alignment.
//
// The interpolation weight comes from the coordinate's fixed-point bits
// (coordinate + 1.5 * 2^13 leaves 10 fractional bits in the FP32 mantissa),
// assembled into the FP16 pair (1 + f, 1 + f) by one integer multiply-add and
// turned into (f, f) and (1 - f, 1 - f) exactly by two packed FP16 ops: no
// float-to-half conversion per update.  ACC selects how products are summed:
//   QACC_F32  FP32 accumulation of every product (mixed fma.rn.f32.f16);
//   QACC_LERP the lerp in packed FP16 (one rounding of the interpolated
//             value), FP32 accumulation via mixed-precision adds;
//   QACC_H16  lerp and sum of 8 consecutive angles in packed FP16, block
//             sums accumulated in FP32.
enum { QACC_F32 = 0, QACC_LERP = 1, QACC_H16 = 2 };

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// 4-D map over [groups][P][cells][4] 32-bit words; box = (4, box_cells, 1, box_groups).
ufob_status make_quad_map(CUtensorMap *map, const void *base, uint32_t cells, uint32_t P, uint32_t groups,
                          uint32_t pitch, uint64_t group_pitch, uint32_t box_cells, uint32_t box_groups)
{
    auto fn = encode_fn();
    if (!fn) return fail(UFOB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    cuuint64_t dims[4] = {4, cells, P, groups};
    cuuint64_t strides[3] = {16, (cuuint64_t)pitch * 16, (cuuint64_t)group_pitch * 16};
    cuuint32_t box[4] = {4, box_cells, 1, box_groups};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(UFOB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): cells=%u P=%u groups=%u pitch=%u box=%u,%u",
                    (int)r, cells, P, groups, pitch, box_cells, box_groups);
    return UFOB_OK;
}

template <int TX, int TY, int ZT, int A, int S>
struct BPQShape {
    static constexpr int kThreads = 256;
    static constexpr int kRY = TY / (kThreads / TX);
    static_assert(TX == 32 && ZT % 4 == 0, "one warp spans the tile width; whole slice groups");
    static_assert(kRY >= 1 && kRY * (kThreads / TX) == TY, "tile height");
    static constexpr int kSpan = tile_span<TX, TY>();
    static constexpr int kWin = (kSpan + 2 + 2 + 1) / 2 * 2;  // + tap + guard on each side
    static constexpr int kGroups = ZT / 4;
    static constexpr int kAngleStride = (kGroups * kWin * 4 + 31) / 32 * 32;  // words; 128-byte aligned boxes
    static constexpr int kStageElems = A * kAngleStride;
    static constexpr size_t kDataBytes = (size_t)S * kStageElems * 4;
    static constexpr size_t kWinOffset = kDataBytes;
    static constexpr size_t kBarOffset = (kWinOffset + (size_t)S * A * 4 + 7) / 8 * 8;
    static constexpr size_t kSmem = kBarOffset + (size_t)S * 8 + 128;
};

__device__ __forceinline__ uint32_t h2_fma(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

__device__ __forceinline__ uint32_t h2_mul(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

__device__ __forceinline__ uint32_t h2_add(uint32_t a, uint32_t b)
{
    uint32_t d;
    asm("add.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// (c0, c1) += (lo(x) * lo(w), hi(x) * lo(w)) with FP32 accumulation
__device__ __forceinline__ void mix_fma2(float &c0, float &c1, uint32_t x, uint32_t w)
{
    asm("{\n\t.reg .b16 xl, xh, wl, wh;\n\tmov.b32 {xl, xh}, %2;\n\tmov.b32 {wl, wh}, %3;\n\t"
        "fma.rn.f32.f16 %0, xl, wl, %0;\n\tfma.rn.f32.f16 %1, xh, wl, %1;\n\t}"
        : "+f"(c0), "+f"(c1)
        : "r"(x), "r"(w));
}

// (c0, c1) += (lo(x), hi(x)) with FP32 accumulation
__device__ __forceinline__ void mix_add2(float &c0, float &c1, uint32_t x)
{
    asm("{\n\t.reg .b16 xl, xh;\n\tmov.b32 {xl, xh}, %2;\n\t"
        "add.rn.f32.f16 %0, xl, %0;\n\tadd.rn.f32.f16 %1, xh, %1;\n\t}"
        : "+f"(c0), "+f"(c1)
        : "r"(x));
}

__device__ __forceinline__ void h2_flush(float &c0, float &c1, uint32_t &h)
{
    mix_add2(c0, c1, h);
    h = 0u;
}

template <int TX, int TY, int ZT, int A, int S, int ACC, bool KAHAN>
__device__ __forceinline__ bool bp_tile_quads(const CUtensorMap *map, const BPArgs &args, int x0, int y0, int z0,
                                              const BPSmem<BPQShape<TX, TY, ZT, A, S>> &sm, uint32_t &g)
{
    using Sh = BPQShape<TX, TY, ZT, A, S>;
    constexpr int WIN = Sh::kWin;
    constexpr int RY = Sh::kRY;
    constexpr int NG = Sh::kGroups;
    constexpr int YSTEP = 256 / TX;
    constexpr int ASTR = Sh::kAngleStride;
    constexpr int KB = ACC == QACC_H16 ? 8 : A;  // angles per FP16 block sum (QACC_H16)
    uint32_t *data = sm.data;
    int *win = sm.win;
    uint64_t *full = sm.full;

    const int tid = threadIdx.x;
    const uint32_t P = args.P;
    const int nblk = (int)((P + A - 1) / A);
    const float axis = args.axis;
    const uint32_t g0 = g;

    auto issue = [&](int blk) {
        const int slot = (int)((g0 + (uint32_t)blk) % S);
        const int p0 = blk * A;
        const int nval = min(A, (int)P - p0);
        mbar_arrive_expect_tx(&full[slot], (uint32_t)(nval * NG * WIN * 16));
        const float cx0 = (float)(args.roi_x + x0) - axis + 0.5f, cx1 = cx0 + (float)(TX - 1);
        const float cy0 = (float)(args.roi_y + y0) - axis + 0.5f, cy1 = cy0 + (float)(TY - 1);
        for (int a = 0; a < nval; a++) {
            const float2 sc = args.sincos[p0 + a];
            float h0 = fmaf(cy0, sc.x, fmaf(cx0, sc.y, axis));
            float h1 = fmaf(cy0, sc.x, fmaf(cx1, sc.y, axis));
            float h2 = fmaf(cy1, sc.x, fmaf(cx0, sc.y, axis));
            float h3 = fmaf(cy1, sc.x, fmaf(cx1, sc.y, axis));
            float hmin = fminf(fminf(h0, h1), fminf(h2, h3));
            // first cell needed: floor(hmin - 0.5) + 1, minus one guard cell
            int e = (int)floorf(hmin - 0.5f);
            e = max(min(e, 1 << 24), -(1 << 24));
            win[slot * A + a] = e;
            tma_load_4d(data + (size_t)(slot * A + a) * ASTR, map, &full[slot], 0, e, p0 + a, z0 / 4);
        }
    };

    if (tid == 0)
        for (int b = 0; b < S - 1 && b < nblk; b++) issue(b);

    const int lx = tid % TX, ly = tid / TX;
    const float bx = (float)(args.roi_x + x0 + lx) - axis + 0.5f;
    float by[RY];
#pragma unroll
    for (int j = 0; j < RY; j++) by[j] = (float)(args.roi_y + y0 + ly + j * YSTEP) - axis + 0.5f;

    float acc[RY][ZT], comp[RY][ZT];
#pragma unroll
    for (int j = 0; j < RY; j++)
#pragma unroll
        for (int z = 0; z < ZT; z++) acc[j][z] = comp[j][z] = 0.f;

    const float kFix = 12288.0f;  // 1.5 * 2^13: 10 fractional bits left in the mantissa
    const uint32_t kFixBits = __float_as_uint(kFix);
    const float toff = axis + 0.5f;  // cell coordinate = h - 0.5 + 1 - window origin
    bool aborted = false;
    // FP32 accumulation: partial sums run over FOLD angle blocks before they are added
    // (compensated) into the totals
    constexpr int FOLD = ACC == QACC_F32 ? 2 : 1;
    float part[RY][ZT];
#pragma unroll
    for (int j = 0; j < RY; j++)
#pragma unroll
        for (int z = 0; z < ZT; z++) part[j][z] = 0.f;

    for (int blk = 0; blk < nblk; blk++) {
        if (tid == 0 && blk + S - 1 < nblk) issue(blk + S - 1);
        const int slot = (int)((g0 + (uint32_t)blk) % S);
        const uint32_t parity = ((g0 + (uint32_t)blk) / S) & 1u;
        const bool ok = mbar_wait_bounded(&full[slot], parity, kWaitLimitNs);
        const int p0 = blk * A;
        const int nval = min(A, (int)P - p0);
        const uint32_t *sdata = data + (size_t)slot * A * ASTR;

        if (ok) {
            for (int a0 = 0; a0 < nval; a0 += KB) {
                uint32_t hs[RY][ZT / 2];
#pragma unroll
                for (int j = 0; j < RY; j++)
#pragma unroll
                    for (int q = 0; q < ZT / 2; q++) hs[j][q] = 0u;
                const int a1 = min(a0 + KB, nval);
#pragma unroll 2
                for (int a = a0; a < a1; a++) {
                    const float2 sc = __ldg(&args.sincos[p0 + a]);
                    const int xs = win[slot * A + a];
                    const float t = fmaf(bx, sc.y, toff - (float)xs);
                    const uint32_t *row = sdata + a * ASTR;
#pragma unroll
                    for (int j = 0; j < RY; j++) {
                        const float u = fmaf(by[j], sc.x, t);
                        const uint32_t bits = __float_as_uint(u + kFix);
                        const uint32_t e = min((uint32_t)((int)(bits - kFixBits) >> 10), (uint32_t)(WIN - 1));
                        const uint32_t pat = (bits & 1023u) * 0x00010001u + 0x3C003C00u;  // (1 + f, 1 + f)
                        const uint32_t whi = h2_add(pat, 0xBC00BC00u);                    // (f, f)
                        const uint32_t wlo = h2_fma(pat, 0xBC00BC00u, 0x40004000u);       // (1 - f, 1 - f)
#pragma unroll
                        for (int q = 0; q < NG; q++) {
                            const uint4 v = *reinterpret_cast<const uint4 *>(row + (q * WIN + (int)e) * 4);
                            float *pz = &part[j][4 * q];
                            if (ACC == QACC_F32) {
                                mix_fma2(pz[0], pz[1], v.x, wlo);
                                mix_fma2(pz[0], pz[1], v.z, whi);
                                mix_fma2(pz[2], pz[3], v.y, wlo);
                                mix_fma2(pz[2], pz[3], v.w, whi);
                            } else if (ACC == QACC_LERP) {
                                mix_add2(pz[0], pz[1], h2_fma(v.z, whi, h2_mul(v.x, wlo)));
                                mix_add2(pz[2], pz[3], h2_fma(v.w, whi, h2_mul(v.y, wlo)));
                            } else {
                                hs[j][2 * q] = h2_fma(v.z, whi, h2_fma(v.x, wlo, hs[j][2 * q]));
                                hs[j][2 * q + 1] = h2_fma(v.w, whi, h2_fma(v.y, wlo, hs[j][2 * q + 1]));
                            }
                        }
                    }
                }
                if (ACC == QACC_H16) {
#pragma unroll
                    for (int j = 0; j < RY; j++)
#pragma unroll
                        for (int q = 0; q < ZT / 2; q++) h2_flush(part[j][2 * q], part[j][2 * q + 1], hs[j][q]);
                }
            }
        }
        if ((blk + 1) % FOLD == 0 || blk + 1 == nblk) {
#pragma unroll
            for (int j = 0; j < RY; j++)
#pragma unroll
                for (int z = 0; z < ZT; z++) {
                    if (KAHAN) {
                        const float yk = part[j][z] - comp[j][z];
                        const float tk = acc[j][z] + yk;
                        comp[j][z] = (tk - acc[j][z]) - yk;
                        acc[j][z] = tk;
                    } else {
                        acc[j][z] += part[j][z];
                    }
                    part[j][z] = 0.f;
                }
        }
        if (__syncthreads_or(!ok)) {
            aborted = true;
            break;
        }
    }

    if (aborted) {
        if (tid == 0) {
            atomicExch(args.err, kErrTmaTimeout);
            for (int s = 0; s < S; s++) {
                for (int k = 0; k < 2; k++) mbar_wait_bounded(&full[s], (uint32_t)k, kWaitLimitNs / 8);
            }
        }
        return false;
    }
    g = g0 + (uint32_t)nblk;

    const float norm = args.norm;
#pragma unroll
    for (int j = 0; j < RY; j++) {
        const int y = y0 + ly + j * YSTEP;
        const int x = x0 + lx;
        if (y >= (int)args.roi_h || x >= (int)args.roi_w) continue;
#pragma unroll
        for (int z = 0; z < ZT; z++) {
            if (z0 + z >= (int)args.nz) break;
            args.out[((size_t)(z0 + z) * args.roi_h + y) * args.roi_w + x] = acc[j][z] * norm;
        }
    }
    return true;
}

template <int TX, int TY, int ZT, int A, int S, int ACC, bool KAHAN>
__global__ void __launch_bounds__(256, 2) k_bp_quads(const __grid_constant__ CUtensorMap map, const BPArgs args)
{
    using Sh = BPQShape<TX, TY, ZT, A, S>;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const BPSmem<Sh> sm(smem_dyn);
    init_ring<S>(sm.full);
    uint32_t g = 0;
    // Tiles in bands of 16 tile columns (8 for 8-row tiles), walked top to bottom: the CTAs
    // resident at one time cover a compact region whose projection spans ~30% of the detector
    // instead of a full-width strip (which re-read a whole slice group, larger than L2, once per
    // wave).  With 32x8 tiles, 8-column bands read 2.60 GB from DRAM for a 32-slice launch where
    // 16-column bands read 4.76 GB (393 MB of cells), in the same time.
    constexpr int GW = TY >= 16 ? 16 : 8;
    const int id = blockIdx.y * gridDim.x + blockIdx.x, band_tiles = GW * gridDim.y;
    const int band = id / band_tiles, r = id - band * band_tiles;
    const int bw = min(GW, (int)gridDim.x - band * GW);
    const int tx = band * GW + r % bw, ty = r / bw;
    bp_tile_quads<TX, TY, ZT, A, S, ACC, KAHAN>(&map, args, tx * TX, ty * TY, blockIdx.z * ZT, sm, g);
}

// ------------------------------------------------------------------ nearest kernel

// backproject.cl:24-48: index the flat sinogram with the OUTPUT width as row
// stride, truncating; indices outside the sinogram read 0 here (the reference
// has no bounds check).
__global__ void k_bp_nearest(const float *__restrict__ sino, uint32_t W, uint32_t P, uint32_t pitch,
                             uint64_t slice_pitch, uint32_t nz, const float2 *__restrict__ sincos, uint32_t roi_x,
                             uint32_t roi_y, uint32_t roi_w, uint32_t roi_h, float axis, float norm,
                             float *__restrict__ out)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const uint32_t z = blockIdx.z;
    if (x >= roi_w || y >= roi_h) return;
    const float bx = (float)x - axis + (float)roi_x + 0.5f;
    const float by = (float)y - axis + (float)roi_y + 0.5f;
    const float *s = sino + (size_t)z * slice_pitch;
    float sum = 0.f;
    for (uint32_t p = 0; p < P; p++) {
        const float2 sc = __ldg(&sincos[p]);
        const float h = fmaf(by, sc.x, fmaf(bx, sc.y, axis));  // axis + bx*cos + by*sin
        const float fi = __fadd_rn((float)(p * roi_w), h);
        const long long k = (long long)fi;
        if (k >= 0 && k < (long long)W * P) {
            // element k of the flat [P][W] sinogram, honouring the caller's pitch
            const long long row = k / W, col = k % W;
            sum += __ldg(s + row * pitch + col);
        }
    }
    out[((size_t)z * roi_h + y) * roi_w + x] = sum * norm;
}

ufob_status bp_nearest_launch(const BPGeometry &g, const float *d_sino, uint32_t pitch, uint64_t slice_pitch,
                              float *d_out, cudaStream_t stream)
{
    dim3 blk(32, 8), grd((g.roi_w + 31) / 32, (g.roi_h + 7) / 8, g.nz);
    if (!g.roi_w || !g.roi_h || !g.nz) return UFOB_OK;
    k_bp_nearest<<<grd, blk, 0, stream>>>(d_sino, g.W, g.P, pitch, slice_pitch, g.nz, g.d_sincos, g.roi_x, g.roi_y,
                                          g.roi_w, g.roi_h, g.axis, g.norm, d_out);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

// ------------------------------------------------------------------ dispatch

template <int TX, int TY, int ZT, int A, int S, int KIND, bool KAHAN>
static ufob_status launch_linear(const BPGeometry &g, const void *d_sino, uint32_t elems, uint32_t pitch,
                                 uint64_t slice_pitch, float *d_out, cudaStream_t stream, uint32_t zstride = 0)
{
    using Sh = BPShape<TX, TY, ZT, A, S>;
    auto kern = k_bp_linear<TX, TY, ZT, A, S, KIND, KAHAN>;
    static std::atomic<uint64_t> attr_devs{0};
    UFOB_CUDA_TRY(smem_limit_per_device(kern, (int)Sh::kSmem, attr_devs));
    CUtensorMap map;
    UFOB_TRY(make_sino_map(&map, d_sino, elems, g.P, g.nz, pitch, slice_pitch, Sh::kWin, ZT));
    BPArgs a;
    a.P = g.P;
    a.nz = g.nz;
    a.roi_x = g.roi_x;
    a.roi_y = g.roi_y;
    a.roi_w = g.roi_w;
    a.roi_h = g.roi_h;
    a.axis = g.axis;
    a.norm = g.norm;
    a.sincos = g.d_sincos;
    a.out = d_out;
    a.err = device_error_word();
    a.sincos_zstride = zstride;
    dim3 grid((g.roi_w + TX - 1) / TX, (g.roi_h + TY - 1) / TY, (g.nz + ZT - 1) / ZT);
    kern<<<grid, Sh::kThreads, Sh::kSmem, stream>>>(map, a);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

template <int KIND, bool KAHAN>
static ufob_status dispatch_tile(int tile, const BPGeometry &g, const void *d_sino, uint32_t elems, uint32_t pitch,
                                 uint64_t slice_pitch, float *d_out, cudaStream_t stream, uint32_t zstride = 0)
{
    switch (tile) {
    // single-slice shapes (ZT = 1), also the slices of an angle-group split (zstride: table rows
    // per group)
    case 0: return launch_linear<32, 16, 1, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream, zstride);
    case 8: return launch_linear<32, 96, 1, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream, zstride);
    case 9: return launch_linear<32, 32, 1, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream, zstride);
    case 10: return launch_linear<32, 64, 1, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream, zstride);
    case 11: return launch_linear<32, 128, 1, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream, zstride);
    case 1: return launch_linear<32, 32, 2, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    case 2: return launch_linear<32, 32, 4, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    case 3: return launch_linear<32, 16, 4, 16, 4, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    case 4: return launch_linear<32, 32, 8, 8, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    case 5: return launch_linear<32, 16, 8, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    case 6: return launch_linear<32, 32, 8, 16, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    case 7: return launch_linear<32, 16, 4, 32, 3, KIND, KAHAN>(g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    default: return fail(UFOB_ERR_INVALID, "backproject: unknown tile id %d", tile);
    }
}

// ------------------------------------------------------------------ batch dispatch

// Tile-shape variants of the persistent batch kernel (single slices, ZT = 1):
// (tile height, angles per stage).  The autotuner picks one per batch.
static const int kBatchVariants[][2] = {{16, 32}, {32, 16}, {8, 32}, {16, 16}, {64, 16}, {64, 32}, {128, 16}, {96, 16}};

int bp_batch_variants() { return (int)(sizeof(kBatchVariants) / sizeof(kBatchVariants[0])); }

template <int TY, int A>
static int batch_window()
{
    return BPShape<32, TY, 1, A, 3>::kWin;
}

void bp_batch_tile(int v, int *tx, int *ty, int *window)
{
    *tx = 32;
    *ty = kBatchVariants[v][0];
    switch (v) {
    case 0: *window = batch_window<16, 32>(); break;
    case 1: *window = batch_window<32, 16>(); break;
    case 2: *window = batch_window<8, 32>(); break;
    case 3: *window = batch_window<16, 16>(); break;
    case 4: *window = batch_window<64, 16>(); break;
    case 5: *window = batch_window<64, 32>(); break;
    case 6: *window = batch_window<128, 16>(); break;
    default: *window = batch_window<96, 16>(); break;
    }
}

template <int TY, int A, int KIND, bool KAHAN>
static ufob_status launch_batch_t(const BatchBP *d_jobs, const uint2 *d_items, uint32_t n_items, uint32_t *counter,
                                  cudaStream_t s)
{
    using Sh = BPShape<32, TY, 1, A, 3>;
    auto kern = k_bp_batch<32, TY, A, 3, KIND, KAHAN>;
    UFOB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::kSmem));
    int per_sm = 0;
    UFOB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, Sh::kSmem));
    if (per_sm < 1) return fail(UFOB_ERR_UNSUPPORTED, "backproject batch: kernel does not fit on an SM");
    const uint32_t grid = std::min<uint32_t>((uint32_t)num_sms() * (uint32_t)per_sm, n_items);
    if (!grid) return UFOB_OK;
    kern<<<grid, 256, Sh::kSmem, s>>>(d_jobs, d_items, n_items, counter);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

template <int KIND, bool KAHAN>
static ufob_status batch_variant(int v, const BatchBP *j, const uint2 *it, uint32_t n, uint32_t *c, cudaStream_t s)
{
    switch (v) {
    case 0: return launch_batch_t<16, 32, KIND, KAHAN>(j, it, n, c, s);
    case 1: return launch_batch_t<32, 16, KIND, KAHAN>(j, it, n, c, s);
    case 2: return launch_batch_t<8, 32, KIND, KAHAN>(j, it, n, c, s);
    case 3: return launch_batch_t<16, 16, KIND, KAHAN>(j, it, n, c, s);
    case 4: return launch_batch_t<64, 16, KIND, KAHAN>(j, it, n, c, s);
    case 5: return launch_batch_t<64, 32, KIND, KAHAN>(j, it, n, c, s);
    case 6: return launch_batch_t<128, 16, KIND, KAHAN>(j, it, n, c, s);
    case 7: return launch_batch_t<96, 16, KIND, KAHAN>(j, it, n, c, s);
    default: return fail(UFOB_ERR_INVALID, "backproject batch: unknown variant %d", v);
    }
}

ufob_status bp_batch_launch(const BatchBP *d_jobs, const uint2 *d_items, uint32_t n_items, uint32_t *d_counter,
                            SinoKind kind, bool kahan, int variant, cudaStream_t s)
{
    if (kind == SINO_F32) return batch_variant<SINO_F32, false>(variant, d_jobs, d_items, n_items, d_counter, s);
    if (kind == SINO_F16_PAIRS)
        return kahan ? batch_variant<SINO_F16_PAIRS, true>(variant, d_jobs, d_items, n_items, d_counter, s)
                     : batch_variant<SINO_F16_PAIRS, false>(variant, d_jobs, d_items, n_items, d_counter, s);
    return kahan ? batch_variant<SINO_BF16_PAIRS, true>(variant, d_jobs, d_items, n_items, d_counter, s)
                 : batch_variant<SINO_BF16_PAIRS, false>(variant, d_jobs, d_items, n_items, d_counter, s);
}

template <int TX, int TY, int ZT, int A, int S, int ACC, bool KAHAN>
static ufob_status launch_quads_t(const BPGeometry &g, const void *d_sino, uint32_t pitch, uint64_t group_pitch,
                                  float *d_out, cudaStream_t stream)
{
    using Sh = BPQShape<TX, TY, ZT, A, S>;
    auto kern = k_bp_quads<TX, TY, ZT, A, S, ACC, KAHAN>;
    static std::atomic<uint64_t> attr_devs{0};
    UFOB_CUDA_TRY(smem_limit_per_device(kern, (int)Sh::kSmem, attr_devs));
    CUtensorMap map;
    UFOB_TRY(make_quad_map(&map, d_sino, g.W + 1, g.P, (g.nz + 3) / 4, pitch, group_pitch, Sh::kWin, Sh::kGroups));
    BPArgs a;
    a.P = g.P;
    a.nz = g.nz;
    a.roi_x = g.roi_x;
    a.roi_y = g.roi_y;
    a.roi_w = g.roi_w;
    a.roi_h = g.roi_h;
    a.axis = g.axis;
    a.norm = g.norm;
    a.sincos = g.d_sincos;
    a.out = d_out;
    a.err = device_error_word();
    dim3 grid((g.roi_w + TX - 1) / TX, (g.roi_h + TY - 1) / TY, (g.nz + ZT - 1) / ZT);
    kern<<<grid, Sh::kThreads, Sh::kSmem, stream>>>(map, a);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

template <int ACC, bool KAHAN>
static ufob_status quads_tile(int tile, const BPGeometry &g, const void *d, uint32_t pitch, uint64_t gp, float *o,
                              cudaStream_t s)
{
    switch (tile) {
    case 0: return launch_quads_t<32, 16, 4, 16, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 1: return launch_quads_t<32, 32, 4, 16, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 2: return launch_quads_t<32, 16, 8, 16, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 3: return launch_quads_t<32, 32, 8, 16, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 4: return launch_quads_t<32, 16, 8, 32, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 5: return launch_quads_t<32, 8, 8, 32, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 6: return launch_quads_t<32, 32, 8, 32, 2, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 7: return launch_quads_t<32, 16, 8, 32, 2, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 8: return launch_quads_t<32, 16, 16, 16, 2, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 9: return launch_quads_t<32, 16, 16, 8, 3, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 10: return launch_quads_t<32, 8, 16, 16, 2, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 11: return launch_quads_t<32, 8, 32, 8, 2, ACC, KAHAN>(g, d, pitch, gp, o, s);
    case 12: return launch_quads_t<32, 8, 32, 16, 2, ACC, KAHAN>(g, d, pitch, gp, o, s);
    default: return fail(UFOB_ERR_INVALID, "backproject: unknown slice-quad tile id %d", tile);
    }
}

int bp_quad_tiles() { return 13; }

// Slice-quad FP16 backprojection.  pitch = cells per angle row (>= W + 1),
// group_pitch = cells per group of four slices (>= P * pitch).  `tile` < 0
// picks the default shape; `acc` is one of QACC_*.
ufob_status bp_quads_launch(const BPGeometry &g, const void *d_sino, uint32_t pitch, uint64_t group_pitch,
                            float *d_out, bool kahan, int acc, int tile, cudaStream_t stream)
{
    if (!g.roi_w || !g.roi_h || !g.nz || !g.P) return UFOB_OK;
    if ((uintptr_t)d_sino & 15) return fail(UFOB_ERR_INVALID, "backproject: slice-quad base must be 16-byte aligned");
    if (pitch < g.W + 1 || group_pitch < (uint64_t)pitch * g.P)
        return fail(UFOB_ERR_INVALID, "backproject: slice-quad pitches too small");
    // Measured on B200 (2048^2 x 1500): with compensated block sums 32x16 px x 16 slices, 2 stages of
    // 16 angles (tile 8) is fastest; with FP32 block sums 32x8 px x 32 slices, 2 stages of 8 angles
    // (tile 11: each coordinate serves 32 slices) ran at 6644 against 6482 GUPS, so it is taken
    // unless rounding the stack up to 32 slices costs more than that.
    if (tile < 0) {
        if (g.nz <= 4) {
            tile = 0;
        } else if (g.nz <= 8) {
            tile = 2;
        } else {
            const uint64_t w32 = (g.nz + 31) / 32 * 32, w16 = (g.nz + 15) / 16 * 16;
            tile = !kahan && w32 * 6482 <= w16 * 6644 ? 11 : 8;
        }
    }
    switch (acc) {
    case QACC_F32:
        return kahan ? quads_tile<QACC_F32, true>(tile, g, d_sino, pitch, group_pitch, d_out, stream)
                     : quads_tile<QACC_F32, false>(tile, g, d_sino, pitch, group_pitch, d_out, stream);
    case QACC_LERP:
        return kahan ? quads_tile<QACC_LERP, true>(tile, g, d_sino, pitch, group_pitch, d_out, stream)
                     : quads_tile<QACC_LERP, false>(tile, g, d_sino, pitch, group_pitch, d_out, stream);
    case QACC_H16:
        return kahan ? quads_tile<QACC_H16, true>(tile, g, d_sino, pitch, group_pitch, d_out, stream)
                     : quads_tile<QACC_H16, false>(tile, g, d_sino, pitch, group_pitch, d_out, stream);
    default: return fail(UFOB_ERR_INVALID, "backproject: unknown accumulation mode %d", acc);
    }
}

static int default_tile(const BPGeometry &g)
{
    // one slice: 96-row tiles share each angle's setup across 12 rows per thread, when the
    // slice still gives every SM two of them; else 32-row tiles when it gives every SM one;
    // else the 16-row tile (measured on 256^2 to 2048^2 slices)
    if (g.nz == 1) {
        const uint64_t tx = (g.roi_w + 31) / 32, sms = (uint64_t)num_sms();
        if (tx * ((g.roi_h + 95) / 96) >= 2 * sms) return 8;
        return tx * ((g.roi_h + 31) / 32) >= sms ? 9 : 0;
    }
    if (g.nz == 2) return 1;
    return 2;
}

ufob_status bp_linear_launch(const BPGeometry &g, const void *d_sino, SinoKind kind, uint32_t pitch,
                             uint64_t slice_pitch, float *d_out, bool kahan, int tile, cudaStream_t stream)
{
    if (!g.roi_w || !g.roi_h || !g.nz || !g.P) return UFOB_OK;
    if (((uintptr_t)d_sino & 15) || (pitch & 3) || (slice_pitch & 3))
        return fail(UFOB_ERR_INVALID, "backproject: sinogram base/pitches must be 16-byte aligned");
    if (tile < 0) tile = default_tile(g);
    const uint32_t elems = kind == SINO_F32 ? g.W : g.W + 1;  // pairs: (s[j-1], s[j]) for j = 0..W
    if (kind == SINO_F32) {
        return kahan ? dispatch_tile<SINO_F32, true>(tile, g, d_sino, elems, pitch, slice_pitch, d_out, stream)
                     : dispatch_tile<SINO_F32, false>(tile, g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    } else if (kind == SINO_F16_PAIRS) {
        return kahan ? dispatch_tile<SINO_F16_PAIRS, true>(tile, g, d_sino, elems, pitch, slice_pitch, d_out, stream)
                     : dispatch_tile<SINO_F16_PAIRS, false>(tile, g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    } else {
        return kahan ? dispatch_tile<SINO_BF16_PAIRS, true>(tile, g, d_sino, elems, pitch, slice_pitch, d_out, stream)
                     : dispatch_tile<SINO_BF16_PAIRS, false>(tile, g, d_sino, elems, pitch, slice_pitch, d_out, stream);
    }
}

// out[i] = sum over the angle groups of part[k][i], in group order; four pixels per thread
// (plane % 4 == 0, 16-byte aligned buffers) or one
template <int V>
__global__ void k_sum_groups(const float *__restrict__ part, uint64_t plane, uint32_t groups, float *__restrict__ out)
{
    const uint64_t n = plane / V;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (V == 4) {
            float4 v = reinterpret_cast<const float4 *>(part)[i];
            for (uint32_t k = 1; k < groups; k++) {
                const float4 w = reinterpret_cast<const float4 *>(part + (uint64_t)k * plane)[i];
                v.x += w.x;
                v.y += w.y;
                v.z += w.z;
                v.w += w.w;
            }
            reinterpret_cast<float4 *>(out)[i] = v;
        } else {
            float v = part[i];
            for (uint32_t k = 1; k < groups; k++) v += part[(uint64_t)k * plane + i];
            out[i] = v;
        }
    }
}

ufob_status bp_linear_split_launch(const BPGeometry &g, const void *d_sino, SinoKind kind, uint32_t pitch,
                                   uint32_t groups, int tile, float *d_part, float *d_out, bool kahan,
                                   cudaStream_t stream)
{
    if (!groups || g.nz != 1 || g.P % groups)
        return fail(UFOB_ERR_INVALID, "backproject: %u angle groups for %u rows of one sinogram", groups, g.P);
    if (!(tile == 0 || tile == 8 || tile == 9 || tile == 10 || tile == 11))
        return fail(UFOB_ERR_INVALID, "backproject: angle groups need a single-slice tile (0, 8, 9, 10, 11), not %d",
                    tile);
    if (((uintptr_t)d_sino & 15) || (pitch & 3))
        return fail(UFOB_ERR_INVALID, "backproject: sinogram base/pitches must be 16-byte aligned");
    BPGeometry gg = g;
    gg.P = g.P / groups;  // rows per group; the norm stays pi / (all rows)
    gg.nz = groups;
    const uint32_t elems = kind == SINO_F32 ? g.W : g.W + 1;
    const uint64_t sp = (uint64_t)gg.P * pitch;
    ufob_status st;
    if (kind == SINO_F32)
        st = kahan ? dispatch_tile<SINO_F32, true>(tile, gg, d_sino, elems, pitch, sp, d_part, stream, gg.P)
                   : dispatch_tile<SINO_F32, false>(tile, gg, d_sino, elems, pitch, sp, d_part, stream, gg.P);
    else if (kind == SINO_F16_PAIRS)
        st = kahan ? dispatch_tile<SINO_F16_PAIRS, true>(tile, gg, d_sino, elems, pitch, sp, d_part, stream, gg.P)
                   : dispatch_tile<SINO_F16_PAIRS, false>(tile, gg, d_sino, elems, pitch, sp, d_part, stream, gg.P);
    else
        st = kahan ? dispatch_tile<SINO_BF16_PAIRS, true>(tile, gg, d_sino, elems, pitch, sp, d_part, stream, gg.P)
                   : dispatch_tile<SINO_BF16_PAIRS, false>(tile, gg, d_sino, elems, pitch, sp, d_part, stream, gg.P);
    UFOB_TRY(st);
    const uint64_t plane = (uint64_t)g.roi_w * g.roi_h;
    const bool vec = !(plane & 3) && !(((uintptr_t)d_part | (uintptr_t)d_out) & 15);
    const uint64_t items = vec ? plane / 4 : plane;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((items + 255) / 256, (uint64_t)num_sms() * 8);
    if (vec)
        k_sum_groups<4><<<grid, 256, 0, stream>>>(d_part, plane, groups, d_out);
    else
        k_sum_groups<1><<<grid, 256, 0, stream>>>(d_part, plane, groups, d_out);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}


}  // namespace ufob
