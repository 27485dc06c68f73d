// General backprojection (the `general-backproject` task): parallel beam,
// cone beam and laminography with arbitrary tilted axis, detector and volume.
//
// Reference: src/ufo-general-backproject-task.c.  The reference generates an
// OpenCL kernel per geometry class (make_kernel :1069-1180) whose per-voxel
// code is, per projection (make_transformations :909-1048):
//   voxel_0 = (x0 + ix*dx, y0 + iy*dy, z)      (region mapping, general_bp_body.in)
//   cone: voxel_0 *= -s.y / (d.y - s.y)        (magnification)
//   voxel_0 = Rx(vol_x) Ry(vol_y) Rz(vol_z) voxel_0   (volume rotation)
//   V = Rx(axis_x) Ry(axis_y) Rz(tomo_p) voxel_0     (tomographic rotation, tilted axis)
//   project V onto the detector plane (parallel or from the source s), shift
//   by -d, rotate by the inverse detector angles, add the centre, sample the
//   projection bilinearly; cone beam weighs by coeff^2 = ((s.y-d.y)/(s.y-V.y))^2.
//   volume (store-type) += norm * sum over each burst of projections.
//
// B200 design.  Every step before the sampling is affine in
// X = (ix, iy, z, 1), and the cone-beam projection divides two affine forms,
// so the whole chain of one projection is four rows of a 4x4 table:
//   u = Nu.X / D.X,  v = Nv.X / D.X,  weight = (K / C.X)^2 (cone)  (D = C = e4, K = 1 parallel)
// The tables are built on the device in FP64 (one thread per projection, or
// per projection and slice when the swept parameter is not z) and cast to the
// compute type.  The backprojection kernel gives each thread a column of ZT
// voxels along z (8 cone, 4 otherwise), so the x/y part of every dot product is
// formed once per projection; table blocks are staged in shared memory.  With
// the FP32 compute type each sample is one texture gather of the 2x2 footprint
// (texture border/clamp addressing = the reference's CLAMP / CLAMP_TO_EDGE) and
// the cone divisions are approximate reciprocals; interpolation weights are
// exact FP32 in every path.
#include <cuda_fp16.h>
#include <math.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <string>

#include "f32x2.cuh"
#include "tma.cuh"
#include "ufob_internal.h"

namespace ufob {

enum { GC_TOMO = 0, GC_AXIS_X, GC_AXIS_Y, GC_VOL_X, GC_VOL_Y, GC_VOL_Z, GC_DET_AX, GC_DET_AY, GC_DET_AZ,
       GC_CENTER_X, GC_CENTER_Z, GC_SRC_X, GC_SRC_Y, GC_SRC_Z, GC_DET_X, GC_DET_Y, GC_DET_Z, GC_NCOLS };

enum { GF_WITH_AXIS = 1, GF_WITH_VOLUME = 2, GF_PERPENDICULAR = 4, GF_SHIFTED_DETECTOR = 8, GF_SHIFTED_SOURCE = 16,
       GF_PARALLEL = 32 };

enum StoreKind { ST_HALF = 0, ST_FLOAT, ST_DOUBLE, ST_UCHAR, ST_USHORT, ST_UINT };
enum ResultKind { RT_HALF = 0, RT_FLOAT, RT_DOUBLE };
enum AddrKind { AD_NONE = 0, AD_CLAMP_TO_EDGE, AD_CLAMP, AD_REPEAT, AD_MIRRORED_REPEAT };

static constexpr int kTab = 20;  // Nu[4] Nv[4] D[4] C[4] K pad[3]

__device__ __forceinline__ float fmaf_ct(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmaf_ct(double a, double b, double c) { return fma(a, b, c); }

struct d3 {
    double x, y, z;
};
__host__ __device__ inline d3 rx(double s, double c, d3 p) { return {p.x, c * p.y - s * p.z, s * p.y + c * p.z}; }
__host__ __device__ inline d3 ry(double s, double c, d3 p) { return {c * p.x + s * p.z, p.y, -s * p.x + c * p.z}; }
__host__ __device__ inline d3 rz(double s, double c, d3 p) { return {c * p.x - s * p.y, s * p.x + c * p.y, p.z}; }

// 4-component row vectors of affine forms in X = (ix, iy, z, 1)
struct Row {
    double a[4];
};
__host__ __device__ inline Row rsc(Row r, double k)
{
    for (int i = 0; i < 4; i++) r.a[i] *= k;
    return r;
}
__host__ __device__ inline Row radd(Row p, Row q)
{
    for (int i = 0; i < 4; i++) p.a[i] += q.a[i];
    return p;
}
__host__ __device__ inline Row rconst(double k)
{
    Row r = {{0.0, 0.0, 0.0, k}};
    return r;
}
struct Rows3 {
    Row x, y, z;
};
// rotate a triple of rows (a linear map applied component-wise)
__host__ __device__ inline Rows3 rot_rows(int axis, double s, double c, Rows3 p)
{
    Rows3 o = p;
    if (axis == 0) {
        o.y = radd(rsc(p.y, c), rsc(p.z, -s));
        o.z = radd(rsc(p.y, s), rsc(p.z, c));
    } else if (axis == 1) {
        o.x = radd(rsc(p.x, c), rsc(p.z, s));
        o.z = radd(rsc(p.x, -s), rsc(p.z, c));
    } else {
        o.x = radd(rsc(p.x, c), rsc(p.y, -s));
        o.y = radd(rsc(p.x, s), rsc(p.y, c));
    }
    return o;
}

// The table of one projection (and slice): the chain of make_transformations
// (src/ufo-general-backproject-task.c:909-1048) for geometry row g [GC_NCOLS],
// as rows Nu, Nv, D, C of affine forms in X = (ix, iy, z, 1) and K, in FP64.
// Shared by the device table builder and the host's staging plan.
__host__ __device__ inline void gbp_table_entry(const double *g, int flags, double x0, double dxs, double y0,
                                                double dys, double vals[kTab])
{
    const bool parallel = flags & GF_PARALLEL, perp = flags & GF_PERPENDICULAR;
    const double sx = g[GC_SRC_X], sy = g[GC_SRC_Y], sz = g[GC_SRC_Z];
    const double dx = g[GC_DET_X], dy = g[GC_DET_Y], dz = g[GC_DET_Z];
    double s_, c_;

    // columns of the affine map X -> voxel_0, pushed through the linear chain
    d3 col[4] = {{dxs, 0.0, 0.0}, {0.0, dys, 0.0}, {0.0, 0.0, 1.0}, {x0, y0, 0.0}};
    for (int j = 0; j < 4; j++) {
        d3 v = col[j];
        if (!parallel) {
            const double m = -sy / (dy - sy);
            v = {v.x * m, v.y * m, v.z * m};
        }
        if (flags & GF_WITH_VOLUME) {
            sincos(g[GC_VOL_Z], &s_, &c_); v = rz(s_, c_, v);
            sincos(g[GC_VOL_Y], &s_, &c_); v = ry(s_, c_, v);
            sincos(g[GC_VOL_X], &s_, &c_); v = rx(s_, c_, v);
        }
        sincos(g[GC_TOMO], &s_, &c_); v = rz(s_, c_, v);
        if (flags & GF_WITH_AXIS) {
            sincos(g[GC_AXIS_Y], &s_, &c_); v = ry(s_, c_, v);
            sincos(g[GC_AXIS_X], &s_, &c_); v = rx(s_, c_, v);
        }
        col[j] = v;
    }
    Rows3 M;
    for (int j = 0; j < 4; j++) {
        M.x.a[j] = col[j].x;
        M.y.a[j] = col[j].y;
        M.z.a[j] = col[j].z;
    }
    // detector normal and offset (make_static_transformations)
    d3 n = {0.0, -1.0, 0.0};
    double det_off = 0.0;
    if (!perp) {
        sincos(g[GC_DET_AZ], &s_, &c_); n = rz(s_, c_, n);
        sincos(g[GC_DET_AY], &s_, &c_); n = ry(s_, c_, n);
        sincos(g[GC_DET_AX], &s_, &c_); n = rx(s_, c_, n);
        det_off = -(dx * n.x + dy * n.y + dz * n.z);
    }
    // inverse detector rotation applied after the shift: x, then y, then z with negated sines
    auto det_rot = [&](Rows3 r) {
        double s0, c0;
        sincos(g[GC_DET_AX], &s0, &c0); r = rot_rows(0, -s0, c0, r);
        sincos(g[GC_DET_AY], &s0, &c0); r = rot_rows(1, -s0, c0, r);
        sincos(g[GC_DET_AZ], &s0, &c0); r = rot_rows(2, -s0, c0, r);
        return r;
    };
    const double cx = g[GC_CENTER_X], cz = g[GC_CENTER_Z];
    Row Nu, Nv, D = rconst(1.0), C = rconst(1.0);
    double K = 1.0;
    if (perp && parallel) {
        const double dxs_ = (flags & GF_SHIFTED_DETECTOR) ? dx : 0.0, dzs_ = (flags & GF_SHIFTED_DETECTOR) ? dz : 0.0;
        Nu = radd(M.x, rconst(cx - dxs_));
        Nv = radd(M.z, rconst(cz - dzs_));
    } else if (perp) {
        const double dxs_ = (flags & GF_SHIFTED_DETECTOR) ? dx : 0.0, dzs_ = (flags & GF_SHIFTED_DETECTOR) ? dz : 0.0;
        const double ssx = (flags & GF_SHIFTED_SOURCE) ? sx : 0.0, ssz = (flags & GF_SHIFTED_SOURCE) ? sz : 0.0;
        const Row w = radd(M.y, rconst(-sy));  // V.y - s.y
        Nu = radd(rsc(radd(M.x, rconst(-ssx)), dy - sy), rsc(w, sx - dxs_ + cx));
        Nv = radd(rsc(radd(M.z, rconst(-ssz)), dy - sy), rsc(w, sz - dzs_ + cz));
        D = w;
        C = w;
        K = dy - sy;
    } else if (parallel) {
        Rows3 P;
        P.x = radd(M.x, rconst(-dx));
        // V.y on the detector plane: -(V.z n.z + V.x n.x + off) / n.y
        P.y = radd(rsc(radd(radd(rsc(M.z, n.z), rsc(M.x, n.x)), rconst(det_off)), -1.0 / n.y), rconst(-dy));
        P.z = radd(M.z, rconst(-dz));
        P = det_rot(P);
        Nu = radd(P.x, rconst(cx));
        Nv = radd(P.z, rconst(cz));
    } else {
        const double T = -(det_off + (sx * n.x + sy * n.y + sz * n.z));
        Rows3 Q;
        Q.x = radd(M.x, rconst(-sx));
        Q.y = radd(M.y, rconst(-sy));
        Q.z = radd(M.z, rconst(-sz));
        const Row w = radd(radd(rsc(Q.x, n.x), rsc(Q.y, n.y)), rsc(Q.z, n.z));
        const Rows3 RQ = det_rot(Q);
        Rows3 sd;
        sd.x = rconst(sx - dx);
        sd.y = rconst(sy - dy);
        sd.z = rconst(sz - dz);
        sd = det_rot(sd);
        Nu = radd(rsc(RQ.x, T), rsc(w, sd.x.a[3] + cx));
        Nv = radd(rsc(RQ.z, T), rsc(w, sd.z.a[3] + cz));
        D = w;
        C = radd(rconst(sy), rsc(M.y, -1.0));  // s.y - V.y
        K = sy - dy;
    }
    const double v[kTab] = {Nu.a[0], Nu.a[1], Nu.a[2], Nu.a[3], Nv.a[0], Nv.a[1], Nv.a[2], Nv.a[3],
                            D.a[0],  D.a[1],  D.a[2],  D.a[3],  C.a[0],  C.a[1],  C.a[2],  C.a[3], K, 0.0, 0.0, 0.0};
    for (int i = 0; i < kTab; i++) vals[i] = v[i];
}

// One table entry per (slice-or-0, projection).  geom: [n_proj][GC_NCOLS]
// FP64; when param_col >= 0 the column is replaced by slice_values[slice].
__global__ void k_gbp_tables(const double *__restrict__ geom, uint32_t n_proj, uint32_t n_tab_slices, int param_col,
                             const double *__restrict__ slice_values, int flags, double x0, double dxs, double y0,
                             double dys, float *__restrict__ tf, double *__restrict__ td)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t sl = blockIdx.y;
    if (p >= n_proj || sl >= n_tab_slices) return;
    double g[GC_NCOLS];
    for (int i = 0; i < GC_NCOLS; i++) g[i] = geom[(size_t)p * GC_NCOLS + i];
    if (param_col >= 0) g[param_col] = slice_values[sl];
    double vals[kTab];
    gbp_table_entry(g, flags, x0, dxs, y0, dys, vals);
    const size_t o = ((size_t)sl * n_proj + p) * kTab;
    for (int i = 0; i < kTab; i++) {
        td[o + i] = vals[i];
        tf[o + i] = (float)vals[i];
    }
}

// ---------------------------------------------------------------- sampling

__device__ __forceinline__ float texel(const float *__restrict__ img, int W, int H, int i, int j, int addr)
{
    if (addr == AD_CLAMP) {
        if ((unsigned)i >= (unsigned)W || (unsigned)j >= (unsigned)H) return 0.f;
    } else {
        i = min(max(i, 0), W - 1);
        j = min(max(j, 0), H - 1);
    }
    return __ldg(img + (size_t)j * W + i);
}

// OpenCL linear sampler with unnormalised coordinates: texel centres at +0.5.
template <typename CT>
__device__ __forceinline__ float bilinear(const float *__restrict__ img, int W, int H, CT u, CT v, int addr)
{
    const float uu = (float)u - 0.5f, vv = (float)v - 0.5f;
    const float fu = floorf(uu), fv = floorf(vv);
    const float a = uu - fu, b = vv - fv;
    const int i = (int)fu, j = (int)fv;
    float t00, t10, t01, t11;
    if (i >= 0 && j >= 0 && i + 1 < W && j + 1 < H) {
        const float *q = img + (size_t)j * W + i;
        t00 = __ldg(q);
        t10 = __ldg(q + 1);
        t01 = __ldg(q + W);
        t11 = __ldg(q + W + 1);
    } else {
        t00 = texel(img, W, H, i, j, addr);
        t10 = texel(img, W, H, i + 1, j, addr);
        t01 = texel(img, W, H, i, j + 1, addr);
        t11 = texel(img, W, H, i + 1, j + 1, addr);
    }
    const float top = fmaf(a, t10 - t00, t00), bot = fmaf(a, t11 - t01, t01);
    return fmaf(b, bot - top, top);
}

// Fast path of bilinear() for FP32 coordinates: floor and fraction from the
// 1.5 * 2^23 rounding trick (i = rint(x - 1) with x = coordinate, which is
// floor(x - 0.5) except at exact ties, where the fraction becomes 1 and the
// interpolated value is the same), no float-to-int conversion.  Coordinates
// beyond +-4e6 (outside any detector) and NaN take the general path.
__device__ __forceinline__ float bilinear_fast(const float *__restrict__ img, int W, int H, float u, float v,
                                               int addr)
{
    const float M = 12582912.0f;  // 1.5 * 2^23
    if (!(fabsf(u) < 4.0e6f && fabsf(v) < 4.0e6f)) return bilinear<float>(img, W, H, u, v, addr);
    const float ru = u + (M - 1.0f), rv = v + (M - 1.0f);
    const int i = __float_as_int(ru) - __float_as_int(M), j = __float_as_int(rv) - __float_as_int(M);
    const float a = (u - 0.5f) - (ru - M), b = (v - 0.5f) - (rv - M);
    float t00, t10, t01, t11;
    if ((unsigned)i < (unsigned)(W - 1) && (unsigned)j < (unsigned)(H - 1)) {
        const float *q = img + (size_t)j * W + i;
        t00 = __ldg(q);
        t10 = __ldg(q + 1);
        t01 = __ldg(q + W);
        t11 = __ldg(q + W + 1);
    } else {
        t00 = texel(img, W, H, i, j, addr);
        t10 = texel(img, W, H, i + 1, j, addr);
        t01 = texel(img, W, H, i, j + 1, addr);
        t11 = texel(img, W, H, i + 1, j + 1, addr);
    }
    const float top = fmaf(a, t10 - t00, t00), bot = fmaf(a, t11 - t01, t01);
    return fmaf(b, bot - top, top);
}

// Bilinear sample through the texture unit: tex2Dgather returns the 2x2
// footprint (x: (i0, j0+1), y: (i0+1, j0+1), z: (i0+1, j0), w: (i0, j0)).  It is
// queried at the centre of the footprint chosen here in software, so the
// texel selection never depends on the unit's coordinate rounding; the weights
// are exact FP32.  The texture's border (0) / clamp addressing implements the
// reference's CLAMP / CLAMP_TO_EDGE; coordinates are first clamped to
// [-2, size + 2], which leaves both modes' results unchanged.
__device__ __forceinline__ float bilinear_tex(cudaTextureObject_t t, int W, int H, float u, float v)
{
    const float M = 12582912.0f;  // 1.5 * 2^23
    u = fminf(fmaxf(u, -2.0f), (float)W + 2.0f);
    v = fminf(fmaxf(v, -2.0f), (float)H + 2.0f);
    // gu = rint(u) = floor(u - 0.5) + 1 but ties: the footprint's centre; the weights
    // a = (u + 0.5) - gu equal (u - 0.5) - floor(u - 0.5), both steps exact for |u| < 2^22
    const float gu = (u + (M - 1.0f)) - (M - 1.0f), gv = (v + (M - 1.0f)) - (M - 1.0f);
    const float a = (u + 0.5f) - gu, b = (v + 0.5f) - gv;
    const float4 g = tex2Dgather<float4>(t, gu, gv, 0);
    const float top = fmaf(a, g.z - g.w, g.w), bot = fmaf(a, g.y - g.x, g.x);
    return fmaf(b, bot - top, top);
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ---------------------------------------------------------------- accumulation semantics

struct StoreParams {
    int kind;          // StoreKind
    double gray_min;   // gray_limit.x
    double gray_scale; // gray_limit.y = max / (gray_max - gray_min)
    double maxval;
};

__device__ __forceinline__ float to_half_f(float x) { return __half2float(__float2half_rn(x)); }

// volume (store type) += convert(norm * burst_sum), as the generated kernel
// does once per burst (general_bp_body.in, make_type_conversion :705-719).
template <typename CT>
__device__ __forceinline__ void store_accumulate(double &acc, CT contrib_norm, const StoreParams &sp)
{
    switch (sp.kind) {
    case ST_FLOAT: acc = (double)((float)acc + (float)contrib_norm); break;
    case ST_DOUBLE: acc += (double)contrib_norm; break;
    case ST_HALF: acc = (double)to_half_f(to_half_f((float)acc) + to_half_f((float)contrib_norm)); break;
    default: {
        CT gv = (CT)sp.gray_scale * (contrib_norm - (CT)sp.gray_min);
        gv = gv < (CT)0 ? (CT)0 : (gv > (CT)sp.maxval ? (CT)sp.maxval : gv);
        const uint64_t add = (uint64_t)gv;  // C cast: truncation toward zero
        const uint64_t mod = sp.kind == ST_UCHAR ? 0x100ull : (sp.kind == ST_USHORT ? 0x10000ull : 0x100000000ull);
        acc = (double)(((uint64_t)acc + add) % mod);
    }
    }
}

__device__ __forceinline__ void store_write(void *vol, size_t idx, double acc, int kind)
{
    switch (kind) {
    case ST_FLOAT: reinterpret_cast<float *>(vol)[idx] = (float)acc; break;
    case ST_DOUBLE: reinterpret_cast<double *>(vol)[idx] = acc; break;
    case ST_HALF: reinterpret_cast<__half *>(vol)[idx] = __float2half_rn((float)acc); break;
    case ST_UCHAR: reinterpret_cast<uint8_t *>(vol)[idx] = (uint8_t)acc; break;
    case ST_USHORT: reinterpret_cast<uint16_t *>(vol)[idx] = (uint16_t)acc; break;
    default: reinterpret_cast<uint32_t *>(vol)[idx] = (uint32_t)acc; break;
    }
}

// result-type accumulation of one sample into the burst sum
template <int RT, typename CT>
__device__ __forceinline__ void result_add(CT &r, CT val)
{
    if (RT == RT_HALF) r = (CT)to_half_f((float)r + (float)val);
    else r += val;
}

struct GBPArgs {
    const float *proj;  // [n][H][W]
    uint32_t W, H, n_proj;
    uint32_t nx, ny, nz;
    uint32_t burst;
    const void *tab;     // [n_tab_slices][n_proj][kTab] of CT
    const double *zvals; // z value of each slice (parameter z) or the constant slice z
    double norm;
    StoreParams sp;
    int addr;
    void *vol;
    const cudaTextureObject_t *tex;  // one per projection (FP32 compute type), or null: global loads
    int hw_interp;                   // 1: the texture unit's linear filter (8-bit weights) samples
};

template <bool CONE, typename CT, int RT, bool PARAMZ, int ZT, bool TEX, bool HW = false>
__global__ void __launch_bounds__(256) k_gbp(const GBPArgs a)
{
    constexpr int PB = 16;  // projections per staged table block
    __shared__ __align__(16) CT s_tab[PB * kTab];
    const int ix = blockIdx.x * 32 + (threadIdx.x & 31);
    const int iy = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int z0 = blockIdx.z * ZT;
    const CT fx = (CT)ix, fy = (CT)iy;
    CT zv[ZT];
#pragma unroll
    for (int k = 0; k < ZT; k++) zv[k] = (CT)a.zvals[min(z0 + k, (int)a.nz - 1)];
    const CT *tab = reinterpret_cast<const CT *>(a.tab) + (PARAMZ ? 0 : (size_t)z0 * a.n_proj * kTab);
    double acc[ZT];
    CT bsum[ZT];
#pragma unroll
    for (int k = 0; k < ZT; k++) {
        acc[k] = 0.0;
        bsum[k] = (CT)0;
    }
    const size_t plane = (size_t)a.W * a.H;
    uint32_t in_burst = 0;
    for (uint32_t p0 = 0; p0 < a.n_proj; p0 += PB) {
        const uint32_t nb = min((uint32_t)PB, a.n_proj - p0);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nb * kTab; i += blockDim.x) s_tab[i] = tab[(size_t)p0 * kTab + i];
        __syncthreads();
        for (uint32_t q = 0; q < nb; q++) {
            CT t[kTab];
            if (sizeof(CT) == 4) {
                // the projection's table as five 16-byte shared loads (broadcast)
#pragma unroll
                for (int r = 0; r < kTab / 4; r++)
                    *reinterpret_cast<float4 *>(&t[4 * r]) = reinterpret_cast<const float4 *>(s_tab + q * kTab)[r];
            } else {
#pragma unroll
                for (int r = 0; r < kTab; r++) t[r] = s_tab[q * kTab + r];
            }
            const float *img = a.proj + (size_t)(p0 + q) * plane;
            cudaTextureObject_t tx = 0;
            if (TEX) tx = a.tex[p0 + q];
            const CT u_xy = fmaf_ct(t[0], fx, fmaf_ct(t[1], fy, t[3]));
            const CT v_xy = fmaf_ct(t[4], fx, fmaf_ct(t[5], fy, t[7]));
            CT d_xy = (CT)1, c_xy = (CT)1;
            if (CONE) {
                d_xy = fmaf_ct(t[8], fx, fmaf_ct(t[9], fy, t[11]));
                c_xy = fmaf_ct(t[12], fx, fmaf_ct(t[13], fy, t[15]));
            }
#pragma unroll
            for (int k = 0; k < ZT; k++) {
                CT u = fmaf_ct(t[2], zv[k], u_xy), v = fmaf_ct(t[6], zv[k], v_xy);
                CT wgt = (CT)1;
                if (CONE) {
                    if (sizeof(CT) == 4) {
                        // approximate reciprocals (1 ulp): u = Nu.X / D.X, weight = (K / C.X)^2
                        const float inv = rcp_approx((float)fmaf_ct(t[10], zv[k], d_xy));
                        u *= (CT)inv;
                        v *= (CT)inv;
                        const float cc = (float)t[16] * rcp_approx((float)fmaf_ct(t[14], zv[k], c_xy));
                        wgt = (CT)(cc * cc);
                    } else {
                        const CT inv = (CT)1 / fmaf_ct(t[10], zv[k], d_xy);
                        u *= inv;
                        v *= inv;
                        const CT cc = t[16] / fmaf_ct(t[14], zv[k], c_xy);
                        wgt = cc * cc;
                    }
                }
                const float val = TEX ? (HW ? tex2D<float>(tx, (float)u, (float)v)
                                            : bilinear_tex(tx, (int)a.W, (int)a.H, (float)u, (float)v))
                                  : sizeof(CT) == 4 ? bilinear_fast(img, (int)a.W, (int)a.H, (float)u, (float)v, a.addr)
                                                    : bilinear<CT>(img, (int)a.W, (int)a.H, u, v, a.addr);
                result_add<RT, CT>(bsum[k], CONE ? (CT)val * wgt : (CT)val);
            }
            if (++in_burst == a.burst || p0 + q + 1 == a.n_proj) {
#pragma unroll
                for (int k = 0; k < ZT; k++) {
                    store_accumulate<CT>(acc[k], (CT)a.norm * bsum[k], a.sp);
                    bsum[k] = (CT)0;
                }
                in_burst = 0;
            }
        }
    }
    if (ix >= (int)a.nx || iy >= (int)a.ny) return;
#pragma unroll
    for (int k = 0; k < ZT; k++) {
        if (z0 + k >= (int)a.nz) break;
        store_write(a.vol, ((size_t)(z0 + k) * a.ny + iy) * a.nx + ix, acc[k], a.sp.kind);
    }
}

// ---------------------------------------------------------------- TMA-staged column kernel
//
// Geometries whose u coordinate and cone denominators do not depend on z
// (Nu.z = D.z = C.z = 0 in every projection's table: circular orbits with the
// rotation axis parallel to the detector columns, laminography tilted about x,
// parallel beam) give each z-column of voxels one u, one weight and a v affine
// in z per projection.  A CTA owns 32 x 8 columns of ZT voxels.  Per projection
// the detector window its samples reach (bw x bh texels, bw a multiple of 4,
// from the host's plan) is staged by one TMA copy into an S-stage ring of PB
// projections per stage (warp 0 finds the windows, one lane per projection,
// from the stage's tables, which a bulk copy brought into a ring of S + 1 table
// slots one stage earlier; each warp releases a stage through an mbarrier, so
// warps drift up to S - 1 stages apart instead of meeting at a CTA barrier per
// stage).  Samples are
// interpolated from shared memory with exact FP32 weights (floor and fraction
// by the round-down 1.5 * 2^23 trick, v' = v - 1/2 one affine function of z per
// column).  TMA's zero fill outside the detector is the reference's CLAMP
// addressing.  A projection whose window for the tile exceeds the staged box
// (where the plan underestimated it) is sampled from global memory instead.

struct GBPColArgs {
    const float *proj;    // [n][H][W]
    const float *tab;     // [n][kTab] FP32 tables
    const double *zvals;  // z value of each slice
    uint32_t W, H, n_proj, nx, ny, nz, burst;
    uint32_t bw, bh, slot_floats;  // staged window (texels, rows) and its shared-memory stride (floats)
    float norm;
    float *vol;
    int *err;
};

template <int PB, int S>
struct GBPColSmem {
    float *data;     // [S][PB][slot_floats] staged windows
    float4 *tab;     // [S + 1][PB][kTab / 4] tables of the staged projections (one stage ahead)
    int2 *org;       // [S][PB] window origin (u0, v0) in texels
    uint64_t *full;  // [S] mbarriers: the stage's window copies have landed
    uint64_t *empty; // [S] mbarriers: all 8 warps are done with the stage
    uint64_t *tfull; // [S + 1] mbarriers: the table slot's copy has landed
    static size_t bytes(uint32_t slot_floats)
    {
        return (size_t)S * PB * slot_floats * 4 + (size_t)(S + 1) * PB * kTab * 4 + (size_t)S * PB * 8 +
               (size_t)(3 * S + 1) * 8 + 128;
    }
    __device__ __forceinline__ GBPColSmem(unsigned char *dyn, uint32_t slot_floats)
    {
        unsigned char *raw = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(dyn) + 127) & ~(uintptr_t)127);
        data = reinterpret_cast<float *>(raw);
        tab = reinterpret_cast<float4 *>(data + (size_t)S * PB * slot_floats);
        org = reinterpret_cast<int2 *>(tab + (S + 1) * PB * (kTab / 4));
        full = reinterpret_cast<uint64_t *>(org + S * PB);
        empty = full + S;
        tfull = empty + S;
    }
};

template <bool CONE, int ZT, int PB, int S>
__global__ void __launch_bounds__(256, 2) k_gbp_col(const __grid_constant__ CUtensorMap map, const GBPColArgs c)
{
    static_assert(PB <= 32 && kTab % 4 == 0, "one producer lane per projection of a stage");
    static_assert(ZT % 2 == 0, "the voxels of a column are processed in packed pairs");
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const GBPColSmem<PB, S> sm(smem_dyn, c.slot_floats);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8, z0 = blockIdx.z * ZT;
    // a warp covers 16 x 2 columns: its samples of one row then span fewer than 32 banks
    const int ix = x0 + (warp & 1) * 16 + (lane & 15), iy = y0 + (warp >> 1) * 2 + (lane >> 4);
    const float fx = (float)ix, fy = (float)iy;
    // z of the column's voxels as packed pairs (2j, 2j + 1)
    uint64_t zz[ZT / 2];
#pragma unroll
    for (int j = 0; j < ZT / 2; j++)
        zz[j] = f2pack((float)c.zvals[min(z0 + 2 * j, (int)c.nz - 1)], (float)c.zvals[min(z0 + 2 * j + 1, (int)c.nz - 1)]);
    float zlo, zhi, zdummy;
    f2unpack(zz[0], zlo, zdummy);
    f2unpack(zz[ZT / 2 - 1], zdummy, zhi);
    if (tid == 0) {
        for (int q = 0; q < S; q++) {
            mbar_init(&sm.full[q], 1);
            mbar_init(&sm.empty[q], 8);
        }
        for (int q = 0; q <= S; q++) mbar_init(&sm.tfull[q], 1);
        fence_barrier_init();
    }
    __syncthreads();

    const int n = (int)c.n_proj, nblk = (n + PB - 1) / PB;
    // lane 0 of warp 0: bulk copy of the tables of stage blk (contiguous, 80 bytes each) into
    // table slot blk % (S + 1), whose previous stage (blk - S - 1) every warp has released
    auto issue_tab = [&](int blk) {
        const int ts = blk % (S + 1), nval = min(PB, n - blk * PB);
        mbar_arrive_expect_tx(&sm.tfull[ts], (uint32_t)nval * kTab * 4u);
        bulk_load_1d(sm.tab + ts * PB * (kTab / 4), c.tab + (size_t)blk * PB * kTab, (uint32_t)nval * kTab * 4u,
                     &sm.tfull[ts]);
    };
    // Producer, all lanes of warp 0: lane q stages projection blk * PB + q once every warp has
    // released the slot's previous stage, and the tables of stage blk + 1 are requested.
    // Returns false if a wait gave up.
    auto issue = [&](int blk) {
        const int slot = blk % S, ts = blk % (S + 1), p = blk * PB + lane;
        const int nval = min(PB, n - blk * PB);
        if (blk >= S && !mbar_wait_bounded(&sm.empty[slot], (uint32_t)(blk / S - 1) & 1u, kWaitLimitNs)) return false;
        if (lane == 0 && blk + 1 < nblk) issue_tab(blk + 1);
        if (!mbar_wait_bounded(&sm.tfull[ts], (uint32_t)(blk / (S + 1)) & 1u, kWaitLimitNs)) return false;
        int u0 = 0, v0 = 0;
        if (lane < nval) {
            float t[kTab];
#pragma unroll
            for (int r = 0; r < kTab / 4; r++) {
                const float4 w = sm.tab[(ts * PB + lane) * (kTab / 4) + r];
                t[4 * r] = w.x;
                t[4 * r + 1] = w.y;
                t[4 * r + 2] = w.z;
                t[4 * r + 3] = w.w;
            }
            // the extremes of a projective (or affine) map over the tile's box are at its corners
            // (a cone denominator that changes sign inside the box has no such bound: not staged)
            float umin = FLT_MAX, vmin = FLT_MAX, umax = -FLT_MAX, vmax = -FLT_MAX, dmin = 1.0f, dmax = 1.0f;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float cx = (float)(x0 + (i & 1) * 31), cy = (float)(y0 + (i >> 1) * 7);
                const float uxy = fmaf(t[0], cx, fmaf(t[1], cy, t[3])), vxy = fmaf(t[4], cx, fmaf(t[5], cy, t[7]));
                const float d = CONE ? fmaf(t[8], cx, fmaf(t[9], cy, t[11])) : 1.0f;
                dmin = i ? fminf(dmin, d) : d;
                dmax = i ? fmaxf(dmax, d) : d;
                const float inv = 1.0f / d;
                const float va = fmaf(t[6], zlo, vxy) * inv, vb = fmaf(t[6], zhi, vxy) * inv;
                umin = fminf(umin, uxy * inv);
                umax = fmaxf(umax, uxy * inv);
                vmin = fminf(vmin, fminf(va, vb));
                vmax = fmaxf(vmax, fmaxf(va, vb));
            }
            // left / upper tap = floor(x - 0.5) (rint(x) - 1 in the samples), one guard texel on
            // each side for the samples' approximate reciprocals; x origin on a 16-byte boundary.
            // A window larger than the staged box (or a degenerate one) sends the projection's
            // samples of this tile to global memory.
            const bool finite = fabsf(umin) < 4.0e6f && fabsf(umax) < 4.0e6f && fabsf(vmin) < 4.0e6f &&
                                fabsf(vmax) < 4.0e6f && (dmin > 0.0f || dmax < 0.0f);
            if (finite) {
                u0 = ((int)floorf(umin - 0.5f) - 1) & ~3;
                v0 = (int)floorf(vmin - 0.5f) - 1;
            }
            const bool fits = finite && (int)floorf(umax - 0.5f) + 2 - u0 <= (int)c.bw - 1 &&
                              (int)floorf(vmax - 0.5f) + 2 - v0 <= (int)c.bh - 1;
            sm.org[slot * PB + lane] = make_int2(fits ? u0 : INT_MIN, v0);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&sm.full[slot], (uint32_t)nval * c.bw * c.bh * 4u);
        __syncwarp();
        if (lane < nval) tma_load_3d(sm.data + (size_t)(slot * PB + lane) * c.slot_floats, &map, &sm.full[slot], u0, v0, p);
        return true;
    };
    if (tid == 0 && nblk > 0) issue_tab(0);
    bool aborted = false;
    if (tid < 32)
        for (int b = 0; b < S - 1 && b < nblk; b++)
            if (!issue(b)) aborted = true;

    const float M1 = 12582911.0f;  // 1.5 * 2^23 - 1: (x + M1) - M1 = rint(x) for |x| < 2^22
    const int M1b = __float_as_int(M1);
    const float M = 12582912.0f;  // 1.5 * 2^23: x + M rounded down = floor(x) + M for |x| < 2^22
    const int Mb = __float_as_int(M);
    const float Wf = (float)c.W + 2.0f, Hf = (float)c.H + 2.0f;
    const int bw = (int)c.bw;
    float acc[ZT];
    uint64_t bsum[ZT / 2];  // burst sums of voxels (2j, 2j + 1)
#pragma unroll
    for (int k = 0; k < ZT; k++) acc[k] = 0.f;
#pragma unroll
    for (int j = 0; j < ZT / 2; j++) bsum[j] = 0;  // (+0, +0)
    uint32_t in_burst = 0;
    for (int blk = 0; blk < nblk && !aborted; blk++) {
        // the warps run up to S - 1 stages apart: no CTA-wide barrier per stage
        if (tid < 32 && blk + S - 1 < nblk && !issue(blk + S - 1)) {
            aborted = true;
            break;
        }
        const int slot = blk % S, ts = blk % (S + 1);
        // the stage's windows, and its tables (whose copy the producer saw land before it issued them)
        const bool ok = mbar_wait_bounded(&sm.full[slot], (uint32_t)(blk / S) & 1u, kWaitLimitNs) &&
                        mbar_wait_bounded(&sm.tfull[ts], (uint32_t)(blk / (S + 1)) & 1u, kWaitLimitNs);
        const int nval = min(PB, n - blk * PB);
        if (ok) {
            for (int q = 0; q < nval; q++) {
                const int p = blk * PB + q;
                float t[kTab];
#pragma unroll
                for (int r = 0; r < kTab / 4; r++)
                    *reinterpret_cast<float4 *>(&t[4 * r]) = sm.tab[(ts * PB + q) * (kTab / 4) + r];
                const int2 o = sm.org[slot * PB + q];
                const float *win = sm.data + (size_t)(slot * PB + q) * c.slot_floats;
                const float uxy = fmaf(t[0], fx, fmaf(t[1], fy, t[3]));
                const float vxy = fmaf(t[4], fx, fmaf(t[5], fy, t[7]));
                float inv = 1.0f, wgt = 1.0f;
                if (CONE) {
                    // approximate reciprocals (1 ulp), as the texture-gather path: u = Nu.X / D.X,
                    // weight = (K / C.X)^2
                    inv = rcp_approx(fmaf(t[8], fx, fmaf(t[9], fy, t[11])));
                    const float cc = t[16] * rcp_approx(fmaf(t[12], fx, fmaf(t[13], fy, t[15])));
                    wgt = cc * cc;
                }
                if (o.x != INT_MIN) {
                    // the tile's footprints lie inside the staged window (one guard texel each side):
                    // x' = x - 0.5 per axis, tap = floor(x') by adding 1.5 * 2^23 rounded down,
                    // weight = x' - tap; v' is affine in z: v' = Av * z + Bv.  Two voxels of the
                    // column per packed FP32 operation (each lane rounds as the scalar form).
                    const float up = fmaf(uxy, inv, -0.5f);
                    const float ru = __fadd_rd(up, M);
                    const float a = up - (ru - M);
                    const int iu = min(max(__float_as_int(ru) - Mb - o.x, 0), bw - 2);
                    const float Av = t[6] * inv, Bv = fmaf(vxy, inv, -0.5f);
                    const int vbase = Mb + o.y;
                    const float *col = win + iu;
                    const uint64_t AA = f2pack(a, a), AV = f2pack(Av, Av), BV = f2pack(Bv, Bv);
                    const uint64_t MM = f2pack(M, M), WG = f2pack(wgt, wgt);
#pragma unroll
                    for (int j = 0; j < ZT / 2; j++) {
                        const uint64_t vp = f2fma(AV, zz[j], BV);
                        const uint64_t rv = f2add_rd(vp, MM);
                        const uint64_t bb = f2sub(vp, f2sub(rv, MM));
                        float r0, r1;
                        f2unpack(rv, r0, r1);
                        // one unsigned clamp keeps every read inside the window (the plan's guard
                        // texels already do for every in-range footprint)
                        const uint32_t i0 = min((uint32_t)(__float_as_int(r0) - vbase), c.bh - 2u);
                        const uint32_t i1 = min((uint32_t)(__float_as_int(r1) - vbase), c.bh - 2u);
                        const float *p0 = col + i0 * (uint32_t)bw, *p1 = col + i1 * (uint32_t)bw;
                        const uint64_t t00 = f2pack(p0[0], p1[0]), t10 = f2pack(p0[1], p1[1]);
                        const uint64_t t01 = f2pack(p0[bw], p1[bw]), t11 = f2pack(p0[bw + 1], p1[bw + 1]);
                        const uint64_t top = f2fma(AA, f2sub(t10, t00), t00), bot = f2fma(AA, f2sub(t11, t01), t01);
                        const uint64_t val = f2fma(bb, f2sub(bot, top), top);
                        bsum[j] = CONE ? f2fma(val, WG, bsum[j]) : f2add(bsum[j], val);
                    }
                } else {
                    // window not staged: the same footprints and weights from global memory
                    const float *img = c.proj + (size_t)p * c.W * c.H;
                    const float u = fminf(fmaxf(uxy * inv, -2.0f), Wf);
                    const float ru = u + M1;
                    const float a = (u + 0.5f) - (ru - M1);
                    const int i0 = __float_as_int(ru) - M1b - 1;
                    auto texel0 = [&](int i, int j) {
                        return ((unsigned)i < c.W && (unsigned)j < c.H) ? __ldg(img + (size_t)j * c.W + i) : 0.f;
                    };
                    for (int j = 0; j < ZT / 2; j++) {
                        float zp[2], bs[2];
                        f2unpack(zz[j], zp[0], zp[1]);
                        f2unpack(bsum[j], bs[0], bs[1]);
                        for (int h = 0; h < 2; h++) {
                            const float v = fminf(fmaxf(fmaf(t[6], zp[h], vxy) * inv, -2.0f), Hf);
                            const float rv = v + M1;
                            const float b = (v + 0.5f) - (rv - M1);
                            const int j0 = __float_as_int(rv) - M1b - 1;
                            const float t00 = texel0(i0, j0), t10 = texel0(i0 + 1, j0);
                            const float t01 = texel0(i0, j0 + 1), t11 = texel0(i0 + 1, j0 + 1);
                            const float top = fmaf(a, t10 - t00, t00), bot = fmaf(a, t11 - t01, t01);
                            const float val = fmaf(b, bot - top, top);
                            bs[h] = CONE ? fmaf(val, wgt, bs[h]) : bs[h] + val;
                        }
                        bsum[j] = f2pack(bs[0], bs[1]);
                    }
                }
                if (++in_burst == c.burst || p + 1 == n) {
#pragma unroll
                    for (int j = 0; j < ZT / 2; j++) {
                        float b0, b1;
                        f2unpack(bsum[j], b0, b1);
                        acc[2 * j] = acc[2 * j] + __fmul_rn(c.norm, b0);
                        acc[2 * j + 1] = acc[2 * j + 1] + __fmul_rn(c.norm, b1);
                        bsum[j] = 0;
                    }
                    in_burst = 0;
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.empty[slot]);
        if (!ok) {
            aborted = true;
            break;
        }
    }
    // every loop above ends (all waits are bounded); a CTA that gave up lets its copies in
    // flight land before it exits
    if (__syncthreads_or(aborted)) {
        if (tid == 0) {
            atomicExch(c.err, kErrTmaTimeout);
            for (int q = 0; q < S; q++)
                for (int k = 0; k < 2; k++) mbar_wait_bounded(&sm.full[q], (uint32_t)k, kWaitLimitNs / 8);
            for (int q = 0; q <= S; q++)
                for (int k = 0; k < 2; k++) mbar_wait_bounded(&sm.tfull[q], (uint32_t)k, kWaitLimitNs / 8);
        }
        return;
    }
    if (ix >= (int)c.nx || iy >= (int)c.ny) return;
#pragma unroll
    for (int k = 0; k < ZT; k++) {
        if (z0 + k >= (int)c.nz) break;
        c.vol[((size_t)(z0 + k) * c.ny + iy) * c.nx + ix] = acc[k];
    }
}

// Staged-window plan of the column kernel for one geometry: whether every projection's table has
// Nu.z = D.z = C.z = 0, and the window (bw x bh texels) that covers the 2x2 footprints of every
// sample of a 32 x 8 x ZT voxel tile, from the tiles at 0, 1/4 .. 1 of the volume along each axis
// (all projections), plus two texels of margin each way.
struct GBPColPlan {
    bool ok = false;
    uint32_t bw = 0, bh = 0;
};

// voxels per column: 16 share each projection's setup (tables, reciprocals, v coefficients)
// between twice the voxels of 8 and measured 910 / 1014 / 1103 against 805 / 961 / 999 GUPS on
// configuration 2 (cone / laminography / parallel); the taller window costs ring depth, not speed
static constexpr int kColZT = 16;

static GBPColPlan gbp_col_plan(const std::vector<double> &tabs, uint32_t n, bool cone, uint32_t nx, uint32_t ny,
                               const std::vector<double> &zvals, uint32_t W, uint32_t H)
{
    GBPColPlan plan;
    for (uint32_t p = 0; p < n; p++) {
        const double *t = &tabs[(size_t)p * kTab];
        if (t[2] != 0.0 || (cone && (t[10] != 0.0 || t[14] != 0.0))) return plan;
    }
    const uint32_t nz = (uint32_t)zvals.size();
    const uint32_t tx = (nx + 31) / 32, ty = (ny + 7) / 8, tz = (nz + kColZT - 1) / kColZT;
    auto picks = [](uint32_t m) {
        std::vector<uint32_t> v;
        for (int i = 0; i <= 4; i++) v.push_back((uint32_t)((uint64_t)(m - 1) * i / 4));
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        return v;
    };
    double wmax = 0, hmax = 0;
    for (uint32_t bx : picks(tx))
        for (uint32_t by : picks(ty))
            for (uint32_t bz : picks(tz)) {
                const double zl = zvals[bz * kColZT], zh = zvals[std::min(bz * kColZT + kColZT - 1, nz - 1)];
                for (uint32_t p = 0; p < n; p++) {
                    const double *t = &tabs[(size_t)p * kTab];
                    double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
                    for (int i = 0; i < 4; i++) {
                        const double cx = bx * 32.0 + (i & 1) * 31.0, cy = by * 8.0 + (i >> 1) * 7.0;
                        const double inv = cone ? 1.0 / (t[8] * cx + t[9] * cy + t[11]) : 1.0;
                        const double u = (t[0] * cx + t[1] * cy + t[3]) * inv;
                        const double vxy = t[4] * cx + t[5] * cy + t[7];
                        const double va = (vxy + t[6] * zl) * inv, vb = (vxy + t[6] * zh) * inv;
                        umin = std::min(umin, u);
                        umax = std::max(umax, u);
                        vmin = std::min({vmin, va, vb});
                        vmax = std::max({vmax, va, vb});
                    }
                    auto clampd = [](double x, double hi) { return std::min(std::max(x, -4.0), hi + 4.0); };
                    umin = clampd(umin, W), umax = clampd(umax, W), vmin = clampd(vmin, H), vmax = clampd(vmax, H);
                    const double u0 = std::floor(std::floor(umin - 0.5) - 1.0 - 3.0);  // worst case of the & ~3
                    const double v0 = std::floor(vmin - 0.5) - 1.0;
                    wmax = std::max(wmax, std::floor(umax - 0.5) + 2.0 - u0);
                    hmax = std::max(hmax, std::floor(vmax - 0.5) + 2.0 - v0);
                }
            }
    const double bw = std::ceil((wmax + 2.0) / 4.0) * 4.0, bh = hmax + 2.0;
    if (!(bw >= 4 && bw <= 256 && bh >= 2 && bh <= 256)) return plan;
    plan.ok = true;
    plan.bw = (uint32_t)bw;
    plan.bh = (uint32_t)bh;
    return plan;
}

template <bool CONE, int PB, int S>
static ufob_status launch_gbp_col_t(const GBPColArgs &c, cudaStream_t s)
{
    using Sm = GBPColSmem<PB, S>;
    auto kern = k_gbp_col<CONE, kColZT, PB, S>;
    static std::atomic<uint64_t> attr_devs{0};
    const size_t smem = Sm::bytes(c.slot_floats);
    UFOB_CUDA_TRY(smem_limit_per_device(kern, 227 * 1024, attr_devs));
    CUtensorMap map;
    UFOB_TRY(make_image_map(&map, c.proj, c.W, c.H, c.n_proj, c.W, (uint64_t)c.W * c.H, c.bw, c.bh));
    dim3 grid((c.nx + 31) / 32, (c.ny + 7) / 8, (c.nz + kColZT - 1) / kColZT);
    kern<<<grid, 256, smem, s>>>(map, c);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

// Launches the column kernel with a ring that keeps two CTAs per SM; false when the window is too
// large for that.
static ufob_status launch_gbp_col(GBPColArgs c, bool cone, bool *launched, cudaStream_t s)
{
    *launched = false;
    c.slot_floats = (c.bw * c.bh + 31) / 32 * 32;  // 128-byte aligned TMA destinations
    constexpr size_t kBudget = 110 * 1024;           // two CTAs per SM
    if (GBPColSmem<8, 3>::bytes(c.slot_floats) <= kBudget) {
        *launched = true;
        return cone ? launch_gbp_col_t<true, 8, 3>(c, s) : launch_gbp_col_t<false, 8, 3>(c, s);
    }
    // three stages of 6 before two of 8 (configuration-2 laminography: 1055 against 1013 GUPS)
    if (GBPColSmem<6, 3>::bytes(c.slot_floats) <= kBudget) {
        *launched = true;
        return cone ? launch_gbp_col_t<true, 6, 3>(c, s) : launch_gbp_col_t<false, 6, 3>(c, s);
    }
    if (GBPColSmem<8, 2>::bytes(c.slot_floats) <= kBudget) {
        *launched = true;
        return cone ? launch_gbp_col_t<true, 8, 2>(c, s) : launch_gbp_col_t<false, 8, 2>(c, s);
    }
    if (GBPColSmem<4, 3>::bytes(c.slot_floats) <= kBudget) {
        *launched = true;
        return cone ? launch_gbp_col_t<true, 4, 3>(c, s) : launch_gbp_col_t<false, 4, 3>(c, s);
    }
    // a third stage of 3 projections beats 2 stages of 4 (configuration-2 cone: 950 against 915
    // GUPS; 2 projections per stage, 4 or 5 stages: 876 / 880)
    if (GBPColSmem<3, 3>::bytes(c.slot_floats) <= kBudget) {
        *launched = true;
        return cone ? launch_gbp_col_t<true, 3, 3>(c, s) : launch_gbp_col_t<false, 3, 3>(c, s);
    }
    if (GBPColSmem<4, 2>::bytes(c.slot_floats) <= kBudget) {
        *launched = true;
        return cone ? launch_gbp_col_t<true, 4, 2>(c, s) : launch_gbp_col_t<false, 4, 2>(c, s);
    }
    return UFOB_OK;
}

template <bool CONE, typename CT, int RT, bool PARAMZ>
static ufob_status launch_gbp_t(const GBPArgs &a, cudaStream_t s)
{
    // voxels per thread along z: 8 for cone beam (two reciprocals per sample make the per-voxel
    // x/y work worth sharing), 4 otherwise (fewer detector rows per warp); measured on B200
    constexpr int ZT = PARAMZ ? (CONE ? 8 : 4) : 1;
    dim3 grid((a.nx + 31) / 32, (a.ny + 7) / 8, (a.nz + ZT - 1) / ZT);
    if (a.tex && a.hw_interp)
        k_gbp<CONE, CT, RT, PARAMZ, ZT, true, true><<<grid, 256, 0, s>>>(a);
    else if (a.tex)
        k_gbp<CONE, CT, RT, PARAMZ, ZT, true><<<grid, 256, 0, s>>>(a);
    else
        k_gbp<CONE, CT, RT, PARAMZ, ZT, false><<<grid, 256, 0, s>>>(a);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

template <bool CONE, typename CT>
static ufob_status launch_gbp_rt(const GBPArgs &a, int rt, bool paramz, cudaStream_t s)
{
    switch (rt) {
    case RT_HALF: return paramz ? launch_gbp_t<CONE, CT, RT_HALF, true>(a, s) : launch_gbp_t<CONE, CT, RT_HALF, false>(a, s);
    case RT_DOUBLE: return paramz ? launch_gbp_t<CONE, CT, RT_DOUBLE, true>(a, s) : launch_gbp_t<CONE, CT, RT_DOUBLE, false>(a, s);
    default: return paramz ? launch_gbp_t<CONE, CT, RT_FLOAT, true>(a, s) : launch_gbp_t<CONE, CT, RT_FLOAT, false>(a, s);
    }
}

}  // namespace ufob

using namespace ufob;

// =================================================================== task object

namespace {

const char *kParamNames[] = {"axis-angle-x",        "axis-angle-y",        "axis-angle-z",        "volume-angle-x",
                             "volume-angle-y",      "volume-angle-z",      "detector-angle-x",    "detector-angle-y",
                             "detector-angle-z",    "detector-position-x", "detector-position-y", "detector-position-z",
                             "source-position-x",   "source-position-y",   "source-position-z",   "center-position-x",
                             "center-position-z",   "z"};
// geometry column of each `parameter` value (-1: z); axis-angle-z is not sweepable here
const int kParamCol[] = {GC_AXIS_X, GC_AXIS_Y, -2,         GC_VOL_X,   GC_VOL_Y,  GC_VOL_Z,    GC_DET_AX, GC_DET_AY,  GC_DET_AZ,
                         GC_DET_X,  GC_DET_Y,  GC_DET_Z,   GC_SRC_X,   GC_SRC_Y,  GC_SRC_Z,    GC_CENTER_X, GC_CENTER_Z, -1};
const char *kGeomNames[GC_NCOLS] = {"axis-angle-z",     "axis-angle-x",     "axis-angle-y",      "volume-angle-x",
                                    "volume-angle-y",   "volume-angle-z",   "detector-angle-x",  "detector-angle-y",
                                    "detector-angle-z", "center-position-x", "center-position-z", "source-position-x",
                                    "source-position-y", "source-position-z", "detector-position-x",
                                    "detector-position-y", "detector-position-z"};
const char *kStoreNames[] = {"half", "float", "double", "uchar", "ushort", "uint"};
const char *kResultNames[] = {"half", "float", "double"};
const char *kAddrNames[] = {"none", "clamp_to_edge", "clamp", "repeat", "mirrored_repeat"};

bool name_is(const char *name, const char *canon)
{
    if (!name) return false;
    for (; *name && *canon; name++, canon++) {
        char a = *name == '_' ? '-' : *name;
        if (a != *canon) return false;
    }
    return *name == 0 && *canon == 0;
}

int lookup(const char *v, const char *const *names, int n)
{
    for (int i = 0; i < n; i++)
        if (v && strcmp(v, names[i]) == 0) return i;
    return -1;
}

bool almost_zero(const std::vector<double> &v)
{
    for (double x : v)
        if (!(fabs(x) < 1e-7)) return false;
    return true;
}

}  // namespace

struct ufob_gbp {
    // properties (src/ufo-general-backproject-task.c:2087-2359)
    uint32_t burst = 0;
    int parameter = 17;  // z
    double z = 0.0;
    std::vector<double> region{0, 0, 0}, x_region{0, 0, 0}, y_region{0, 0, 0};
    std::vector<double> geom[GC_NCOLS];
    uint32_t num_projections = 0;
    int compute_type = 0;  // 0 float, 1 double, 2 half (FP16 projection samples, FP32 arithmetic)
    int result_type = RT_FLOAT;
    int store_type = ST_FLOAT;
    double overall_angle = 2 * M_PI;
    int addressing_mode = AD_CLAMP;
    double gray_map_min = 0.0, gray_map_max = 0.0;
    int interpolation = 0;  // engine property: 0 exact FP32 weights, 1 the texture unit's linear filter
    int staging = 1;        // engine property: 1 TMA-staged detector windows where the geometry allows, 0 never
    // staging plan of the last geometry (host FP64 tables, window size), keyed by its inputs
    std::vector<double> col_key;
    GBPColPlan col_plan;
    // device state
    DevBuf d_geom, d_zvals, d_tab_f, d_tab_d, d_proj, d_vol, d_proj16;
    DevBuf d_proj_h;  // compute-type half on the staged kernel: the projections rounded to FP16, as FP32
    uint32_t pushed = 0, pw = 0, ph = 0;
    bool volume_ready = false;
    // texture objects over the projections of the last call (rebuilt when base/shape/mode change)
    std::vector<cudaTextureObject_t> tex;
    DevBuf d_tex;
    const void *tex_base = nullptr;
    uint32_t tex_w = 0, tex_h = 0;
    int tex_addr = -1, tex_filter = -1, tex_half = -1;
    ufob_gbp()
    {
        for (int i = 0; i < GC_NCOLS; i++) geom[i] = {0.0};
        geom[GC_SRC_Y] = {-INFINITY};
    }
    void drop_textures()
    {
        for (cudaTextureObject_t t : tex) cudaDestroyTextureObject(t);
        tex.clear();
        tex_base = nullptr;
    }
    ~ufob_gbp() { drop_textures(); }
};

// [n][H][W] FP32 -> [n][H][pitch] FP16 (round to nearest), planes `plane` elements apart.
__global__ void k_proj_to_half(const float *__restrict__ in, uint32_t W, uint32_t H, uint32_t n, size_t pitch,
                               size_t plane, __half *__restrict__ out)
{
    const uint64_t total = (uint64_t)n * H * W;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % W);
        const uint64_t r = i / W;
        const uint32_t y = (uint32_t)(r % H), p = (uint32_t)(r / H);
        out[(size_t)p * plane + (size_t)y * pitch + x] = __float2half_rn(__ldg(in + i));
    }
}

// The projections rounded to FP16 and widened back to FP32 (both conversions exact for the values
// kept), four per thread: the very samples the FP16 gathers of compute-type half read.
__global__ void k_proj_round_half(const float4 *__restrict__ in, uint64_t n4, float4 *__restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x) {
        float4 v = __ldg(in + i);
        v.x = __half2float(__float2half_rn(v.x));
        v.y = __half2float(__float2half_rn(v.y));
        v.z = __half2float(__float2half_rn(v.z));
        v.w = __half2float(__float2half_rn(v.w));
        out[i] = v;
    }
}

// One 2-D texture object per projection of a [n][H][W] stack: FP32 with row
// pitch W * 4 bytes, or (half) FP16 with the given row pitch and plane size in
// elements.  Border or clamp addressing; point sampling (the gather path) or the
// unit's linear filter.  Returns false when the stack does not meet the texture
// alignment rules.
static bool gbp_textures(ufob_gbp *g, const void *base, uint32_t W, uint32_t H, uint32_t n, int addr,
                         cudaStream_t s, int linear = 0, bool half = false, size_t pitch16 = 0, size_t plane16 = 0)
{
    if (g->tex_base == base && g->tex_w == W && g->tex_h == H && g->tex.size() == n && g->tex_addr == addr &&
        g->tex_filter == linear && g->tex_half == (int)half)
        return true;
    g->drop_textures();
    int dev = 0, align = 0, palign = 0, maxw = 0, maxh = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&align, cudaDevAttrTextureAlignment, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&palign, cudaDevAttrTexturePitchAlignment, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxTexture2DLinearWidth, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maxh, cudaDevAttrMaxTexture2DLinearHeight, dev) != cudaSuccess)
        return false;
    const size_t esize = half ? 2 : 4, pitch = half ? pitch16 * 2 : (size_t)W * 4;
    const size_t plane = half ? plane16 * 2 : (size_t)W * H * 4;
    if (((uintptr_t)base % align) || (plane % align) || (pitch % palign) || W > (uint32_t)maxw ||
        H > (uint32_t)maxh || W < 2 || H < 2)
        return false;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = addr == AD_CLAMP ? cudaAddressModeBorder : cudaAddressModeClamp;
    td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    g->tex.reserve(n);
    for (uint32_t p = 0; p < n; p++) {
        cudaResourceDesc rd = {};
        rd.resType = cudaResourceTypePitch2D;
        rd.res.pitch2D.devPtr = const_cast<char *>(static_cast<const char *>(base)) + (size_t)p * plane;
        rd.res.pitch2D.desc = half ? cudaCreateChannelDescHalf() : cudaCreateChannelDesc<float>();
        rd.res.pitch2D.width = W;
        rd.res.pitch2D.height = H;
        rd.res.pitch2D.pitchInBytes = pitch;
        (void)esize;
        cudaTextureObject_t t = 0;
        if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
            cudaGetLastError();
            g->drop_textures();
            return false;
        }
        g->tex.push_back(t);
    }
    if (g->d_tex.ensure(n * sizeof(cudaTextureObject_t)) != UFOB_OK ||
        cudaMemcpyAsync(g->d_tex.ptr, g->tex.data(), n * sizeof(cudaTextureObject_t), cudaMemcpyHostToDevice, s) !=
            cudaSuccess) {
        g->drop_textures();
        return false;
    }
    g->tex_base = base;
    g->tex_w = W;
    g->tex_h = H;
    g->tex_addr = addr;
    g->tex_filter = linear;
    g->tex_half = (int)half;
    return true;
}

static int geom_col(const char *name)
{
    for (int i = 0; i < GC_NCOLS; i++)
        if (name_is(name, kGeomNames[i])) return i;
    return -1;
}

static size_t store_size(int st)
{
    static const size_t sz[] = {2, 4, 8, 1, 2, 4};
    return sz[st];
}

extern "C" ufob_status ufob_gbp_create(ufob_gbp **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "gbp_create: out is NULL");
    *out = new ufob_gbp;
    return UFOB_OK;
}

extern "C" ufob_status ufob_gbp_set_array(ufob_gbp *g, const char *name, const double *values, uint32_t n)
{
    if (!g || (!values && n)) return fail(UFOB_ERR_INVALID, "gbp_set_array: NULL argument");
    std::vector<double> v(values, values + n);
    if (name_is(name, "region") || name_is(name, "x-region") || name_is(name, "y-region")) {
        if (n != 3) return fail(UFOB_ERR_INVALID, "%s needs 3 values (from, to, step)", name);
        if (name_is(name, "region")) g->region = v;
        else if (name_is(name, "x-region")) g->x_region = v;
        else g->y_region = v;
        g->volume_ready = false;
        return UFOB_OK;
    }
    const int c = geom_col(name);
    if (c < 0) return fail(UFOB_ERR_INVALID, "general-backproject: no array property named '%s'", name ? name : "(null)");
    if (!n) return fail(UFOB_ERR_INVALID, "%s needs at least one value", name);
    g->geom[c] = v;
    g->volume_ready = false;
    return UFOB_OK;
}

extern "C" ufob_status ufob_gbp_set_property(ufob_gbp *g, const char *name, double v)
{
    if (!g) return fail(UFOB_ERR_INVALID, "gbp handle is NULL");
    g->volume_ready = false;
    if (name_is(name, "burst")) {
        if (v < 0 || v > 128) return fail(UFOB_ERR_INVALID, "burst outside [0, 128]");
        g->burst = (uint32_t)v;
    } else if (name_is(name, "z")) g->z = v;
    else if (name_is(name, "num-projections")) {
        if (v < 0 || v > 32768) return fail(UFOB_ERR_INVALID, "num-projections outside [0, 32768]");
        g->num_projections = (uint32_t)v;
    } else if (name_is(name, "overall-angle")) g->overall_angle = v;
    else if (name_is(name, "gray-map-min")) g->gray_map_min = v;
    else if (name_is(name, "gray-map-max")) g->gray_map_max = v;
    else if (geom_col(name) >= 0) return ufob_gbp_set_array(g, name, &v, 1);
    else return fail(UFOB_ERR_INVALID, "general-backproject: no numeric property named '%s'", name ? name : "(null)");
    return UFOB_OK;
}

extern "C" ufob_status ufob_gbp_set_property_string(ufob_gbp *g, const char *name, const char *value)
{
    if (!g) return fail(UFOB_ERR_INVALID, "gbp handle is NULL");
    g->volume_ready = false;
    int i;
    if (name_is(name, "parameter")) {
        if ((i = lookup(value, kParamNames, 18)) < 0) return fail(UFOB_ERR_INVALID, "unknown parameter '%s'", value);
        if (kParamCol[i] == -2)
            return fail(UFOB_ERR_UNSUPPORTED, "parameter axis-angle-z (the tomographic angle) cannot be swept");
        g->parameter = i;
    } else if (name_is(name, "compute-type")) {
        if ((i = lookup(value, kResultNames, 3)) < 0) return fail(UFOB_ERR_INVALID, "unknown compute-type '%s'", value);
        g->compute_type = i == 0 ? 2 : i - 1;
    } else if (name_is(name, "result-type")) {
        if ((i = lookup(value, kResultNames, 3)) < 0) return fail(UFOB_ERR_INVALID, "unknown result-type '%s'", value);
        g->result_type = i;
    } else if (name_is(name, "store-type")) {
        if ((i = lookup(value, kStoreNames, 6)) < 0) return fail(UFOB_ERR_INVALID, "unknown store-type '%s'", value);
        g->store_type = i;
    } else if (name_is(name, "addressing-mode")) {
        if ((i = lookup(value, kAddrNames, 5)) < 0) return fail(UFOB_ERR_INVALID, "unknown addressing-mode '%s'", value);
        g->addressing_mode = i;
    } else if (name_is(name, "interpolation")) {  // engine property
        static const char *const kInterp[] = {"exact", "texture"};
        if ((i = lookup(value, kInterp, 2)) < 0) return fail(UFOB_ERR_INVALID, "unknown interpolation '%s'", value);
        g->interpolation = i;
    } else if (name_is(name, "staging")) {  // engine property
        static const char *const kStaging[] = {"texture", "auto"};
        if ((i = lookup(value, kStaging, 2)) < 0) return fail(UFOB_ERR_INVALID, "unknown staging '%s'", value);
        g->staging = i;
    } else {
        char *end = nullptr;
        double v = value ? strtod(value, &end) : 0.0;
        if (!value || end == value) return fail(UFOB_ERR_INVALID, "'%s' is not a number", value ? value : "(null)");
        return ufob_gbp_set_property(g, name, v);
    }
    return UFOB_OK;
}

extern "C" ufob_status ufob_gbp_setup(ufob_gbp *g)
{
    if (!g) return fail(UFOB_ERR_INVALID, "gbp handle is NULL");
    if (!g->num_projections) return fail(UFOB_ERR_SETUP, "Number of projections not set");
    if (g->gray_map_min >= g->gray_map_max && g->store_type >= ST_UCHAR)
        return fail(UFOB_ERR_SETUP, "Gray mapping minimum must be less then the maximum");
    for (int c = 0; c < GC_NCOLS; c++) {
        size_t n = g->geom[c].size();
        if (c == GC_TOMO) continue;
        if (n != 1 && n != g->num_projections)
            return fail(UFOB_ERR_SETUP, "%s has %zu values; it needs 1 or num-projections (%u)", kGeomNames[c], n,
                        g->num_projections);
    }
    if (g->addressing_mode == AD_REPEAT || g->addressing_mode == AD_MIRRORED_REPEAT)
        return fail(UFOB_ERR_UNSUPPORTED, "addressing-mode %s is undefined for unnormalised coordinates",
                    kAddrNames[g->addressing_mode]);
    return UFOB_OK;
}

static uint32_t region_size(const std::vector<double> &r) { return (uint32_t)ceil((r[1] - r[0]) / r[2]); }

extern "C" ufob_status ufob_gbp_get_requisition(ufob_gbp *g, uint32_t width, uint32_t height, uint32_t *ow,
                                                uint32_t *oh, uint32_t *ns)
{
    if (!g) return fail(UFOB_ERR_INVALID, "gbp handle is NULL");
    if (!width || !height) return fail(UFOB_ERR_REQUISITION, "empty projection %ux%u", width, height);
    // :1495-1507: default slice size is the full detector width (both x and y)
    const uint32_t w = g->x_region[2] == 0.0 ? width : region_size(g->x_region);
    const uint32_t h = g->y_region[2] == 0.0 ? width : region_size(g->y_region);
    uint32_t n = 1;
    if (!(fabs(g->region[2]) < 1e-7)) n = (uint32_t)ceil((g->region[1] - g->region[0]) / g->region[2]);
    if (!w || !h || !n) return fail(UFOB_ERR_REQUISITION, "empty output region");
    if (ow) *ow = w;
    if (oh) *oh = h;
    if (ns) *ns = n;
    return UFOB_OK;
}

// FP16 copy of the projections for compute-type half, rows and planes padded to
// the texture pitch and base alignment.
static ufob_status half_projections(ufob_gbp *g, const float *d_proj, uint32_t W, uint32_t H, uint32_t n,
                                    cudaStream_t s, size_t *pitch16, size_t *plane16)
{
    int dev = 0, align = 0, palign = 0;
    UFOB_CUDA_TRY(cudaGetDevice(&dev));
    UFOB_CUDA_TRY(cudaDeviceGetAttribute(&align, cudaDevAttrTextureAlignment, dev));
    UFOB_CUDA_TRY(cudaDeviceGetAttribute(&palign, cudaDevAttrTexturePitchAlignment, dev));
    const size_t pe = (size_t)std::max(palign, 2) / 2, ae = (size_t)std::max(align, 2) / 2;
    *pitch16 = ((size_t)W + pe - 1) / pe * pe;
    *plane16 = (*pitch16 * H + ae - 1) / ae * ae;
    UFOB_TRY(g->d_proj16.ensure((size_t)n * *plane16 * sizeof(__half)));
    const uint64_t total = (uint64_t)n * H * W;
    if (!total) return UFOB_OK;
    const uint32_t grid = (uint32_t)std::min<uint64_t>((total + 255) / 256, (uint64_t)num_sms() * 16);
    k_proj_to_half<<<grid, 256, 0, s>>>(d_proj, W, H, n, *pitch16, *plane16, g->d_proj16.as<__half>());
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

static ufob_status gbp_compute(ufob_gbp *g, const float *d_proj, uint32_t W, uint32_t H, void *d_vol, cudaStream_t s)
{
    UFOB_TRY(ufob_gbp_setup(g));
    uint32_t nx, ny, nz;
    UFOB_TRY(ufob_gbp_get_requisition(g, W, H, &nx, &ny, &nz));
    const uint32_t n = g->num_projections;
    // geometry table [n][GC_NCOLS]; scalars broadcast (ufo-scarray.c:95-108); tomographic angles
    // default to i / n * overall-angle (:1435-1446)
    std::vector<double> table((size_t)n * GC_NCOLS);
    for (uint32_t p = 0; p < n; p++)
        for (int c = 0; c < GC_NCOLS; c++) {
            const std::vector<double> &v = g->geom[c];
            double val;
            if (c == GC_TOMO) val = v.size() == n ? v[p] : (double)p / n * g->overall_angle;
            else val = v.size() == 1 ? v[0] : v[p];
            table[(size_t)p * GC_NCOLS + c] = val;
        }
    // geometry class (node_setup :1294-1320)
    const int pcol = kParamCol[g->parameter];
    const bool is_axis = pcol == GC_AXIS_X || pcol == GC_AXIS_Y;
    const bool is_vol = pcol == GC_VOL_X || pcol == GC_VOL_Y || pcol == GC_VOL_Z;
    const bool is_det_rot = pcol == GC_DET_AX || pcol == GC_DET_AY || pcol == GC_DET_AZ;
    const bool is_det_pos = pcol == GC_DET_X || pcol == GC_DET_Y || pcol == GC_DET_Z;
    int flags = 0;
    if (is_axis || !(almost_zero(g->geom[GC_AXIS_X]) && almost_zero(g->geom[GC_AXIS_Y]))) flags |= GF_WITH_AXIS;
    if (is_vol || !(almost_zero(g->geom[GC_VOL_X]) && almost_zero(g->geom[GC_VOL_Y]) && almost_zero(g->geom[GC_VOL_Z])))
        flags |= GF_WITH_VOLUME;
    if (!(almost_zero(g->geom[GC_DET_X]) && almost_zero(g->geom[GC_DET_Z]))) flags |= GF_SHIFTED_DETECTOR;
    if (!(almost_zero(g->geom[GC_SRC_X]) && almost_zero(g->geom[GC_SRC_Z]))) flags |= GF_SHIFTED_SOURCE;
    if (!is_det_rot && !is_det_pos && almost_zero(g->geom[GC_DET_AX]) && almost_zero(g->geom[GC_DET_AY]) &&
        almost_zero(g->geom[GC_DET_AZ]))
        flags |= GF_PERPENDICULAR;
    bool parallel = true;
    for (uint32_t p = 0; p < n; p++) parallel = parallel && std::isinf(table[(size_t)p * GC_NCOLS + GC_SRC_Y]);
    if (parallel) flags |= GF_PARALLEL;
    // regions (compute_slice_region :280-291)
    auto reg = [](const std::vector<double> &r, uint32_t len, double *start, double *step) {
        if (r[2] != 0.0) {
            *start = r[0];
            *step = r[2];
        } else {
            *start = -((double)(float)len / 2.0);
            *step = 1.0;
        }
    };
    double x0, dxs, y0, dys;
    reg(g->x_region, nx, &x0, &dxs);
    reg(g->y_region, ny, &y0, &dys);
    double rs = 0.0, rstep = 1.0;
    if (!(fabs(g->region[2]) < 1e-7)) {
        rs = g->region[0];
        rstep = g->region[2];
    }
    std::vector<double> slice_values(nz);
    for (uint32_t k = 0; k < nz; k++) slice_values[k] = rs + k * rstep;
    const bool paramz = pcol == -1;
    std::vector<double> zvals(nz, g->z);
    if (paramz) zvals = slice_values;
    const uint32_t tab_slices = paramz ? 1 : nz;
    UFOB_TRY(g->d_geom.ensure(table.size() * sizeof(double) + nz * sizeof(double)));
    UFOB_TRY(g->d_zvals.ensure(nz * sizeof(double) * 2));
    UFOB_TRY(g->d_tab_f.ensure((size_t)tab_slices * n * kTab * sizeof(float)));
    UFOB_TRY(g->d_tab_d.ensure((size_t)tab_slices * n * kTab * sizeof(double)));
    double *d_table = g->d_geom.as<double>(), *d_slicev = d_table + table.size();
    UFOB_CUDA_TRY(cudaMemcpyAsync(d_table, table.data(), table.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    UFOB_CUDA_TRY(cudaMemcpyAsync(d_slicev, slice_values.data(), nz * sizeof(double), cudaMemcpyHostToDevice, s));
    UFOB_CUDA_TRY(cudaMemcpyAsync(g->d_zvals.ptr, zvals.data(), nz * sizeof(double), cudaMemcpyHostToDevice, s));
    k_gbp_tables<<<dim3((n + 127) / 128, tab_slices), 128, 0, s>>>(d_table, n, tab_slices, paramz ? -1 : pcol, d_slicev,
                                                                  flags, x0, dxs, y0, dys, g->d_tab_f.as<float>(),
                                                                  g->d_tab_d.as<double>());
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();

    GBPArgs a;
    a.proj = d_proj;
    a.W = W;
    a.H = H;
    a.n_proj = n;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.burst = g->burst ? g->burst : 8;  // "GENERIC" entry of the node table (ufo-conebeam.c:21-26)
    a.zvals = g->d_zvals.as<double>();
    a.norm = fabs(g->overall_angle) / n;  // :292
    a.sp.kind = g->store_type;
    a.sp.gray_min = g->gray_map_min;
    const double maxv = g->store_type == ST_UCHAR ? 255.0 : g->store_type == ST_USHORT ? 65535.0 : 4294967295.0;
    a.sp.maxval = maxv;
    a.sp.gray_scale = g->store_type >= ST_UCHAR ? maxv / (g->gray_map_max - g->gray_map_min) : 0.0;
    a.addr = g->addressing_mode == AD_CLAMP ? AD_CLAMP : AD_CLAMP_TO_EDGE;  // "none": defined as clamp-to-edge
    a.vol = d_vol;
    a.tex = nullptr;
    a.hw_interp = 0;
    const bool cone = !parallel;
    if (g->compute_type == 1) {
        a.tab = g->d_tab_d.ptr;
        return cone ? launch_gbp_rt<true, double>(a, g->result_type, paramz, s)
                    : launch_gbp_rt<false, double>(a, g->result_type, paramz, s);
    }
    a.tab = g->d_tab_f.ptr;
    if ((g->compute_type == 0 || g->compute_type == 2) && !g->interpolation && g->staging &&
        g->result_type == RT_FLOAT && g->store_type == ST_FLOAT && paramz && a.addr == AD_CLAMP && W % 4 == 0 &&
        !((uintptr_t)d_proj & 15)) {
        // TMA-staged detector windows for geometries whose u does not depend on z; the plan (host
        // FP64 tables, window size) is kept while the geometry stays the same
        std::vector<double> key(table);
        key.insert(key.end(), {(double)flags, x0, dxs, y0, dys, (double)nx, (double)ny, (double)W, (double)H});
        key.insert(key.end(), zvals.begin(), zvals.end());
        if (key != g->col_key) {
            std::vector<double> tabs((size_t)n * kTab);
            for (uint32_t p = 0; p < n; p++)
                gbp_table_entry(&table[(size_t)p * GC_NCOLS], flags, x0, dxs, y0, dys, &tabs[(size_t)p * kTab]);
            g->col_plan = gbp_col_plan(tabs, n, cone, nx, ny, zvals, W, H);
            g->col_key.swap(key);
        }
        if (g->col_plan.ok) {
            const float *src = d_proj;
            if (g->compute_type == 2) {
                // compute-type half: FP16 samples with FP32 coordinates, weights and sums, the
                // arithmetic of the FP16 gathers, staged from a rounded FP32 copy
                const uint64_t n4 = (uint64_t)n * H * W / 4;
                UFOB_TRY(g->d_proj_h.ensure(n4 * 16));
                if (n4) {
                    const uint32_t grid = (uint32_t)std::min<uint64_t>((n4 + 255) / 256, (uint64_t)num_sms() * 16);
                    k_proj_round_half<<<grid, 256, 0, s>>>(reinterpret_cast<const float4 *>(d_proj), n4,
                                                           g->d_proj_h.as<float4>());
                    UFOB_CUDA_TRY(cudaGetLastError());
                    note_launch();
                }
                src = g->d_proj_h.as<float>();
            }
            GBPColArgs c;
            c.proj = src;
            c.tab = g->d_tab_f.as<float>();
            c.zvals = a.zvals;
            c.W = W;
            c.H = H;
            c.n_proj = n;
            c.nx = nx;
            c.ny = ny;
            c.nz = nz;
            c.burst = a.burst;
            c.bw = g->col_plan.bw;
            c.bh = g->col_plan.bh;
            c.norm = (float)a.norm;
            c.vol = static_cast<float *>(d_vol);
            c.err = device_error_word();
            bool launched = false;
            UFOB_TRY(launch_gbp_col(c, cone, &launched, s));
            if (launched) return UFOB_OK;
        }
    }
    if (g->compute_type == 2) {
        // FP16 samples: the gather unit returns 16-bit texels at twice the FP32 rate;
        // coordinates, weights and sums stay FP32
        size_t pitch16 = 0, plane16 = 0;
        UFOB_TRY(half_projections(g, d_proj, W, H, n, s, &pitch16, &plane16));
        if (!gbp_textures(g, g->d_proj16.ptr, W, H, n, a.addr, s, g->interpolation, true, pitch16, plane16))
            return fail(UFOB_ERR_UNSUPPORTED, "compute-type half needs texture-compatible projections (%ux%u)", W, H);
        a.tex = g->d_tex.as<cudaTextureObject_t>();
        a.hw_interp = g->interpolation;
        return cone ? launch_gbp_rt<true, float>(a, g->result_type, paramz, s)
                    : launch_gbp_rt<false, float>(a, g->result_type, paramz, s);
    }
    if (gbp_textures(g, d_proj, W, H, n, a.addr, s, g->interpolation)) {
        a.tex = g->d_tex.as<cudaTextureObject_t>();
        a.hw_interp = g->interpolation;
    } else if (g->interpolation) {
        return fail(UFOB_ERR_UNSUPPORTED, "interpolation=texture needs texture-compatible projections");
    }
    return cone ? launch_gbp_rt<true, float>(a, g->result_type, paramz, s)
                : launch_gbp_rt<false, float>(a, g->result_type, paramz, s);
}

extern "C" ufob_status ufob_gbp_run(ufob_gbp *g, const float *d_proj, uint32_t W, uint32_t H, void *d_vol,
                                    void *stream)
{
    if (!g || !d_proj || !d_vol) return fail(UFOB_ERR_INVALID, "gbp_run: NULL argument");
    UFOB_TRY(ensure_device());
    return gbp_compute(g, d_proj, W, H, d_vol, (cudaStream_t)stream);
}

extern "C" ufob_status ufob_gbp_process(ufob_gbp *g, const float *d_projection, uint32_t W, uint32_t H, void *stream)
{
    if (!g || !d_projection) return fail(UFOB_ERR_INVALID, "gbp_process: NULL argument");
    UFOB_TRY(ensure_device());
    UFOB_TRY(ufob_gbp_setup(g));
    cudaStream_t s = (cudaStream_t)stream;
    if (g->pushed == 0) {
        g->pw = W;
        g->ph = H;
        UFOB_TRY(g->d_proj.ensure((size_t)g->num_projections * W * H * sizeof(float)));
    }
    if (W != g->pw || H != g->ph) return fail(UFOB_ERR_INVALID, "projection size changed within the stream");
    if (g->pushed >= g->num_projections)
        return fail(UFOB_ERR_INVALID, "received more than num-projections (%u) projections", g->num_projections);
    UFOB_CUDA_TRY(cudaMemcpyAsync(g->d_proj.as<float>() + (size_t)g->pushed * W * H, d_projection,
                                  (size_t)W * H * sizeof(float), cudaMemcpyDeviceToDevice, s));
    g->pushed++;
    if (g->pushed == g->num_projections) {
        uint32_t nx, ny, nz;
        UFOB_TRY(ufob_gbp_get_requisition(g, W, H, &nx, &ny, &nz));
        UFOB_TRY(g->d_vol.ensure((size_t)nx * ny * nz * store_size(g->store_type)));
        UFOB_TRY(gbp_compute(g, g->d_proj.as<float>(), W, H, g->d_vol.ptr, s));
        g->volume_ready = true;
    }
    return UFOB_OK;
}

extern "C" ufob_status ufob_gbp_generate(ufob_gbp *g, void *d_slice, uint32_t index, void *stream)
{
    if (!g || !d_slice) return fail(UFOB_ERR_INVALID, "gbp_generate: NULL argument");
    if (g->pushed != g->num_projections || !g->volume_ready)
        return fail(UFOB_ERR_INVALID,
                    "general-backproject received only %u projections out of %u specified, no output will be generated",
                    g->pushed, g->num_projections);
    uint32_t nx, ny, nz;
    UFOB_TRY(ufob_gbp_get_requisition(g, g->pw, g->ph, &nx, &ny, &nz));
    if (index >= nz) return fail(UFOB_ERR_INVALID, "slice %u of %u", index, nz);
    const size_t bytes = (size_t)nx * ny * store_size(g->store_type);
    UFOB_CUDA_TRY(cudaMemcpyAsync(d_slice, g->d_vol.as<char>() + bytes * index, bytes, cudaMemcpyDeviceToDevice,
                                  (cudaStream_t)stream));
    return UFOB_OK;
}

extern "C" void ufob_gbp_destroy(ufob_gbp *g) { delete g; }

// ------------------------------------------------------------------ lamino-backproject
//
// src/ufo-lamino-backproject-task.c (setup :164-237, get_requisition :239-256,
// process :280-500, properties :690-811) with the kernels generated from
// src/kernels/templates/{z,center,lamino,roll}_template.in, common.in and
// definitions.in.  Per voxel (idx, idy, idz) and projection (sin, cos of the
// tomographic angle):
//   vx = idx * x_step + x_from, vy = idy * y_step + y_from, vz = z (or the z region)
//   px = vx cos + vy sin + xc                     (xc per slice for parameter x-center)
//   py = (vx cosL) sin + (-vy cosL) cos + vz sinL + yc
//   rotate(): px -= xc0; py -= yc; px = px cosR + py sinR; py = -px sinR + py cosR
//             (the updated px enters the second line); px += xc0; py += yc
//   volume += norm * sample(px, py)    (linear, texel centres at +1/2)
// with sin/cos of the lamino angle per slice for parameter lamino-angle and of
// minus the roll angle per slice for parameter roll-angle.  Every step is
// affine in (idx, idy, vz), so each (slice, projection) becomes one table of
// the general backprojector (k_gbp, FP32 texture gathers, exact weights); the
// FP32 scalars are formed as the task forms them on the host.

struct ufob_lamino {
    int x_region[3] = {0, 0, 0}, y_region[3] = {0, 0, 0};  // (from, to, step), integers
    float region[3] = {0.f, 0.f, 0.f};
    float z = 0.f;
    int projection_offset[2] = {0, 0};
    float center[2] = {0.f, 0.f};
    uint32_t num_projections = 0;
    float overall_angle = (float)M_PI;
    float tomo_angle = -FLT_MAX;
    float lamino_angle = 0.f, roll_angle = 0.f;
    int parameter = 0;  // z, x-center, lamino-angle, roll-angle
    int addressing_mode = AD_CLAMP;
    ufob_gbp g;  // tables, textures
    uint32_t pushed = 0, pw = 0, ph = 0;
    bool generated = false;
    DevBuf d_proj;
};

namespace {
const char *kLaminoParams[] = {"z", "x-center", "lamino-angle", "roll-angle"};

uint32_t lamino_region_size(const int r[3])
{
    // REGION_SIZE, src/ufo-lamino-backproject-task.c:41-43 (integer arithmetic)
    return r[2] == 0 ? 0u : (uint32_t)std::max(0, (r[1] - r[0] - 1) / r[2] + 1);
}
}  // namespace

extern "C" ufob_status ufob_lamino_create(ufob_lamino **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "lamino_create: out is NULL");
    *out = new ufob_lamino;
    return UFOB_OK;
}

extern "C" ufob_status ufob_lamino_set_array(ufob_lamino *l, const char *name, const double *v, uint32_t n)
{
    if (!l || (!v && n)) return fail(UFOB_ERR_INVALID, "lamino_set_array: NULL argument");
    if (name_is(name, "x-region") || name_is(name, "y-region")) {
        if (n != 3) return fail(UFOB_ERR_INVALID, "%s needs 3 values (from, to, step)", name);
        // set_region (:110-123): from > to is refused with a warning and the old value kept
        if ((int)v[0] > (int)v[1]) return UFOB_OK;
        int *r = name_is(name, "x-region") ? l->x_region : l->y_region;
        for (int i = 0; i < 3; i++) r[i] = (int)v[i];
    } else if (name_is(name, "region")) {
        if (n != 3) return fail(UFOB_ERR_INVALID, "region needs 3 values (from, to, step)");
        for (int i = 0; i < 3; i++) l->region[i] = (float)v[i];
    } else if (name_is(name, "projection-offset")) {
        if (n != 2) return fail(UFOB_ERR_INVALID, "projection-offset needs 2 values");
        for (int i = 0; i < 2; i++) l->projection_offset[i] = (int)v[i];
    } else if (name_is(name, "center")) {
        if (n != 2) return fail(UFOB_ERR_INVALID, "center needs 2 values (x, y)");
        for (int i = 0; i < 2; i++) l->center[i] = (float)v[i];
    } else {
        return fail(UFOB_ERR_INVALID, "lamino-backproject: no array property named '%s'", name ? name : "(null)");
    }
    return UFOB_OK;
}

extern "C" ufob_status ufob_lamino_set_property(ufob_lamino *l, const char *name, double v)
{
    if (!l) return fail(UFOB_ERR_INVALID, "lamino handle is NULL");
    if (name_is(name, "z")) l->z = (float)v;
    else if (name_is(name, "num-projections")) {
        if (v < 0 || v > 32768) return fail(UFOB_ERR_INVALID, "num-projections outside [0, 32768]");
        l->num_projections = (uint32_t)v;
    } else if (name_is(name, "overall-angle")) l->overall_angle = (float)v;
    else if (name_is(name, "tomo-angle")) l->tomo_angle = (float)v;
    else if (name_is(name, "lamino-angle")) l->lamino_angle = (float)v;
    else if (name_is(name, "roll-angle")) l->roll_angle = (float)v;
    else if (name_is(name, "parameter")) {
        if (!(v >= 0 && v <= 3)) return fail(UFOB_ERR_INVALID, "parameter %g", v);
        l->parameter = (int)v;
    } else return fail(UFOB_ERR_INVALID, "lamino-backproject: no numeric property named '%s'", name ? name : "(null)");
    return UFOB_OK;
}

extern "C" ufob_status ufob_lamino_set_property_string(ufob_lamino *l, const char *name, const char *value)
{
    if (!l) return fail(UFOB_ERR_INVALID, "lamino handle is NULL");
    int i;
    if (name_is(name, "parameter")) {
        if ((i = lookup(value, kLaminoParams, 4)) < 0) return fail(UFOB_ERR_INVALID, "unknown parameter '%s'", value);
        l->parameter = i;
        return UFOB_OK;
    }
    if (name_is(name, "addressing-mode")) {
        if ((i = lookup(value, kAddrNames, 5)) < 0) return fail(UFOB_ERR_INVALID, "unknown addressing-mode '%s'", value);
        l->addressing_mode = i;
        return UFOB_OK;
    }
    char *end = nullptr;
    double v = value ? strtod(value, &end) : 0.0;
    if (!value || end == value) return fail(UFOB_ERR_INVALID, "'%s' is not a number", value ? value : "(null)");
    return ufob_lamino_set_property(l, name, v);
}

extern "C" ufob_status ufob_lamino_setup(ufob_lamino *l)
{
    if (!l) return fail(UFOB_ERR_INVALID, "lamino handle is NULL");
    if (!l->num_projections) return fail(UFOB_ERR_SETUP, "Number of projections has not been set");
    if (l->region[2] == 0.0f) return fail(UFOB_ERR_SETUP, "Step in region is 0");
    if (l->addressing_mode == AD_REPEAT || l->addressing_mode == AD_MIRRORED_REPEAT)
        return fail(UFOB_ERR_UNSUPPORTED, "addressing-mode %s is undefined for unnormalised coordinates",
                    kAddrNames[l->addressing_mode]);
    return UFOB_OK;
}

extern "C" ufob_status ufob_lamino_get_requisition(ufob_lamino *l, uint32_t *nx, uint32_t *ny, uint32_t *nz)
{
    if (!l) return fail(UFOB_ERR_INVALID, "lamino handle is NULL");
    const uint32_t x = lamino_region_size(l->x_region), y = lamino_region_size(l->y_region);
    const float n = ceilf((l->region[1] - l->region[0]) / l->region[2]);
    const uint32_t z = l->region[2] == 0.0f || !(n > 0) ? 0u : (uint32_t)n;
    if (nx) *nx = x;
    if (ny) *ny = y;
    if (nz) *nz = z;
    return UFOB_OK;
}

static ufob_status lamino_compute(ufob_lamino *l, const float *d_proj, uint32_t W, uint32_t H, float *d_vol,
                                  cudaStream_t s)
{
    UFOB_TRY(ufob_lamino_setup(l));
    uint32_t nx, ny, nz;
    UFOB_TRY(ufob_lamino_get_requisition(l, &nx, &ny, &nz));
    if (!nx || !ny || !nz) return fail(UFOB_ERR_REQUISITION, "lamino-backproject: empty output region");
    const uint32_t n = l->num_projections;
    const int par = l->parameter;
    const bool paramz = par == 0;
    const uint32_t tab_slices = paramz ? 1 : nz;
    // FP32 scalars as the task forms them (process :300-360)
    const float norm = (float)(fabs((double)l->overall_angle) / n);
    const float xs = (float)l->x_region[2], x0 = (float)l->x_region[0];
    const float ys = (float)l->y_region[2], y0 = (float)l->y_region[0];
    const float xc0 = par == 1 ? l->region[0] - (float)l->projection_offset[0]
                               : l->center[0] - (float)l->projection_offset[0];
    const float xcs = par == 1 ? l->region[2] : xc0;
    const float yc = l->center[1] - (float)l->projection_offset[1];
    std::vector<double> zvals(nz);
    for (uint32_t k = 0; k < nz; k++)
        zvals[k] = paramz ? (double)fmaf((float)k, l->region[2], l->region[0]) : (double)l->z;
    std::vector<float> tab((size_t)tab_slices * n * kTab, 0.0f);
    for (uint32_t sl = 0; sl < tab_slices; sl++) {
        float sinL = sinf(l->lamino_angle), cosL = cosf(l->lamino_angle);
        float sinR = sinf(-l->roll_angle), cosR = cosf(-l->roll_angle);
        float xcc = xc0;
        if (par == 1) xcc = fmaf((float)sl, xcs, xc0);
        if (par == 2) {
            const float a = fmaf((float)sl, l->region[2], l->region[0]);
            sinL = sinf(a);
            cosL = cosf(a);
        }
        if (par == 3) {
            const float a = fmaf((float)sl, -l->region[2], -l->region[0]);
            sinR = sinf(a);
            cosR = cosf(a);
        }
        for (uint32_t p = 0; p < n; p++) {
            const float t = l->tomo_angle > -FLT_MAX ? l->tomo_angle : l->overall_angle * (float)p / (float)n;
            const double sn = (double)(float)sin((double)t), cs = (double)(float)cos((double)t);
            // rows over X = (idx, idy, vz, 1)
            const double VX[4] = {xs, 0.0, 0.0, x0}, VY[4] = {0.0, ys, 0.0, y0}, VZ[4] = {0.0, 0.0, 1.0, 0.0};
            double px[4], py[4], u[4], v[4];
            for (int i = 0; i < 4; i++) {
                px[i] = VX[i] * cs + VY[i] * sn + (i == 3 ? (double)xcc : 0.0);
                py[i] = VX[i] * (double)cosL * sn - VY[i] * (double)cosL * cs + VZ[i] * (double)sinL +
                        (i == 3 ? (double)yc : 0.0);
            }
            for (int i = 0; i < 4; i++) {  // rotate() with its sequential update
                const double a = px[i] - (i == 3 ? (double)xc0 : 0.0), b = py[i] - (i == 3 ? (double)yc : 0.0);
                const double a2 = a * cosR + b * sinR;
                const double b2 = -a2 * sinR + b * cosR;
                u[i] = a2 + (i == 3 ? (double)xc0 : 0.0);
                v[i] = b2 + (i == 3 ? (double)yc : 0.0);
            }
            float *e = &tab[((size_t)sl * n + p) * kTab];
            for (int i = 0; i < 4; i++) {
                e[i] = (float)u[i];
                e[4 + i] = (float)v[i];
            }
        }
    }
    ufob_gbp &g = l->g;
    UFOB_TRY(g.d_tab_f.ensure(tab.size() * sizeof(float)));
    UFOB_TRY(g.d_zvals.ensure(nz * sizeof(double)));
    UFOB_CUDA_TRY(cudaMemcpyAsync(g.d_tab_f.ptr, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    UFOB_CUDA_TRY(cudaMemcpyAsync(g.d_zvals.ptr, zvals.data(), nz * sizeof(double), cudaMemcpyHostToDevice, s));
    // the host vectors must outlive the copies: pageable sources are staged before the calls return
    GBPArgs a;
    a.proj = d_proj;
    a.W = W;
    a.H = H;
    a.n_proj = n;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.burst = 16;  // BURST, meson option lamino_backproject_burst_mode (default 16)
    a.tab = g.d_tab_f.ptr;
    a.zvals = g.d_zvals.as<double>();
    a.norm = norm;
    a.sp.kind = ST_FLOAT;
    a.sp.gray_min = 0.0;
    a.sp.maxval = 0.0;
    a.sp.gray_scale = 0.0;
    a.addr = l->addressing_mode == AD_CLAMP ? AD_CLAMP : AD_CLAMP_TO_EDGE;
    a.vol = d_vol;
    a.tex = nullptr;
    a.hw_interp = 0;
    if (paramz && a.addr == AD_CLAMP && W % 4 == 0 && !((uintptr_t)d_proj & 15)) {
        // TMA-staged detector windows when u does not depend on z (no roll angle); the plan is
        // kept while the tables stay the same
        std::vector<double> key(tab.begin(), tab.end());
        key.insert(key.end(), {(double)nx, (double)ny, (double)W, (double)H});
        key.insert(key.end(), zvals.begin(), zvals.end());
        if (key != g.col_key) {
            g.col_plan = gbp_col_plan(std::vector<double>(tab.begin(), tab.end()), n, false, nx, ny, zvals, W, H);
            g.col_key.swap(key);
        }
        if (g.col_plan.ok) {
            GBPColArgs c;
            c.proj = d_proj;
            c.tab = g.d_tab_f.as<float>();
            c.zvals = a.zvals;
            c.W = W;
            c.H = H;
            c.n_proj = n;
            c.nx = nx;
            c.ny = ny;
            c.nz = nz;
            c.burst = a.burst;
            c.bw = g.col_plan.bw;
            c.bh = g.col_plan.bh;
            c.norm = norm;
            c.vol = d_vol;
            c.err = device_error_word();
            bool launched = false;
            UFOB_TRY(launch_gbp_col(c, false, &launched, s));
            if (launched) return UFOB_OK;
        }
    }
    if (gbp_textures(&g, d_proj, W, H, n, a.addr, s)) a.tex = g.d_tex.as<cudaTextureObject_t>();
    return launch_gbp_rt<false, float>(a, RT_FLOAT, paramz, s);
}

extern "C" ufob_status ufob_lamino_run(ufob_lamino *l, const float *d_proj, uint32_t W, uint32_t H, float *d_vol,
                                       void *stream)
{
    if (!l || !d_proj || !d_vol) return fail(UFOB_ERR_INVALID, "lamino_run: NULL argument");
    UFOB_TRY(ensure_device());
    return lamino_compute(l, d_proj, W, H, d_vol, (cudaStream_t)stream);
}

extern "C" ufob_status ufob_lamino_process(ufob_lamino *l, const float *d_projection, uint32_t W, uint32_t H,
                                           void *stream)
{
    if (!l || !d_projection) return fail(UFOB_ERR_INVALID, "lamino_process: NULL argument");
    UFOB_TRY(ensure_device());
    UFOB_TRY(ufob_lamino_setup(l));
    if (l->pushed == 0) {
        l->pw = W;
        l->ph = H;
        UFOB_TRY(l->d_proj.ensure((size_t)l->num_projections * W * H * sizeof(float)));
    }
    if (W != l->pw || H != l->ph) return fail(UFOB_ERR_INVALID, "projection size changed within the stream");
    if (l->pushed >= l->num_projections)
        return fail(UFOB_ERR_INVALID, "received more than num-projections (%u) projections", l->num_projections);
    UFOB_CUDA_TRY(cudaMemcpyAsync(l->d_proj.as<float>() + (size_t)l->pushed * W * H, d_projection,
                                  (size_t)W * H * sizeof(float), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    l->pushed++;
    return UFOB_OK;
}

extern "C" ufob_status ufob_lamino_generate(ufob_lamino *l, float *d_vol, void *stream)
{
    if (!l || !d_vol) return fail(UFOB_ERR_INVALID, "lamino_generate: NULL argument");
    if (l->generated) return fail(UFOB_ERR_INVALID, "lamino-backproject: the volume was already generated");
    if (l->pushed != l->num_projections)
        return fail(UFOB_ERR_INVALID, "lamino-backproject received %u projections out of %u", l->pushed,
                    l->num_projections);
    UFOB_TRY(lamino_compute(l, l->d_proj.as<float>(), l->pw, l->ph, d_vol, (cudaStream_t)stream));
    l->generated = true;
    return UFOB_OK;
}

extern "C" void ufob_lamino_destroy(ufob_lamino *l) { delete l; }
