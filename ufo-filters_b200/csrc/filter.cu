// Ramp-filter stage: the reference's `fft ! filter ! ifft` chain fused into one
// kernel per pair of sinogram rows.
//
// Reference behaviour restated here:
//  * src/ufo-fft-task.c:123-196,293-304 and src/kernels/fft.cl:20-48 -- each
//    row of width W is zero-padded to the FFT width N (fft "size-x", default W)
//    and transformed forward (e^{-2 pi i ...}).
//  * src/ufo-filter-task.c:162-336 -- a vector of 2N interleaved float
//    coefficients c is built once; src/kernels/filter.cl:20-29 multiplies the
//    real part of bin k by c[2k] and the imaginary part by c[2k+1].
//  * src/ufo-ifft-task.c:287-311 and src/kernels/fft.cl:50-82 -- backward FFT,
//    real part, crop to "crop-width", scale by 1/N.
//
// B200 formulation.  The real part of the inverse transform only depends on
// the Hermitian part of the filtered spectrum, so for a real row with spectrum
// X the result equals C2R(G . X) with per-bin gains
//   G[k] = ((c[2k] + c[2(N-k)]) / 2, (c[2k+1] + c[2(N-k)+1]) / 2),  k = 0..N/2,
// applied to the real and imaginary parts separately.  This is exact for every
// coefficient vector the reference can build (also the non-symmetric
// faris-byer one).  Two real rows a, b are transformed as one complex signal
// z = a + i b; their spectra are separated, filtered and recombined in shared
// memory, so one complex FFT pair serves two rows.  The FFT is a radix-4 (plus
// one radix-2 pass for odd log2 N) Stockham transform in shared memory, with
// twiddles computed in FP64 and staged into shared memory once per CTA.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include <algorithm>
#include <cstdlib>

#include "f32x2.cuh"
#include "tma.cuh"
#include "ufob_internal.h"

namespace ufob {

static constexpr uint32_t kMaxFusedFFT = 8192;
static constexpr int kFilterThreads = 256;

// The register-radix kernel serves FFT widths 256..4096 unless UFOB_FILTER_RADIX4=1 selects the
// shared-memory radix-4 kernel for every width (comparison and fallback).
static bool fast_filter_enabled()
{
    static const int on = [] {
        const char *e = getenv("UFOB_FILTER_RADIX4");
        return (e && e[0] == '1') ? 0 : 1;
    }();
    return on != 0;
}

// ------------------------------------------------------------ host coefficient code

static uint32_t padding_value(uint32_t x)  // src/ufo-filter-task.c:242-252
{
    uint32_t padding = 2 * x, result = 1;
    while (result < padding) result *= 2;
    return result;
}

bool build_filter_coefficients(const ufob_filter_props &p, uint32_t nfft, std::vector<float> &f)
{
    const uint32_t width = 2 * nfft;  // interleaved float width, as the reference's requisition
    if (!is_pow2(width)) {
        set_error("Invalid filter input width %u, must be a power of two", width);
        return false;
    }
    f.assign(width, 0.f);
    f[0] = f[1] = (float)(0.5 / width);
    const double scale = p.scale, cutoff = p.cutoff, order = p.order, tau = p.tau, theta = p.theta;
    const double step = 2.0 / width;
    switch (p.filter) {
    case UFOB_FILTER_RAMP:
        for (uint32_t k = 1; k < width / 4 + 1; k++) f[2 * k] = f[2 * k + 1] = (float)(k * step * scale);
        break;
    case UFOB_FILTER_RAMP_FROMREAL:
        f[0] = f[1] = (float)(0.25 * scale);
        for (uint32_t k = 1; k < width / 4 + 1; k++)
            f[2 * k] = f[2 * k + 1] = (k % 2) ? (float)(-scale / ((double)k * k * M_PI * M_PI)) : 0.f;
        break;
    case UFOB_FILTER_BUTTERWORTH:
        for (uint32_t k = 0; k < width / 4 + 1; k++) {
            double fr = k * step;
            f[2 * k] = f[2 * k + 1] = (float)(fr / (1.0 + pow(fr / cutoff, 2.0 * order)) * scale);
        }
        break;
    case UFOB_FILTER_FARIS_BYER: {
        const double pi_squared_tau = M_PI * M_PI * tau;
        const double sin_theta_2 = -sin(theta) / 2;
        const uint32_t padding = padding_value(width);
        f[0] = 0;
        for (uint32_t x = 1; x <= width / 2; x++)
            if (x % 2 != 0) f[x] = (float)(1 / (pi_squared_tau * x));
        for (uint32_t i = width / 2 + 1; i < width; i++) {
            uint32_t x = width + 1 - i;
            if (x % 2 != 0) f[padding - width - i - 1] = (float)(sin_theta_2 / ((double)x * x * pi_squared_tau));
        }
        break;
    }
    case UFOB_FILTER_HAMMING:
        for (uint32_t k = 0; k < width / 4 + 1; k++) {
            double fr = k * step;
            f[2 * k] = f[2 * k + 1] =
                fr < cutoff ? (float)(fr * (0.54 + 0.46 * cos(M_PI * fr / cutoff)) * scale) : 0.f;
        }
        break;
    case UFOB_FILTER_BH3:
        for (uint32_t k = 1; k < width / 4 + 1; k++) {
            double fr = k * step;
            f[2 * k] = f[2 * k + 1] =
                (float)(fr * (0.42 + 0.5 * cos(fr * M_PI) + 0.08 * cos(2.0 * fr * M_PI)) * scale);
        }
        break;
    default:
        set_error("unknown filter type %d", p.filter);
        return false;
    }
    // mirror_coefficients, src/ufo-filter-task.c:162-169
    for (uint32_t k = width / 2 + 2; k < width; k += 2) {
        f[k] = f[width - k];
        f[k + 1] = f[width - k + 1];
    }
    return true;
}

// ------------------------------------------------------------ FP64 table kernels

__global__ void k_twiddles(float2 *tw, uint32_t n)
{
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double s, c;
    sincospi(-2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_float2((float)c, (float)s);
}

// Per-pass twiddles of the register-radix kernel: [0, 64) pass 2, w^(2^b k) =
// exp(-2 pi i 2^b k / 256) at b * 16 + k; then pass 3, exp(-2 pi i 2^b k / (256 R3))
// at 64 + b * 256 + k for b < log2 R3 (R3 = n / 256).
__global__ void k_pass_twiddles(float2 *tab, uint32_t n, uint32_t count)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t b, k;
    double den;
    if (i < 64) {
        b = i / 16;
        k = i % 16;
        den = 256.0;
    } else {
        b = (i - 64) / 256;
        k = (i - 64) % 256;
        den = (double)n;
    }
    double s, c;
    sincospi(-2.0 * (double)(k << b) / den, &s, &c);
    tab[i] = make_float2((float)c, (float)s);
}

static uint32_t pass_twiddle_count(uint32_t n)
{
    const uint32_t r3 = n / 256;
    return 64 + 256 * (r3 >= 16 ? 4 : r3 >= 8 ? 3 : r3 >= 4 ? 2 : r3 >= 2 ? 1 : 0);
}

// In-place forward DFT of the interleaved pairs (ramp-fromreal, src/ufo-filter-task.c:317-334),
// FP64, direct summation over an exact index m = j*k mod n.
__global__ void k_dft_pairs_fp64(const float *in, float *out, uint32_t n)
{
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double re = 0.0, im = 0.0;
    for (uint32_t j = 0; j < n; j++) {
        uint32_t m = (uint32_t)(((uint64_t)j * k) & (n - 1));
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        double a = in[2 * j], b = in[2 * j + 1];
        re += a * c - b * s;
        im += a * s + b * c;
    }
    out[2 * k] = (float)re;
    out[2 * k + 1] = (float)im;
}

// Symmetrised gains with the 1/N of the inverse transform folded in (exact: N is a power of two).
__global__ void k_gains(const float *coeff, float2 *gains, uint32_t n)
{
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > n / 2) return;
    uint32_t m = (n - k) & (n - 1);
    double inv = 1.0 / (double)n;
    double gr = 0.5 * ((double)coeff[2 * k] + (double)coeff[2 * m]) * inv;
    double gi = 0.5 * ((double)coeff[2 * k + 1] + (double)coeff[2 * m + 1]) * inv;
    gains[k] = make_float2((float)gr, (float)gi);
}

ufob_status filter_plan_build(const ufob_filter_props &p, uint32_t nfft, FilterPlan &plan, cudaStream_t stream)
{
    if (plan.nfft == nfft && !plan.coeff.empty()) return UFOB_OK;
    std::vector<float> c;
    if (!build_filter_coefficients(p, nfft, c)) return UFOB_ERR_REQUISITION;
    UFOB_TRY(plan.d_coeff.ensure(sizeof(float) * 2 * nfft));
    UFOB_TRY(plan.d_gains.ensure(sizeof(float2) * (nfft / 2 + 1)));
    UFOB_TRY(plan.d_twiddle.ensure(sizeof(float2) * nfft));
    const int T = 256;
    if (p.filter == UFOB_FILTER_RAMP_FROMREAL) {
        DevBuf tmp;
        UFOB_TRY(tmp.ensure(sizeof(float) * 2 * nfft));
        UFOB_CUDA_TRY(cudaMemcpyAsync(tmp.ptr, c.data(), sizeof(float) * 2 * nfft, cudaMemcpyHostToDevice, stream));
        k_dft_pairs_fp64<<<(nfft + T - 1) / T, T, 0, stream>>>(tmp.as<float>(), plan.d_coeff.as<float>(), nfft);
        UFOB_CUDA_TRY(cudaGetLastError());
        note_launch();
        UFOB_CUDA_TRY(cudaMemcpyAsync(c.data(), plan.d_coeff.ptr, sizeof(float) * 2 * nfft, cudaMemcpyDeviceToHost,
                                      stream));
        UFOB_CUDA_TRY(cudaStreamSynchronize(stream));
    } else {
        UFOB_CUDA_TRY(
            cudaMemcpyAsync(plan.d_coeff.ptr, c.data(), sizeof(float) * 2 * nfft, cudaMemcpyHostToDevice, stream));
    }
    k_gains<<<(nfft / 2 + 1 + T - 1) / T, T, 0, stream>>>(plan.d_coeff.as<float>(), plan.d_gains.as<float2>(), nfft);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    k_twiddles<<<(nfft + T - 1) / T, T, 0, stream>>>(plan.d_twiddle.as<float2>(), nfft);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    if (nfft >= 256 && nfft <= 4096) {
        const uint32_t cnt = pass_twiddle_count(nfft);
        UFOB_TRY(plan.d_pass_tw.ensure(sizeof(float2) * cnt));
        k_pass_twiddles<<<(cnt + T - 1) / T, T, 0, stream>>>(plan.d_pass_tw.as<float2>(), nfft, cnt);
        UFOB_CUDA_TRY(cudaGetLastError());
        note_launch();
    }
    UFOB_CUDA_TRY(cudaStreamSynchronize(stream));
    plan.coeff.swap(c);
    plan.nfft = nfft;
    return UFOB_OK;
}

// ------------------------------------------------------------ fused row kernel

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// complex add / subtract as one packed FP32 operation (each lane rounds as the scalar add)
__device__ __forceinline__ float2 cadd(float2 a, float2 b)
{
    float2 r;
    f2unpack(f2add(f2pack(a.x, a.y), f2pack(b.x, b.y)), r.x, r.y);
    return r;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b)
{
    float2 r;
    f2unpack(f2sub(f2pack(a.x, a.y), f2pack(b.x, b.y)), r.x, r.y);
    return r;
}

// One Stockham pass of radix R over N points: src -> dst (both shared).
// Twiddle for leg r of butterfly j in a sub-transform of size Ns*R is
// w_N^(r * k * N / (Ns * R)) with k = j mod Ns (Govindaraju et al., SC'08).
template <int R, bool INV>
__device__ __forceinline__ void stockham_pass(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                              const float2 *__restrict__ tw, uint32_t N, uint32_t Ns, int twshift)
{
    const uint32_t nb = N / R;
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        const uint32_t k = j & (Ns - 1);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src[j + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                float2 w = tw[(r * k) << twshift];
                if (INV) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        if (R == 2) {
            float2 a = v[0], b = v[1];
            v[0] = cadd(a, b);
            v[1] = csub(a, b);
        } else {
            float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
            float2 t2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
            // forward: d * (-i) = (d.y, -d.x); inverse: d * i = (-d.y, d.x)
            float2 t3 = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
            v[0] = cadd(t0, t2);
            v[2] = csub(t0, t2);
            v[1] = cadd(t1, t3);
            v[3] = csub(t1, t3);
        }
        const uint32_t base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[base + r * Ns] = v[r];
    }
}

// Full transform; returns the buffer holding the result.
template <bool INV>
__device__ float2 *fft_smem(float2 *a, float2 *b, const float2 *tw, uint32_t N, int log2N)
{
    uint32_t Ns = 1;
    int l = log2N;
    if (l & 1) {
        stockham_pass<2, INV>(a, b, tw, N, Ns, l - 1);
        __syncthreads();
        float2 *t = a; a = b; b = t;
        Ns = 2;
        l -= 1;
    }
    while (l > 0) {
        // twiddle index scale N / (Ns * 4) = 2^(log2N - log2(Ns) - 2)
        int shift = log2N - (31 - __clz(Ns)) - 2;
        stockham_pass<4, INV>(a, b, tw, N, Ns, shift);
        __syncthreads();
        float2 *t = a; a = b; b = t;
        Ns *= 4;
        l -= 2;
    }
    return a;
}

enum OutKind { OUT_F32 = 0, OUT_F16 = 1, OUT_BF16 = 2, OUT_F16_PAIRS = 3, OUT_BF16_PAIRS = 4, OUT_F16_QUADS = 5 };

template <int OUT>
__device__ __forceinline__ void store_value(void *out, size_t idx, float v)
{
    if (OUT == OUT_F32) reinterpret_cast<float *>(out)[idx] = v;
    if (OUT == OUT_F16) reinterpret_cast<__half *>(out)[idx] = __float2half_rn(v);
    if (OUT == OUT_BF16) reinterpret_cast<__nv_bfloat16 *>(out)[idx] = __float2bfloat16_rn(v);
}

template <int OUT>
__device__ __forceinline__ uint32_t pack_pair(float lo, float hi)
{
    if (OUT == OUT_F16_PAIRS || OUT == OUT_F16_QUADS) {
        __half2 h = __floats2half2_rn(lo, hi);
        return *reinterpret_cast<uint32_t *>(&h);
    } else {
        __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        return *reinterpret_cast<uint32_t *>(&h);
    }
}

// Rows of one work item (one complex FFT of a + i b): rows 2*pair and
// 2*pair+1, or for the slice-quad layout (OUT_F16_QUADS, `P` angles per slice)
// item pair = (group * P + angle) * 2 + half, i.e. slices 4*group + 2*half and
// 4*group + 2*half + 1 at one angle.
struct PairMap {
    uint32_t ra, rb, half;
    bool hasa, hasb;
    size_t cell0;
};

template <int OUT>
__device__ __forceinline__ PairMap map_pair(uint32_t pair, uint32_t rows, uint32_t P, uint32_t out_pitch)
{
    PairMap m;
    m.ra = 2 * pair;
    m.rb = 2 * pair + 1;
    m.half = 0;
    m.cell0 = 0;
    m.hasa = m.ra < rows;
    if (OUT == OUT_F16_QUADS) {
        const uint32_t gp = pair >> 1;  // group * P + angle
        m.half = pair & 1u;
        const uint32_t grp = gp / P, ang = gp - grp * P;
        m.ra = (4 * grp + 2 * m.half) * P + ang;
        m.rb = m.ra + P;
        m.hasa = m.ra < rows;
        m.cell0 = (size_t)gp * out_pitch;
    }
    m.hasb = m.rb < rows;
    return m;
}

// Store the filtered pair (X(n) = complex sample n: real = row a, imag = row b)
// in the output layout; threads t0, t0 + step, ... share the row.
template <int OUT, typename GET>
__device__ __forceinline__ void store_pair(const PairMap &m, GET X, void *__restrict__ out, uint32_t out_w,
                                           uint32_t out_pitch, uint32_t t0, uint32_t step)
{
    if (OUT == OUT_F16_QUADS) {
        // words `half` (taps j-1) and 2 + `half` (taps j) of cell j; rows a, b in the low, high halves
        uint32_t *o = reinterpret_cast<uint32_t *>(out) + m.cell0 * 4;
        for (uint32_t j = t0; j < out_pitch; j += step) {
            float2 lo = (j >= 1 && j - 1 < out_w) ? X(j - 1) : make_float2(0.f, 0.f);
            float2 hi = (j < out_w) ? X(j) : make_float2(0.f, 0.f);
            if (!m.hasa) lo.x = hi.x = 0.f;  // slices past the stack: exact zeros, not FFT round-off
            if (!m.hasb) lo.y = hi.y = 0.f;
            o[(size_t)j * 4 + m.half] = pack_pair<OUT>(lo.x, lo.y);
            o[(size_t)j * 4 + 2 + m.half] = pack_pair<OUT>(hi.x, hi.y);
        }
    } else if (OUT == OUT_F16_PAIRS || OUT == OUT_BF16_PAIRS) {
        uint32_t *o = reinterpret_cast<uint32_t *>(out);
        for (uint32_t j = t0; j < out_pitch; j += step) {
            float2 lo = (j >= 1 && j - 1 < out_w) ? X(j - 1) : make_float2(0.f, 0.f);
            float2 hi = (j < out_w) ? X(j) : make_float2(0.f, 0.f);
            o[(size_t)m.ra * out_pitch + j] = pack_pair<OUT>(lo.x, hi.x);
            if (m.hasb) o[(size_t)m.rb * out_pitch + j] = pack_pair<OUT>(lo.y, hi.y);
        }
    } else {
        for (uint32_t n = t0; n < out_w; n += step) {
            float2 v = X(n);
            store_value<OUT>(out, (size_t)m.ra * out_pitch + n, v.x);
            if (m.hasb) store_value<OUT>(out, (size_t)m.rb * out_pitch + n, v.y);
        }
    }
}

// Filter one work item in shared memory with the radix-4 Stockham transform
// (any power-of-two N up to 8192).
template <int OUT, bool PRE>
__device__ __forceinline__ void filter_pair(const RowSource &src, uint32_t width, uint32_t rows, uint32_t pair,
                                            float2 *bufA, float2 *bufB, const float2 *tw, const float2 *gains,
                                            uint32_t N, int log2N, void *__restrict__ out, uint32_t out_w,
                                            uint32_t out_pitch, uint32_t P = 0)
{
    const PairMap m = map_pair<OUT>(pair, rows, P, out_pitch);
    uint32_t ya, pa_proj, yb, pb_proj;
    const float *pa = row_start(src, m.hasa ? m.ra : 0, ya, pa_proj);
    const float *pb = row_start(src, m.hasb ? m.rb : 0, yb, pb_proj);
    __syncthreads();  // previous pair's output reads of bufA/bufB (and table loads) are done
    for (uint32_t n = threadIdx.x; n < N; n += blockDim.x) {
        float a = 0.f, b = 0.f;
        if (n < width) {  // zero padding to N comes after the preprocessing
            if (m.hasa) a = __ldg(pa + n);
            if (m.hasb) b = __ldg(pb + n);
            if (PRE) {
                if (m.hasa) a = preprocess_value(src, a, n, ya, pa_proj);
                if (m.hasb) b = preprocess_value(src, b, n, yb, pb_proj);
            }
        }
        bufA[n] = make_float2(a, b);
    }
    __syncthreads();
    float2 *Z = fft_smem<false>(bufA, bufB, tw, N, log2N);
    // separate, filter, recombine (pairs (k, N-k) are disjoint across threads)
    for (uint32_t k = threadIdx.x; k <= N / 2; k += blockDim.x) {
        const uint32_t mm = (N - k) & (N - 1);
        float2 zk = Z[k], zm = Z[mm], g = gains[k];
        float ax = 0.5f * (zk.x + zm.x), ay = 0.5f * (zk.y - zm.y);
        float bx = 0.5f * (zk.y + zm.y), by = -0.5f * (zk.x - zm.x);
        ax *= g.x; ay *= g.y; bx *= g.x; by *= g.y;
        Z[k] = make_float2(ax - by, ay + bx);
        if (mm != k) Z[mm] = make_float2(ax + by, bx - ay);
    }
    __syncthreads();
    float2 *other = (Z == bufA) ? bufB : bufA;
    float2 *X = fft_smem<true>(Z, other, tw, N, log2N);
    store_pair<OUT>(m, [X](uint32_t i) { return X[i]; }, out, out_w, out_pitch, threadIdx.x, blockDim.x);
}

template <int OUT, bool PRE>
__global__ void __launch_bounds__(kFilterThreads) k_filter_rows(const RowSource src, uint32_t width, uint32_t rows,
                                                                const float2 *__restrict__ g_tw,
                                                                const float2 *__restrict__ g_gains, uint32_t N,
                                                                int log2N, void *__restrict__ out, uint32_t out_w,
                                                                uint32_t out_pitch, uint32_t npairs, uint32_t P)
{
    extern __shared__ float4 smem_f4[];
    float2 *bufA = reinterpret_cast<float2 *>(smem_f4);
    float2 *bufB = bufA + N;
    float2 *tw = bufB + N;
    float2 *gains = tw + N;

    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) tw[i] = g_tw[i];
    for (uint32_t i = threadIdx.x; i <= N / 2; i += blockDim.x) gains[i] = g_gains[i];

    for (uint32_t pair = blockIdx.x; pair < npairs; pair += gridDim.x)
        filter_pair<OUT, PRE>(src, width, rows, pair, bufA, bufB, tw, gains, N, log2N, out, out_w, out_pitch, P);
}

// ------------------------------------------------------------ register-radix kernel (N = 256 .. 4096)
//
// A team of T = N / 16 threads transforms one work item; every thread holds 16
// complex values in registers and each Stockham pass is a radix-16 (or, for the
// last pass, radix N / 256) DFT in registers followed by one exchange through
// shared memory: 2 or 3 passes per transform instead of log4 N radix-4 passes,
// 7 barriers per work item.  Shared indices are XOR-swizzled, i ^ ((i >> 4) &
// 15), which makes the stride-16 stores of the first pass conflict-free.
// Twiddles of pass p come from a per-pass table w^(2^b * k), b < log2 radix,
// and the others are products of at most three of them.  Two or more teams
// share a 256-thread CTA and move in lock step.

static constexpr int kFastThreads = 256;

__device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ ((i >> 4) & 15u); }

template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a)  // a * (-i) forward, a * (+i) inverse
{
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// a * (c, s) with s negated for the inverse transform
template <bool INV>
__device__ __forceinline__ float2 mulc(float2 a, float c, float s)
{
    if (INV) s = -s;
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2 &x0, float2 &x1, float2 &x2, float2 &x3)
{
    const float2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), d = csub(x1, x3);
    x0 = cadd(t0, t2);
    x2 = csub(t0, t2);
    // t3 = d * (-i) forward, d * (+i) inverse; x1 = t1 + t3 and x3 = t1 - t3 cross the lanes, so they
    // stay scalar (a + (-b) and a - b round alike)
    if (!INV) {
        x1 = make_float2(t1.x + d.y, t1.y - d.x);
        x3 = make_float2(t1.x - d.y, t1.y + d.x);
    } else {
        x1 = make_float2(t1.x - d.y, t1.y + d.x);
        x3 = make_float2(t1.x + d.y, t1.y - d.x);
    }
}

// In-place DFT of R points in natural order (R = 2, 4, 8, 16), forward e^{-2 pi i nk/R}.
template <int R, bool INV>
__device__ __forceinline__ void dft(float2 *v)
{
    constexpr float r2 = 0.70710678118654752440f;
    constexpr float c1 = 0.92387953251128675613f;  // cos(pi/8)
    constexpr float s1 = 0.38268343236508977173f;  // sin(pi/8)
    if (R == 2) {
        const float2 a = v[0];
        v[0] = cadd(a, v[1]);
        v[1] = csub(a, v[1]);
    } else if (R == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3]);
    } else if (R == 8) {
        // x[n1 + 2 n2]: DFT4 over n2, twiddle W8^(n1 k2), DFT2 over n1 -> X[k2 + 4 k1]
        dft4<INV>(v[0], v[2], v[4], v[6]);
        dft4<INV>(v[1], v[3], v[5], v[7]);
        v[3] = mulc<INV>(v[3], r2, -r2);
        v[5] = mul_mi<INV>(v[5]);
        v[7] = mulc<INV>(v[7], -r2, -r2);
        float2 o[8];
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) {
            o[k2] = cadd(v[2 * k2], v[2 * k2 + 1]);
            o[k2 + 4] = csub(v[2 * k2], v[2 * k2 + 1]);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = o[i];
    } else {
        // x[n1 + 4 n2]: DFT4 over n2, twiddle W16^(n1 k2), DFT4 over n1 -> X[k2 + 4 k1]
#pragma unroll
        for (int n1 = 0; n1 < 4; n1++) dft4<INV>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
        // y[n1][k2] sits in v[n1 + 4 k2]
        v[1 + 4] = mulc<INV>(v[1 + 4], c1, -s1);    // W^1
        v[1 + 8] = mulc<INV>(v[1 + 8], r2, -r2);    // W^2
        v[1 + 12] = mulc<INV>(v[1 + 12], s1, -c1);  // W^3
        v[2 + 4] = mulc<INV>(v[2 + 4], r2, -r2);    // W^2
        v[2 + 8] = mul_mi<INV>(v[2 + 8]);           // W^4
        v[2 + 12] = mulc<INV>(v[2 + 12], -r2, -r2); // W^6
        v[3 + 4] = mulc<INV>(v[3 + 4], s1, -c1);    // W^3
        v[3 + 8] = mulc<INV>(v[3 + 8], -r2, -r2);   // W^6
        v[3 + 12] = mulc<INV>(v[3 + 12], -c1, s1);  // W^9
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) dft4<INV>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
        // X[k2 + 4 k1] sits in v[k1 + 4 k2]: transpose the 4x4 block
        float2 o[16];
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++)
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) o[k2 + 4 * k1] = v[k1 + 4 * k2];
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = o[i];
    }
}

// v[m] *= w^(m k) for m < R, with w^(2^b k) = tab[b * Ns + k]
template <int R, bool INV>
__device__ __forceinline__ void twiddle(float2 *v, const float2 *tab, uint32_t k, uint32_t Ns)
{
    float2 w[R];
    w[1] = tab[k];
    if (R >= 4) w[2] = tab[Ns + k];
    if (R >= 8) w[4] = tab[2 * Ns + k];
    if (R >= 16) w[8] = tab[3 * Ns + k];
    if (INV) {
        w[1].y = -w[1].y;
        if (R >= 4) w[2].y = -w[2].y;
        if (R >= 8) w[4].y = -w[4].y;
        if (R >= 16) w[8].y = -w[8].y;
    }
    if (R >= 4) w[3] = cmul(w[1], w[2]);
    if (R >= 8) {
        w[5] = cmul(w[1], w[4]);
        w[6] = cmul(w[2], w[4]);
        w[7] = cmul(w[3], w[4]);
    }
    if (R >= 16) {
#pragma unroll
        for (int m = 9; m < 16; m++) w[m] = cmul(w[m - 8], w[8]);
    }
#pragma unroll
    for (int m = 1; m < R; m++) v[m] = cmul(v[m], w[m]);
}

// One Stockham pass (Ns > 1) of radix R over N points, shared src -> shared dst;
// thread t of a team of T handles butterflies t, t + T, ... (16 / R of them).
// LIN writes dst in natural order: the last pass of a transform stores runs of
// consecutive elements across lanes, conflict-free without the swizzle, and a
// linear result serves the filter step's mirrored reads and the output's
// (j - 1, j) reads without bank conflicts.
template <int R, bool INV, bool LIN>
__device__ __forceinline__ void fast_pass(const float2 *src, float2 *dst, const float2 *tab, uint32_t N, uint32_t Ns,
                                          uint32_t t, uint32_t T)
{
#pragma unroll
    for (int q = 0; q < 16 / R; q++) {
        const uint32_t j = t + q * T;
        const uint32_t k = j & (Ns - 1);
        float2 v[R];
#pragma unroll
        for (int m = 0; m < R; m++) v[m] = src[swz(j + m * (N / R))];
        twiddle<R, INV>(v, tab, k, Ns);
        dft<R, INV>(v);
        const uint32_t base = (j - k) * R + k;
#pragma unroll
        for (int m = 0; m < R; m++) dst[LIN ? base + m * Ns : swz(base + m * Ns)] = v[m];
    }
}

// Lanes of this thread's group of G <= 32 threads (groups are aligned within the warp).
template <uint32_t G>
__device__ __forceinline__ uint32_t group_lanes()
{
    if constexpr (G >= 32)
        return 0xffffffffu;
    else
        return ((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(G - 1u));
}

// Barrier of G threads (aligned, contiguous): the CTA barrier when G is the whole CTA, named
// barrier `id` (1 .. 15: teams take 1 .. TEAMS, team pairs the ids after them) for several warps,
// a warp-level barrier for one warp or part of one.  The teams of a CTA only meet where
// they share data.
template <uint32_t G>
__device__ __forceinline__ void group_sync(uint32_t id)
{
    if constexpr (G >= kFastThreads)
        __syncthreads();
    else if constexpr (G > 32)
        asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(G) : "memory");
    else
        __syncwarp(group_lanes<G>());
}

// The same barrier, returning whether `pred` held in any of the G threads.
template <uint32_t G>
__device__ __forceinline__ bool group_sync_or(uint32_t id, bool pred)
{
    if constexpr (G >= kFastThreads) {
        return __syncthreads_or(pred) != 0;
    } else if constexpr (G > 32) {
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}"
            : "=r"(r)
            : "r"((uint32_t)pred), "r"(id), "n"(G)
            : "memory");
        return r != 0;
    } else {
        const uint32_t mask = group_lanes<G>();
        __syncwarp(mask);
        return __any_sync(mask, pred) != 0;
    }
}

// Passes 2 and 3 (Ns = 16, 256) of an N-point transform, src -> ... ; returns the result buffer,
// which holds the transform in natural (unswizzled) order.  The team synchronises between passes;
// the barrier after the last pass spans LASTG threads (id `last_id`), so that a partner team can
// read the result.
template <int LOGN, bool INV, uint32_t LASTG>
__device__ __forceinline__ float2 *fast_tail(float2 *a, float2 *b, const float2 *tab2, const float2 *tab3,
                                             uint32_t t, uint32_t team, uint32_t last_id)
{
    constexpr uint32_t N = 1u << LOGN, T = N / 16;
    constexpr int R3 = (int)(N / 256);
    fast_pass<16, INV, R3 == 1>(a, b, tab2, N, 16, t, T);
    if (R3 == 1) {
        group_sync<LASTG>(last_id);
        return b;
    }
    group_sync<T>(1 + team);
    fast_pass<(R3 > 1 ? R3 : 2), INV, true>(b, a, tab3, N, 256, t, T);
    group_sync<LASTG>(last_id);
    return a;
}

// With STG, each team's two input rows of the next work item are fetched by bulk copies into a
// staging buffer while the current item is transformed (one mbarrier per team, bounded waits),
// so the first pass reads shared memory instead of waiting on global loads; the host selects it
// for plain FP32 rows whose starts and lengths are 16-byte multiples when it costs no resident CTA.
template <int OUT, bool PRE, int LOGN, bool STG>
__global__ void __launch_bounds__(kFastThreads, 2) k_filter_fast(const RowSource src, uint32_t width, uint32_t rows,
                                                             const float2 *__restrict__ g_tab,
                                                             const float2 *__restrict__ g_gains,
                                                             void *__restrict__ out, uint32_t out_w,
                                                             uint32_t out_pitch, uint32_t npairs, uint32_t P,
                                                             int *__restrict__ err)
{
    constexpr uint32_t N = 1u << LOGN, T = N / 16, TEAMS = kFastThreads / T;
    constexpr uint32_t R3 = N / 256, LR3 = R3 >= 16 ? 4 : R3 >= 8 ? 3 : R3 >= 4 ? 2 : R3 >= 2 ? 1 : 0;
    constexpr uint32_t NTAB = 4 * 16 + LR3 * 256;
    static_assert(!(STG && PRE), "staged rows carry no preprocessing");
    extern __shared__ float4 smem_f4[];
    __shared__ uint64_t s_bar[TEAMS];
    float2 *sm = reinterpret_cast<float2 *>(smem_f4);
    float2 *tab2 = sm, *tab3 = sm + 64, *gains = sm + NTAB;
    const uint32_t team = threadIdx.x / T, t = threadIdx.x - team * T;
    float2 *bufA = gains + (N / 2 + 2) + team * 2 * N, *bufB = bufA + N;
    float *stg = reinterpret_cast<float *>(gains + (N / 2 + 2) + TEAMS * 2 * N) + team * 2 * N;
    for (uint32_t i = threadIdx.x; i < NTAB; i += kFastThreads) sm[i] = g_tab[i];
    for (uint32_t i = threadIdx.x; i <= N / 2; i += kFastThreads) gains[i] = g_gains[i];

    const uint32_t iters = (npairs + gridDim.x * TEAMS - 1) / (gridDim.x * TEAMS);
    const uint32_t wl = width < N ? width : N;  // samples read per row
    // leader of the team: expect and issue the rows of iteration i (nothing for a pair past the
    // end; a row past the stack is not copied and reads as zero)
    auto issue = [&](uint32_t i) {
        const uint32_t pr = (i * gridDim.x + blockIdx.x) * TEAMS + team;
        if (pr >= npairs) return;
        const PairMap mm = map_pair<OUT>(pr, rows, P, out_pitch);
        uint32_t y, p;
        mbar_arrive_expect_tx(&s_bar[team], ((mm.hasa ? 1u : 0u) + (mm.hasb ? 1u : 0u)) * wl * 4u);
        if (mm.hasa) bulk_load_1d(stg, row_start(src, mm.ra, y, p), wl * 4u, &s_bar[team]);
        if (mm.hasb) bulk_load_1d(stg + N, row_start(src, mm.rb, y, p), wl * 4u, &s_bar[team]);
    };
    if (STG && t == 0) {
        mbar_init(&s_bar[team], 1);
        fence_barrier_init();
    }
    __syncthreads();  // tables, gains and barriers are ready; from here on the teams meet only in
                      // pairs, where a quad output cell takes both teams' results
    if (STG && t == 0 && iters > 0) issue(0);
    // the cell store of the slice-quad output reads the partner team's result
    constexpr bool CELLS = OUT == OUT_F16_QUADS && TEAMS % 2 == 0;
    static_assert(2 * T <= 32 || TEAMS + TEAMS / 2 <= 15, "named barrier ids 1 .. 15");
    constexpr uint32_t SG = CELLS ? 2 * T : T;  // threads that share a result buffer
    const uint32_t sid = CELLS ? 1 + TEAMS + (team >> 1) : 1 + team;
    for (uint32_t it = 0; it < iters; it++) {
        const uint32_t pair = (it * gridDim.x + blockIdx.x) * TEAMS + team;
        const bool live = pair < npairs;
        const PairMap m = map_pair<OUT>(live ? pair : 0, live ? rows : 0, P, out_pitch);
        // pass 1 loads elements t + m N/16 of rows a, b (staged, or straight from global memory)
        float2 v[16];
        bool failed = false;
        if (STG) {
            // live pairs come first in every team, so the barrier's phase is the iteration's parity
            if (live && !mbar_wait_bounded(&s_bar[team], it & 1u, kWaitLimitNs)) failed = true;
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const uint32_t n = t + q * T;
                const bool in = n < wl;
                v[q] = make_float2(in && m.hasa ? stg[n] : 0.f, in && m.hasb ? stg[N + n] : 0.f);
            }
        } else {
            uint32_t ya, pa_, yb, pb_;
            const float *ra = row_start(src, m.hasa ? m.ra : 0, ya, pa_);
            const float *rb = row_start(src, m.hasb ? m.rb : 0, yb, pb_);
            if (!PRE) {
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const uint32_t n = t + q * T;
                    float a = 0.f, b = 0.f;
                    if (n < width) {
                        if (m.hasa) a = __ldg(ra + n);
                        if (m.hasb) b = __ldg(rb + n);
                    }
                    v[q] = make_float2(a, b);
                }
            } else {
                // every load of a half (data, dark, flat) is issued before the dependent divisions
                // and logarithms; rows past the stack read row 0 and are zeroed afterwards
                const float *da = src.dark ? src.dark + (size_t)ya * src.corr_pitch : nullptr;
                const float *fa = src.dark ? src.flat + (size_t)ya * src.corr_pitch : nullptr;
                const float *db = src.dark ? src.dark + (size_t)yb * src.corr_pitch : nullptr;
                const float *fb = src.dark ? src.flat + (size_t)yb * src.corr_pitch : nullptr;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float xa[8], xb[8], dka[8], fla[8], dkb[8], flb[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const uint32_t n = t + (8 * h + i) * T;
                        const uint32_t nn = n < width ? n : 0;
                        xa[i] = __ldg(ra + nn);
                        xb[i] = __ldg(rb + nn);
                        if (src.dark) {
                            dka[i] = __ldg(da + nn);
                            fla[i] = __ldg(fa + nn);
                            dkb[i] = __ldg(db + nn);
                            flb[i] = __ldg(fb + nn);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const uint32_t n = t + (8 * h + i) * T;
                        float a = xa[i], b = xb[i];
                        if (src.dark) {
                            a = ffc_value(src, a, dka[i], fla[i]);
                            b = ffc_value(src, b, dkb[i], flb[i]);
                        }
                        if (src.cone) {
                            a = preprocess_value(src.cone_only(), a, n, ya, pa_);
                            b = preprocess_value(src.cone_only(), b, n, yb, pb_);
                        }
                        const bool in = n < width;
                        v[8 * h + i] = make_float2(in && m.hasa ? a : 0.f, in && m.hasb ? b : 0.f);
                    }
                }
            }
        }
        // the previous item's output reads (the partner team's too, for quad cells) and this item's
        // staged reads are done; teams that share buffers leave together on a failed wait
        if (STG) {
            if (group_sync_or<SG>(sid, failed)) {
                if (t == 0) {
                    atomicExch(err, kErrTmaTimeout);
                    mbar_wait_bounded(&s_bar[team], it & 1u, kWaitLimitNs);  // the copy in flight
                }
                return;
            }
            if (t == 0 && it + 1 < iters) issue(it + 1);
        } else {
            group_sync<SG>(sid);
        }
        dft<16, false>(v);
#pragma unroll
        for (int q = 0; q < 16; q++) bufA[swz(t * 16 + q)] = v[q];
        group_sync<T>(1 + team);
        const float2 *Z = fast_tail<LOGN, false, T>(bufA, bufB, tab2, tab3, t, team, 1 + team);
        float2 *O = (Z == bufA) ? bufB : bufA;
        // separate the two rows' spectra, apply the gains, recombine (element e = t + q N/16)
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const uint32_t e = t + q * T;
            const bool lower = e <= N / 2;
            const uint32_t k = lower ? e : N - e;
            const float2 zk = Z[k], zm = Z[(N - k) & (N - 1)], g = gains[k];
            // a = (zk + conj zm) / 2, b = (zk - conj zm) / 2i are the two rows' spectra at k; with
            // (hx, hy) = g / 2 and S = zk + zm, D = zk - zm, the filtered recombination is
            // (S.x hx + D.x hy, S.y hx + D.y hy) at e <= N/2 and (S.x hx - D.x hy, S.y hx - D.y hy)
            // above: one packed product and one packed FMA (D negated exactly for the upper half)
            const float2 S = cadd(zk, zm), D = lower ? csub(zk, zm) : csub(zm, zk);
            float hx, hy;
            f2unpack(f2mul(f2pack(g.x, g.y), f2pack(0.5f, 0.5f)), hx, hy);
            const uint64_t ab = f2mul(f2pack(S.x, S.y), f2pack(hx, hx));
            f2unpack(f2fma(f2pack(D.x, D.y), f2pack(hy, hy), ab), v[q].x, v[q].y);
        }
        dft<16, true>(v);
#pragma unroll
        for (int q = 0; q < 16; q++) O[swz(t * 16 + q)] = v[q];
        group_sync<T>(1 + team);
        const float2 *X = fast_tail<LOGN, true, SG>(O, O == bufA ? bufB : bufA, tab2, tab3, t, team, sid);
        if constexpr (CELLS) {
            // teams 2u and 2u + 1 hold the two halves (slices 4g, 4g+1 and 4g+2, 4g+3 at one angle)
            // of the same cells, and the barrier that ended the transform made both results visible:
            // the pair's 2T threads write whole 16-byte cells, consecutive across threads
            if (live) {
                const uint32_t u = team >> 1, i0 = threadIdx.x - u * 2 * T;
                const uint32_t pair0 = pair - (team & 1u);
                const PairMap m0 = map_pair<OUT>(pair0, rows, P, out_pitch);
                const PairMap m1 = map_pair<OUT>(pair0 + 1, rows, P, out_pitch);
                const size_t xoff = (size_t)(X - bufA);  // this team's result: bufA or bufB
                const float2 *X0 = gains + (N / 2 + 2) + (size_t)(2 * u) * 2 * N + xoff;
                const float2 *X1 = X0 + 2 * N;
                uint4 *o = reinterpret_cast<uint4 *>(out) + m0.cell0;
                auto taps = [&](const float2 *Xh, const PairMap &mh, uint32_t j, bool prev) {
                    const uint32_t e = prev ? j - 1 : j;
                    float2 v = ((!prev || j >= 1) && e < out_w) ? Xh[e] : make_float2(0.f, 0.f);
                    if (!mh.hasa) v.x = 0.f;  // slices past the stack: exact zeros, not FFT round-off
                    if (!mh.hasb) v.y = 0.f;
                    return pack_pair<OUT>(v.x, v.y);
                };
                for (uint32_t j = i0; j < out_pitch; j += 2 * T)
                    o[j] = make_uint4(taps(X0, m0, j, true), taps(X1, m1, j, true), taps(X0, m0, j, false),
                                      taps(X1, m1, j, false));
            }
        } else {
            if (live) store_pair<OUT>(m, [X](uint32_t i) { return X[i]; }, out, out_w, out_pitch, t, T);
        }
    }
}

// Persistent filter stage of an uneven batch: work items (job, row pair) are
// grouped by FFT width and taken from a device counter; a CTA reloads its
// shared twiddles/gains only when the width changes between its items.
template <int OUT>
__global__ void __launch_bounds__(kFilterThreads) k_filter_batch(const BatchFilter *__restrict__ jobs,
                                                                 const uint2 *__restrict__ items, uint32_t n_items,
                                                                 uint32_t maxN, uint32_t *__restrict__ counter)
{
    extern __shared__ float4 smem_f4[];
    float2 *bufA = reinterpret_cast<float2 *>(smem_f4);
    float2 *bufB = bufA + maxN;
    float2 *tw = bufB + maxN;
    float2 *gains = tw + maxN;
    __shared__ uint32_t s_item;
    const float2 *loaded = nullptr;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= n_items) break;
        const uint2 w = items[it];  // (job, row pair)
        const BatchFilter &j = jobs[w.x];
        if (j.tw != loaded) {
            for (uint32_t i = threadIdx.x; i < j.N; i += blockDim.x) tw[i] = j.tw[i];
            for (uint32_t i = threadIdx.x; i <= j.N / 2; i += blockDim.x) gains[i] = j.gains[i];
            loaded = j.tw;
        }
        filter_pair<OUT, false>(plain_rows(j.in, j.in_pitch), j.width, j.rows, w.y, bufA, bufB, tw, gains, j.N,
                                j.log2N, j.out, j.out_w, j.out_pitch);
    }
}

template <int OUT, bool PRE>
static ufob_status launch_rows_t(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t rows,
                                 void *d_out, uint32_t out_w, uint32_t out_pitch, cudaStream_t s, uint32_t P)
{
    const uint32_t N = plan.nfft;
    const size_t smem = sizeof(float2) * (3 * (size_t)N + N / 2 + 1);
    auto kern = k_filter_rows<OUT, PRE>;
    static std::atomic<uint64_t> attr_devs{0};
    UFOB_CUDA_TRY(smem_limit_per_device(
        kern, (int)(sizeof(float2) * (3 * (size_t)kMaxFusedFFT + kMaxFusedFFT / 2 + 1)), attr_devs));
    const int log2N = ilog2(N);
    int per_sm = 0;
    UFOB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFilterThreads, smem));
    if (per_sm < 1) return fail(UFOB_ERR_UNSUPPORTED, "filter: FFT width %u does not fit in shared memory", N);
    // slice-quad layout: two items per (group of four slices, angle)
    const uint32_t npairs = OUT == OUT_F16_QUADS ? (rows / P + 3) / 4 * P * 2 : (rows + 1) / 2;
    uint32_t grid = (uint32_t)num_sms() * (uint32_t)per_sm * 4;
    if (grid > npairs) grid = npairs;
    if (grid == 0) return UFOB_OK;
    kern<<<grid, kFilterThreads, smem, s>>>(src, width, rows, plan.d_twiddle.as<float2>(), plan.d_gains.as<float2>(),
                                            N, log2N, d_out, out_w, out_pitch, npairs, P);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

// Shared memory of k_filter_fast: pass twiddles, gains, two exchange buffers per team and, when
// rows are staged, two input rows per team.
template <int LOGN, bool STG>
static size_t fast_smem()
{
    constexpr uint32_t N = 1u << LOGN, TEAMS = kFastThreads / (N / 16);
    return sizeof(float2) * (pass_twiddle_count(N) + N / 2 + 2 + (size_t)TEAMS * 2 * N) +
           (STG ? sizeof(float) * TEAMS * 2 * N : 0);
}

template <int OUT, bool PRE, int LOGN, bool STG>
static ufob_status fast_occupancy(int &per_sm)
{
    auto kern = k_filter_fast<OUT, PRE, LOGN, STG>;
    static std::atomic<uint64_t> attr_devs{0};
    UFOB_CUDA_TRY(smem_limit_per_device(kern, (int)fast_smem<LOGN, STG>(), attr_devs));
    UFOB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFastThreads, fast_smem<LOGN, STG>()));
    return UFOB_OK;
}

// Bulk copies need 16-byte aligned row starts and lengths.
static bool rows_stageable(const RowSource &src, uint32_t width, uint32_t N)
{
    const uint32_t wl = std::min(width, N);
    return !src.has_pre() && wl % 4 == 0 && ((uintptr_t)src.base & 15u) == 0 && src.outer_stride % 4 == 0 &&
           src.inner_stride % 4 == 0;
}

template <int OUT, bool PRE, int LOGN>
static ufob_status launch_fast_t(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t rows,
                                 void *d_out, uint32_t out_w, uint32_t out_pitch, cudaStream_t s, uint32_t P)
{
    constexpr uint32_t N = 1u << LOGN, TEAMS = kFastThreads / (N / 16);
    int per_sm = 0, per_sm_stg = 0;
    UFOB_TRY((fast_occupancy<OUT, PRE, LOGN, false>(per_sm)));
    if (per_sm < 1) return fail(UFOB_ERR_UNSUPPORTED, "filter: FFT width %u does not fit in shared memory", N);
    // stage the rows only where the staging buffers cost no resident CTA
    bool stg = !PRE && rows_stageable(src, width, N);
    if (stg) {
        UFOB_TRY((fast_occupancy<OUT, false, LOGN, true>(per_sm_stg)));
        stg = per_sm_stg >= per_sm;
    }
    const uint32_t npairs = OUT == OUT_F16_QUADS ? (rows / P + 3) / 4 * P * 2 : (rows + 1) / 2;
    uint32_t grid = (uint32_t)num_sms() * (uint32_t)per_sm;
    grid = std::min(grid, (npairs + TEAMS - 1) / TEAMS);
    if (grid == 0) return UFOB_OK;
    const float2 *tab = plan.d_pass_tw.as<float2>(), *gains = plan.d_gains.as<float2>();
    if (stg)
        k_filter_fast<OUT, false, LOGN, true><<<grid, kFastThreads, fast_smem<LOGN, true>(), s>>>(
            src, width, rows, tab, gains, d_out, out_w, out_pitch, npairs, P, device_error_word());
    else
        k_filter_fast<OUT, PRE, LOGN, false><<<grid, kFastThreads, fast_smem<LOGN, false>(), s>>>(
            src, width, rows, tab, gains, d_out, out_w, out_pitch, npairs, P, device_error_word());
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

template <int OUT, bool PRE>
static ufob_status launch_rows_p(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t rows,
                                 void *d_out, uint32_t out_w, uint32_t out_pitch, cudaStream_t s, uint32_t P)
{
    if (fast_filter_enabled()) switch (plan.nfft) {
        case 256: return launch_fast_t<OUT, PRE, 8>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
        case 512: return launch_fast_t<OUT, PRE, 9>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
        case 1024: return launch_fast_t<OUT, PRE, 10>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
        case 2048: return launch_fast_t<OUT, PRE, 11>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
        case 4096: return launch_fast_t<OUT, PRE, 12>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
        default: break;
        }
    return launch_rows_t<OUT, PRE>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
}

template <int OUT>
static ufob_status launch_rows(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t rows,
                               void *d_out, uint32_t out_w, uint32_t out_pitch, cudaStream_t s, uint32_t P = 0)
{
    if (src.has_pre()) return launch_rows_p<OUT, true>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
    return launch_rows_p<OUT, false>(plan, src, width, rows, d_out, out_w, out_pitch, s, P);
}

ufob_status filter_rows_launch_src(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t rows,
                                   void *d_out, ufob_dtype out_dtype, ufob_layout out_layout, uint32_t out_w,
                                   uint32_t out_pitch, cudaStream_t stream)
{
    const uint32_t N = plan.nfft;
    if (N > kMaxFusedFFT || N < 4)
        return fail(UFOB_ERR_UNSUPPORTED, "filter: FFT width %u outside the supported range [4, %u]", N, kMaxFusedFFT);
    if (width > N) return fail(UFOB_ERR_INVALID, "filter: input width %u exceeds FFT width %u", width, N);
    if (out_w > N) return fail(UFOB_ERR_INVALID, "filter: crop width %u exceeds FFT width %u", out_w, N);
    if (out_layout == UFOB_LAYOUT_PAIRS) {
        if (out_pitch < out_w + 1) return fail(UFOB_ERR_INVALID, "filter: pair pitch %u < crop width + 1", out_pitch);
        if (out_dtype == UFOB_F16) return launch_rows<OUT_F16_PAIRS>(plan, src, width, rows, d_out, out_w, out_pitch, stream);
        if (out_dtype == UFOB_BF16) return launch_rows<OUT_BF16_PAIRS>(plan, src, width, rows, d_out, out_w, out_pitch, stream);
        return fail(UFOB_ERR_INVALID, "filter: the pair layout needs F16 or BF16 output");
    }
    if (out_pitch < out_w) return fail(UFOB_ERR_INVALID, "filter: output pitch %u < crop width %u", out_pitch, out_w);
    switch (out_dtype) {
    case UFOB_F32: return launch_rows<OUT_F32>(plan, src, width, rows, d_out, out_w, out_pitch, stream);
    case UFOB_F16: return launch_rows<OUT_F16>(plan, src, width, rows, d_out, out_w, out_pitch, stream);
    case UFOB_BF16: return launch_rows<OUT_BF16>(plan, src, width, rows, d_out, out_w, out_pitch, stream);
    default: return fail(UFOB_ERR_INVALID, "filter: unsupported output dtype %d", (int)out_dtype);
    }
}

ufob_status filter_rows_launch(const FilterPlan &plan, const float *d_in, uint32_t width, uint32_t rows,
                               uint32_t in_pitch, void *d_out, ufob_dtype out_dtype, ufob_layout out_layout,
                               uint32_t out_w, uint32_t out_pitch, cudaStream_t stream)
{
    if (in_pitch < width) return fail(UFOB_ERR_INVALID, "filter: input pitch %u < width %u", in_pitch, width);
    return filter_rows_launch_src(plan, plain_rows(d_in, in_pitch), width, rows, d_out, out_dtype, out_layout, out_w,
                                  out_pitch, stream);
}

// Filter a stack of `nz` sinograms of P rows into the slice-quad FP16 layout
// ([ceil(nz/4)][P][out_pitch] cells of 16 bytes; see backproject.cu).
ufob_status filter_quads_launch_src(const FilterPlan &plan, const RowSource &src, uint32_t width, uint32_t P,
                                    uint32_t nz, void *d_out, uint32_t out_w, uint32_t out_pitch,
                                    cudaStream_t stream)
{
    const uint32_t N = plan.nfft;
    if (N > kMaxFusedFFT || N < 4)
        return fail(UFOB_ERR_UNSUPPORTED, "filter: FFT width %u outside the supported range [4, %u]", N, kMaxFusedFFT);
    if (width > N || out_w > N || out_pitch < out_w + 1 || !P)
        return fail(UFOB_ERR_INVALID, "filter: bad slice-quad sizes (width %u, N %u, crop %u, pitch %u)", width, N,
                    out_w, out_pitch);
    return launch_rows<OUT_F16_QUADS>(plan, src, width, P * nz, d_out, out_w, out_pitch, stream, P);
}

ufob_status filter_quads_launch(const FilterPlan &plan, const float *d_in, uint32_t width, uint32_t P, uint32_t nz,
                                uint32_t in_pitch, void *d_out, uint32_t out_w, uint32_t out_pitch,
                                cudaStream_t stream)
{
    if (in_pitch < width) return fail(UFOB_ERR_INVALID, "filter: input pitch %u < width %u", in_pitch, width);
    return filter_quads_launch_src(plan, plain_rows(d_in, in_pitch), width, P, nz, d_out, out_w, out_pitch, stream);
}

// The reference `filter` kernel alone (filter.cl:20-29): out[y][x] = in[y][x] * coeff[x].
__global__ void k_filter_spectrum(const float *__restrict__ coeff, const float *__restrict__ in,
                                  float *__restrict__ out, uint32_t width2, uint32_t rows)
{
    size_t n = (size_t)width2 * rows;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = in[i] * __ldg(coeff + (i % width2));
}

ufob_status filter_spectrum_launch(const float *d_coeff, const float *d_in, float *d_out, uint32_t width2,
                                   uint32_t rows, cudaStream_t stream)
{
    size_t n = (size_t)width2 * rows;
    if (!n) return UFOB_OK;
    uint32_t grid = (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)num_sms() * 16);
    k_filter_spectrum<<<grid, 256, 0, stream>>>(d_coeff, d_in, d_out, width2, rows);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

template <int OUT>
static ufob_status launch_batch(const BatchFilter *d_jobs, const uint2 *d_items, uint32_t n_items, uint32_t maxN,
                                uint32_t *d_counter, cudaStream_t s)
{
    const size_t smem = sizeof(float2) * (3 * (size_t)maxN + maxN / 2 + 1);
    UFOB_CUDA_TRY(cudaFuncSetAttribute(k_filter_batch<OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    UFOB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_filter_batch<OUT>, kFilterThreads, smem));
    if (per_sm < 1) return fail(UFOB_ERR_UNSUPPORTED, "filter: FFT width %u does not fit in shared memory", maxN);
    uint32_t grid = std::min<uint32_t>((uint32_t)num_sms() * (uint32_t)per_sm, n_items);
    if (!grid) return UFOB_OK;
    k_filter_batch<OUT><<<grid, kFilterThreads, smem, s>>>(d_jobs, d_items, n_items, maxN, d_counter);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

ufob_status filter_batch_launch(const BatchFilter *d_jobs, const uint2 *d_items, uint32_t n_items, uint32_t maxN,
                                uint32_t *d_counter, int out_kind, cudaStream_t s)
{
    if (maxN > kMaxFusedFFT) return fail(UFOB_ERR_UNSUPPORTED, "filter: FFT width %u above %u", maxN, kMaxFusedFFT);
    switch (out_kind) {
    case OUT_F32: return launch_batch<OUT_F32>(d_jobs, d_items, n_items, maxN, d_counter, s);
    case OUT_F16_PAIRS: return launch_batch<OUT_F16_PAIRS>(d_jobs, d_items, n_items, maxN, d_counter, s);
    case OUT_BF16_PAIRS: return launch_batch<OUT_BF16_PAIRS>(d_jobs, d_items, n_items, maxN, d_counter, s);
    default: return fail(UFOB_ERR_INVALID, "filter batch: unsupported output kind %d", out_kind);
    }
}

}  // namespace ufob
