// 3x3 convolutions for the sparse-view correction network on the 5th-gen
// tensor cores (tcgen05): BF16 operands, FP32 accumulation in tensor memory.
//
// Layouts: activations NHWC bf16 with C a multiple of 16; forward weights
// [Cout][9][Cin] bf16 (tap t = 3*(dy+1) + (dx+1)).
//
// Forward (and data-gradient) convolution as an implicit GEMM:
//   D[p][co] = sum_{t, ci} A[p][(t, ci)] * B[co][(t, ci)]
//   A[p][(t, ci)] = in[p shifted by tap t][ci] (zero outside the image),
// M = 128 consecutive pixels per CTA, N = Cout (the whole output width,
// <= 256 TMEM columns), K walked tap by tap in chunks of <= 64 channels.  The
// data gradient is the same GEMM on the output gradient with the weights
// transposed and tap-flipped ([Cin][9][Cout], t -> 8 - t).
// Weight gradient: dW[co][t][ci] = sum_p dZ[p][co] * in[p + off(t)][ci], a GEMM
// with M = 128 output channels (zero-padded), N = Cin, K = pixels, fed from the
// NHWC tensors as MN-major operands; each CTA reduces a pixel range and adds
// its tile to the FP32 gradient with atomics.
//
// Operand tiles are staged by the CTA's threads into the canonical
// no-swizzle core-matrix layout (8 rows x 16 bytes per core matrix) and made
// visible to the tensor core with fence.proxy.async; one thread issues
// tcgen05.mma (M=128, N=Cout, K=16 per instruction) and tcgen05.commit arrives
// on an mbarrier per shared-memory stage (two stages), so loads of the next K
// chunk overlap the running MMAs.  The epilogue reads the accumulators with
// tcgen05.ld (32 lanes x 32 bit, 8 columns at a time), one pixel per thread.
// Descriptor encodings follow the SM100 UMMA shared-memory and instruction
// descriptor formats (start address>>4, leading/stride byte offsets>>4,
// version 1, no swizzle; c=F32, a=b=BF16, N>>3, M>>4, K- or MN-major bits).
#include <cuda_bf16.h>

#include "ufob_internal.h"

namespace ufob {

// ------------------------------------------------------------------ tcgen05 / mbarrier helpers

__device__ __forceinline__ uint32_t cvta_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cnn_mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(cvta_smem(bar)) : "memory");
}

// Bounded wait (2 s); the timer is read only every 256 polls so that its
// latency does not delay noticing the phase flip.
__device__ __forceinline__ bool cnn_mbar_wait(uint64_t *bar, uint32_t parity)
{
    uint64_t t0 = 0;
    for (uint32_t i = 1;; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(cvta_smem(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 255u) == 0) {
            uint64_t t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (!t0)
                t0 = t;
            else if (t - t0 > 2000000000ull)
                return false;
        }
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(cvta_smem(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version
    return d;
}

// Instruction descriptor of kind::f16: D = F32, A = B = BF16, M x N, majorness bits.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N, uint32_t a_mn_major, uint32_t b_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn_major << 15) | (b_mn_major << 16) | ((N >> 3) << 17) |
           ((M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(cvta_smem(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

static constexpr int kErrConvTimeout = 0x2001;

// ------------------------------------------------------------------ forward / data-gradient conv

struct ConvArgs {
    const __nv_bfloat16 *in;  // [NB][H][W][Cin]
    const __nv_bfloat16 *w;   // [Cout][9][Cin]
    const float *bias;        // [Cout] or null
    const __nv_bfloat16 *residual;  // [NB][H][W][Cout] added after the activation, or null
    __nv_bfloat16 *out;       // [NB][H][W][Cout] or null
    float *out_f32;           // [NB][H][W][Cout] or null
    int NB, H, W, Cin, Cout, relu;
    int *err;
};

// Core-matrix (8 rows x 16 B) no-swizzle K-major layout of a rows x BK tile:
// chunk k (8 bf16 along K) of row r at  k*LBO + (r/8)*128 + (r%8)*16.
__global__ void __launch_bounds__(128) k_conv3x3(const ConvArgs a)
{
    constexpr int BK = 64;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Cin = a.Cin, Cout = a.Cout;
    const int bk = Cin < BK ? Cin : BK;  // channels per K chunk (multiple of 16)
    const int kchunks = bk / 8;
    const uint32_t A_BYTES = 128 * BK * 2, B_BYTES = 256 * BK * 2;
    unsigned char *sA[2] = {smem, smem + A_BYTES + B_BYTES};
    unsigned char *sB[2] = {smem + A_BYTES, smem + 2 * A_BYTES + B_BYTES};
    const uint32_t lboA = 16 * 128, lboB = (uint32_t)(Cout / 8) * 128;
    const uint32_t ncols = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : (Cout <= 128 ? 128 : 256));

    if (warp == 0) tmem_alloc(&tslot, ncols);
    if (tid == 0) {
        cnn_mbar_init(&bars[0]);
        cnn_mbar_init(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;

    const long long npix = (long long)a.NB * a.H * a.W;
    const long long p = (long long)blockIdx.x * 128 + tid;  // this thread's pixel for loading and output
    int pb = 0, py = 0, px = 0;
    const bool pvalid = p < npix;
    if (pvalid) {
        px = (int)(p % a.W);
        py = (int)((p / a.W) % a.H);
        pb = (int)(p / ((long long)a.W * a.H));
    }
    const uint32_t idesc = idesc_bf16(128, (uint32_t)Cout, 0, 0);
    const int cblocks = Cin / bk;
    const int nk = 9 * cblocks;
    bool ok = true;
    for (int i = 0; i < nk && ok; i++) {
        const int st = i & 1;
        if (i >= 2) ok = cnn_mbar_wait(&bars[st], (uint32_t)(((i - 2) >> 1) & 1));  // MMAs of chunk i-2 done
        const int t = i / cblocks, c0 = (i % cblocks) * bk;
        const int dy = t / 3 - 1, dx = t % 3 - 1;
        // A: this thread's pixel, shifted by the tap, bk channels
        {
            const int yy = py + dy, xx = px + dx;
            const bool in = pvalid && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
            const uint4 *src =
                reinterpret_cast<const uint4 *>(a.in + ((((size_t)pb * a.H + yy) * a.W + xx) * Cin + c0));
            for (int k = 0; k < kchunks; k++) {
                uint4 v = in ? __ldg(src + k) : make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4 *>(sA[st] + k * lboA + (tid >> 3) * 128 + (tid & 7) * 16) = v;
            }
        }
        // B: Cout rows x bk channels of tap t
        for (int idx = tid; idx < Cout * kchunks; idx += 128) {
            const int row = idx / kchunks, k = idx % kchunks;
            const uint4 v = __ldg(reinterpret_cast<const uint4 *>(a.w + ((size_t)row * 9 + t) * Cin + c0) + k);
            *reinterpret_cast<uint4 *>(sB[st] + k * lboB + (row >> 3) * 128 + (row & 7) * 16) = v;
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = cvta_smem(sA[st]), b0 = cvta_smem(sB[st]);
            for (int s = 0; s < bk / 16; s++)
                umma_bf16(tmem, smem_desc(a0 + s * 2 * lboA, lboA, 128), smem_desc(b0 + s * 2 * lboB, lboB, 128),
                          idesc, (i > 0 || s > 0) ? 1u : 0u);
            umma_commit(&bars[st]);
        }
    }
    // the last chunk's commit covers every earlier MMA of this thread
    if (ok) ok = cnn_mbar_wait(&bars[(nk - 1) & 1], (uint32_t)(((nk - 1) >> 1) & 1));
    tc_fence_after();
    if (!ok) {
        if (tid == 0) atomicExch(a.err, kErrConvTimeout);
    } else {
        // epilogue: warp w owns TMEM lanes (pixels) 32w .. 32w+31
        const long long q = (long long)blockIdx.x * 128 + warp * 32 + lane;
        for (int c = 0; c < Cout; c += 8) {
            float v[8];
            tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            if (q < npix) {
                if (a.bias)
#pragma unroll
                    for (int j = 0; j < 8; j++) v[j] += a.bias[c + j];
                if (a.relu)
#pragma unroll
                    for (int j = 0; j < 8; j++) v[j] = fmaxf(v[j], 0.f);
                if (a.residual) {
                    const uint4 r = *reinterpret_cast<const uint4 *>(a.residual + q * Cout + c);
                    const __nv_bfloat162 *rh = reinterpret_cast<const __nv_bfloat162 *>(&r);
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float2 f = __bfloat1622float2(rh[j]);
                        v[2 * j] += f.x;
                        v[2 * j + 1] += f.y;
                    }
                }
                if (a.out) {
                    uint4 o;
                    __nv_bfloat162 *oh = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
                    for (int j = 0; j < 4; j++) oh[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    *reinterpret_cast<uint4 *>(a.out + q * Cout + c) = o;
                }
                if (a.out_f32)
#pragma unroll
                    for (int j = 0; j < 8; j++) a.out_f32[q * Cout + c + j] = v[j];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ------------------------------------------------------------------ weight gradient

struct WgradArgs {
    const __nv_bfloat16 *in;  // [NB][H][W][Cin]   (layer input)
    const __nv_bfloat16 *dz;  // [NB][H][W][Cout]  (gradient at the pre-activation)
    float *dw;                // [Cout][9][Cin] FP32, accumulated with atomics
    int NB, H, W, Cin, Cout;
    long long pix_per_cta;    // K range of one CTA (multiple of 64)
    int *err;
};

// MN-major no-swizzle layout of an R x 64 (rows x K) tile fed from NHWC data:
// the 16-byte chunk of rows 8g..8g+7 at K index k sits at g*128 + (k/8)*LBO + (k%8)*16.
__global__ void __launch_bounds__(128) k_conv3x3_wgrad(const WgradArgs a)
{
    constexpr int BK = 64;  // pixels per K chunk
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t = blockIdx.y, mt = blockIdx.z;  // tap, output-channel tile
    const int dy = t / 3 - 1, dx = t % 3 - 1;
    const int Cin = a.Cin, Cout = a.Cout;
    const uint32_t A_BYTES = 128 * BK * 2, B_BYTES = 256 * BK * 2;
    unsigned char *sA[2] = {smem, smem + A_BYTES + B_BYTES};
    unsigned char *sB[2] = {smem + A_BYTES, smem + 2 * A_BYTES + B_BYTES};
    const uint32_t lboA = 16 * 128, lboB = (uint32_t)(Cin / 8) * 128;  // K-group strides
    const uint32_t ncols = Cin <= 32 ? 32 : (Cin <= 64 ? 64 : (Cin <= 128 ? 128 : 256));
    const int co0 = mt * 128;
    const int mvalid = min(128, Cout - co0);

    if (warp == 0) tmem_alloc(&tslot, ncols);
    if (tid == 0) {
        cnn_mbar_init(&bars[0]);
        cnn_mbar_init(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // rows co >= Cout of the A tiles stay zero for the whole kernel
    for (int i = tid; i < (int)(2 * (A_BYTES + B_BYTES) / 16); i += 128)
        reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;

    const long long npix = (long long)a.NB * a.H * a.W;
    const long long p_begin = (long long)blockIdx.x * a.pix_per_cta;
    const long long p_end = min(npix, p_begin + a.pix_per_cta);
    const int nk = p_end > p_begin ? (int)((p_end - p_begin + BK - 1) / BK) : 0;
    const uint32_t idesc = idesc_bf16(128, (uint32_t)Cin, 1, 1);
    const int ca = mvalid / 8, cb = Cin / 8;  // 16-byte chunks per pixel for A and B
    bool ok = true;
    for (int i = 0; i < nk && ok; i++) {
        const int st = i & 1;
        if (i >= 2) ok = cnn_mbar_wait(&bars[st], (uint32_t)(((i - 2) >> 1) & 1));
        const long long pk0 = p_begin + (long long)i * BK;
        // A: dz[p][co0 .. co0+mvalid) for the 64 pixels of the chunk
        for (int idx = tid; idx < BK * ca; idx += 128) {
            const int k = idx / ca, g = idx % ca;
            const long long p = pk0 + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < p_end) v = __ldg(reinterpret_cast<const uint4 *>(a.dz + p * Cout + co0) + g);
            *reinterpret_cast<uint4 *>(sA[st] + g * 128 + (k >> 3) * lboA + (k & 7) * 16) = v;
        }
        // B: in[p + off(t)][0 .. Cin)
        for (int idx = tid; idx < BK * cb; idx += 128) {
            const int k = idx / cb, g = idx % cb;
            const long long p = pk0 + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < p_end) {
                const int x = (int)(p % a.W), y = (int)((p / a.W) % a.H);
                const long long b = p / ((long long)a.W * a.H);
                const int yy = y + dy, xx = x + dx;
                if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
                    v = __ldg(reinterpret_cast<const uint4 *>(a.in + (((b * a.H + yy) * a.W + xx) * Cin)) + g);
            }
            *reinterpret_cast<uint4 *>(sB[st] + g * 128 + (k >> 3) * lboB + (k & 7) * 16) = v;
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = cvta_smem(sA[st]), b0 = cvta_smem(sB[st]);
            // MN-major: leading offset = K-group stride, stride offset = 8-row group stride
            for (int s = 0; s < BK / 16; s++)
                umma_bf16(tmem, smem_desc(a0 + s * 2 * lboA, lboA, 128), smem_desc(b0 + s * 2 * lboB, lboB, 128),
                          idesc, (i > 0 || s > 0) ? 1u : 0u);
            umma_commit(&bars[st]);
        }
    }
    if (nk > 0 && ok) ok = cnn_mbar_wait(&bars[(nk - 1) & 1], (uint32_t)(((nk - 1) >> 1) & 1));
    tc_fence_after();
    if (!ok) {
        if (tid == 0) atomicExch(a.err, kErrConvTimeout);
    } else if (nk > 0) {
        const int co = co0 + warp * 32 + lane;  // TMEM lane = output channel
        for (int c = 0; c < Cin; c += 8) {
            float v[8];
            tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
            if (co < Cout)
#pragma unroll
                for (int j = 0; j < 8; j++) atomicAdd(a.dw + ((size_t)co * 9 + t) * Cin + c + j, v[j]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ------------------------------------------------------------------ host launchers

static size_t conv_smem_bytes() { return 2 * (128 * 64 * 2 + 256 * 64 * 2); }

ufob_status conv3x3_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                           const __nv_bfloat16 *residual, __nv_bfloat16 *out, float *out_f32, int NB, int H, int W,
                           int Cin, int Cout, int relu, cudaStream_t s)
{
    if (Cin % 16 || Cout % 16 || Cin < 16 || Cout < 16 || Cin > 256 || Cout > 256 || (Cin > 64 && Cin % 64))
        return fail(UFOB_ERR_INVALID, "conv3x3: channels must be multiples of 16 in [16, 256] (Cin > 64: of 64)");
    static std::atomic<uint64_t> attr_devs{0};
    UFOB_CUDA_TRY(smem_limit_per_device(k_conv3x3, (int)conv_smem_bytes(), attr_devs));
    ConvArgs a;
    a.in = in;
    a.w = w;
    a.bias = bias;
    a.residual = residual;
    a.out = out;
    a.out_f32 = out_f32;
    a.NB = NB;
    a.H = H;
    a.W = W;
    a.Cin = Cin;
    a.Cout = Cout;
    a.relu = relu;
    a.err = device_error_word();
    const long long npix = (long long)NB * H * W;
    const unsigned grid = (unsigned)((npix + 127) / 128);
    k_conv3x3<<<grid, 128, conv_smem_bytes(), s>>>(a);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

ufob_status conv3x3_wgrad_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *dz, float *dw, int NB, int H, int W,
                                 int Cin, int Cout, cudaStream_t s)
{
    if (Cin % 16 || Cout % 16 || Cin < 16 || Cout < 16 || Cin > 256 || Cout > 256)
        return fail(UFOB_ERR_INVALID, "conv3x3 wgrad: channels must be multiples of 16 in [16, 256]");
    static std::atomic<uint64_t> attr_devs{0};
    UFOB_CUDA_TRY(smem_limit_per_device(k_conv3x3_wgrad, (int)conv_smem_bytes(), attr_devs));
    const long long npix = (long long)NB * H * W;
    // about two waves of CTAs over (pixel ranges x 9 taps x channel tiles)
    const int mt = (Cout + 127) / 128;
    long long ranges = std::max<long long>(1, (long long)num_sms() * 4 / (9 * mt));
    long long per = (npix + ranges - 1) / ranges;
    per = (per + 63) / 64 * 64;
    ranges = (npix + per - 1) / per;
    WgradArgs a;
    a.in = in;
    a.dz = dz;
    a.dw = dw;
    a.NB = NB;
    a.H = H;
    a.W = W;
    a.Cin = Cin;
    a.Cout = Cout;
    a.pix_per_cta = per;
    a.err = device_error_word();
    k_conv3x3_wgrad<<<dim3((unsigned)ranges, 9, mt), 128, conv_smem_bytes(), s>>>(a);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

}  // namespace ufob

using namespace ufob;

// Low-level entry points (used by the network and by the gradient tests).
extern "C" ufob_status ufob_conv3x3_forward(const void *d_in, const void *d_w, const float *d_bias,
                                            const void *d_residual, void *d_out, float *d_out_f32, int nb, int h,
                                            int w, int cin, int cout, int relu, void *stream)
{
    UFOB_TRY(ensure_device());
    return conv3x3_launch((const __nv_bfloat16 *)d_in, (const __nv_bfloat16 *)d_w, d_bias,
                          (const __nv_bfloat16 *)d_residual, (__nv_bfloat16 *)d_out, d_out_f32, nb, h, w, cin, cout,
                          relu, (cudaStream_t)stream);
}

extern "C" ufob_status ufob_conv3x3_wgrad(const void *d_in, const void *d_dz, float *d_dw, int nb, int h, int w,
                                          int cin, int cout, void *stream)
{
    UFOB_TRY(ensure_device());
    return conv3x3_wgrad_launch((const __nv_bfloat16 *)d_in, (const __nv_bfloat16 *)d_dz, d_dw, nb, h, w, cin, cout,
                                (cudaStream_t)stream);
}
