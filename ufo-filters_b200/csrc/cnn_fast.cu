// Inference path of the sparse-view correction network: persistent,
// warp-specialised tcgen05 convolutions over a padded channel-group layout.
//
// Activation layout "CG": a tensor of B images, H x W pixels, C channels is
// stored as C/8 planes; plane g holds channels 8g..8g+7 of every pixel as one
// 16-byte row, rows ordered by the flattened PADDED image index
//   q = (b * (H + 2) + y + 1) * (W + 2) + x + 1,
// preceded by guard rows and followed by a tail, all zero.  The
// one-pixel zero border makes a 3x3 convolution a 1-D convolution over q with
// the nine row offsets (dy * (W + 2) + dx), so for a tile of consecutive rows
// the operand of every tap is the same staged halo block read at a different
// start row: a K-major UMMA operand whose 8-row core matrices are 128
// contiguous bytes.  Every load is therefore a plain 1-D bulk copy
// (cp.async.bulk) of one plane's row range, and the weights, pre-arranged as
// [tap][channel group][Cout][8], are one contiguous bulk copy per tap.
//
// CTA roles (320 threads): warp 0 lane 0 issues the bulk copies into an
// A ring (halo blocks, 2 stages) and a B ring of per-tap weight tiles (as deep
// as shared memory allows; small layers keep all nine taps resident);
// warp 1 allocates tensor memory and lane 0 issues tcgen05.mma (M = 128 rows
// per MMA, MT row blocks per tile, N = Cout, K = 16) and tcgen05.commit;
// warps 2-9 (two per TMEM lane quarter, one channel half each) drain the
// double-buffered accumulators (tcgen05.ld, up to 32 columns per load) and run the
// fused epilogue: bias + ReLU + BF16 store, or the decoder's nearest 2x
// up-sampling plus skip connection, or the output depth-to-space plus the
// residual FBP image.  Border rows of the padded grid are never written, so
// they stay zero.  Every mbarrier wait is bounded; on expiry the CTA raises a
// shared abort flag, records an error code and winds down.
#include <cuda_bf16.h>

#include <algorithm>

#include "ufob_internal.h"

namespace ufob {

typedef __nv_bfloat16 bf16;

namespace {

constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;  // producer warp, MMA warp, epilogue warps
constexpr int kAStages = 2;
constexpr int kMaxBStages = 16;
constexpr int kErrFastTimeout = 0x2101;
constexpr size_t kMaxSmem = 220 * 1024;
constexpr uint64_t kLimitNs = 2000000000ull;

__device__ __forceinline__ uint32_t sa(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t *b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa(b)), "r"(count) : "memory");
}

__device__ __forceinline__ bool bar_try(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(sa(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t now_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait that also gives up as soon as another role raised the abort flag.
// The timer and the flag are checked only every 256 polls: a %globaltimer read
// per poll delays noticing the phase flip by the read's latency.
__device__ __forceinline__ bool bar_wait(uint64_t *b, uint32_t parity, volatile int *abort_flag)
{
    uint64_t t0 = 0;
    for (uint32_t i = 1;; i++) {
        if (bar_try(b, parity)) return true;
        if ((i & 255u) == 0) {
            if (*abort_flag) return false;
            const uint64_t t = now_ns();
            if (!t0) {
                t0 = t;
            } else if (t - t0 > kLimitNs) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}

// Programmatic dependent launch: the next kernel of the forward pass may be scheduled as soon as
// every CTA of this one has started (launch_dependents); a kernel launched that way waits for its
// predecessor, and hence for every earlier kernel of the stream, to complete and become visible
// (wait) before it reads their outputs.  Both are no-ops without the launch attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void bar_arrive(uint64_t *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa(b)) : "memory");
}

__device__ __forceinline__ void bar_expect(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *b)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sa(dst)),
                 "l"(src), "r"(bytes), "r"(sa(b))
                 : "memory");
}

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

__host__ __device__ constexpr uint32_t idesc_f16_bf16(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void commit(uint64_t *b)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sa(b))
                 : "memory");
}

// tcgen05.ld of N consecutive 32-bit columns (32 lanes x 32 bit), no wait
template <int N>
__device__ __forceinline__ void tld(uint32_t taddr, float (&v)[N]);

template <>
__device__ __forceinline__ void tld<8>(uint32_t taddr, float (&v)[8])
{
    uint32_t *r = reinterpret_cast<uint32_t *>(v);
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

template <>
__device__ __forceinline__ void tld<16>(uint32_t taddr, float (&v)[16])
{
    uint32_t *r = reinterpret_cast<uint32_t *>(v);
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
}

template <>
__device__ __forceinline__ void tld<32>(uint32_t taddr, float (&v)[32])
{
    uint32_t *r = reinterpret_cast<uint32_t *>(v);
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                 "[%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
}

__device__ __forceinline__ int ilog2_dev(int v) { return 31 - __clz(v); }

__device__ __forceinline__ void tld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint4 pack8(const float (&v)[8])
{
    uint4 o;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
    for (int j = 0; j < 4; j++) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
    return o;
}

__device__ __forceinline__ void unpack8_add(const uint4 &u, float (&v)[8])
{
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float2 f = __bfloat1622float2(h[j]);
        v[2 * j] += f.x;
        v[2 * j + 1] += f.y;
    }
}

}  // namespace

enum { EPI_STORE = 0, EPI_UPADD = 1, EPI_FINAL = 2 };

// One padded-grid geometry (B images of H x W interior pixels).
struct CGGeom {
    int B, H, W;
    long long rows;   // B * (H + 2) * (W + 2)
    long long alloc;  // rows per plane including guard and tail
    int guard;        // zero rows before q = 0
};

struct FastConvArgs {
    const bf16 *in;   // CG, Cin channels, geometry gi
    const bf16 *wt;   // [9][Cin/8][Cout][8]
    const float *bias;
    bf16 *out;        // EPI_STORE: CG at gi; EPI_UPADD: CG at 2x (go)
    const bf16 *skip; // EPI_UPADD: CG at 2x (go)
    const float *fbp; // EPI_FINAL: [B][4H][4W]
    float *img;       // EPI_FINAL output
    float scale;
    CGGeom gi, go;
    int Cin, Cout, MT, relu, mode;
    int bstages;   // weight ring depth; == 9 * chunks: all weights resident, loaded once
    long long ntiles;
    int *err;
};

// The MMAs of one tap, fully unrolled: MT row blocks x KS K-steps of 16
// channels.  The descriptors of the tap are built once; each MMA adds a
// compile-time row / channel-group offset to the 16-byte start-address field
// (smem addresses stay below 256 KB, so the field never carries).  A single
// thread issues every MMA, so its per-MMA instruction count bounds the
// tensor-core rate for small N.
template <int MT, int KS>
__device__ __forceinline__ void issue_tap(uint32_t dcol, uint32_t Cout, uint64_t dA, uint64_t dB, uint32_t a16,
                                          uint32_t b16, uint32_t idesc, bool first)
{
#pragma unroll
    for (int m = 0; m < MT; m++)
#pragma unroll
        for (int k = 0; k < KS; k++)
            mma(dcol + (uint32_t)m * Cout, dA + (uint64_t)(m * 128) + (uint64_t)(2 * k) * a16,
                dB + (uint64_t)(2 * k) * b16, idesc, (first && k == 0) ? 0u : 1u);
}

template <int MT, int KS>
__global__ void __launch_bounds__(kThreads, 1) k_conv_cg(const FastConvArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t a_full[kAStages], a_empty[kAStages], b_full[kMaxBStages], b_empty[kMaxBStages];
    __shared__ uint64_t t_full[2], t_empty[2];
    __shared__ uint32_t tslot;
    __shared__ int abort_flag;
    __shared__ float s_bias[256];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    pdl_launch_dependents();
    const int Cin = a.Cin, Cout = a.Cout;
    const int cgc = Cin < 64 ? Cin / 8 : 8;  // channel groups per K chunk
    const int nchunks = Cin / (cgc * 8);
    const int nbs = a.bstages;
    const bool resident = nbs == 9 * nchunks;
    const int Wp = a.gi.W + 2;
    const int halo = Wp + 1;
    const int arows = MT * 128 + 2 * halo;  // rows of one staged plane
    const uint32_t a_plane = (uint32_t)arows * 16;
    const uint32_t a_stage = a_plane * (uint32_t)cgc;
    const uint32_t b_stage = (uint32_t)cgc * (uint32_t)Cout * 16;
    unsigned char *sA = smem;
    unsigned char *sB = smem + (size_t)kAStages * a_stage;
    const uint32_t acc_cols = (uint32_t)(MT * Cout);
    uint32_t ncols = 32;
    while (ncols < 2 * acc_cols) ncols <<= 1;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kAStages; i++) {
            bar_init(&a_full[i], 1);
            bar_init(&a_empty[i], 1);
        }
        for (int i = 0; i < nbs; i++) {
            bar_init(&b_full[i], 1);
            bar_init(&b_empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            bar_init(&t_full[i], 1);
            bar_init(&t_empty[i], kEpiWarps);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < Cout; i += blockDim.x) s_bias[i] = a.bias[i];
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa(&tslot)), "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tslot;
    volatile int *abort_p = &abort_flag;

    // offsets of the nine taps in padded rows
    const long long plane_elems = a.gi.alloc * 8;  // bf16 per input plane

    if (warp == 0) {
        if (lane == 0) {
            uint32_t ka = 0, kb = 0;
            int last_a[kAStages], last_b[kMaxBStages];  // running index of each stage's last copy
            for (int i = 0; i < kAStages; i++) last_a[i] = -1;
            for (int i = 0; i < nbs; i++) last_b[i] = -1;
            bool ok = true;
            if (resident && blockIdx.x < a.ntiles) {
                // every (chunk, tap) weight tile once, kept for the whole kernel
                for (int kc = 0; kc < nchunks; kc++)
                    for (int t = 0; t < 9; t++) {
                        const int sb = kc * 9 + t;
                        bar_expect(&b_full[sb], b_stage);
                        const bf16 *src = a.wt + ((size_t)t * (Cin / 8) + (size_t)kc * cgc) * Cout * 8;
                        bulk_g2s(sB + (size_t)sb * b_stage, src, b_stage, &b_full[sb]);
                        last_b[sb] = 0;
                    }
            }
            pdl_wait();  // the activations are the previous kernels' outputs
            for (long long tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x) {
                const long long q0 = tile * (long long)(MT * 128);
                for (int kc = 0; kc < nchunks && ok; kc++) {
                    const int s = (int)(ka % kAStages);
                    ok = bar_wait(&a_empty[s], ((ka / kAStages) & 1u) ^ 1u, abort_p);
                    if (!ok) break;
                    bar_expect(&a_full[s], a_stage);
                    for (int g = 0; g < cgc; g++) {
                        const bf16 *src = a.in + (size_t)(kc * cgc + g) * plane_elems +
                                          (size_t)(a.gi.guard + q0 - halo) * 8;
                        bulk_g2s(sA + (size_t)s * a_stage + (size_t)g * a_plane, src, a_plane, &a_full[s]);
                    }
                    last_a[s] = (int)ka;
                    ka++;
                    for (int t = 0; t < 9 && ok && !resident; t++) {
                        const int sb = (int)(kb % nbs);
                        ok = bar_wait(&b_empty[sb], ((kb / nbs) & 1u) ^ 1u, abort_p);
                        if (!ok) break;
                        bar_expect(&b_full[sb], b_stage);
                        const bf16 *src = a.wt + ((size_t)t * (Cin / 8) + (size_t)kc * cgc) * Cout * 8;
                        bulk_g2s(sB + (size_t)sb * b_stage, src, b_stage, &b_full[sb]);
                        last_b[sb] = (int)kb;
                        kb++;
                    }
                }
            }
            if (!ok) {
                atomicExch(a.err, kErrFastTimeout);
                // let copies already in flight land before the CTA can exit (bounded)
                for (int s = 0; s < kAStages; s++) {
                    const uint64_t t0 = now_ns();
                    if (last_a[s] >= 0)
                        while (!bar_try(&a_full[s], ((uint32_t)last_a[s] / kAStages) & 1u) &&
                               now_ns() - t0 < kLimitNs / 8) {
                        }
                }
                for (int s = 0; s < nbs; s++) {
                    const uint64_t t0 = now_ns();
                    if (last_b[s] >= 0)
                        while (!bar_try(&b_full[s], ((uint32_t)last_b[s] / nbs) & 1u) &&
                               now_ns() - t0 < kLimitNs / 8) {
                        }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_f16_bf16(128, (uint32_t)Cout);
            uint32_t ka = 0, kb = 0, it = 0;
            bool ok = true;
            for (long long tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x, it++) {
                const uint32_t ab = it & 1u;
                ok = bar_wait(&t_empty[ab], ((it >> 1) & 1u) ^ 1u, abort_p);
                if (!ok) break;
                fence_after();
                const uint32_t dcol = tmem + ab * acc_cols;
                for (int kc = 0; kc < nchunks && ok; kc++) {
                    const int s = (int)(ka % kAStages);
                    ok = bar_wait(&a_full[s], (ka / kAStages) & 1u, abort_p);
                    if (!ok) break;
                    fence_after();
                    const uint32_t abase = sa(sA + (size_t)s * a_stage);
                    for (int t = 0; t < 9 && ok; t++) {
                        const int sb = resident ? kc * 9 + t : (int)(kb % nbs);
                        if (!resident || it == 0) {
                            ok = bar_wait(&b_full[sb], resident ? 0u : (kb / nbs) & 1u, abort_p);
                            if (!ok) break;
                            fence_after();
                        }
                        const uint32_t bbase = sa(sB + (size_t)sb * b_stage);
                        const int off = halo + (t / 3 - 1) * Wp + (t % 3 - 1);
                        issue_tap<MT, KS>(dcol, (uint32_t)Cout, desc_kmajor(abase + (uint32_t)off * 16, a_plane, 128),
                                          desc_kmajor(bbase, (uint32_t)Cout * 16, 128), a_plane >> 4, (uint32_t)Cout,
                                          idesc, kc == 0 && t == 0);
                        if (!resident) commit(&b_empty[sb]);  // frees the weight stage once these MMAs finish
                        kb++;
                    }
                    commit(&a_empty[s]);
                    ka++;
                }
                commit(&t_full[ab]);
            }
            if (!ok) atomicExch(a.err, kErrFastTimeout);
        }
    } else {
        // epilogue warps 2..9: TMEM lane quarter = warp % 4, channel half = (warp - 2) / 4
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const int ch = Cout / 2;  // channels per epilogue warp
        uint32_t it = 0;
        const uint32_t Hp = (uint32_t)a.gi.H + 2;
        const uint32_t img_rows = Hp * (uint32_t)Wp;
        const uint32_t rows = (uint32_t)a.gi.rows;
        pdl_wait();  // skip tensors and the FBP image come from earlier kernels
        for (long long tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, it++) {
            const uint32_t ab = it & 1u;
            if (!bar_wait(&t_full[ab], (it >> 1) & 1u, abort_p)) {
                if (lane == 0) atomicExch(a.err, kErrFastTimeout);
                break;
            }
            fence_after();
            const uint32_t q0 = (uint32_t)tile * (uint32_t)(MT * 128) + (uint32_t)(quarter * 32 + lane);
            const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + ab * acc_cols + (uint32_t)(half * ch);
            // pixel of row q of the padded grid: (b, y, x), inside = interior pixel
            auto locate = [&](uint32_t q, int &b, int &y, int &x) -> bool {
                if (q >= rows) return false;
                b = (int)(q / img_rows);
                const uint32_t r = q - (uint32_t)b * img_rows;
                const int yy = (int)(r / (uint32_t)Wp);
                y = yy - 1;
                x = (int)r - yy * Wp - 1;
                return y >= 0 && y < a.gi.H && x >= 0 && x < a.gi.W;
            };
            if (a.mode == EPI_FINAL) {
                // Cout = 16 = 4 x 4 sub-pixels; this warp: sub-rows 2*half, 2*half + 1.  The FBP loads
                // and TMEM loads of up to 4 row blocks are in flight before each wait.
                constexpr int MG = MT < 4 ? MT : 4;
                const int W4 = 4 * a.gi.W;
#pragma unroll
                for (int m0 = 0; m0 < MT; m0 += MG) {
                    float v[MG][8];
                    float4 f[MG][2];
                    size_t base[MG];
                    bool in[MG];
#pragma unroll
                    for (int i = 0; i < MG; i++) {
                        int b = 0, y = 0, x = 0;
                        in[i] = locate(q0 + (uint32_t)((m0 + i) * 128), b, y, x);
                        base[i] = ((size_t)b * 4 * a.gi.H + 4 * y + 2 * half) * W4 + 4 * x;
                        if (in[i]) {
                            f[i][0] = *reinterpret_cast<const float4 *>(a.fbp + base[i]);
                            f[i][1] = *reinterpret_cast<const float4 *>(a.fbp + base[i] + W4);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < MG; i++) tld<8>(tb + (uint32_t)((m0 + i) * Cout), v[i]);
                    tld_wait();
#pragma unroll
                    for (int i = 0; i < MG; i++) {
                        if (!in[i]) continue;
#pragma unroll
                        for (int dy = 0; dy < 2; dy++) {
                            const float *bb = s_bias + 8 * half + 4 * dy;
                            float4 o;
                            o.x = f[i][dy].x + a.scale * (v[i][4 * dy + 0] + bb[0]);
                            o.y = f[i][dy].y + a.scale * (v[i][4 * dy + 1] + bb[1]);
                            o.z = f[i][dy].z + a.scale * (v[i][4 * dy + 2] + bb[2]);
                            o.w = f[i][dy].w + a.scale * (v[i][4 * dy + 3] + bb[3]);
                            *reinterpret_cast<float4 *>(a.img + base[i] + (size_t)dy * W4) = o;
                        }
                    }
                }
            } else if (a.mode == EPI_STORE) {
                // interior flags of this thread's MT rows, once per tile
                uint32_t inmask = 0;
#pragma unroll
                for (int m = 0; m < MT; m++) {
                    int b, y, x;
                    if (locate(q0 + (uint32_t)(m * 128), b, y, x)) inmask |= 1u << m;
                }
                // chunks of 8 channels over (row block, channel group); chunks per block is a power
                // of two (Cout / 16); 4 chunks in flight per wait
                const int lcpm = ilog2_dev(ch >> 3), nch = MT << lcpm;
                for (int c0 = 0; c0 < nch; c0 += 4) {
                    float v[4][8];
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        if (c0 + i < nch) {
                            const int m = (c0 + i) >> lcpm, cc = (c0 + i) & ((1 << lcpm) - 1);
                            tld<8>(tb + (uint32_t)(m * Cout + cc * 8), v[i]);
                        }
                    tld_wait();
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        if (c0 + i >= nch) break;
                        const int m = (c0 + i) >> lcpm, cc = (c0 + i) & ((1 << lcpm) - 1);
                        if (!((inmask >> m) & 1u)) continue;
                        const uint32_t q = q0 + (uint32_t)(m * 128);
                        const int c = half * ch + cc * 8;
                        float w[8];
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            w[j] = v[i][j] + s_bias[c + j];
                            if (a.relu) w[j] = fmaxf(w[j], 0.f);
                        }
                        bf16 *dst = a.out + ((size_t)(c >> 3) * a.gi.alloc + a.gi.guard + q) * 8;
                        *reinterpret_cast<uint4 *>(dst) = pack8(w);
                    }
                }
            } else {
                // decoder: nearest 2x up-sampling plus the skip tensor at the output grid; the skip loads
                // and TMEM loads of 2 chunks are in flight before the wait.  The decoder activation is
                // rounded to BF16 first, as where it is stored.
                const int lcpm = ilog2_dev(ch >> 3), nch = MT << lcpm;
                const uint32_t Wo = (uint32_t)a.go.W + 2, Ho = (uint32_t)a.go.H + 2;
                for (int c0 = 0; c0 < nch; c0 += 2) {
                    float v[2][8];
                    uint4 sk[2][4];
                    size_t off[2];
                    bool in[2];
#pragma unroll
                    for (int i = 0; i < 2; i++) {
                        in[i] = false;
                        if (c0 + i >= nch) continue;
                        const int m = (c0 + i) >> lcpm, cc = (c0 + i) & ((1 << lcpm) - 1);
                        int b = 0, y = 0, x = 0;
                        in[i] = locate(q0 + (uint32_t)(m * 128), b, y, x);
                        const int g = (half * ch + cc * 8) >> 3;
                        const uint32_t qo = ((uint32_t)b * Ho + 2 * y + 1) * Wo + 2 * x + 1;
                        off[i] = ((size_t)g * a.go.alloc + a.go.guard + qo) * 8;
                        if (in[i]) {
                            const bf16 *sp = a.skip + off[i];
                            sk[i][0] = *reinterpret_cast<const uint4 *>(sp);
                            sk[i][1] = *reinterpret_cast<const uint4 *>(sp + 8);
                            sk[i][2] = *reinterpret_cast<const uint4 *>(sp + (size_t)Wo * 8);
                            sk[i][3] = *reinterpret_cast<const uint4 *>(sp + (size_t)Wo * 8 + 8);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 2; i++)
                        if (c0 + i < nch) {
                            const int m = (c0 + i) >> lcpm, cc = (c0 + i) & ((1 << lcpm) - 1);
                            tld<8>(tb + (uint32_t)(m * Cout + cc * 8), v[i]);
                        }
                    tld_wait();
#pragma unroll
                    for (int i = 0; i < 2; i++) {
                        if (!in[i]) continue;
                        const int cc = (c0 + i) & ((1 << lcpm) - 1);
                        const int c = half * ch + cc * 8;
                        float w[8];
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            w[j] = v[i][j] + s_bias[c + j];
                            if (a.relu) w[j] = fmaxf(w[j], 0.f);
                            w[j] = __bfloat162float(__float2bfloat16(w[j]));
                        }
#pragma unroll
                        for (int r = 0; r < 4; r++) {
                            float o[8];
#pragma unroll
                            for (int k = 0; k < 8; k++) o[k] = w[k];
                            unpack8_add(sk[i][r], o);
                            const size_t d = off[i] + (size_t)(r >> 1) * Wo * 8 + (size_t)(r & 1) * 8;
                            *reinterpret_cast<uint4 *>(a.out + d) = pack8(o);
                        }
                    }
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) bar_arrive(&t_empty[ab]);
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

// ------------------------------------------------------------------ small CG kernels

#define CG_LOOP(i, n) for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// The per-pixel kernels below run on a 2-D grid: y walks the images (slices, or channel planes x
// slices), x one image's output pixels, so every index is 32-bit arithmetic (one image holds at
// most 2^31 pixels; 64-bit divisions by runtime sizes cost more than these kernels' loads).

// fbp [B][4H][4W] -> CG x0 (16 channels, two planes): channel 4*dy + dx = fbp[4y+dy][4x+dx] / s
__global__ void k_cg_unshuffle(const float *__restrict__ fbp, bf16 *__restrict__ x0, CGGeom g, float inv_s)
{
    pdl_launch_dependents();
    const uint32_t hw = (uint32_t)g.H * (uint32_t)g.W;
    const size_t W4 = (size_t)4 * g.W;
    for (uint32_t b = blockIdx.y; b < (uint32_t)g.B; b += gridDim.y)
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < hw; i += gridDim.x * blockDim.x) {
            const uint32_t y = i / (uint32_t)g.W, x = i - y * (uint32_t)g.W;
            const float *src = fbp + ((size_t)b * 4 * g.H + 4 * y) * W4 + 4 * x;
            float v[16];
#pragma unroll
            for (int dy = 0; dy < 4; dy++) {
                const float4 f = *reinterpret_cast<const float4 *>(src + dy * W4);
                v[4 * dy] = f.x * inv_s;
                v[4 * dy + 1] = f.y * inv_s;
                v[4 * dy + 2] = f.z * inv_s;
                v[4 * dy + 3] = f.w * inv_s;
            }
            const long long q = ((long long)b * (g.H + 2) + y + 1) * (g.W + 2) + x + 1;
            float lo[8], hi[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                lo[k] = v[k];
                hi[k] = v[8 + k];
            }
            *reinterpret_cast<uint4 *>(x0 + ((size_t)g.guard + q) * 8) = pack8(lo);
            *reinterpret_cast<uint4 *>(x0 + ((size_t)g.alloc + g.guard + q) * 8) = pack8(hi);
        }
}

// 2x2 average pool between CG tensors (gi -> go = gi / 2), C/8 planes
__global__ void k_cg_pool(const bf16 *__restrict__ in, bf16 *__restrict__ out, CGGeom gi, CGGeom go, int planes)
{
    pdl_launch_dependents();
    pdl_wait();
    const uint32_t hw = (uint32_t)go.H * (uint32_t)go.W, images = (uint32_t)planes * (uint32_t)go.B;
    for (uint32_t img = blockIdx.y; img < images; img += gridDim.y) {
        const uint32_t p = img / (uint32_t)go.B, b = img - p * (uint32_t)go.B;
        const bf16 *ip = in + ((size_t)p * gi.alloc + gi.guard) * 8;
        bf16 *op = out + ((size_t)p * go.alloc + go.guard) * 8;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < hw; i += gridDim.x * blockDim.x) {
            const uint32_t y = i / (uint32_t)go.W, x = i - y * (uint32_t)go.W;
            const long long qi = ((long long)b * (gi.H + 2) + 2 * y + 1) * (gi.W + 2) + 2 * x + 1;
            const bf16 *s = ip + (size_t)qi * 8;
            const uint4 r0 = *reinterpret_cast<const uint4 *>(s);
            const uint4 r1 = *reinterpret_cast<const uint4 *>(s + 8);
            const uint4 r2 = *reinterpret_cast<const uint4 *>(s + (size_t)(gi.W + 2) * 8);
            const uint4 r3 = *reinterpret_cast<const uint4 *>(s + (size_t)(gi.W + 3) * 8);
            float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            unpack8_add(r0, v);
            unpack8_add(r1, v);
            unpack8_add(r2, v);
            unpack8_add(r3, v);
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] *= 0.25f;
            const long long qo = ((long long)b * (go.H + 2) + y + 1) * (go.W + 2) + x + 1;
            *reinterpret_cast<uint4 *>(op + (size_t)qo * 8) = pack8(v);
        }
    }
}

// [Cout][9][Cin] FP32 master weights -> [9][Cin/8][Cout][8] BF16 (K-major tiles per tap)
__global__ void k_cg_arrange(const float *__restrict__ w, bf16 *__restrict__ wt, int Cout, int Cin)
{
    const long long n = (long long)Cout * 9 * Cin;
    CG_LOOP(i, n) {
        const int ci = (int)(i % Cin), t = (int)((i / Cin) % 9), co = (int)(i / (9LL * Cin));
        wt[(((size_t)t * (Cin / 8) + ci / 8) * Cout + co) * 8 + (ci & 7)] = __float2bfloat16(w[i]);
    }
}

// ------------------------------------------------------------------ host side

static CGGeom cg_geom(int B, int H, int W, int max_tile_rows)
{
    CGGeom g;
    g.B = B;
    g.H = H;
    g.W = W;
    g.rows = (long long)B * (H + 2) * (W + 2);
    g.guard = (W + 3 + 7) / 8 * 8;
    // tail: the last tile may extend max_tile_rows past the end, plus its halo
    g.alloc = g.guard + g.rows + max_tile_rows + W + 3 + 8;
    return g;
}

struct CGBuf {
    DevBuf buf;
    CGGeom g;
    int C = 0;
    bf16 *ptr() const { return buf.as<bf16>(); }
};

static ufob_status cg_alloc(CGBuf &t, int B, int H, int W, int C, cudaStream_t s)
{
    const CGGeom g = cg_geom(B, H, W, 8 * 128);  // largest tile of plan_conv
    const size_t bytes = (size_t)(C / 8) * g.alloc * 16;
    const bool same = t.C == C && t.g.B == B && t.g.H == H && t.g.W == W && t.buf.ptr;
    if (!same) {
        UFOB_TRY(t.buf.ensure(bytes));
        UFOB_CUDA_TRY(cudaMemsetAsync(t.buf.ptr, 0, bytes, s));  // border, guard and tail rows stay zero
        t.g = g;
        t.C = C;
    }
    return UFOB_OK;
}

struct FastNet {
    DevBuf wt[8];
    CGBuf x0, e1, p1, e2, p2, e3, p3, e4, u3, u2, u1;
    uint32_t smem_attr = 0;  // bit (3 log2 MT + log2 KS): shared-memory attribute set for that instance
};

// Tile plan of one layer: row blocks per tile (two accumulator buffers of
// MT * Cout columns in the 512 TMEM columns), weight ring depth, smem bytes.
struct ConvPlan {
    int MT, bstages;
    size_t smem;
    long long ntiles;
};

static ConvPlan plan_conv(int Cin, int Cout, const CGGeom &g)
{
    const int cgc = Cin < 64 ? Cin / 8 : 8;
    const int nchunks = Cin / (cgc * 8);
    const size_t b_stage = (size_t)cgc * Cout * 16;
    const int sms = num_sms();
    ConvPlan best{0, 0, 0, 0};
    for (int mt = 8; mt >= 1; mt >>= 1) {
        if (2 * mt * Cout > 512) continue;
        const size_t arows = (size_t)mt * 128 + 2 * (g.W + 3);
        const size_t abytes = (size_t)kAStages * arows * 16 * cgc + 1024;
        if (abytes + 2 * b_stage > kMaxSmem) continue;
        ConvPlan p;
        p.MT = mt;
        p.ntiles = (g.rows + mt * 128 - 1) / (mt * 128);
        const int nres = 9 * nchunks;
        if (nres <= kMaxBStages && abytes + nres * b_stage <= kMaxSmem)
            p.bstages = nres;  // all weights resident
        else
            p.bstages = (int)std::min<size_t>(kMaxBStages, std::min<size_t>(nres - 1, (kMaxSmem - abytes) / b_stage));
        p.smem = abytes + (size_t)p.bstages * b_stage;
        // largest tile that still gives every SM work; else the one with most tiles
        if (!best.MT || (best.ntiles < sms && p.ntiles > best.ntiles)) best = p;
        if (p.ntiles >= sms) {
            best = p;
            break;
        }
    }
    return best;
}

typedef void (*ConvKernel)(const FastConvArgs);

static ConvKernel conv_kernel(int mt, int ks)
{
#define UFOB_CONV_CASE(M, K) \
    if (mt == M && ks == K) return k_conv_cg<M, K>;
    UFOB_CONV_CASE(1, 1) UFOB_CONV_CASE(1, 2) UFOB_CONV_CASE(1, 4)
    UFOB_CONV_CASE(2, 1) UFOB_CONV_CASE(2, 2) UFOB_CONV_CASE(2, 4)
    UFOB_CONV_CASE(4, 1) UFOB_CONV_CASE(4, 2) UFOB_CONV_CASE(4, 4)
    UFOB_CONV_CASE(8, 1) UFOB_CONV_CASE(8, 2) UFOB_CONV_CASE(8, 4)
#undef UFOB_CONV_CASE
    return nullptr;
}

static ufob_status conv_cg(FastNet *f, const CGBuf &in, const bf16 *wt, const float *bias, int Cout, int relu,
                           int mode, CGBuf *out, const CGBuf *skip, const float *fbp, float *img, float scale,
                           cudaStream_t s)
{
    FastConvArgs a{};
    a.in = in.ptr();
    a.wt = wt;
    a.bias = bias;
    a.gi = in.g;
    a.Cin = in.C;
    a.Cout = Cout;
    a.relu = relu;
    a.mode = mode;
    if (in.g.alloc >= (1ll << 31) || (mode == EPI_UPADD && out->g.alloc >= (1ll << 31)))
        return fail(UFOB_ERR_UNSUPPORTED, "cnn: batch too large for 32-bit row indices");
    const ConvPlan pl = plan_conv(in.C, Cout, in.g);
    if (!pl.MT) return fail(UFOB_ERR_UNSUPPORTED, "cnn: convolution tile does not fit in shared memory");
    a.MT = pl.MT;
    a.bstages = pl.bstages;
    a.err = device_error_word();
    a.scale = scale;
    if (mode == EPI_STORE) a.out = out->ptr();
    if (mode == EPI_UPADD) {
        a.out = out->ptr();
        a.skip = skip->ptr();
        a.go = out->g;
    }
    a.fbp = fbp;
    a.img = img;
    a.ntiles = pl.ntiles;
    const size_t smem = pl.smem;
    const int ks = (in.C < 64 ? in.C / 8 : 8) / 2;
    auto kern = conv_kernel(a.MT, ks);
    if (!kern) return fail(UFOB_ERR_UNSUPPORTED, "cnn: no convolution kernel for %d row blocks x %d K-steps", a.MT, ks);
    const uint32_t bit = 1u << (ilog2((uint64_t)a.MT) * 3 + ilog2((uint64_t)ks));
    if (!(f->smem_attr & bit)) {
        UFOB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
        cudaFuncAttributes fa;
        UFOB_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
        if (fa.maxThreadsPerBlock < kThreads)
            return fail(UFOB_ERR_UNSUPPORTED,
                        "cnn: convolution kernel (%d row blocks, %d K-steps) takes %d registers: at most %d threads "
                        "per block, %d needed",
                        a.MT, ks, fa.numRegs, fa.maxThreadsPerBlock, kThreads);
        f->smem_attr |= bit;
    }
    // one CTA per SM: the two accumulator buffers may take all 512 TMEM columns
    const long long grid = std::min<long long>(a.ntiles, num_sms());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = std::max<size_t>(smem, 116 * 1024);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, a);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess)
        return fail(UFOB_ERR_CUDA, "cnn: convolution launch (%d row blocks, %d K-steps, %zu B shared) failed: %s", a.MT,
                    ks, std::max<size_t>(smem, 116 * 1024), cudaGetErrorString(le));
    note_launch();
    return UFOB_OK;
}

static unsigned grid_for(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, (long long)num_sms() * 16); }

// 256-thread CTAs over one image's pixels (x) and the images (y)
static dim3 grid_images(const CGGeom &g, int images)
{
    const unsigned hw = (unsigned)g.H * (unsigned)g.W;
    return dim3((hw + 255) / 256, (unsigned)std::min(images, 65535));
}

// 2x2 average pool between CG tensors, launched as a programmatic dependent of the convolution
// before it
static ufob_status pool_launch(const CGBuf &in, const CGBuf &out, int planes, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid_images(out.g, planes * out.g.B);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    UFOB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_cg_pool, (const bf16 *)in.ptr(), out.ptr(), in.g, out.g, planes));
    note_launch();
    return UFOB_OK;
}

void *cnn_fast_create() { return new FastNet; }
void cnn_fast_destroy(void *p) { delete static_cast<FastNet *>(p); }

// Re-arrange the FP32 master weights of the 8 layers into the per-tap BF16 tiles.
ufob_status cnn_fast_weights(void *fp, const float *const *w, const int (*shape)[2], cudaStream_t s)
{
    FastNet *f = static_cast<FastNet *>(fp);
    for (int i = 0; i < 8; i++) {
        const int cin = shape[i][0], cout = shape[i][1];
        const size_t n = (size_t)cout * 9 * cin;
        UFOB_TRY(f->wt[i].ensure(n * 2));
        k_cg_arrange<<<grid_for((long long)n), 256, 0, s>>>(w[i], f->wt[i].as<bf16>(), cout, cin);
        UFOB_CUDA_TRY(cudaGetLastError());
        note_launch();
    }
    return UFOB_OK;
}

// Whole network on B slices [B][4H][4W] (H, W = quarter-resolution sides).
ufob_status cnn_fast_forward(void *fp, const float *const *bias, const float *fbp, float *out, int B, int H, int W,
                             float scale, cudaStream_t s)
{
    FastNet *f = static_cast<FastNet *>(fp);
    UFOB_TRY(cg_alloc(f->x0, B, H, W, 16, s));
    UFOB_TRY(cg_alloc(f->e1, B, H, W, 32, s));
    UFOB_TRY(cg_alloc(f->p1, B, H / 2, W / 2, 32, s));
    UFOB_TRY(cg_alloc(f->e2, B, H / 2, W / 2, 64, s));
    UFOB_TRY(cg_alloc(f->p2, B, H / 4, W / 4, 64, s));
    UFOB_TRY(cg_alloc(f->e3, B, H / 4, W / 4, 128, s));
    UFOB_TRY(cg_alloc(f->p3, B, H / 8, W / 8, 128, s));
    UFOB_TRY(cg_alloc(f->e4, B, H / 8, W / 8, 256, s));
    UFOB_TRY(cg_alloc(f->u3, B, H / 4, W / 4, 128, s));
    UFOB_TRY(cg_alloc(f->u2, B, H / 2, W / 2, 64, s));
    UFOB_TRY(cg_alloc(f->u1, B, H, W, 32, s));
    k_cg_unshuffle<<<grid_images(f->x0.g, B), 256, 0, s>>>(fbp, f->x0.ptr(), f->x0.g, 1.f / scale);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    auto wt = [&](int i) { return f->wt[i].as<bf16>(); };
    UFOB_TRY(conv_cg(f, f->x0, wt(0), bias[0], 32, 1, EPI_STORE, &f->e1, nullptr, nullptr, nullptr, 0.f, s));
    UFOB_TRY(pool_launch(f->e1, f->p1, 4, s));
    UFOB_TRY(conv_cg(f, f->p1, wt(1), bias[1], 64, 1, EPI_STORE, &f->e2, nullptr, nullptr, nullptr, 0.f, s));
    UFOB_TRY(pool_launch(f->e2, f->p2, 8, s));
    UFOB_TRY(conv_cg(f, f->p2, wt(2), bias[2], 128, 1, EPI_STORE, &f->e3, nullptr, nullptr, nullptr, 0.f, s));
    UFOB_TRY(pool_launch(f->e3, f->p3, 16, s));
    UFOB_TRY(conv_cg(f, f->p3, wt(3), bias[3], 256, 1, EPI_STORE, &f->e4, nullptr, nullptr, nullptr, 0.f, s));
    UFOB_TRY(conv_cg(f, f->e4, wt(4), bias[4], 128, 1, EPI_UPADD, &f->u3, &f->e3, nullptr, nullptr, 0.f, s));
    UFOB_TRY(conv_cg(f, f->u3, wt(5), bias[5], 64, 1, EPI_UPADD, &f->u2, &f->e2, nullptr, nullptr, 0.f, s));
    UFOB_TRY(conv_cg(f, f->u2, wt(6), bias[6], 32, 1, EPI_UPADD, &f->u1, &f->e1, nullptr, nullptr, 0.f, s));
    UFOB_TRY(conv_cg(f, f->u1, wt(7), bias[7], 16, 0, EPI_FINAL, nullptr, nullptr, fbp, out, scale, s));
    UFOB_CUDA_TRY(cudaGetLastError());
    return UFOB_OK;
}

}  // namespace ufob
