// Sparse-view correction network: a 4-level U-Net (32/64/128/256 channels,
// 3x3 convolutions) that maps a 90-angle FBP slice to a correction added to
// it, trained toward the 1800-angle FBP of the same phantom.  For a 512^2
// slice:
//   x0 = space-to-depth4(fbp / s)            128^2 x 16
//   e1 = relu(conv(x0, 16->32))              128^2 x 32
//   e2 = relu(conv(pool(e1), 32->64))         64^2 x 64
//   e3 = relu(conv(pool(e2), 64->128))        32^2 x 128
//   e4 = relu(conv(pool(e3), 128->256))       16^2 x 256
//   d3 = relu(conv(e4, 256->128));  u3 = up(d3) + e3       32^2 x 128
//   d2 = relu(conv(u3, 128->64));   u2 = up(d2) + e2       64^2 x 64
//   d1 = relu(conv(u2, 64->32));    u1 = up(d1) + e1      128^2 x 32
//   o  = conv(u1, 32->16)                                 128^2 x 16 (FP32)
//   out = fbp + s * depth-to-space4(o)
// Every convolution runs on the tcgen05 kernels of cnn_conv.cu (BF16 weights
// and activations, FP32 accumulation); the backward pass uses the same
// kernels for data gradients (transposed, tap-flipped weights) and the
// weight-gradient kernel; the rest (pooling, up-sampling, ReLU masks, loss,
// bias gradients, Adam on FP32 master weights) are small CUDA-core kernels.
// About 1.2 GFLOP per 512^2 slice forward.
#include <cuda_bf16.h>
#include <math.h>

#include <random>
#include <vector>

#include "ufob_internal.h"

namespace ufob {

ufob_status conv3x3_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
                           const __nv_bfloat16 *residual, __nv_bfloat16 *out, float *out_f32, int NB, int H, int W,
                           int Cin, int Cout, int relu, cudaStream_t s);
ufob_status conv3x3_wgrad_launch(const __nv_bfloat16 *in, const __nv_bfloat16 *dz, float *dw, int NB, int H, int W,
                                 int Cin, int Cout, cudaStream_t s);

typedef __nv_bfloat16 bf16;

static inline unsigned blocks_for(size_t n, unsigned t = 256)
{
    size_t b = (n + t - 1) / t;
    return (unsigned)std::min<size_t>(b, (size_t)num_sms() * 32);
}

#define GRID_STRIDE(i, n) for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

// Space-to-depth by kS = 4: fbp [B][4H][4W] f32 -> x [B][H][W][16] bf16,
// channel 4*dy + dx = fbp[4y+dy][4x+dx] / s.
constexpr int kS = 4;

__global__ void k_unshuffle_in(const float *__restrict__ fbp, bf16 *__restrict__ x, int B, int H, int W, float inv_s)
{
    const size_t n = (size_t)B * H * W;
    GRID_STRIDE(i, n) {
        const int xx = (int)(i % W), yy = (int)((i / W) % H);
        const size_t b = i / ((size_t)W * H);
        const size_t row = (size_t)kS * W;
        const float *src = fbp + (b * kS * H + kS * yy) * row + kS * xx;
        __nv_bfloat162 v[8];
#pragma unroll
        for (int dy = 0; dy < kS; dy++) {
            const float4 q = *reinterpret_cast<const float4 *>(src + dy * row);
            v[2 * dy] = __floats2bfloat162_rn(q.x * inv_s, q.y * inv_s);
            v[2 * dy + 1] = __floats2bfloat162_rn(q.z * inv_s, q.w * inv_s);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(x + i * 16);
        dst[0] = *reinterpret_cast<uint4 *>(&v[0]);
        dst[1] = *reinterpret_cast<uint4 *>(&v[4]);
    }
}

// out = fbp + s * depth-to-space(o)   (o FP32 [B][H][W][16])
__global__ void k_shuffle_out(const float *__restrict__ o, const float *__restrict__ fbp, float *__restrict__ out, int B,
                              int H, int W, float s)
{
    const size_t n = (size_t)B * kS * kS * H * W;
    GRID_STRIDE(i, n) {
        const int X = (int)(i % (kS * W)), Y = (int)((i / (kS * W)) % (kS * H));
        const size_t b = i / ((size_t)kS * kS * H * W);
        const int c = kS * (Y % kS) + (X % kS);
        out[i] = fbp[i] + s * o[((b * H + Y / kS) * W + X / kS) * 16 + c];
    }
}

// gradient at o (bf16 [B][H][W][16]) of the loss from d_out: s * space-to-depth(d_out)
__global__ void k_shuffle_out_grad(const float *__restrict__ dout, bf16 *__restrict__ dz, int B, int H, int W, float s)
{
    const size_t n = (size_t)B * H * W;
    GRID_STRIDE(i, n) {
        const int xx = (int)(i % W), yy = (int)((i / W) % H);
        const size_t b = i / ((size_t)W * H);
        const size_t row = (size_t)kS * W;
        const float *src = dout + (b * kS * H + kS * yy) * row + kS * xx;
        __nv_bfloat162 v[8];
#pragma unroll
        for (int dy = 0; dy < kS; dy++) {
            const float4 q = *reinterpret_cast<const float4 *>(src + dy * row);
            v[2 * dy] = __floats2bfloat162_rn(s * q.x, s * q.y);
            v[2 * dy + 1] = __floats2bfloat162_rn(s * q.z, s * q.w);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(dz + i * 16);
        dst[0] = *reinterpret_cast<uint4 *>(&v[0]);
        dst[1] = *reinterpret_cast<uint4 *>(&v[4]);
    }
}

// 2x2 average pool, NHWC
__global__ void k_pool(const bf16 *__restrict__ in, bf16 *__restrict__ out, int B, int H, int W, int C)
{
    const int h = H / 2, w = W / 2;
    const size_t n = (size_t)B * h * w * C;
    GRID_STRIDE(i, n) {
        const int c = (int)(i % C);
        const size_t pix = i / C;
        const int x = (int)(pix % w), y = (int)((pix / w) % h);
        const size_t b = pix / ((size_t)w * h);
        const bf16 *s = in + ((b * H + 2 * y) * W + 2 * x) * C + c;
        const float v = __bfloat162float(s[0]) + __bfloat162float(s[C]) + __bfloat162float(s[(size_t)W * C]) +
                        __bfloat162float(s[(size_t)W * C + C]);
        out[i] = __float2bfloat16(0.25f * v);
    }
}

// pool backward: d_in[2y+i][2x+j] (+)= d_out[y][x] / 4 ; accumulate into an FP32 buffer
__global__ void k_pool_grad(const float *__restrict__ dout, float *__restrict__ din, int B, int H, int W, int C)
{
    const size_t n = (size_t)B * H * W * C;  // over the full-resolution gradient
    GRID_STRIDE(i, n) {
        const int c = (int)(i % C);
        const size_t pix = i / C;
        const int x = (int)(pix % W), y = (int)((pix / W) % H);
        const size_t b = pix / ((size_t)W * H);
        din[i] += 0.25f * dout[((b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
    }
}

// out = up2(low) + skip  (nearest), NHWC bf16
__global__ void k_up_add(const bf16 *__restrict__ low, const bf16 *__restrict__ skip, bf16 *__restrict__ out, int B,
                         int H, int W, int C)
{
    const size_t n = (size_t)B * H * W * C;
    GRID_STRIDE(i, n) {
        const int c = (int)(i % C);
        const size_t pix = i / C;
        const int x = (int)(pix % W), y = (int)((pix / W) % H);
        const size_t b = pix / ((size_t)W * H);
        out[i] = __float2bfloat16(__bfloat162float(low[((b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]) +
                                  __bfloat162float(skip[i]));
    }
}

// up backward into the low-resolution FP32 gradient: d_low[y][x] = sum of the 2x2 block
__global__ void k_up_grad(const float *__restrict__ dout, float *__restrict__ dlow, int B, int H, int W, int C)
{
    const int h = H / 2, w = W / 2;
    const size_t n = (size_t)B * h * w * C;
    GRID_STRIDE(i, n) {
        const int c = (int)(i % C);
        const size_t pix = i / C;
        const int x = (int)(pix % w), y = (int)((pix / w) % h);
        const size_t b = pix / ((size_t)w * h);
        const float *s = dout + ((b * H + 2 * y) * W + 2 * x) * C + c;
        dlow[i] = s[0] + s[C] + s[(size_t)W * C] + s[(size_t)W * C + C];
    }
}

// dz = dy * (y > 0) as bf16 (y = the layer's ReLU output), dy FP32
__global__ void k_relu_grad(const float *__restrict__ dy, const bf16 *__restrict__ y, bf16 *__restrict__ dz, size_t n)
{
    GRID_STRIDE(i, n) dz[i] = __float2bfloat16(__bfloat162float(y[i]) > 0.f ? dy[i] : 0.f);
}

__global__ void k_bf16_to_f32_add(const bf16 *__restrict__ a, float *__restrict__ out, size_t n)
{
    GRID_STRIDE(i, n) out[i] += __bfloat162float(a[i]);
}

__global__ void k_f32_to_bf16(const float *__restrict__ a, bf16 *__restrict__ out, size_t n)
{
    GRID_STRIDE(i, n) out[i] = __float2bfloat16(a[i]);
}

// db[c] += sum_p dz[p][c]
__global__ void k_bias_grad(const bf16 *__restrict__ dz, float *__restrict__ db, size_t npix, int C)
{
    const int c = threadIdx.x % C, lane_group = threadIdx.x / C, groups = blockDim.x / C;
    float acc = 0.f;
    for (size_t p = (size_t)blockIdx.x * groups + lane_group; p < npix; p += (size_t)gridDim.x * groups)
        acc += __bfloat162float(dz[p * C + c]);
    atomicAdd(db + c, acc);
}

// loss = mean (pred - target)^2 ; d_pred = 2 (pred - target) / n
__global__ void k_mse(const float *__restrict__ pred, const float *__restrict__ target, float *__restrict__ dpred,
                      double *__restrict__ loss, size_t n)
{
    double acc = 0.0;
    const float inv = 2.0f / (float)n;
    GRID_STRIDE(i, n) {
        const float d = pred[i] - target[i];
        dpred[i] = inv * d;
        acc += (double)d * d;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc / (double)n);
}

// Adam on FP32 master weights; writes the BF16 forward weights [Cout][9][Cin]
// and the data-gradient weights [Cin][9][Cout] (taps flipped).
__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v, const float *__restrict__ g,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2, bf16 *__restrict__ wf,
                       bf16 *__restrict__ wd, int Cout, int Cin)
{
    GRID_STRIDE(i, n) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        w[i] = wi;
        if (wf) {
            const int ci = (int)(i % Cin), t = (int)((i / Cin) % 9), co = (int)(i / ((size_t)9 * Cin));
            wf[i] = __float2bfloat16(wi);
            wd[((size_t)ci * 9 + (8 - t)) * Cout + co] = __float2bfloat16(wi);
        }
    }
}

__global__ void k_cast_weights(const float *__restrict__ w, size_t n, bf16 *__restrict__ wf, bf16 *__restrict__ wd,
                               int Cout, int Cin)
{
    GRID_STRIDE(i, n) {
        const int ci = (int)(i % Cin), t = (int)((i / Cin) % 9), co = (int)(i / ((size_t)9 * Cin));
        wf[i] = __float2bfloat16(w[i]);
        wd[((size_t)ci * 9 + (8 - t)) * Cout + co] = __float2bfloat16(w[i]);
    }
}

}  // namespace ufob

using namespace ufob;

namespace {

struct Layer {
    int cin, cout, relu;
    size_t nw() const { return (size_t)cout * 9 * cin; }
    DevBuf w, b, m_w, v_w, m_b, v_b, gw, gb, wf, wd;  // master FP32, Adam moments, gradients, BF16 copies
};

// Layer table: enc1..enc4, dec3, dec2, dec1, out
const int kLayers[8][3] = {{16, 32, 1}, {32, 64, 1}, {64, 128, 1}, {128, 256, 1},
                           {256, 128, 1}, {128, 64, 1}, {64, 32, 1}, {32, 16, 0}};

}  // namespace

// Inference path (cnn_fast.cu): persistent tcgen05 convolutions over padded
// channel-group activations, with per-tap BF16 weight tiles.
namespace ufob {
void *cnn_fast_create();
void cnn_fast_destroy(void *);
ufob_status cnn_fast_weights(void *f, const float *const *w, const int (*shape)[2], cudaStream_t s);
ufob_status cnn_fast_forward(void *f, const float *const *bias, const float *fbp, float *out, int B, int H, int W,
                             float scale, cudaStream_t s);
}  // namespace ufob

struct ufob_cnn {
    Layer L[8];
    float scale = 1.f;  // input/output scaling s
    int step = 0;
    void *fast = nullptr;     // inference workspace and weight tiles
    bool fast_dirty = true;   // weight tiles stale after a parameter change
    ~ufob_cnn() { cnn_fast_destroy(fast); }
    int B = 0, H = 0, W = 0;  // training workspace shape (quarter resolution)
    // activations (bf16) and gradient buffers (f32)
    DevBuf x0, e1, p1, e2, p2, e3, p3, e4, d3, u3, d2, u2, d1, u1, o, pred, dpred, loss;
    DevBuf g_a, g_b, g_c, dz;  // scratch gradients
    DevBuf g_e1, g_e2, g_e3;   // FP32 gradients of the skip tensors
};

static ufob_status cnn_workspace(ufob_cnn *c, int B, int H, int W)
{
    if (c->B == B && c->H == H && c->W == W) return UFOB_OK;
    const size_t P0 = (size_t)B * H * W, P1 = P0 / 4, P2 = P1 / 4, P3 = P2 / 4;
    UFOB_TRY(c->x0.ensure(P0 * 16 * 2));
    UFOB_TRY(c->e1.ensure(P0 * 32 * 2));
    UFOB_TRY(c->p1.ensure(P1 * 32 * 2));
    UFOB_TRY(c->e2.ensure(P1 * 64 * 2));
    UFOB_TRY(c->p2.ensure(P2 * 64 * 2));
    UFOB_TRY(c->e3.ensure(P2 * 128 * 2));
    UFOB_TRY(c->p3.ensure(P3 * 128 * 2));
    UFOB_TRY(c->e4.ensure(P3 * 256 * 2));
    UFOB_TRY(c->d3.ensure(P3 * 128 * 2));
    UFOB_TRY(c->u3.ensure(P2 * 128 * 2));
    UFOB_TRY(c->d2.ensure(P2 * 64 * 2));
    UFOB_TRY(c->u2.ensure(P1 * 64 * 2));
    UFOB_TRY(c->d1.ensure(P1 * 32 * 2));
    UFOB_TRY(c->u1.ensure(P0 * 32 * 2));
    UFOB_TRY(c->o.ensure(P0 * 16 * 4));
    UFOB_TRY(c->pred.ensure(P0 * kS * kS * 4));
    UFOB_TRY(c->dpred.ensure(P0 * kS * kS * 4));
    UFOB_TRY(c->loss.ensure(sizeof(double)));
    const size_t big = P0 * 32 * 4;  // largest FP32 gradient (256^2 x 32)
    UFOB_TRY(c->g_a.ensure(big));
    UFOB_TRY(c->g_b.ensure(big));
    UFOB_TRY(c->g_c.ensure(big));
    UFOB_TRY(c->dz.ensure(P0 * 32 * 2));
    UFOB_TRY(c->g_e1.ensure(P0 * 32 * 4));
    UFOB_TRY(c->g_e2.ensure(P1 * 64 * 4));
    UFOB_TRY(c->g_e3.ensure(P2 * 128 * 4));
    c->B = B;
    c->H = H;
    c->W = W;
    return UFOB_OK;
}

#define LAUNCH(kernel, n, ...)                                             \
    do {                                                                   \
        kernel<<<blocks_for(n), 256, 0, s>>>(__VA_ARGS__);                 \
        UFOB_CUDA_TRY(cudaGetLastError());                                 \
        note_launch();                                                     \
    } while (0)

static ufob_status cnn_forward(ufob_cnn *c, const float *fbp, float *out, int B, int H2, int W2, cudaStream_t s)
{
    const int H = H2 / kS, W = W2 / kS;
    UFOB_TRY(cnn_workspace(c, B, H, W));
    auto bw = [&](DevBuf &d) { return d.as<bf16>(); };
    Layer *L = c->L;
    const size_t P0 = (size_t)B * H * W;
    LAUNCH(k_unshuffle_in, P0, fbp, bw(c->x0), B, H, W, 1.f / c->scale);
    UFOB_TRY(conv3x3_launch(bw(c->x0), L[0].wf.as<bf16>(), L[0].b.as<float>(), nullptr, bw(c->e1), nullptr, B, H, W, 16,
                            32, 1, s));
    LAUNCH(k_pool, P0 / 4 * 32, bw(c->e1), bw(c->p1), B, H, W, 32);
    UFOB_TRY(conv3x3_launch(bw(c->p1), L[1].wf.as<bf16>(), L[1].b.as<float>(), nullptr, bw(c->e2), nullptr, B, H / 2,
                            W / 2, 32, 64, 1, s));
    LAUNCH(k_pool, P0 / 16 * 64, bw(c->e2), bw(c->p2), B, H / 2, W / 2, 64);
    UFOB_TRY(conv3x3_launch(bw(c->p2), L[2].wf.as<bf16>(), L[2].b.as<float>(), nullptr, bw(c->e3), nullptr, B, H / 4,
                            W / 4, 64, 128, 1, s));
    LAUNCH(k_pool, P0 / 64 * 128, bw(c->e3), bw(c->p3), B, H / 4, W / 4, 128);
    UFOB_TRY(conv3x3_launch(bw(c->p3), L[3].wf.as<bf16>(), L[3].b.as<float>(), nullptr, bw(c->e4), nullptr, B, H / 8,
                            W / 8, 128, 256, 1, s));
    UFOB_TRY(conv3x3_launch(bw(c->e4), L[4].wf.as<bf16>(), L[4].b.as<float>(), nullptr, bw(c->d3), nullptr, B, H / 8,
                            W / 8, 256, 128, 1, s));
    LAUNCH(k_up_add, P0 / 16 * 128, bw(c->d3), bw(c->e3), bw(c->u3), B, H / 4, W / 4, 128);
    UFOB_TRY(conv3x3_launch(bw(c->u3), L[5].wf.as<bf16>(), L[5].b.as<float>(), nullptr, bw(c->d2), nullptr, B, H / 4,
                            W / 4, 128, 64, 1, s));
    LAUNCH(k_up_add, P0 / 4 * 64, bw(c->d2), bw(c->e2), bw(c->u2), B, H / 2, W / 2, 64);
    UFOB_TRY(conv3x3_launch(bw(c->u2), L[6].wf.as<bf16>(), L[6].b.as<float>(), nullptr, bw(c->d1), nullptr, B, H / 2,
                            W / 2, 64, 32, 1, s));
    LAUNCH(k_up_add, P0 * 32, bw(c->d1), bw(c->e1), bw(c->u1), B, H, W, 32);
    UFOB_TRY(conv3x3_launch(bw(c->u1), L[7].wf.as<bf16>(), L[7].b.as<float>(), nullptr, nullptr, c->o.as<float>(), B, H,
                            W, 32, 16, 0, s));
    LAUNCH(k_shuffle_out, P0 * kS * kS, c->o.as<float>(), fbp, out, B, H, W, c->scale);
    return UFOB_OK;
}

// Backward of one conv layer: dy (FP32, at the layer output) -> dz (bf16, masked by ReLU),
// weight/bias gradients, and optionally dx (FP32) via the data-gradient convolution.
static ufob_status conv_backward(ufob_cnn *c, Layer &l, const bf16 *x, const bf16 *y, const float *dy, float *dx,
                                 int B, int H, int W, cudaStream_t s)
{
    const size_t n = (size_t)B * H * W * l.cout;
    bf16 *dz = c->dz.as<bf16>();
    if (l.relu) {
        LAUNCH(k_relu_grad, n, dy, y, dz, n);
    } else {
        LAUNCH(k_f32_to_bf16, n, dy, dz, n);
    }
    UFOB_TRY(conv3x3_wgrad_launch(x, dz, l.gw.as<float>(), B, H, W, l.cin, l.cout, s));
    const int threads = 256 / l.cout * l.cout;
    k_bias_grad<<<num_sms() * 2, threads, 0, s>>>(dz, l.gb.as<float>(), (size_t)B * H * W, l.cout);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    if (dx) UFOB_TRY(conv3x3_launch(dz, l.wd.as<bf16>(), nullptr, nullptr, nullptr, dx, B, H, W, l.cout, l.cin, 0, s));
    return UFOB_OK;
}

static ufob_status cnn_backward(ufob_cnn *c, int B, cudaStream_t s)
{
    const int H = c->H, W = c->W;
    const size_t P0 = (size_t)B * H * W;
    auto bw = [&](DevBuf &d) { return d.as<bf16>(); };
    Layer *L = c->L;
    float *ga = c->g_a.as<float>(), *gb = c->g_b.as<float>(), *gc = c->g_c.as<float>();
    bf16 *dzo = c->dz.as<bf16>();
    // out layer: gradient at o from d_pred
    LAUNCH(k_shuffle_out_grad, P0, c->dpred.as<float>(), dzo, B, H, W, c->scale);
    UFOB_TRY(conv3x3_wgrad_launch(bw(c->u1), dzo, L[7].gw.as<float>(), B, H, W, 32, 16, s));
    k_bias_grad<<<num_sms() * 2, 256, 0, s>>>(dzo, L[7].gb.as<float>(), P0, 16);
    UFOB_CUDA_TRY(cudaGetLastError());
    UFOB_TRY(conv3x3_launch(dzo, L[7].wd.as<bf16>(), nullptr, nullptr, nullptr, ga, B, H, W, 16, 32, 0, s));  // d u1
    // u1 = up(d1) + e1
    UFOB_CUDA_TRY(cudaMemcpyAsync(c->g_e1.ptr, ga, P0 * 32 * 4, cudaMemcpyDeviceToDevice, s));
    LAUNCH(k_up_grad, P0 / 4 * 32, ga, gb, B, H, W, 32);  // d d1
    UFOB_TRY(conv_backward(c, L[6], bw(c->u2), bw(c->d1), gb, ga, B, H / 2, W / 2, s));  // d u2 -> ga
    UFOB_CUDA_TRY(cudaMemcpyAsync(c->g_e2.ptr, ga, P0 / 4 * 64 * 4, cudaMemcpyDeviceToDevice, s));
    LAUNCH(k_up_grad, P0 / 16 * 64, ga, gb, B, H / 2, W / 2, 64);  // d d2
    UFOB_TRY(conv_backward(c, L[5], bw(c->u3), bw(c->d2), gb, ga, B, H / 4, W / 4, s));  // d u3
    UFOB_CUDA_TRY(cudaMemcpyAsync(c->g_e3.ptr, ga, P0 / 16 * 128 * 4, cudaMemcpyDeviceToDevice, s));
    LAUNCH(k_up_grad, P0 / 64 * 128, ga, gb, B, H / 4, W / 4, 128);  // d d3
    UFOB_TRY(conv_backward(c, L[4], bw(c->e4), bw(c->d3), gb, ga, B, H / 8, W / 8, s));  // d e4
    UFOB_TRY(conv_backward(c, L[3], bw(c->p3), bw(c->e4), ga, gb, B, H / 8, W / 8, s));  // d p3
    // e3 gradient = skip part + pool backward of d p3
    LAUNCH(k_pool_grad, P0 / 16 * 128, gb, c->g_e3.as<float>(), B, H / 4, W / 4, 128);
    UFOB_TRY(conv_backward(c, L[2], bw(c->p2), bw(c->e3), c->g_e3.as<float>(), gc, B, H / 4, W / 4, s));  // d p2
    LAUNCH(k_pool_grad, P0 / 4 * 64, gc, c->g_e2.as<float>(), B, H / 2, W / 2, 64);
    UFOB_TRY(conv_backward(c, L[1], bw(c->p1), bw(c->e2), c->g_e2.as<float>(), gc, B, H / 2, W / 2, s));  // d p1
    LAUNCH(k_pool_grad, P0 * 32, gc, c->g_e1.as<float>(), B, H, W, 32);
    UFOB_TRY(conv_backward(c, L[0], bw(c->x0), bw(c->e1), c->g_e1.as<float>(), nullptr, B, H, W, s));
    return UFOB_OK;
}

extern "C" ufob_status ufob_cnn_create(uint64_t seed, float scale, ufob_cnn **out)
{
    if (!out) return fail(UFOB_ERR_INVALID, "cnn_create: out is NULL");
    UFOB_TRY(ensure_device());
    ufob_cnn *c = new ufob_cnn;
    c->fast = cnn_fast_create();
    c->scale = scale > 0.f ? scale : 1.f;
    std::mt19937_64 rng(seed);
    for (int i = 0; i < 8; i++) {
        Layer &l = c->L[i];
        l.cin = kLayers[i][0];
        l.cout = kLayers[i][1];
        l.relu = kLayers[i][2];
        const size_t nw = l.nw();
        // He initialisation; the output layer starts small so the network starts near identity
        const double fan_in = 9.0 * l.cin;
        std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / fan_in) * (i == 7 ? 0.1 : 1.0));
        std::vector<float> w(nw);
        for (size_t k = 0; k < nw; k++) w[k] = (float)nd(rng);
        ufob_status st = UFOB_OK;
        if (st == UFOB_OK) st = l.w.ensure(nw * 4);
        if (st == UFOB_OK) st = l.m_w.ensure(nw * 4);
        if (st == UFOB_OK) st = l.v_w.ensure(nw * 4);
        if (st == UFOB_OK) st = l.gw.ensure(nw * 4);
        if (st == UFOB_OK) st = l.b.ensure(l.cout * 4);
        if (st == UFOB_OK) st = l.m_b.ensure(l.cout * 4);
        if (st == UFOB_OK) st = l.v_b.ensure(l.cout * 4);
        if (st == UFOB_OK) st = l.gb.ensure(l.cout * 4);
        if (st == UFOB_OK) st = l.wf.ensure(nw * 2);
        if (st == UFOB_OK) st = l.wd.ensure(nw * 2);
        if (st != UFOB_OK) {
            delete c;
            return st;
        }
        cudaMemcpy(l.w.ptr, w.data(), nw * 4, cudaMemcpyHostToDevice);
        cudaMemset(l.m_w.ptr, 0, nw * 4);
        cudaMemset(l.v_w.ptr, 0, nw * 4);
        cudaMemset(l.b.ptr, 0, l.cout * 4);
        cudaMemset(l.m_b.ptr, 0, l.cout * 4);
        cudaMemset(l.v_b.ptr, 0, l.cout * 4);
        k_cast_weights<<<blocks_for(nw), 256>>>(l.w.as<float>(), nw, l.wf.as<bf16>(), l.wd.as<bf16>(), l.cout, l.cin);
        note_launch();
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cnn_create");
    }
    *out = c;
    return UFOB_OK;
}

extern "C" void ufob_cnn_destroy(ufob_cnn *c) { delete c; }

static ufob_status check_shape(int B, int H2, int W2)
{
    if (B < 1 || H2 % (8 * kS) || W2 % (8 * kS) || H2 < 8 * kS || W2 < 8 * kS)
        return fail(UFOB_ERR_INVALID, "cnn: image sides must be positive multiples of 32");
    return UFOB_OK;
}

extern "C" ufob_status ufob_cnn_forward(ufob_cnn *c, const float *d_fbp, float *d_out, int B, int H, int W,
                                        void *stream)
{
    if (!c || !d_fbp || !d_out) return fail(UFOB_ERR_INVALID, "cnn_forward: NULL argument");
    UFOB_TRY(check_shape(B, H, W));
    cudaStream_t s = (cudaStream_t)stream;
    if (c->fast_dirty) {
        const float *w[8];
        int shape[8][2];
        for (int i = 0; i < 8; i++) {
            w[i] = c->L[i].w.as<float>();
            shape[i][0] = c->L[i].cin;
            shape[i][1] = c->L[i].cout;
        }
        UFOB_TRY(cnn_fast_weights(c->fast, w, shape, s));
        c->fast_dirty = false;
    }
    const float *bias[8];
    for (int i = 0; i < 8; i++) bias[i] = c->L[i].b.as<float>();
    return cnn_fast_forward(c->fast, bias, d_fbp, d_out, B, H / kS, W / kS, c->scale, s);
}

// The training path's forward pass (NHWC kernels of cnn_conv.cu), for checks of the inference path.
extern "C" ufob_status ufob_cnn_forward_nhwc(ufob_cnn *c, const float *d_fbp, float *d_out, int B, int H, int W,
                                             void *stream)
{
    if (!c || !d_fbp || !d_out) return fail(UFOB_ERR_INVALID, "cnn_forward_nhwc: NULL argument");
    UFOB_TRY(check_shape(B, H, W));
    return cnn_forward(c, d_fbp, d_out, B, H, W, (cudaStream_t)stream);
}

extern "C" ufob_status ufob_cnn_train_step(ufob_cnn *c, const float *d_fbp, const float *d_target, int B, int H,
                                           int W, float lr, double *loss_out, void *stream)
{
    if (!c || !d_fbp || !d_target) return fail(UFOB_ERR_INVALID, "cnn_train_step: NULL argument");
    UFOB_TRY(check_shape(B, H, W));
    cudaStream_t s = (cudaStream_t)stream;
    // size the workspace before taking any of its pointers (a shape change reallocates it)
    UFOB_TRY(cnn_workspace(c, B, H / kS, W / kS));
    UFOB_TRY(cnn_forward(c, d_fbp, c->pred.as<float>(), B, H, W, s));
    const size_t n = (size_t)B * H * W;
    UFOB_CUDA_TRY(cudaMemsetAsync(c->loss.ptr, 0, sizeof(double), s));
    LAUNCH(k_mse, n, c->pred.as<float>(), d_target, c->dpred.as<float>(), c->loss.as<double>(), n);
    for (auto &l : c->L) {
        UFOB_CUDA_TRY(cudaMemsetAsync(l.gw.ptr, 0, l.nw() * 4, s));
        UFOB_CUDA_TRY(cudaMemsetAsync(l.gb.ptr, 0, l.cout * 4, s));
    }
    UFOB_TRY(cnn_backward(c, B, s));
    c->step++;
    c->fast_dirty = true;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f / (1.f - powf(b1, (float)c->step)), c2 = 1.f / (1.f - powf(b2, (float)c->step));
    for (auto &l : c->L) {
        const size_t nw = l.nw();
        LAUNCH(k_adam, nw, l.w.as<float>(), l.m_w.as<float>(), l.v_w.as<float>(), l.gw.as<float>(), nw, lr, b1, b2,
               eps, c1, c2, l.wf.as<bf16>(), l.wd.as<bf16>(), l.cout, l.cin);
        LAUNCH(k_adam, (size_t)l.cout, l.b.as<float>(), l.m_b.as<float>(), l.v_b.as<float>(), l.gb.as<float>(),
               (size_t)l.cout, lr, b1, b2, eps, c1, c2, (bf16 *)nullptr, (bf16 *)nullptr, l.cout, l.cin);
    }
    if (loss_out) {
        UFOB_CUDA_TRY(cudaMemcpyAsync(loss_out, c->loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
        UFOB_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return UFOB_OK;
}

// State vectors, one FP32 vector each, per layer weights [Cout][9][Cin] then
// bias [Cout]: which = 0 parameters, 1 gradients of the last train step,
// 2 Adam first moments, 3 Adam second moments.
extern "C" uint64_t ufob_cnn_num_params(void)
{
    uint64_t n = 0;
    for (int i = 0; i < 8; i++) n += (uint64_t)kLayers[i][1] * 9 * kLayers[i][0] + kLayers[i][1];
    return n;
}

static void state_bufs(Layer &l, int which, DevBuf *&w, DevBuf *&b)
{
    switch (which) {
    case 0: w = &l.w; b = &l.b; break;
    case 1: w = &l.gw; b = &l.gb; break;
    case 2: w = &l.m_w; b = &l.m_b; break;
    default: w = &l.v_w; b = &l.v_b; break;
    }
}

extern "C" ufob_status ufob_cnn_get_state(ufob_cnn *c, int which, float *host, uint64_t n)
{
    if (!c || !host || n < ufob_cnn_num_params()) return fail(UFOB_ERR_INVALID, "cnn_get_state: bad buffer");
    if (which < 0 || which > 3) return fail(UFOB_ERR_INVALID, "cnn_get_state: which must be 0..3");
    UFOB_CUDA_TRY(cudaDeviceSynchronize());
    size_t off = 0;
    for (auto &l : c->L) {
        DevBuf *w, *b;
        state_bufs(l, which, w, b);
        UFOB_CUDA_TRY(cudaMemcpy(host + off, w->ptr, l.nw() * 4, cudaMemcpyDeviceToHost));
        off += l.nw();
        UFOB_CUDA_TRY(cudaMemcpy(host + off, b->ptr, l.cout * 4, cudaMemcpyDeviceToHost));
        off += l.cout;
    }
    return UFOB_OK;
}

extern "C" ufob_status ufob_cnn_set_state(ufob_cnn *c, int which, const float *host, uint64_t n)
{
    if (!c || !host || n < ufob_cnn_num_params()) return fail(UFOB_ERR_INVALID, "cnn_set_state: bad buffer");
    if (which < 0 || which > 3 || which == 1) return fail(UFOB_ERR_INVALID, "cnn_set_state: which must be 0, 2 or 3");
    UFOB_CUDA_TRY(cudaDeviceSynchronize());
    size_t off = 0;
    for (auto &l : c->L) {
        DevBuf *w, *b;
        state_bufs(l, which, w, b);
        UFOB_CUDA_TRY(cudaMemcpy(w->ptr, host + off, l.nw() * 4, cudaMemcpyHostToDevice));
        off += l.nw();
        UFOB_CUDA_TRY(cudaMemcpy(b->ptr, host + off, l.cout * 4, cudaMemcpyHostToDevice));
        off += l.cout;
        if (which == 0) {
            c->fast_dirty = true;
            k_cast_weights<<<blocks_for(l.nw()), 256>>>(l.w.as<float>(), l.nw(), l.wf.as<bf16>(), l.wd.as<bf16>(),
                                                        l.cout, l.cin);
            UFOB_CUDA_TRY(cudaGetLastError());
            note_launch();
        }
    }
    UFOB_CUDA_TRY(cudaDeviceSynchronize());
    return UFOB_OK;
}

// Adam step counter (bias correction), saved and restored with the moments.
extern "C" int64_t ufob_cnn_get_step(const ufob_cnn *c) { return c ? c->step : -1; }
extern "C" ufob_status ufob_cnn_set_step(ufob_cnn *c, int64_t step)
{
    if (!c || step < 0) return fail(UFOB_ERR_INVALID, "cnn_set_step: bad argument");
    c->step = (int)step;
    return UFOB_OK;
}
