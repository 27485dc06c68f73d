// Micro-benchmarks of the two on-chip ceilings that bound voxel-driven
// backprojection: shared-memory load bandwidth (32-bit loads, one wavefront of
// 128 bytes per warp instruction when conflict-free) and FP32 FMA throughput.
// They report what this device sustains, for roofline fractions.
#include "ufob_internal.h"

namespace ufob {

__global__ void __launch_bounds__(1024) k_smem_bw(int iters, float *sink)
{
    __shared__ float buf[8192];
    for (int i = threadIdx.x; i < 8192; i += blockDim.x) buf[i] = (float)i;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
    uint32_t off = (threadIdx.x >> 5) * 32 + lane;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint32_t base = (off + (uint32_t)(k * 256)) & 8191u;
            acc0 += buf[base];
            acc1 += buf[base ^ 1024u];
            acc2 += buf[base ^ 2048u];
            acc3 += buf[base ^ 4096u];
        }
        off = (off + 37u * 32u) & 8191u;
    }
    if (acc0 + acc1 + acc2 + acc3 == -1.f) sink[threadIdx.x] = acc0;
}

__global__ void __launch_bounds__(512) k_fp32(int iters, float *sink)
{
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = threadIdx.x * 1e-9f + i;
    const float m = 0.9999f, c = 1e-7f;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 32; k++) {
#pragma unroll
            for (int i = 0; i < 8; i++) a[i] = fmaf(a[i], m, c);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; i++) s += a[i];
    if (s == -1.f) sink[threadIdx.x] = s;
}

}  // namespace ufob

using namespace ufob;

extern "C" ufob_status ufob_measure_peaks(double *smem_gbs, double *fp32_tflops)
{
    UFOB_TRY(ensure_device());
    DevBuf sink;
    UFOB_TRY(sink.ensure(4096 * sizeof(float)));
    cudaEvent_t e0, e1;
    UFOB_CUDA_TRY(cudaEventCreate(&e0));
    UFOB_CUDA_TRY(cudaEventCreate(&e1));
    const int sms = num_sms();
    float ms = 0.f;
    // shared memory: 4 loads x 16 per iteration per thread, 4 bytes each
    {
        const int blocks = sms * 2, threads = 1024, iters = 4000;
        k_smem_bw<<<blocks, threads>>>(10, sink.as<float>());
        UFOB_CUDA_TRY(cudaEventRecord(e0));
        k_smem_bw<<<blocks, threads>>>(iters, sink.as<float>());
        UFOB_CUDA_TRY(cudaEventRecord(e1));
        UFOB_CUDA_TRY(cudaEventSynchronize(e1));
        UFOB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        const double bytes = (double)blocks * threads * iters * 64.0 * 4.0;
        if (smem_gbs) *smem_gbs = bytes / (ms * 1e-3) / 1e9;
    }
    {
        const int blocks = sms * 4, threads = 512, iters = 20000;
        k_fp32<<<blocks, threads>>>(10, sink.as<float>());
        UFOB_CUDA_TRY(cudaEventRecord(e0));
        k_fp32<<<blocks, threads>>>(iters, sink.as<float>());
        UFOB_CUDA_TRY(cudaEventRecord(e1));
        UFOB_CUDA_TRY(cudaEventSynchronize(e1));
        UFOB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        const double flops = (double)blocks * threads * iters * 32.0 * 8.0 * 2.0;
        if (fp32_tflops) *fp32_tflops = flops / (ms * 1e-3) / 1e12;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    UFOB_CUDA_TRY(cudaGetLastError());
    return UFOB_OK;
}
