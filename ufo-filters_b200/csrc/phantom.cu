// Analytic parallel-beam projection of ellipse phantoms on the device: the
// engine's own synthetic-input generator (the same line-integral formula the
// CPU oracle uses for its known-answer tests).
#include <math.h>

#include "ufob_internal.h"

namespace ufob {

struct Ellipse {
    double cx, cy, a, b, phi, rho;
};

// sino[p][i] = scale * sum_e 2 rho a b sqrt(r2 - s^2) / r2, with
// t = (i + 0.5 - axis) / scale, s = t - (cx cos + cy sin),
// r2 = a^2 cos^2(theta - phi) + b^2 sin^2(theta - phi).
__global__ void k_ellipse_sinogram(const Ellipse *__restrict__ ell, uint32_t n, uint32_t W, uint32_t P, double step,
                                   double axis, double scale, float *__restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, p = blockIdx.y;
    if (i >= W || p >= P) return;
    const double theta = p * step;
    double s, c;
    sincos(theta, &s, &c);
    const double t = ((double)i + 0.5 - axis) / scale;
    double acc = 0.0;
    for (uint32_t e = 0; e < n; e++) {
        const Ellipse q = ell[e];
        const double sp = t - (q.cx * c + q.cy * s);
        double sa, ca;
        sincos(theta - q.phi, &sa, &ca);
        const double r2 = q.a * q.a * ca * ca + q.b * q.b * sa * sa;
        const double d = r2 - sp * sp;
        if (d > 0.0) acc += 2.0 * q.rho * q.a * q.b * sqrt(d) / r2;
    }
    out[(size_t)p * W + i] = (float)(acc * scale);
}

// Stack of parallel-beam sinograms of an ellipsoid phantom (rows cx, cy, cz,
// a, b, c, phi, rho; rotation phi about z).  Slice z (centre height
// (z + 0.5 - nz/2) / scale) cuts each ellipsoid in an ellipse with semi-axes
// scaled by sqrt(1 - ((z - cz) / c)^2); those ellipses are projected as above.
// One block per (angle, slice); the per-ellipse terms that do not depend on the
// detector bin are formed once per block in shared memory.
__global__ void k_ellipsoid_stack(const double *__restrict__ ell, uint32_t n, uint32_t W, uint32_t P, uint32_t nz,
                                  double step, double axis, double scale, float *__restrict__ out)
{
    __shared__ double s_off[64], s_r2[64], s_amp[64];
    __shared__ int s_n;
    const uint32_t p = blockIdx.x, z = blockIdx.y;
    const double theta = p * step;
    if (threadIdx.x == 0) {
        double s, c;
        sincos(theta, &s, &c);
        const double zu = ((double)z + 0.5 - 0.5 * nz) / scale;
        int m = 0;
        for (uint32_t e = 0; e < n && m < 64; e++) {
            const double *q = ell + 8 * e;
            const double dz = (zu - q[2]) / q[5];
            if (dz * dz >= 1.0) continue;
            const double f = sqrt(1.0 - dz * dz), a = q[3] * f, b = q[4] * f;
            double sa, ca;
            sincos(theta - q[6], &sa, &ca);
            s_off[m] = q[0] * c + q[1] * s;
            s_r2[m] = a * a * ca * ca + b * b * sa * sa;
            s_amp[m] = 2.0 * q[7] * a * b;
            m++;
        }
        s_n = m;
    }
    __syncthreads();
    const int m = s_n;
    for (uint32_t i = threadIdx.x; i < W; i += blockDim.x) {
        const double t = ((double)i + 0.5 - axis) / scale;
        double acc = 0.0;
        for (int e = 0; e < m; e++) {
            const double sp = t - s_off[e];
            const double d = s_r2[e] - sp * sp;
            if (d > 0.0) acc += s_amp[e] * sqrt(d) / s_r2[e];
        }
        out[((size_t)z * P + p) * W + i] = (float)(acc * scale);
    }
}

}  // namespace ufob

using namespace ufob;

extern "C" ufob_status ufob_phantom_stack(const double *h_ell, uint32_t n, uint32_t W, uint32_t P, uint32_t nz,
                                          double angle_step, double axis, double scale, float *d_sino, void *stream)
{
    if (!h_ell || !d_sino) return fail(UFOB_ERR_INVALID, "phantom_stack: NULL argument");
    if (n > 64) return fail(UFOB_ERR_INVALID, "phantom_stack: at most 64 ellipsoids");
    UFOB_TRY(ensure_device());
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf d;
    UFOB_TRY(d.ensure(sizeof(double) * 8 * (n ? n : 1)));
    UFOB_CUDA_TRY(cudaMemcpyAsync(d.ptr, h_ell, sizeof(double) * 8 * n, cudaMemcpyHostToDevice, s));
    k_ellipsoid_stack<<<dim3(P, nz), 256, 0, s>>>(d.as<double>(), n, W, P, nz, angle_step, axis, scale, d_sino);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    UFOB_CUDA_TRY(cudaStreamSynchronize(s));
    return UFOB_OK;
}

extern "C" ufob_status ufob_phantom_sinogram(const double *h_ell, uint32_t n, uint32_t W, uint32_t P,
                                             double angle_step, double axis, double scale, float *d_sino,
                                             void *stream)
{
    if (!h_ell || !d_sino) return fail(UFOB_ERR_INVALID, "phantom_sinogram: NULL argument");
    UFOB_TRY(ensure_device());
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf d;
    UFOB_TRY(d.ensure(sizeof(Ellipse) * (n ? n : 1)));
    UFOB_CUDA_TRY(cudaMemcpyAsync(d.ptr, h_ell, sizeof(Ellipse) * n, cudaMemcpyHostToDevice, s));
    dim3 blk(256), grd((W + 255) / 256, P);
    k_ellipse_sinogram<<<grd, blk, 0, s>>>(d.as<Ellipse>(), n, W, P, angle_step, axis, scale, d_sino);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    UFOB_CUDA_TRY(cudaStreamSynchronize(s));  // `d` is freed on return
    return UFOB_OK;
}
