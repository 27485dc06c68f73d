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

}  // namespace ufob

using namespace ufob;

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
    UFOB_CUDA_TRY(cudaStreamSynchronize(s));  // `d` is freed on return
    return UFOB_OK;
}
