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

// Ray-marching forward projector, src/kernels/forwardproject.cl:24-58: for
// detector pixel idx and angle idy*step, walk unit steps along the ray through
// the circle of radius min(axis, W - axis) and sum linear samples (texel
// centres at +0.5, zero outside the image).  Exact FP32 weights; the angle's
// sin/cos are taken in FP64.
__global__ void k_forwardproject(const float *__restrict__ img, uint32_t W, uint32_t n_angles, float axis,
                                 double step, float *__restrict__ sino)
{
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x, idy = blockIdx.y;
    if (idx >= W || idy >= n_angles) return;
    double sd, cd;
    sincos((double)idy * step, &sd, &cd);
    const float r = fminf(axis, (float)W - axis);
    const float d = (float)idx - axis + 0.5f;
    const float l = sqrtf(4.0f * r * r - 4.0f * d * d);  // NaN outside the circle: no samples
    float Dx = (float)cd, Dy = (float)sd;
    const float nrm = rsqrtf(Dx * Dx + Dy * Dy);
    Dx *= nrm;
    Dy *= nrm;
    const float Nx = Dy, Ny = -Dx;
    float sx = d * Dx - l / 2.0f * Nx + axis, sy = d * Dy - l / 2.0f * Ny + axis;
    float sum = 0.f;
    for (int i = 0; (float)i < l; i++) {
        const float u = sx - 0.5f, v = sy - 0.5f;
        const float fu = floorf(u), fv = floorf(v);
        const float a = u - fu, b = v - fv;
        const int i0 = (int)fu, j0 = (int)fv;
        float t00 = 0.f, t10 = 0.f, t01 = 0.f, t11 = 0.f;
        if (j0 >= 0 && j0 < (int)W) {
            if (i0 >= 0 && i0 < (int)W) t00 = __ldg(img + (size_t)j0 * W + i0);
            if (i0 + 1 >= 0 && i0 + 1 < (int)W) t10 = __ldg(img + (size_t)j0 * W + i0 + 1);
        }
        if (j0 + 1 >= 0 && j0 + 1 < (int)W) {
            if (i0 >= 0 && i0 < (int)W) t01 = __ldg(img + (size_t)(j0 + 1) * W + i0);
            if (i0 + 1 >= 0 && i0 + 1 < (int)W) t11 = __ldg(img + (size_t)(j0 + 1) * W + i0 + 1);
        }
        sum += (1.f - a) * (1.f - b) * t00 + a * (1.f - b) * t10 + (1.f - a) * b * t01 + a * b * t11;
        sx += Nx;
        sy += Ny;
    }
    sino[(size_t)idy * W + idx] = sum;
}

// Rasterise ellipse phantoms (cx, cy, a, b, phi, rho) at pixel centres with
// ss x ss supersampling into a stack [n_images][N][N]; ellipse list i is
// ell[offsets[i] .. offsets[i+1]).
__global__ void k_ellipse_images(const Ellipse *__restrict__ ell, const uint32_t *__restrict__ offsets, uint32_t N,
                                 double axis, double scale, int ss, float *__restrict__ out)
{
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, im = blockIdx.z;
    if (x >= N) return;
    const uint32_t e0 = offsets[im], e1 = offsets[im + 1];
    double acc = 0.0;
    for (int sy = 0; sy < ss; sy++)
        for (int sx = 0; sx < ss; sx++) {
            const double px = ((double)x + (sx + 0.5) / ss - axis) / scale;
            const double py = ((double)y + (sy + 0.5) / ss - axis) / scale;
            for (uint32_t e = e0; e < e1; e++) {
                const Ellipse q = ell[e];
                double sp, cp;
                sincos(q.phi, &sp, &cp);
                const double dx = px - q.cx, dy = py - q.cy;
                const double u = dx * cp + dy * sp, v = -dx * sp + dy * cp;
                if (u * u / (q.a * q.a) + v * v / (q.b * q.b) <= 1.0) acc += q.rho;
            }
        }
    out[((size_t)im * N + y) * N + x] = (float)(acc / (ss * ss));
}

}  // namespace ufob

using namespace ufob;

extern "C" ufob_status ufob_forwardproject(const float *d_slice, uint32_t width, uint32_t n_angles, double axis_pos,
                                           double angle_step, float *d_sino, void *stream)
{
    if (!d_slice || !d_sino) return fail(UFOB_ERR_INVALID, "forwardproject: NULL argument");
    if (!width || !n_angles) return fail(UFOB_ERR_INVALID, "forwardproject: empty size");
    UFOB_TRY(ensure_device());
    dim3 blk(128), grd((width + 127) / 128, n_angles);
    k_forwardproject<<<grd, blk, 0, (cudaStream_t)stream>>>(d_slice, width, n_angles, (float)axis_pos, angle_step,
                                                            d_sino);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    return UFOB_OK;
}

extern "C" ufob_status ufob_phantom_images(const double *h_ellipses, const uint32_t *h_offsets, uint32_t n_images,
                                           uint32_t N, double axis, double scale, int supersample, float *d_out,
                                           void *stream)
{
    if (!h_ellipses || !h_offsets || !d_out) return fail(UFOB_ERR_INVALID, "phantom_images: NULL argument");
    if (supersample < 1 || supersample > 8) return fail(UFOB_ERR_INVALID, "phantom_images: supersample in [1, 8]");
    UFOB_TRY(ensure_device());
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t n_ell = h_offsets[n_images];
    DevBuf de, doff;
    UFOB_TRY(de.ensure(sizeof(Ellipse) * (n_ell ? n_ell : 1)));
    UFOB_TRY(doff.ensure(sizeof(uint32_t) * (n_images + 1)));
    UFOB_CUDA_TRY(cudaMemcpyAsync(de.ptr, h_ellipses, sizeof(Ellipse) * n_ell, cudaMemcpyHostToDevice, s));
    UFOB_CUDA_TRY(cudaMemcpyAsync(doff.ptr, h_offsets, sizeof(uint32_t) * (n_images + 1), cudaMemcpyHostToDevice, s));
    k_ellipse_images<<<dim3((N + 127) / 128, N, n_images), 128, 0, s>>>(de.as<Ellipse>(), doff.as<uint32_t>(), N, axis,
                                                                        scale, supersample, d_out);
    UFOB_CUDA_TRY(cudaGetLastError());
    note_launch();
    UFOB_CUDA_TRY(cudaStreamSynchronize(s));  // the staging buffers are freed on return
    return UFOB_OK;
}

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
