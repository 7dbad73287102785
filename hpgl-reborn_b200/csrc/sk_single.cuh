// The single-system SK solve behind hpgl_simple_kriging_weights (misc.cu) and
// hpgl_b200_sk_weights_noalloc (noalloc.cu): SK weights for real coordinates
// with the analytic model (simple_kriging.cpp:67-87 via sk_kriging_weights_3
// on real_location_t), one CTA, FP64, the matrix in the caller's global memory.
#pragma once
#include "kernels.h"

namespace hb
{
// the analytic model of cov_model.h:146-183 on a real displacement, the
// transform applied in the reference's summation order (cov_model.h:63-77)
__device__ __forceinline__ double cov_real_dev(const DevModel &m, double v0, double v1, double v2)
{
    double acc = 0.0;
    for (int i = 0; i < 3; ++i)
    {
        double d = 0.0;
        d = __dadd_rn(d, __dmul_rn(v0, m.T[3 * i + 0]));
        d = __dadd_rn(d, __dmul_rn(v1, m.T[3 * i + 1]));
        d = __dadd_rn(d, __dmul_rn(v2, m.T[3 * i + 2]));
        acc = __dadd_rn(acc, __dmul_rn(d, d));
    }
    const double h = sqrt(acc);
    if (h < 0.0001) return m.sill;
    const double u = h / m.r0;
    if (m.type == 2) return (m.sill - m.nugget) * exp(-3.0 * (u * u));
    if (m.type == 1) return (m.sill - m.nugget) * exp((-3.0 * h) / m.r0);
    if (h > m.r0) return 0.0;
    return (m.sill - m.nugget) * (1.0 - (1.5 * h) / m.r0 + 0.5 * (u * u * u));
}

// Called by every thread of one CTA. pts = centre (3) | xs | ys | zs (n
// each); A has room for n x n doubles and w for n. Builds A and b, factors
// A = L L^T (right-looking, rows of L in A) and, in thread 0, solves for the
// weights into w. Returns, in every thread, true when a pivot was not positive.
__device__ __forceinline__ bool sk_single_solve(const DevModel &m, const double *__restrict__ pts, int n,
                                                double *__restrict__ A, double *__restrict__ w)
{
    const double cx = pts[0], cy = pts[1], cz = pts[2];
    const double *xs = pts + 3, *ys = xs + n, *zs = ys + n;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x)
    {
        const int i = e / n, j = e % n;
        A[e] = cov_real_dev(m, xs[i] - xs[j], ys[i] - ys[j], zs[i] - zs[j]);
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] = cov_real_dev(m, xs[i] - cx, ys[i] - cy, zs[i] - cz);
    __syncthreads();
    bool fail = false;
    for (int j = 0; j < n; ++j)
    {
        const double d = A[(size_t)j * n + j];
        if (!(d > 0.0)) fail = true;
        const double ljj = sqrt(d);
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + j] /= ljj;
        if (threadIdx.x == 0) A[(size_t)j * n + j] = ljj;
        __syncthreads();
        const int span = n - j - 1;
        for (int e = threadIdx.x; e < span * span; e += blockDim.x)
        {
            const int i = j + 1 + e / span, c = j + 1 + e % span;
            if (c <= i) A[(size_t)i * n + c] -= A[(size_t)i * n + j] * A[(size_t)c * n + j];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        for (int i = 0; i < n; ++i)
        {
            double s = w[i];
            for (int c = 0; c < i; ++c) s -= A[(size_t)i * n + c] * w[c];
            w[i] = s / A[(size_t)i * n + i];
        }
        for (int i = n - 1; i >= 0; --i)
        {
            double s = w[i];
            for (int c = i + 1; c < n; ++c) s -= A[(size_t)c * n + i] * w[c];
            w[i] = s / A[(size_t)i * n + i];
        }
    }
    return fail;
}
} // namespace hb
