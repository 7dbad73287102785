// Leave-one-out ordinary kriging of the conditioning points and its adjoint.
//
// No counterpart in the reference (HPGL has no cross-validation and no
// gradients). For every target point i the system is the reference's OK system
// (my_kriging_weights.h:198-361): A[r][c] = C(p_r - p_c), b[r] = C(p_r - p_i),
// x = A^-1 b, y = A^-1 1, mu = (sum x - 1) / sum y, lambda = x - mu y and the
// estimate zhat_i = lambda . z over the neighbours (combiner.h:10-25 with mean 0).
//
// The covariance is evaluated in FP64 from M = diag(1/r0, 1/r1, 1/r2) R, the
// reference's transform divided by ranges[0] (cov_model.h:16-61): u = |M v|,
// C = sill for r0 u < 1e-4, else (sill - nugget) f(u) with
//   spherical   f = 1 - 1.5 u + 0.5 u^3 (u <= 1), 0 beyond
//   exponential f = exp(-3 u)
//   Gaussian    f = exp(-3 u^2)                        (cov_model.h:146-183).
//
// Adjoint. With K = [A 1; 1^T 0] symmetric, zhat = [z; 0]^T K^-1 [b; 1], so
//   d zhat = alpha^T db - alpha^T dA lambda,   d zhat / d z = lambda,
// where [alpha; beta] = K^-1 [z; 0]: alpha = A^-1 z - beta A^-1 1,
// beta = (1^T A^-1 z) / (1^T A^-1 1). The backward kernel recomputes the factor
// (nothing is stored between the passes), forms alpha and lambda, and sums the
// covariance derivatives of every b and A entry weighted by alpha_r and
// -alpha_r lambda_c:
//   dC/dsill = f, dC/dnugget = -f, dC/dM_ab = (sill - nugget) f'(u) (M v)_a v_b / u
// (dC/dsill = 1 and the rest 0 on the C(0) branch). The host maps dM to ranges
// and angles.
//
// One warp per target, lane r owning row r of A (neighbour counts up to 32), FP64
// right-looking Cholesky with the column of each step broadcast through shared
// memory, triangular solves by warp shuffles.
#include "../../include/hpgl_b200.h"
#include "engine_api.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace hb
{
namespace
{
constexpr int kLooWarps = 4; // warps (targets) per block
constexpr int kLooLD = 33;   // shared row stride (doubles)

struct LooParams
{
    const int *pts_xyz; // 3 ints per point
    const double *values;
    int n_pts;
    const int *targets;
    const int *nb_idx; // k point ids per target
    const int *nb_cnt;
    int n_targets;
    int k;
    int cov_type;
    double M[9];
    double r0, sill, nugget;
};

struct CovD
{
    double c;     // covariance
    double f;     // dC/dsill (and -dC/dnugget)
    double gu;    // (sill - nugget) f'(u) / u: dC/dM_ab = gu (M v)_a v_b
    double w[3];  // M v
    bool at_zero; // the C(0) branch
};

__device__ __forceinline__ CovD cov_d(const LooParams &P, int dx, int dy, int dz)
{
    CovD o;
    const double v0 = (double)dx, v1 = (double)dy, v2 = (double)dz;
    o.w[0] = P.M[0] * v0 + P.M[1] * v1 + P.M[2] * v2;
    o.w[1] = P.M[3] * v0 + P.M[4] * v1 + P.M[5] * v2;
    o.w[2] = P.M[6] * v0 + P.M[7] * v1 + P.M[8] * v2;
    const double u = sqrt(o.w[0] * o.w[0] + o.w[1] * o.w[1] + o.w[2] * o.w[2]);
    o.at_zero = P.r0 * u < 0.0001;
    if (o.at_zero)
    {
        o.c = P.sill;
        o.f = 0.0;
        o.gu = 0.0;
        return o;
    }
    const double s = P.sill - P.nugget;
    double f, fp;
    if (P.cov_type == 1)
    {
        f = exp(-3.0 * u);
        fp = -3.0 * f;
    }
    else if (P.cov_type == 2)
    {
        f = exp(-3.0 * u * u);
        fp = -6.0 * u * f;
    }
    else if (u > 1.0)
    {
        f = 0.0;
        fp = 0.0;
    }
    else
    {
        f = 1.0 - 1.5 * u + 0.5 * u * u * u;
        fp = -1.5 + 1.5 * u * u;
    }
    o.c = s * f;
    o.f = f;
    o.gu = s * fp / u;
    return o;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Everything one target's forward pass leaves in registers.
struct LooSolve
{
    int n;
    bool ok;
    int pid;        // this lane's neighbour (row) point id, -1 for padding rows
    int px, py, pz; // its coordinates
    double z;       // its value
    double lambda;  // OK weight
    double alpha;   // adjoint weight
    double zhat;
};

// Assemble, factor and solve the target's system; lane r holds row r.
__device__ LooSolve loo_solve(const LooParams &P, int t, double *Sm)
{
    const int lane = threadIdx.x & 31;
    LooSolve S;
    S.n = min(P.nb_cnt[t], P.k);
    const int n = S.n;
    const bool live = lane < n;
    S.pid = live ? P.nb_idx[(long long)t * P.k + lane] : -1;
    const int tp = P.targets[t];
    const int tx = P.pts_xyz[3 * tp], ty = P.pts_xyz[3 * tp + 1], tz = P.pts_xyz[3 * tp + 2];
    S.px = live ? P.pts_xyz[3 * S.pid] : 0;
    S.py = live ? P.pts_xyz[3 * S.pid + 1] : 0;
    S.pz = live ? P.pts_xyz[3 * S.pid + 2] : 0;
    S.z = live ? P.values[S.pid] : 0.0;

    // row r: lower triangle, padding rows identity
    double row[32];
#pragma unroll
    for (int c = 0; c < 32; ++c)
    {
        const int cx = __shfl_sync(0xffffffffu, S.px, c), cy = __shfl_sync(0xffffffffu, S.py, c),
                  cz = __shfl_sync(0xffffffffu, S.pz, c);
        double a = 0.0;
        if (live && c <= lane) a = cov_d(P, S.px - cx, S.py - cy, S.pz - cz).c;
        if (!live && c == lane) a = 1.0;
        row[c] = a;
    }
    const double b = live ? cov_d(P, S.px - tx, S.py - ty, S.pz - tz).c : 0.0;

    // right-looking Cholesky; Sm row j receives column j of the current matrix
    bool fail = false;
    double inv = 0.0;
#pragma unroll
    for (int j = 0; j < 32; ++j)
    {
        Sm[j * kLooLD + lane] = row[j];
        __syncwarp();
        const double d = Sm[j * kLooLD + j];
        fail |= !(d > 0.0);
        const double is = rsqrt(d);
        const double s = row[j] * is * is;
#pragma unroll
        for (int c = j + 1; c < 32; ++c) row[c] -= s * Sm[j * kLooLD + c];
        row[j] *= is;
        if (lane == j) inv = is;
        __syncwarp();
    }
    // forward: L y = [b, 1, z]
    double acc[3] = {b, live ? 1.0 : 0.0, S.z}, y[3] = {0, 0, 0};
#pragma unroll
    for (int j = 0; j < 32; ++j)
    {
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            if (lane == j) y[q] = acc[q] * inv;
            const double yj = __shfl_sync(0xffffffffu, y[q], j);
            if (lane > j) acc[q] -= row[j] * yj;
        }
    }
    // back: L^T x = y; L[i][r] = Sm[r][i] / sqrt(d_r) (Sm row r holds column r times sqrt(d_r))
    double x[3] = {0, 0, 0};
#pragma unroll
    for (int q = 0; q < 3; ++q) acc[q] = y[q];
#pragma unroll
    for (int i = 31; i >= 0; --i)
    {
        const double l = Sm[lane * kLooLD + i] * inv;
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            if (lane == i) x[q] = acc[q] * inv;
            const double xi = __shfl_sync(0xffffffffu, x[q], i);
            if (lane < i) acc[q] -= l * xi;
        }
    }
    __syncwarp();
    const double sx = warp_sum(live ? x[0] : 0.0), sy = warp_sum(live ? x[1] : 0.0),
                 sz = warp_sum(live ? x[2] : 0.0);
    const double mu = (sx - 1.0) / sy, beta = sz / sy;
    S.lambda = live ? x[0] - mu * x[1] : 0.0;
    S.alpha = live ? x[2] - beta * x[1] : 0.0;
    S.zhat = warp_sum(S.lambda * S.z);
    S.ok = n > 0 && !fail && !(fabs(sy) < 1e-15) && S.zhat == S.zhat;
    return S;
}

__global__ void __launch_bounds__(32 * kLooWarps) k_loo_forward(const LooParams P, double *__restrict__ zhat,
                                                                signed char *__restrict__ status)
{
    __shared__ double sm[kLooWarps][32 * kLooLD];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = blockIdx.x * kLooWarps + warp; t < P.n_targets; t += gridDim.x * kLooWarps)
    {
        const LooSolve S = loo_solve(P, t, sm[warp]);
        if (lane == 0)
        {
            zhat[t] = S.ok ? S.zhat : 0.0;
            if (status) status[t] = S.ok ? 0 : (S.n == 0 ? 1 : 2);
        }
    }
}

// grad_values[p] += g lambda; grad_params[0..8] += g dzhat/dM, [9] sill, [10] nugget.
__global__ void __launch_bounds__(32 * kLooWarps) k_loo_adjoint(const LooParams P, const double *__restrict__ g_zhat,
                                                                double *__restrict__ grad_values,
                                                                double *__restrict__ grad_params)
{
    __shared__ double sm[kLooWarps][32 * kLooLD];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = blockIdx.x * kLooWarps + warp; t < P.n_targets; t += gridDim.x * kLooWarps)
    {
        const double g = g_zhat[t];
        if (g == 0.0) continue; // warp-uniform
        const LooSolve S = loo_solve(P, t, sm[warp]);
        if (!S.ok) continue; // failed targets carry no gradient (warp-uniform)
        const bool live = lane < S.n;
        if (live) atomicAdd(&grad_values[S.pid], g * S.lambda);
        // alpha_r dC(b_r) - alpha_r sum_c lambda_c dC(A_rc), over the full row
        double gs = 0.0, gn = 0.0, gm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        auto add = [&](const CovD &d, int dx, int dy, int dz, double wgt) {
            if (d.at_zero)
            {
                gs += wgt;
                return;
            }
            gs += wgt * d.f;
            gn -= wgt * d.f;
            const double v[3] = {(double)dx, (double)dy, (double)dz};
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int c = 0; c < 3; ++c) gm[3 * a + c] += wgt * d.gu * d.w[a] * v[c];
        };
        const int tp = P.targets[t];
        const int tx = P.pts_xyz[3 * tp], ty = P.pts_xyz[3 * tp + 1], tz = P.pts_xyz[3 * tp + 2];
        if (live)
        {
            const int dx = S.px - tx, dy = S.py - ty, dz = S.pz - tz;
            add(cov_d(P, dx, dy, dz), dx, dy, dz, S.alpha);
        }
        for (int c = 0; c < S.n; ++c)
        {
            const int cx = __shfl_sync(0xffffffffu, S.px, c), cy = __shfl_sync(0xffffffffu, S.py, c),
                      cz = __shfl_sync(0xffffffffu, S.pz, c);
            const double lc = __shfl_sync(0xffffffffu, S.lambda, c);
            if (live)
            {
                const int dx = S.px - cx, dy = S.py - cy, dz = S.pz - cz;
                add(cov_d(P, dx, dy, dz), dx, dy, dz, -S.alpha * lc);
            }
        }
        gs = warp_sum(gs);
        gn = warp_sum(gn);
#pragma unroll
        for (int q = 0; q < 9; ++q) gm[q] = warp_sum(gm[q]);
        if (lane == 0)
        {
#pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(&grad_params[q], g * gm[q]);
            atomicAdd(&grad_params[9], g * gs);
            atomicAdd(&grad_params[10], g * gn);
        }
    }
}

int fill_params(LooParams &P, const int *pts_xyz, const double *values, int n_pts, const int *targets,
                 const int *nb_idx, const int *nb_cnt, int n_targets, int k, int cov_type, const double *M, double r0,
                 double sill, double nugget)
{
    if (!pts_xyz || !values || !targets || !nb_idx || !nb_cnt || !M || n_pts < 0 || n_targets < 0)
    {
        set_error("loo kriging: null array argument or negative size");
        return HPGL_B200_EINVAL;
    }
    if (k < 1)
    {
        set_error("loo kriging: max_neighbours must be >= 1");
        return HPGL_B200_EINVAL;
    }
    if (k > 32)
    {
        set_error("loo kriging: at most 32 neighbours per target are supported");
        return HPGL_B200_ELIMIT;
    }
    if (cov_type < 0 || cov_type > 2)
    {
        set_error("loo kriging: unknown covariance type");
        return HPGL_B200_EINVAL;
    }
    if (!(r0 > 0.0))
    {
        set_error("loo kriging: ranges[0] must be positive");
        return HPGL_B200_EINVAL;
    }
    P.pts_xyz = pts_xyz;
    P.values = values;
    P.n_pts = n_pts;
    P.targets = targets;
    P.nb_idx = nb_idx;
    P.nb_cnt = nb_cnt;
    P.n_targets = n_targets;
    P.k = k;
    P.cov_type = cov_type;
    for (int i = 0; i < 9; ++i) P.M[i] = M[i];
    P.r0 = r0;
    P.sill = sill;
    P.nugget = nugget;
    return HPGL_B200_OK;
}

int grid_for(int n_targets)
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = ((long long)n_targets + kLooWarps - 1) / kLooWarps;
    const long long cap = (long long)sms * 8;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}
} // namespace
} // namespace hb

extern "C" int hpgl_b200_loo_ok(const int *pts_xyz, const double *values, int n_pts, const int *targets,
                                const int *nb_idx, const int *nb_cnt, int n_targets, int k, int cov_type,
                                const double *M, double r0, double sill, double nugget, double *zhat,
                                signed char *status, void *stream)
{
    hb::LooParams P;
    const int rc = hb::fill_params(P, pts_xyz, values, n_pts, targets, nb_idx, nb_cnt, n_targets, k, cov_type, M, r0,
                                   sill, nugget);
    if (rc != HPGL_B200_OK) return rc;
    if (!zhat)
    {
        hb::set_error("loo kriging: null output");
        return HPGL_B200_EINVAL;
    }
    if (n_targets == 0) return HPGL_B200_OK;
    hb::k_loo_forward<<<hb::grid_for(n_targets), 32 * hb::kLooWarps, 0, (cudaStream_t)stream>>>(P, zhat, status);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        hb::set_error(std::string("loo kriging: ") + cudaGetErrorString(e));
        return HPGL_B200_ECUDA;
    }
    return HPGL_B200_OK;
}

extern "C" int hpgl_b200_loo_ok_adjoint(const int *pts_xyz, const double *values, int n_pts, const int *targets,
                                        const int *nb_idx, const int *nb_cnt, int n_targets, int k, int cov_type,
                                        const double *M, double r0, double sill, double nugget,
                                        const double *grad_zhat, double *grad_values, double *grad_params,
                                        void *stream)
{
    hb::LooParams P;
    const int rc = hb::fill_params(P, pts_xyz, values, n_pts, targets, nb_idx, nb_cnt, n_targets, k, cov_type, M, r0,
                                   sill, nugget);
    if (rc != HPGL_B200_OK) return rc;
    if (!grad_zhat || !grad_values || !grad_params)
    {
        hb::set_error("loo kriging adjoint: null gradient argument");
        return HPGL_B200_EINVAL;
    }
    if (n_targets == 0) return HPGL_B200_OK;
    hb::k_loo_adjoint<<<hb::grid_for(n_targets), 32 * hb::kLooWarps, 0, (cudaStream_t)stream>>>(
        P, grad_zhat, grad_values, grad_params);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        hb::set_error(std::string("loo kriging adjoint: ") + cudaGetErrorString(e));
        return HPGL_B200_ECUDA;
    }
    return HPGL_B200_OK;
}
