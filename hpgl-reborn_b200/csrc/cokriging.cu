// Simple collocated cokriging, Markov models I and II
// (simple_cokriging_markI.cpp:19-330).
//
// Every uninformed cell is kriged from the first max_nb informed primary cells
// of the analytic search template (the kriging path's template search over the
// informed-cell bitmap, run for every bin) and the collocated secondary value. The bordered system
//   [ A   c ] [w ]   [ b   ]
//   [ c^T s ] [wn] = [ b_n ]
// (A, b: primary covariances; c: the cross covariances of the target with the
// neighbours; s: the secondary variance; b_n: the cross covariance at 0) is
// solved through A: x = A^-1 b, y = A^-1 c, then wn = (b_n - c.x) / (s - c.y)
// and w = x - wn y, the same solution as the reference's Gaussian elimination
// (gauss_solver.cpp:8-70), which processes the border last. The result is
// combine()'s float accumulation (simple_cokriging_markI.cpp:83-106).
#include "engine.cuh"
#include "fold32.cuh"
#include "kernels.h"

#include <algorithm>
#include <cfloat>
#include <climits>

namespace hb
{
// flag[i] = 1 for the targets (uninformed primary cells)
__global__ void k_cok_prepare(long long n, const uint8_t *__restrict__ pmask, int *__restrict__ flag)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        flag[i] = pmask[i] ? 0 : 1;
}

__global__ void k_cok_targets(long long n, const int *__restrict__ flag, const int *__restrict__ pos,
                              int *__restrict__ targets)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (flag[i]) targets[pos[i]] = (int)i;
}

// informed cells copy the primary value (every output cell ends informed)
__global__ void k_cok_finalize(long long n, const float *__restrict__ pdata, const uint8_t *__restrict__ pmask,
                               float *__restrict__ out_data, uint8_t *__restrict__ out_mask,
                               signed char *__restrict__ status)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (pmask[i])
        {
            out_data[i] = pdata[i];
            out_mask[i] = 1;
            if (status) status[i] = -1;
        }
}

struct CokArgsDev
{
    Geom g;
    const int *targets;
    int n_targets;
    const int2 *nb_rec; // per cell and slot: {pair-table offset, value bits}
    const int *nb_n;    // per cell
    int k;
    const double *pair64;
    const double *cross_tab;
    const float *pdata;
    const float *sdata;
    const uint8_t *smask;
    CokParams p;
    float *out_data;
    uint8_t *out_mask;
    signed char *status;
};

// the cross table's entry of a neighbour given by its pair-table offset
__device__ __forceinline__ int cross_index_of_lin(const Geom &g, int lin)
{
    const long long i = g.pair_center + lin;
    const int dx = (int)(i % g.pnx) - g.phx, dy = (int)((i / g.pnx) % g.pny) - g.phy,
              dz = (int)(i / ((long long)g.pnx * g.pny)) - g.phz;
    return ((dz + g.rz) * (2 * g.ry + 1) + (dy + g.ry)) * (2 * g.rx + 1) + (dx + g.rx);
}

// the reference's fallback and combine, on the target's values
__device__ __forceinline__ void cok_write(const CokArgsDev &a, int cell, int status, float result, float sv)
{
    if (status != 0) result = __fsub_rn(__fadd_rn(a.p.pm, sv), a.p.sm); // pm + sv - sm in float
    a.out_data[cell] = result;
    a.out_mask[cell] = 1;
    if (a.status) a.status[cell] = (signed char)status;
}

// n <= 32: two targets per warp in the folded layout
constexpr int kCokThreads = 256;

// BOUND (k < 32): the factorisation stops at the warp's largest system
template <bool BOUND>
__global__ void __launch_bounds__(kCokThreads, 1) k_cok_solve_fold(const CokArgsDev a)
{
    constexpr int NP = kFold32NP, G = kFold32G;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int h = lane / G, t = lane % G, rb = NP - 1 - t;
    const unsigned gm = 0xFFFFu << (h * G);
    unsigned char *gb = smem + kFold32SysBytes * (warp * 2 + h);
    double *M = reinterpret_cast<double *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + kFold32MBytes);
    const Geom &g = a.g;
    const long long pc = g.pair_center;
    const int stride = gridDim.x * nwarps * 2;
    for (int it0 = (blockIdx.x * nwarps + warp) * 2; it0 < a.n_targets; it0 += stride)
    {
        const int it = it0 + h;
        const bool valid = it < a.n_targets;
        const int cell = valid ? a.targets[it] : 0;
        const int n = valid ? a.nb_n[cell] : 0;
        const bool live_a = t < n, live_b = rb < n;
        int lin_a = 0, lin_b = 0;
        float va = 0.0f, vb = 0.0f;
        double c_a = 0.0, c_b = 0.0;
        if (live_a)
        {
            const int2 rec = a.nb_rec[(long long)cell * a.k + t];
            lin_a = rec.x;
            va = __int_as_float(rec.y);
            c_a = __dmul_rn(a.p.coef, a.cross_tab[cross_index_of_lin(g, lin_a)]);
        }
        if (live_b)
        {
            const int2 rec = a.nb_rec[(long long)cell * a.k + rb];
            lin_b = rec.x;
            vb = __int_as_float(rec.y);
            c_b = __dmul_rn(a.p.coef, a.cross_tab[cross_index_of_lin(g, lin_b)]);
        }
        const float sv = valid ? (a.smask[cell] ? a.sdata[cell] : a.p.sm) : 0.0f;
        LIN[t] = lin_a;
        LIN[rb] = lin_b;
        __syncwarp(gm);
        double b_a = 0.0, b_b = 0.0, xa[2], xb[2];
        auto load_rhs = [&](double(&rhs_a)[2], double(&rhs_b)[2]) {
            b_a = live_a ? __ldg(a.pair64 + pc + lin_a) : 0.0;
            b_b = live_b ? __ldg(a.pair64 + pc + lin_b) : 0.0;
            rhs_a[0] = b_a;
            rhs_a[1] = c_a;
            rhs_b[0] = b_b;
            rhs_b[1] = c_b;
        };
        const int nmax = BOUND ? __reduce_max_sync(0xffffffffu, n) : NP; // both targets of the warp
        const bool fail = fold32_solve<2, true>(a.pair64 + pc, LIN, M, gm, t, live_a, live_b, lin_a, lin_b, load_rhs,
                                                xa, xb, [] {}, [] {}, nullptr, 1.0, 1.0, nmax);
        // the border: wn = (b_n - c.x) / (s - c.y)
        double cx_ = c_a * xa[0] + c_b * xb[0], cy_ = c_a * xa[1] + c_b * xb[1];
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1)
        {
            cx_ += __shfl_xor_sync(gm, cx_, o, G);
            cy_ += __shfl_xor_sync(gm, cy_, o, G);
        }
        const double piv = a.p.sec_var - cy_;
        const bool bad = fail || !(fabs(piv) >= DBL_EPSILON);
        const double wn = bad ? 0.0 : (a.p.b_last - cx_) / piv;
        // combine: result accumulated in double per term, stored as float
        const double ta = __dmul_rn((double)__fsub_rn(va, a.p.pm), __dsub_rn(xa[0], __dmul_rn(wn, xa[1])));
        const double tb = __dmul_rn((double)__fsub_rn(vb, a.p.pm), __dsub_rn(xb[0], __dmul_rn(wn, xb[1])));
        float result = a.p.pm;
#pragma unroll 4
        for (int i = 0; i < NP; ++i)
        {
            const bool lo = i < G;
            const double ti = __shfl_sync(gm, lo ? ta : tb, lo ? i : NP - 1 - i, G);
            if (i < n) result = __double2float_rn(__dadd_rn((double)result, ti));
        }
        result = __double2float_rn(__dadd_rn((double)result, __dmul_rn(wn, (double)__fsub_rn(sv, a.p.sm))));
        if (valid && t == 0) cok_write(a, cell, n == 0 ? 1 : (bad ? 2 : 0), result, sv);
        __syncwarp(gm);
    }
}

// 32 < n <= kSgsBlockMax: one block per target, A in shared memory.
constexpr int kCokBlockThreads = 128;

__global__ void __launch_bounds__(kCokBlockThreads) k_cok_solve_block(const CokArgsDev a)
{
    extern __shared__ double sh[];
    const int kk = a.k;
    double *A = sh;                  // kk * kk
    double *b = A + (size_t)kk * kk; // b
    double *c = b + kk;              // cross covariances
    double *x = c + kk;              // A^-1 b
    double *y = x + kk;              // A^-1 c
    float *vals = reinterpret_cast<float *>(y + kk);
    __shared__ int s_fail;
    const Geom &g = a.g;
    const long long pc = g.pair_center;
    for (int it = blockIdx.x; it < a.n_targets; it += gridDim.x)
    {
        const int cell = a.targets[it];
        const int n = a.nb_n[cell];
        const int2 *row = a.nb_rec + (long long)cell * kk;
        for (int e = threadIdx.x; e < n * n; e += blockDim.x)
        {
            const int i = e / n, j = e % n;
            A[(size_t)i * n + j] = a.pair64[pc + row[i].x - row[j].x];
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            const int2 rec = row[i];
            b[i] = a.pair64[pc + rec.x];
            c[i] = __dmul_rn(a.p.coef, a.cross_tab[cross_index_of_lin(g, rec.x)]);
            vals[i] = __int_as_float(rec.y);
        }
        if (threadIdx.x == 0) s_fail = 0;
        __syncthreads();
        for (int j = 0; j < n; ++j)
        {
            const double d = A[(size_t)j * n + j];
            if (threadIdx.x == 0 && !(d >= DBL_EPSILON)) s_fail = 1;
            const double ljj = sqrt(d);
            __syncthreads();
            for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + j] /= ljj;
            if (threadIdx.x == 0) A[(size_t)j * n + j] = ljj;
            __syncthreads();
            const int span = n - j - 1;
            for (int e = threadIdx.x; e < span * span; e += blockDim.x)
            {
                const int i = j + 1 + e / span, cc = j + 1 + e % span;
                if (cc <= i) A[(size_t)i * n + cc] -= A[(size_t)i * n + j] * A[(size_t)cc * n + j];
            }
            __syncthreads();
        }
        if (threadIdx.x < 2)
        {
            double *xv = threadIdx.x == 0 ? x : y;
            const double *src = threadIdx.x == 0 ? b : c;
            for (int i = 0; i < n; ++i)
            {
                double s = src[i];
                for (int q = 0; q < i; ++q) s -= A[(size_t)i * n + q] * xv[q];
                xv[i] = s / A[(size_t)i * n + i];
            }
            for (int i = n - 1; i >= 0; --i)
            {
                double s = xv[i];
                for (int q = i + 1; q < n; ++q) s -= A[(size_t)q * n + i] * xv[q];
                xv[i] = s / A[(size_t)i * n + i];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            const float sv = a.smask[cell] ? a.sdata[cell] : a.p.sm;
            int status = 1;
            float result = 0.0f;
            if (n > 0)
            {
                double cxs = 0.0, cys = 0.0;
                for (int i = 0; i < n; ++i)
                {
                    cxs += c[i] * x[i];
                    cys += c[i] * y[i];
                }
                const double piv = a.p.sec_var - cys;
                const bool bad = s_fail || !(fabs(piv) >= DBL_EPSILON);
                const double wn = bad ? 0.0 : (a.p.b_last - cxs) / piv;
                result = a.p.pm;
                for (int i = 0; i < n; ++i)
                    result = __double2float_rn(__dadd_rn(
                        (double)result,
                        __dmul_rn((double)__fsub_rn(vals[i], a.p.pm), __dsub_rn(x[i], __dmul_rn(wn, y[i])))));
                result = __double2float_rn(__dadd_rn((double)result, __dmul_rn(wn, (double)__fsub_rn(sv, a.p.sm))));
                status = bad ? 2 : 0;
            }
            cok_write(a, cell, status, result, sv);
        }
        __syncthreads();
    }
}

void launch_cok_prepare(long long n, const uint8_t *pmask, int *flag, cudaStream_t st)
{
    k_cok_prepare<<<1184, 256, 0, st>>>(n, pmask, flag);
}
void launch_cok_targets(long long n, const int *flag, const int *pos, int *targets, cudaStream_t st)
{
    k_cok_targets<<<1184, 256, 0, st>>>(n, flag, pos, targets);
}
void launch_cok_finalize(long long n, const float *pdata, const uint8_t *pmask, float *out_data, uint8_t *out_mask,
                         signed char *status, cudaStream_t st)
{
    k_cok_finalize<<<1184, 256, 0, st>>>(n, pdata, pmask, out_data, out_mask, status);
}

cudaError_t launch_cok_solve(const Geom &g, const int *targets, int n_targets, const int2 *nb_rec, const int *nb_n,
                             int k, const double *pair64, const double *cross_tab, const float *pdata,
                             const float *sdata, const uint8_t *smask, const CokParams &p, float *out_data,
                             uint8_t *out_mask, signed char *status, int n_sm, cudaStream_t st)
{
    if (n_targets <= 0) return cudaSuccess;
    CokArgsDev a{g, targets, n_targets, nb_rec, nb_n, k, pair64, cross_tab, pdata, sdata, smask, p, out_data, out_mask,
                 status};
    if (k <= 32)
    {
        const int spb = kCokThreads / kFold32G;
        const size_t smem = kFold32SysBytes * spb;
        auto kern = k < 32 ? k_cok_solve_fold<true> : k_cok_solve_fold<false>;
        int per_sm = 0;
        cudaError_t e = set_smem_min_carveout(kern, kCokThreads, smem, per_sm);
        if (e != cudaSuccess) return e;
        const int blocks = std::min((n_targets + spb - 1) / spb, n_sm);
        kern<<<blocks, kCokThreads, smem, st>>>(a);
    }
    else
    {
        const size_t smem = (size_t)k * k * 8 + 4 * (size_t)k * 8 + (size_t)k * 4;
        cudaError_t e = cudaFuncSetAttribute(k_cok_solve_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int blocks = std::min(n_targets, n_sm * 8);
        k_cok_solve_block<<<blocks, kCokBlockThreads, smem, st>>>(a);
    }
    return cudaGetLastError();
}
} // namespace hb
