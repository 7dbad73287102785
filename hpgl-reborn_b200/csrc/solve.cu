// Batched per-cell kriging solves (S1/S2/K2 of the hot path).
//
// Reference semantics: sk_kriging_weights_3 / ok_kriging_weights_3
// (my_kriging_weights.h:60-361) build A[i][j] = cov(c_i, c_j),
// b[i] = cov(c_i, centre), factor A with dpotrf and solve; OK solves A x = b and
// A y = 1, mu = (sum x - 1) / sum y (failing when |sum y| < 1e-15), w = x - mu y
// (the Schur complement of the unbiasedness row), variance C(0) - w.b - mu;
// SK: w = x, variance C(0) - w.b. The estimate is mean + sum w_i (v_i - mean)
// (combiner.h:10-25; mean 0 for OK).
//
// Layout: one "group" of NP threads per system (NP in {8, 16, 32, 64}); thread r
// owns row r of the (padded) matrix in registers. Rows past the neighbour count
// n are identity rows with zero right-hand sides, which leaves the solution of
// the first n unknowns unchanged. The search stage hands over, per neighbour,
// its pair-table offset lin(o_i) (o_i = neighbour - centre) and its value, so
// cov(c_i, c_j) = pair[centre + lin_i - lin_j] and cov(c_i, centre) =
// pair[centre + lin_i]: assembly is one subtraction and one gather per entry.
//
// Factorisation: right-looking Cholesky. Step j: every thread stores its
// current A[r][j] in row j of the group's shared matrix M (rows padded to 16
// bytes), then reads row j back with 16-byte broadcast loads and updates
// A[r][c] -= A[r][j] * M[j][c] / M[j][j] (c > j), and scales A[r][j] by
// 1/sqrt(M[j][j]). Afterwards thread r holds row r of L in registers and row r
// of M holds column r of L (times sqrt(M[r][r])), so both triangular solves
// are one broadcast and one FMA per step.
//
// Precision modes:
//   FP64 plain   : T = double throughout.
//   FP32 refined : A assembled from the float pair table, factored and solved
//                  in float for b, (OK) the ones vector and the centred values
//                  v - mean. The estimate and the variance are bilinear forms
//                  u^T A^-1 w; each is corrected with one FP64 residual,
//                    u^T A^-1 w = u^T x_w + x_u^T (w - A64 x_w) + O(|e_u| |e_w|),
//                  (x_w = A32^-1 w), so one residual pass in double against the
//                  double pair table gives quadratically small errors without a
//                  second triangular solve. The relative size of the first-order
//                  correction bounds what remains (its square); above `tol` the
//                  group falls back to classic refinement x += A32^-1 (b - A64 x)
//                  (up to `steps` rounds, each with an FP64 residual), and a
//                  system that still does not converge, or whose float factor
//                  breaks down, is queued for the FP64 kernel (status 4) instead
//                  of being reported singular.
#include "engine.cuh"
#include "kernels.h"

#include <cstdint>

namespace hb
{
template <int NP>
struct Grp
{
    int r;         // thread index inside the group
    unsigned mask; // lanes of the group inside its warp (NP <= 32)
    int bar;       // named barrier id (NP == 64)

    __device__ __forceinline__ void sync() const
    {
        if constexpr (NP <= 32)
            __syncwarp(mask);
        else
            asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(NP) : "memory");
    }
};

template <int NP, typename T>
__device__ __forceinline__ T group_sum(const Grp<NP> &g, T v, T *scratch)
{
    if constexpr (NP <= 32)
    {
#pragma unroll
        for (int o = NP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(g.mask, v, o, NP);
        return v;
    }
    else
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((g.r & 31) == 0) scratch[g.r >> 5] = v;
        g.sync();
        T s = scratch[0] + scratch[1];
        g.sync();
        return s;
    }
}

template <int NP, typename T>
__device__ __forceinline__ T group_max(const Grp<NP> &g, T v, T *scratch)
{
    if constexpr (NP <= 32)
    {
#pragma unroll
        for (int o = NP / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(g.mask, v, o, NP));
        return v;
    }
    else
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((g.r & 31) == 0) scratch[g.r >> 5] = v;
        g.sync();
        T s = fmax(scratch[0], scratch[1]);
        g.sync();
        return s;
    }
}

// value of `v` held by group thread `src`
template <int NP, typename T>
__device__ __forceinline__ T group_bcast(const Grp<NP> &g, T v, int src, T *slot)
{
    if constexpr (NP <= 32)
    {
        return __shfl_sync(g.mask, v, src, NP);
    }
    else
    {
        if (g.r == src) *slot = v;
        g.sync();
        return *slot;
    }
}

template <typename T>
__device__ __forceinline__ T rsqrt_t(T d);
template <>
__device__ __forceinline__ float rsqrt_t<float>(float d) { return rsqrtf(d); }
template <>
__device__ __forceinline__ double rsqrt_t<double>(double d) { return rsqrt(d); }

template <typename T>
__device__ __forceinline__ T pair_get(const float *p32, const double *p64, long long i);
template <>
__device__ __forceinline__ float pair_get<float>(const float *p32, const double *, long long i) { return __ldg(p32 + i); }
template <>
__device__ __forceinline__ double pair_get<double>(const float *, const double *p64, long long i) { return __ldg(p64 + i); }

// 16-byte vectors of T
template <typename T>
struct Vec;
template <>
struct Vec<float>
{
    typedef float4 type;
    static constexpr int n = 4;
    static __device__ __forceinline__ void unpack(const float4 &v, float *o)
    {
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
};
template <>
struct Vec<double>
{
    typedef double2 type;
    static constexpr int n = 2;
    static __device__ __forceinline__ void unpack(const double2 &v, double *o)
    {
        o[0] = v.x;
        o[1] = v.y;
    }
};

// Forward substitution L y = rhs for R right-hand sides (row-oriented).
template <int NP, typename T, int R>
__device__ __forceinline__ void forward_solve(const Grp<NP> &g, const T (&row)[NP], T (&acc)[R], T my_inv,
                                              T *slots, T (&y)[R])
{
#pragma unroll
    for (int q = 0; q < R; ++q) y[q] = 0;
#pragma unroll
    for (int j = 0; j < NP; ++j)
    {
        if (g.r == j)
        {
#pragma unroll
            for (int q = 0; q < R; ++q) y[q] = acc[q] * my_inv;
        }
        T yj[R];
#pragma unroll
        for (int q = 0; q < R; ++q) yj[q] = group_bcast<NP, T>(g, y[q], j, slots + (NP <= 32 ? 0 : (q * NP + j)));
        if (g.r > j)
        {
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q] -= row[j] * yj[q];
        }
    }
    if constexpr (NP > 32) g.sync(); // slots are reused by the next solve
}

// Back substitution L^T x = y; row r of M holds column r of L times sqrt(M[r][r]).
template <int NP, typename T, int R, int LD>
__device__ __forceinline__ void back_solve(const Grp<NP> &g, const T *M, T (&yv)[R], T my_inv, T *slots,
                                           T (&x)[R])
{
    T acc[R];
#pragma unroll
    for (int q = 0; q < R; ++q)
    {
        acc[q] = yv[q];
        x[q] = 0;
    }
    const T *Mr = M + g.r * LD;
#pragma unroll
    for (int i = NP - 1; i >= 0; --i)
    {
        if (g.r == i)
        {
#pragma unroll
            for (int q = 0; q < R; ++q) x[q] = acc[q] * my_inv;
        }
        T xi[R];
#pragma unroll
        for (int q = 0; q < R; ++q) xi[q] = group_bcast<NP, T>(g, x[q], i, slots + (NP <= 32 ? 0 : (q * NP + i)));
        if (g.r < i)
        {
            const T l = Mr[i] * my_inv;
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q] -= l * xi[q];
        }
    }
    if constexpr (NP > 32) g.sync();
}

template <int NP, typename TF>
struct SolveSmem
{
    static constexpr int V = 16 / (int)sizeof(TF);
    static constexpr int LD = NP + V;
    // M (NP x LD of TF), LIN (NP int), X (2 NP double), slots (3 NP TF), scratch (4 double)
    static constexpr size_t m_bytes = (size_t)NP * LD * sizeof(TF);
    static constexpr size_t lin_off = m_bytes;
    static constexpr size_t x_off = (lin_off + NP * sizeof(int) + 15) / 16 * 16;
    static constexpr size_t slot_off = x_off + 2 * NP * sizeof(double);
    static constexpr size_t scr_off = (slot_off + 3 * NP * sizeof(TF) + 15) / 16 * 16;
    static constexpr size_t bytes = (scr_off + 4 * sizeof(double) + 15) / 16 * 16;
};

// Residuals res[q] = rhs[q] - A64 x[q] for the first Q right-hand sides, FP64,
// A64 row r gathered from the double pair table; X holds the solutions.
template <int NP, int Q, int RX>
__device__ __forceinline__ void residuals_fp64(const Grp<NP> &grp, const double *__restrict__ pair64, long long pc,
                                               int lin, const int *LIN, double *X, int n, bool live,
                                               const double (&x)[RX], const double (&rhs)[Q], double (&res)[Q])
{
    const int r = grp.r;
#pragma unroll
    for (int q = 0; q < Q; ++q) X[q * NP + r] = x[q];
    grp.sync();
#pragma unroll
    for (int q = 0; q < Q; ++q) res[q] = rhs[q];
    if (live)
    {
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            if (c < n)
            {
                const double a = __ldg(pair64 + pc + lin - LIN[c]);
#pragma unroll
                for (int q = 0; q < Q; ++q) res[q] -= a * X[q * NP + c];
            }
        }
    }
    else
    {
#pragma unroll
        for (int q = 0; q < Q; ++q) res[q] = -x[q];
    }
    grp.sync();
}

// Minimum resident 256-thread blocks per SM requested for the FP32 kernels
// (caps their registers at 65536 / (256 * blocks)).
#ifndef HB_SOLVE_MIN_BLOCKS_F32
#define HB_SOLVE_MIN_BLOCKS_F32 3
#endif

template <int NP, typename TF, bool ORDINARY, bool REFINE>
__global__ void __launch_bounds__(256, sizeof(TF) == 4 ? HB_SOLVE_MIN_BLOCKS_F32 : 1) k_solve(const Geom g, const int2 *__restrict__ cells,
                                               const int *__restrict__ n_items_ptr, const int2 *__restrict__ nb_rec,
                                               const int *__restrict__ nb_n, int ind_value,
                                               const double *__restrict__ pair64, const float *__restrict__ pair32,
                                               double mean, double c0, int steps, double tol, SolveOut out,
                                               int2 *__restrict__ esc_cells, int *__restrict__ esc_count)
{
    typedef SolveSmem<NP, TF> SM;
    constexpr int LD = SM::LD;
    constexpr int V = SM::V;
    // right-hand sides: b, (OK) the ones vector, and the centred values v - mean
    constexpr int QB = ORDINARY ? 2 : 1; // b and 1: the systems the weights come from
    constexpr int R = QB + 1;            // plus v: the adjoint system of the estimate
    typedef typename Vec<TF>::type VT;
    extern __shared__ __align__(16) unsigned char smem[];
    const int groups_per_block = blockDim.x / NP;
    const int gi = threadIdx.x / NP;
    Grp<NP> grp;
    grp.r = threadIdx.x % NP;
    if constexpr (NP <= 32)
    {
        int lane0 = (threadIdx.x & 31) / NP * NP;
        grp.mask = (NP == 32) ? 0xffffffffu : (((1u << NP) - 1u) << lane0);
    }
    else
        grp.mask = 0xffffffffu;
    grp.bar = 1 + gi;
    const int r = grp.r;

    unsigned char *gb = smem + SM::bytes * gi;
    TF *M = reinterpret_cast<TF *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + SM::lin_off);
    double *X = reinterpret_cast<double *>(gb + SM::x_off);
    TF *slots = reinterpret_cast<TF *>(gb + SM::slot_off);
    double *scr = reinterpret_cast<double *>(gb + SM::scr_off);

    const int n_items = *n_items_ptr;
    const long long pc = g.pair_center;
    const int stride = gridDim.x * groups_per_block;
    const float mf = (float)mean; // mean_t is float (typedefs.h:122)
    // Work items are {cell, n}. The record of item i+1 and the work entry of
    // item i+2 are loaded while item i is solved, so no load the solve waits on
    // depends on another load issued in the same iteration.
    int item = blockIdx.x * groups_per_block + gi;
    int2 w_cur = item < n_items ? cells[item] : make_int2(0, 0);
    int2 w_nxt = item + stride < n_items ? cells[item + stride] : make_int2(0, 0);
    int2 rec = (item < n_items && r < w_cur.y) ? nb_rec[(long long)w_cur.x * g.k + r] : make_int2(0, 0);
    for (; item < n_items; item += stride)
    {
        const int my_cell = w_cur.x, my_n = w_cur.y;
        const int lin = rec.x;
        const bool live = r < my_n;
        const float vraw = __int_as_float(rec.y);
        rec = (item + stride < n_items && r < w_nxt.y) ? nb_rec[(long long)w_nxt.x * g.k + r] : make_int2(0, 0);
        w_cur = w_nxt;
        w_nxt = item + 2 * stride < n_items ? cells[item + 2 * stride] : make_int2(0, 0);
        // neighbour value centred on the (float) mean as combine() does (combiner.h:19-24)
        float v = 0.0f;
        if (live) v = ind_value >= 0 ? (vraw == (float)ind_value ? 1.0f : 0.0f) : vraw;
        const double vc = live ? (double)(v - mf) : 0.0;
        LIN[r] = live ? lin : 0;
        grp.sync();

        // ---- assembly (lower triangle of row r; padding rows are identity)
        TF row[NP];
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            TF a = (TF)0;
            if (live && c <= r) a = pair_get<TF>(pair32, pair64, pc + lin - LIN[c]);
            if (!live && c == r) a = (TF)1;
            row[c] = a;
        }
        const double b64 = live ? __ldg(pair64 + pc + lin) : 0.0;

        // ---- factorisation
        bool fail = false;
        TF my_inv = 0;
#pragma unroll
        for (int j = 0; j < NP; ++j)
        {
            M[j * LD + r] = row[j];
            grp.sync();
            TF mj[NP + V];
            const VT *mv = reinterpret_cast<const VT *>(M + j * LD);
#pragma unroll
            for (int q = j / V; q < NP / V; ++q) Vec<TF>::unpack(mv[q], mj + q * V);
            const TF d = mj[j];
            fail |= !(d > (TF)0);
            const TF inv_s = rsqrt_t<TF>(d);
            const TF s = row[j] * (inv_s * inv_s);
#pragma unroll
            for (int c = j + 1; c < NP; ++c) row[c] -= s * mj[c];
            row[j] *= inv_s;
            if (r == j) my_inv = inv_s;
        }

        // ---- solves: x = A^-1 b, (OK) y = A^-1 1, and lambda = A^-1 (v - mean)
        TF rhs[R], ytmp[R], xs[R];
        rhs[0] = live ? (TF)b64 : (TF)0;
        if constexpr (ORDINARY) rhs[1] = live ? (TF)1 : (TF)0;
        rhs[R - 1] = (TF)vc;
        forward_solve<NP, TF, R>(grp, row, rhs, my_inv, slots, ytmp);
        back_solve<NP, TF, R, LD>(grp, M, ytmp, my_inv, slots, xs);
        double x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = (double)xs[q];
        const double one = live ? 1.0 : 0.0;

        // Bilinear forms u^T A^-1 w of the estimate and variance. With FP32
        // solutions each form gets the dual-weighted residual correction
        //   u^T A^-1 w = u^T x_w + x_u^T (w - A64 x_w) + O(|e_u| |e_w|),
        // x_w = A32^-1 w, x_u = A32^-1 u, the residual in FP64: one residual
        // pass gives quadratically accurate forms without another solve.
        double f_vb = vc * x[0], f_bb = b64 * x[0], f_1b = 0.0, f_v1 = 0.0, f_11 = 0.0;
        if constexpr (ORDINARY)
        {
            f_1b = one * x[0];
            f_v1 = vc * x[1];
            f_11 = one * x[1];
        }
        bool escalate = false;
        double corr_vb = 0.0, corr_bb = 0.0;
        if constexpr (REFINE)
        {
            escalate = fail;
            double rhs64[QB], res[QB];
            rhs64[0] = b64;
            if constexpr (ORDINARY) rhs64[1] = one;
            residuals_fp64<NP, QB, R>(grp, pair64, pc, lin, LIN, X, my_n, live, x, rhs64, res);
            corr_vb = x[R - 1] * res[0];
            corr_bb = x[0] * res[0];
            f_vb += corr_vb;
            f_bb += corr_bb;
            if constexpr (ORDINARY)
            {
                f_1b += x[1] * res[0];
                f_v1 += x[R - 1] * res[1];
                f_11 += x[1] * res[1];
            }
        }
        double s_vb = group_sum<NP, double>(grp, f_vb, scr);
        double s_bb = group_sum<NP, double>(grp, f_bb, scr);
        double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
        if constexpr (ORDINARY)
        {
            s_1b = group_sum<NP, double>(grp, f_1b, scr);
            s_v1 = group_sum<NP, double>(grp, f_v1, scr);
            s_11 = group_sum<NP, double>(grp, f_11, scr);
        }
        if constexpr (REFINE)
        {
            // a-posteriori check: the first-order correction of each form relative
            // to the form's scale; what remains after it is about its square
            const double abs_vb = group_sum<NP, double>(grp, fabs(vc * x[0]), scr) + 1e-300;
            const double abs_bb = group_sum<NP, double>(grp, fabs(b64 * x[0]), scr) + 1e-300;
            const double c1 = fabs(group_sum<NP, double>(grp, corr_vb, scr)) / abs_vb;
            const double c2 = fabs(group_sum<NP, double>(grp, corr_bb, scr)) / abs_bb;
            const double d = fmax(c1, c2);
            if (!(d * d <= tol)) escalate = true;
            if (!(s_vb == s_vb) || !(s_bb == s_bb)) escalate = true;
            if (escalate && steps > 0 && !fail)
            {
                // classic refinement of x (and y): x += A32^-1 (b - A64 x) until the
                // correction stops mattering, then the forms without correction
                double prev = 0.0;
                bool done = false;
                for (int it = 0; it < steps && !done; ++it)
                {
                    double rq[QB], rr64[QB], xq[QB];
#pragma unroll
                    for (int q = 0; q < QB; ++q)
                    {
                        rq[q] = q == 0 ? b64 : one;
                        xq[q] = x[q];
                    }
                    residuals_fp64<NP, QB, QB>(grp, pair64, pc, lin, LIN, X, my_n, live, xq, rq, rr64);
                    TF rr[QB], yy[QB], dd[QB];
#pragma unroll
                    for (int q = 0; q < QB; ++q) rr[q] = (TF)rr64[q];
                    forward_solve<NP, TF, QB>(grp, row, rr, my_inv, slots, yy);
                    back_solve<NP, TF, QB, LD>(grp, M, yy, my_inv, slots, dd);
                    double dmax = 0.0, xmax = 0.0;
#pragma unroll
                    for (int q = 0; q < QB; ++q)
                    {
                        x[q] += (double)dd[q];
                        dmax = fmax(dmax, fabs((double)dd[q]));
                        xmax = fmax(xmax, fabs(x[q]));
                    }
                    dmax = group_max<NP, double>(grp, dmax, scr);
                    xmax = group_max<NP, double>(grp, xmax, scr);
                    const double delta = xmax > 0.0 ? dmax / xmax : 0.0;
                    double err;
                    if (it == 0)
                        err = delta * delta;
                    else
                    {
                        const double rho = prev > 0.0 ? delta / prev : 0.0;
                        err = rho < 0.5 ? delta * rho / (1.0 - rho) : 1.0;
                    }
                    if (!(delta == delta)) err = 1.0;
                    prev = delta;
                    done = err <= tol;
                }
                if (done)
                {
                    escalate = false;
                    s_vb = group_sum<NP, double>(grp, vc * x[0], scr);
                    s_bb = group_sum<NP, double>(grp, b64 * x[0], scr);
                    if constexpr (ORDINARY)
                    {
                        s_1b = group_sum<NP, double>(grp, one * x[0], scr);
                        s_v1 = group_sum<NP, double>(grp, vc * x[1], scr);
                        s_11 = group_sum<NP, double>(grp, one * x[1], scr);
                    }
                }
            }
        }

        if (escalate)
        {
            if (r == 0)
            {
                int slot = atomicAdd(esc_count, 1);
                esc_cells[slot] = make_int2(my_cell, my_n);
                if (out.status) out.status[my_cell] = 4;
            }
            grp.sync();
            continue;
        }

        // ---- estimate and variance from the forms
        //   SK: est = mean + (v-m)^T A^-1 b,        var = C0 - b^T A^-1 b
        //   OK: mu = (1^T A^-1 b - 1) / 1^T A^-1 1,  est = v^T A^-1 b - mu v^T A^-1 1,
        //       var = C0 - b^T A^-1 b + mu 1^T A^-1 b - mu   (my_kriging_weights.h:312-357)
        double est, var;
        if constexpr (ORDINARY)
        {
            if (fabs(s_11) < 1e-15) fail = true;
            const double mu = (s_1b - 1.0) / s_11;
            est = s_vb - mu * s_v1;
            var = c0 - s_bb + mu * s_1b - mu;
        }
        else
        {
            est = (double)mf + s_vb;
            var = c0 - s_bb;
        }
        if (var < 0) var = 0;
        if (r == 0)
        {
            if (!fail)
            {
                if (out.write_cont)
                {
                    out.out_data[my_cell] = (float)est;
                    out.out_mask[my_cell] = 1;
                }
                if (out.prob) out.prob[(long long)my_cell * out.prob_stride] = (float)est;
                if (out.est64) out.est64[my_cell] = est;
                if (out.var) out.var[my_cell] = var;
                if (out.status) out.status[my_cell] = 0;
            }
            else if (out.status)
                out.status[my_cell] = 2;
        }
        grp.sync();
    }
}

template <int NP, typename TF, bool ORD, bool REF>
static cudaError_t launch_one(const Geom &g, const int2 *cells, const int *n_items, int max_items, const int2 *nb_rec,
                              const int *nb_n, int ind_value, const double *pair64, const float *pair32, double mean,
                              double c0, int steps, double tol, const SolveOut &out, int2 *esc_cells, int *esc_count,
                              int n_sm, cudaStream_t st)
{
    constexpr int threads = 256;
    constexpr int gpb = threads / NP;
    const size_t smem = SolveSmem<NP, TF>::bytes * gpb;
    auto kern = k_solve<NP, TF, ORD, REF>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long want = ((long long)max_items + gpb - 1) / gpb;
    long long blocks = (long long)n_sm * per_sm;
    if (want < blocks) blocks = want;
    if (blocks < 1) blocks = 1;
    kern<<<(unsigned)blocks, threads, smem, st>>>(g, cells, n_items, nb_rec, nb_n, ind_value, pair64, pair32, mean, c0,
                                                  steps, tol, out, esc_cells, esc_count);
    return cudaGetLastError();
}

template <int NP>
static cudaError_t launch_np(int precision, bool ordinary, const Geom &g, const int2 *cells, const int *n_items,
                             int max_items, const int2 *nb_rec, const int *nb_n, int ind_value, const double *pair64,
                             const float *pair32, double mean, double c0, int steps, double tol, const SolveOut &out,
                             int2 *esc_cells, int *esc_count, int n_sm, cudaStream_t st)
{
#define HB_ARGS g, cells, n_items, max_items, nb_rec, nb_n, ind_value, pair64, pair32, mean, c0, steps, tol, out, esc_cells, esc_count, n_sm, st
    if (precision == 0)
        return ordinary ? launch_one<NP, double, true, false>(HB_ARGS) : launch_one<NP, double, false, false>(HB_ARGS);
    return ordinary ? launch_one<NP, float, true, true>(HB_ARGS) : launch_one<NP, float, false, true>(HB_ARGS);
#undef HB_ARGS
}

cudaError_t launch_solve_bucket(int np, int precision, bool ordinary, const Geom &g, const int2 *cells,
                                const int *n_items, int max_items, const int2 *nb_rec, const int *nb_n, int ind_value,
                                const double *pair64, const float *pair32, double mean, double c0, int steps,
                                double tol, const SolveOut &out, int2 *esc_cells, int *esc_count, int n_sm,
                                cudaStream_t st)
{
    switch (np)
    {
    case 8:
        return launch_np<8>(precision, ordinary, g, cells, n_items, max_items, nb_rec, nb_n, ind_value, pair64,
                            pair32, mean, c0, steps, tol, out, esc_cells, esc_count, n_sm, st);
    case 16:
        return launch_np<16>(precision, ordinary, g, cells, n_items, max_items, nb_rec, nb_n, ind_value, pair64,
                             pair32, mean, c0, steps, tol, out, esc_cells, esc_count, n_sm, st);
    case 32:
        return launch_np<32>(precision, ordinary, g, cells, n_items, max_items, nb_rec, nb_n, ind_value, pair64,
                             pair32, mean, c0, steps, tol, out, esc_cells, esc_count, n_sm, st);
    case 64:
        return launch_np<64>(precision, ordinary, g, cells, n_items, max_items, nb_rec, nb_n, ind_value, pair64,
                             pair32, mean, c0, steps, tol, out, esc_cells, esc_count, n_sm, st);
    default:
        return cudaErrorInvalidValue;
    }
}
} // namespace hb
