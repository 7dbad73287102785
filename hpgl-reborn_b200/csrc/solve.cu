// Batched per-cell kriging solves (S1/S2/K2 of the hot path).
//
// Reference semantics: sk_kriging_weights_3 / ok_kriging_weights_3
// (my_kriging_weights.h:60-361) build A[i][j] = cov(c_i, c_j),
// b[i] = cov(c_i, centre), factor A with dpotrf and solve; OK solves A x = b and
// A y = 1, mu = (sum x - 1) / sum y (failing when |sum y| < 1e-15), w = x - mu y
// (the Schur complement of the unbiasedness row), variance C(0) - w.b - mu;
// SK: w = x, variance C(0) - w.b. The estimate is mean + sum w_i (v_i - mean)
// (combiner.h:10-25, mean 0 for OK).
//
// Layout: one "group" of NP threads per system (NP in {8, 16, 32, 64}); thread r
// owns row r of the (padded) matrix in registers. Rows past the neighbour count
// n are identity rows with zero right-hand sides, which leaves the solution of
// the first n unknowns unchanged. Covariances come from the pair table: for
// neighbours at centre-relative offsets o_i, cov(c_i, c_j) = pair[centre +
// lin(o_i) - lin(o_j)] (lin is linear in the offset inside the table block),
// so assembly is one subtraction and one gather per entry.
//
// Factorisation: right-looking Cholesky. Step j: every thread writes its
// current A[r][j] into row j of a per-group shared matrix M, then updates
// A[r][c] -= A[r][j] * M[j][c] / M[j][j] for c > j and scales A[r][j] by
// 1/sqrt(M[j][j]). Afterwards thread r holds row r of L in registers and
// M[r][i] * rsqrt(M[r][r]) = L[i][r] (column r) in shared memory, so both
// triangular solves are one broadcast and one FMA per step.
//
// Precision modes:
//   FP64 plain   : T = double throughout.
//   FP32 refined : A assembled from the float pair table, factored and solved in
//                  float; then `steps` rounds of x += A32^-1 (b - A64 x) with the
//                  residual in double against the double pair table. OK refines
//                  both right-hand sides; mu, w, estimate and variance in double.
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
        for (int o = NP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(g.mask, v, o, NP);
        return v;
    }
    else
    {
        // 64 threads: warp sums, then combine the two halves through shared memory
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((g.r & 31) == 0) scratch[g.r >> 5] = v;
        g.sync();
        T s = scratch[0] + scratch[1];
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
        T o = *slot;
        g.sync();
        return o;
    }
}

template <typename T>
__device__ __forceinline__ T rsqrt_t(T d);
template <>
__device__ __forceinline__ float rsqrt_t<float>(float d) { return rsqrtf(d); }
template <>
__device__ __forceinline__ double rsqrt_t<double>(double d) { return rsqrt(d); }

template <typename T>
struct PairTab;
template <>
struct PairTab<float>
{
    static __device__ __forceinline__ float get(const float *p32, const double *, long long i) { return __ldg(p32 + i); }
};
template <>
struct PairTab<double>
{
    static __device__ __forceinline__ double get(const float *, const double *p64, long long i) { return __ldg(p64 + i); }
};

// Forward substitution L y = rhs (row-oriented), in place on `acc`.
template <int NP, typename T>
__device__ __forceinline__ T forward_solve(const Grp<NP> &g, const T (&row)[NP], T acc, T my_inv, T *slot)
{
    T y = 0;
#pragma unroll
    for (int j = 0; j < NP; ++j)
    {
        if (g.r == j) y = acc * my_inv;
        T yj = group_bcast<NP, T>(g, y, j, slot + (NP <= 32 ? 0 : j));
        if (g.r > j) acc -= row[j] * yj;
    }
    return y;
}

// Back substitution L^T x = y using the columns kept in M (row r of M holds
// column r of L scaled by sqrt(M[r][r])).
template <int NP, typename T>
__device__ __forceinline__ T back_solve(const Grp<NP> &g, const T *M, int ld, T y, T my_inv, T *slot)
{
    T acc = y, x = 0;
#pragma unroll
    for (int i = NP - 1; i >= 0; --i)
    {
        if (g.r == i) x = acc * my_inv;
        T xi = group_bcast<NP, T>(g, x, i, slot + (NP <= 32 ? 0 : i));
        if (g.r < i) acc -= (M[g.r * ld + i] * my_inv) * xi;
    }
    return x;
}



template <int NP, typename TF, bool ORDINARY, bool REFINE>
__global__ void __launch_bounds__(256) k_solve(const Geom g, const int *__restrict__ cells,
                                               const int *__restrict__ n_items_ptr, const int *__restrict__ nb_pid,
                                               const int *__restrict__ nb_n,
                                               const unsigned long long *__restrict__ pts_xyz,
                                               const float *__restrict__ pts_val, const uint8_t *__restrict__ pts_cat,
                                               int ind_value, const double *__restrict__ pair64,
                                               const float *__restrict__ pair32, double mean, double c0,
                                               int steps, SolveOut out)
{
    constexpr int LD = NP + 1;
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

    // per-group shared memory: M (NP x LD of TF), LIN (NP ints), X (NP doubles),
    // broadcast slots (NP TF + NP double), scratch (2 double)
    const size_t grp_bytes = (size_t)NP * LD * sizeof(TF) + NP * sizeof(int) + NP * sizeof(double) +
                             NP * sizeof(TF) + NP * sizeof(double) + 4 * sizeof(double);
    unsigned char *gb = smem + ((grp_bytes + 15) / 16 * 16) * gi;
    TF *M = reinterpret_cast<TF *>(gb);
    int *LIN = reinterpret_cast<int *>(M + NP * LD);
    double *X = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(LIN) + ((NP * sizeof(int) + 7) / 8 * 8));
    TF *slotT = reinterpret_cast<TF *>(X + NP);
    double *slotD = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(slotT) + ((NP * sizeof(TF) + 7) / 8 * 8));
    double *scr = slotD + NP;

    const int n_items = *n_items_ptr;
    const long long pc = g.pair_center;
    for (int item = blockIdx.x * groups_per_block + gi; item < n_items; item += gridDim.x * groups_per_block)
    {
        const int cell = cells[item];
        const int n = nb_n[cell];
        const int cxg = cell % g.nx, cyg = cell % (g.nx * g.ny) / g.nx, czg = cell / (g.nx * g.ny);
        int lin = 0;
        double v = 0.0;
        const bool live = r < n;
        if (live)
        {
            int p = nb_pid[(long long)cell * g.k + r];
            int px, py, pz;
            unpack_xyz(pts_xyz[p], px, py, pz);
            lin = pair_lin(g, px - cxg, py - cyg, pz - czg);
            v = pts_val ? (double)pts_val[p] : (pts_cat[p] == ind_value ? 1.0 : 0.0);
        }
        LIN[r] = lin;
        grp.sync();

        // ---- assembly (lower triangle of row r; padding rows are identity)
        TF row[NP];
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            TF a = (TF)0;
            if (live && c <= r) a = PairTab<TF>::get(pair32, pair64, pc + lin - LIN[c]);
            if (!live && c == r) a = (TF)1;
            row[c] = a;
        }
        const double b64 = live ? __ldg(pair64 + pc + lin) : 0.0;
        const TF bT = live ? PairTab<TF>::get(pair32, pair64, pc + lin) : (TF)0;

        // ---- factorisation
        bool fail = false;
        TF my_inv = 0;
#pragma unroll
        for (int j = 0; j < NP; ++j)
        {
            M[j * LD + r] = row[j];
            grp.sync();
            const TF d = M[j * LD + j];
            fail |= !(d > (TF)0);
            const TF inv_s = rsqrt_t<TF>(d);
            const TF s = row[j] * (inv_s * inv_s);
#pragma unroll
            for (int c = j + 1; c < NP; ++c) row[c] -= s * M[j * LD + c];
            row[j] *= inv_s;
            if (r == j) my_inv = inv_s;
        }
        // M rows are complete (each written before the sync of its own step)

        // ---- solves
        double x = 0.0, y = 0.0; // A^-1 b and (OK) A^-1 1, double
        {
            TF yb = forward_solve<NP, TF>(grp, row, bT, my_inv, slotT);
            x = (double)back_solve<NP, TF>(grp, M, LD, yb, my_inv, slotT);
            if constexpr (ORDINARY)
            {
                TF y1 = forward_solve<NP, TF>(grp, row, live ? (TF)1 : (TF)0, my_inv, slotT);
                y = (double)back_solve<NP, TF>(grp, M, LD, y1, my_inv, slotT);
            }
        }
        if constexpr (REFINE)
        {
            for (int it = 0; it < steps; ++it)
            {
                // residuals r = b - A64 x (and 1 - A64 y) in double
                X[r] = x;
                if constexpr (ORDINARY) slotD[r] = y;
                grp.sync();
                double rx = b64, ry = live ? 1.0 : 0.0;
                if (live)
                {
#pragma unroll 8
                    for (int c = 0; c < NP; ++c)
                    {
                        if (c < n)
                        {
                            double a = __ldg(pair64 + pc + lin - LIN[c]);
                            rx -= a * X[c];
                            if constexpr (ORDINARY) ry -= a * slotD[c];
                        }
                    }
                }
                else
                {
                    rx = -x;
                    ry = -y;
                }
                grp.sync();
                TF dx = back_solve<NP, TF>(grp, M, LD, forward_solve<NP, TF>(grp, row, (TF)rx, my_inv, slotT),
                                           my_inv, slotT);
                x += (double)dx;
                if constexpr (ORDINARY)
                {
                    TF dy = back_solve<NP, TF>(grp, M, LD,
                                               forward_solve<NP, TF>(grp, row, (TF)ry, my_inv, slotT), my_inv,
                                               slotT);
                    y += (double)dy;
                }
            }
        }

        // ---- weights, estimate, variance
        double w = x, mu = 0.0;
        if constexpr (ORDINARY)
        {
            double sx = group_sum<NP, double>(grp, live ? x : 0.0, scr);
            double sy = group_sum<NP, double>(grp, live ? y : 0.0, scr);
            if (fabs(sy) < 1e-15) fail = true;
            mu = (sx - 1.0) / sy;
            w = x - mu * y;
        }
        const float mf = (float)mean; // mean_t is float (typedefs.h:122)
        double contrib = live ? w * (double)((float)v - mf) : 0.0;
        double wb = live ? w * b64 : 0.0;
        double est = (double)mf + group_sum<NP, double>(grp, contrib, scr);
        double var = c0 - group_sum<NP, double>(grp, wb, scr) - mu;
        if (var < 0) var = 0;
        if (r == 0)
        {
            if (!fail)
            {
                if (out.write_cont)
                {
                    out.out_data[cell] = (float)est;
                    out.out_mask[cell] = 1;
                }
                if (out.prob) out.prob[(long long)cell * out.prob_stride] = (float)est;
                if (out.est64) out.est64[cell] = est;
                if (out.var) out.var[cell] = var;
                if (out.status) out.status[cell] = 0;
            }
            else if (out.status)
                out.status[cell] = 2;
        }
        grp.sync();
    }
}

template <int NP, typename TF>
size_t solve_smem_per_group()
{
    constexpr int LD = NP + 1;
    size_t b = (size_t)NP * LD * sizeof(TF) + NP * sizeof(int) + NP * sizeof(double) + NP * sizeof(TF) +
               NP * sizeof(double) + 4 * sizeof(double) + 32;
    return (b + 15) / 16 * 16;
}

template <int NP, typename TF, bool ORD, bool REF>
static cudaError_t launch_one(const Geom &g, const int *cells, const int *n_items, int max_items, const int *nb_pid,
                              const int *nb_n, const unsigned long long *pts_xyz, const float *pts_val,
                              const uint8_t *pts_cat, int ind_value, const double *pair64, const float *pair32,
                              double mean, double c0, int steps, const SolveOut &out, int n_sm, cudaStream_t st)
{
    constexpr int threads = 256;
    constexpr int gpb = threads / NP;
    size_t smem = solve_smem_per_group<NP, TF>() * gpb;
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
    kern<<<(unsigned)blocks, threads, smem, st>>>(g, cells, n_items, nb_pid, nb_n, pts_xyz, pts_val, pts_cat,
                                                  ind_value, pair64, pair32, mean, c0, steps, out);
    return cudaGetLastError();
}

template <int NP>
static cudaError_t launch_np(int precision, bool ordinary, const Geom &g, const int *cells, const int *n_items,
                             int max_items, const int *nb_pid, const int *nb_n, const unsigned long long *pts_xyz,
                             const float *pts_val, const uint8_t *pts_cat, int ind_value, const double *pair64,
                             const float *pair32, double mean, double c0, int steps, const SolveOut &out,
                             int n_sm, cudaStream_t st)
{
#define HB_ARGS g, cells, n_items, max_items, nb_pid, nb_n, pts_xyz, pts_val, pts_cat, ind_value, pair64, pair32, mean, c0, steps, out, n_sm, st
    if (precision == 0)
        return ordinary ? launch_one<NP, double, true, false>(HB_ARGS) : launch_one<NP, double, false, false>(HB_ARGS);
    return ordinary ? launch_one<NP, float, true, true>(HB_ARGS) : launch_one<NP, float, false, true>(HB_ARGS);
#undef HB_ARGS
}

cudaError_t launch_solve_bucket(int np, int precision, bool ordinary, const Geom &g, const int *cells,
                                const int *n_items, int max_items, const int *nb_pid, const int *nb_n,
                                const unsigned long long *pts_xyz, const float *pts_val, const uint8_t *pts_cat,
                                int ind_value, const double *pair64, const float *pair32, double mean, double c0,
                                int steps, const SolveOut &out, int n_sm, cudaStream_t st)
{
    switch (np)
    {
    case 8:
        return launch_np<8>(precision, ordinary, g, cells, n_items, max_items, nb_pid, nb_n, pts_xyz, pts_val,
                            pts_cat, ind_value, pair64, pair32, mean, c0, steps, out, n_sm, st);
    case 16:
        return launch_np<16>(precision, ordinary, g, cells, n_items, max_items, nb_pid, nb_n, pts_xyz, pts_val,
                             pts_cat, ind_value, pair64, pair32, mean, c0, steps, out, n_sm, st);
    case 32:
        return launch_np<32>(precision, ordinary, g, cells, n_items, max_items, nb_pid, nb_n, pts_xyz, pts_val,
                             pts_cat, ind_value, pair64, pair32, mean, c0, steps, out, n_sm, st);
    case 64:
        return launch_np<64>(precision, ordinary, g, cells, n_items, max_items, nb_pid, nb_n, pts_xyz, pts_val,
                             pts_cat, ind_value, pair64, pair32, mean, c0, steps, out, n_sm, st);
    default:
        return cudaErrorInvalidValue;
    }
}
} // namespace hb
