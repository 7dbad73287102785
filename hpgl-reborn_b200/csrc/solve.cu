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
// Layout: one system per G = NP / 2 lanes (NP in {8, 16, 32, 64}), lane t
// owning rows t and NP - 1 - t of the (padded) matrix in registers ("folded":
// see the folded kernels below). Rows past the neighbour count n are identity
// rows with zero right-hand sides, which leaves the solution of the first n
// unknowns unchanged. The search stage hands over, per neighbour, its
// pair-table offset lin(o_i) (o_i = neighbour - centre) and its value, so
// cov(c_i, c_j) = pair[centre + lin_i - lin_j] and cov(c_i, centre) =
// pair[centre + lin_i]: assembly is one subtraction and one gather per entry.
//
// Factorisation: right-looking Cholesky with the forward substitution fused in.
// Step j: the owner of column j of each row stores its current A[r][j] in row
// j of the system's shared matrix M and the owner of row j appends its current
// right-hand sides; the row is read back with 16-byte broadcast loads, every
// row r > j is updated A[r][c] -= A[r][j] * M[j][c] / M[j][j] (c > j) and
// rhs_r -= A[r][j] * rhs_j / M[j][j]; row j is scaled by 1/sqrt(M[j][j]) and
// keeps y_j = rhs_j / sqrt(M[j][j]), the forward solution. Afterwards row r
// of M holds column r of L (times sqrt(M[r][r])), which the back substitution
// reads with 16-byte loads of the lane's own rows.
//
// Precision modes:
//   FP64 plain   : T = double throughout. Every kriging quantity is a bilinear
//                  form u^T A^-1 w = (L^-1 u) . (L^-1 w), so the forward
//                  solutions of b, (OK) the ones vector and v - mean suffice:
//                  no back substitution.
//   FP32 refined : the matrix is gathered from the float pair table (the
//                  rounding of the double one), factored and solved in float
//                  for b, (OK) the ones vector and the centred values
//                  v - mean. Each bilinear
//                  form is corrected with one FP64 residual,
//                    u^T A^-1 w = u^T x_w + x_u^T (w - A64 x_w) + O(|e_u| |e_w|),
//                  (x_w = A32^-1 w), so one residual pass in double gives
//                  quadratically small errors without a second triangular solve.
//                  The relative size of the first-order correction bounds what
//                  remains (its square); above `tol` the group falls back to
//                  classic refinement x += A32^-1 (b - A64 x) (up to `steps`
//                  rounds, each with an FP64 residual), and a system that still
//                  does not converge, or whose float factor breaks down, is
//                  queued for the FP64 kernel (status 4) instead of being
//                  reported singular.
#include "engine.cuh"
#include "kernels.h"
#include "solve_common.cuh"
#include "solve_quad.cuh" // static_for

#include <cstdint>

namespace hb
{
// ------------------------------------------------------------------ folded
// FP32-refined systems of up to 64 neighbours, folded: a system is solved by
// G = NP / 2 lanes and lane t owns rows t ("row a", columns 0..t) and
// NP - 1 - t ("row b", columns 0..NP-1-t), so every lane holds NP + 1 entries
// of the lower triangle and a warp solves 32 / G systems at once. Each step of
// the factorisation updates row a over columns j+1..G-1 and row b over
// j+1..NP-1: about 5/8 of the multiply-adds of one row per lane, with the
// shared-memory broadcast, the rsqrt and the synchronisation of a step serving
// two rows. The arithmetic (right-looking Cholesky with the forward
// substitution fused in, FP32 back substitution, dual-weighted FP64 residual
// correction, classic refinement and FP64 escalation) is described at the top
// of this file.
//
// M is stored packed: row j is read and written only from column 4*(j/4) on
// (its first 16-byte chunk holding a column >= j) through the right-hand sides,
// so row j keeps LD/4 - j/4 chunks. Row j's column c sits at float
// 4*row[j] + c; the rows follow one another in order, and each row's start
// is moved forward by whole chunks until the 16-byte chunk index of column 0,
// modulo 8, differs from that of every earlier row of its group of 8 rows.
// The back substitution's 16-byte loads (lanes t..t+7 reading rows t..t+7, or
// NP-1-t down) then keep to distinct banks as in a square layout, at 68%
// (NP = 32) or 60% (NP = 64) of its footprint, which leaves the L1 cache
// the shared memory gives up for the pair-table gathers.
template <int NP>
struct FoldRows
{
    int row[NP]; // chunk index of column 0 of each row
    int chunks;  // 16-byte chunks of the packed matrix
};

template <int NP>
constexpr FoldRows<NP> make_fold_rows()
{
    FoldRows<NP> f{};
    constexpr int C = (NP + 4) / 4; // chunks of a full row
    int end = 0;
    unsigned used = 0;
    for (int j = 0; j < NP; ++j)
    {
        if (j % 8 == 0) used = 0;
        const int a = j / 4;
        int p = end;
        while (used & (1u << ((p - a) & 7))) ++p;
        used |= 1u << ((p - a) & 7);
        f.row[j] = p - a;
        end = p + C - a;
    }
    f.chunks = end;
    return f;
}

__device__ constexpr FoldRows<8> d_fold_rows8 = make_fold_rows<8>();
__device__ constexpr FoldRows<16> d_fold_rows16 = make_fold_rows<16>();
__device__ constexpr FoldRows<32> d_fold_rows32 = make_fold_rows<32>();
__device__ constexpr FoldRows<64> d_fold_rows64 = make_fold_rows<64>();

// Float offset of column 0 of row j of the packed matrix: the tables are
// constant with known contents, so with j known after unrolling the offset
// folds into the shared-memory instruction; a lane's own rows (t, NP-1-t) are
// read once per call.
template <int NP>
__device__ __forceinline__ int fold_row(int j)
{
    if constexpr (NP == 8)
        return 4 * d_fold_rows8.row[j];
    else if constexpr (NP == 16)
        return 4 * d_fold_rows16.row[j];
    else if constexpr (NP == 32)
        return 4 * d_fold_rows32.row[j];
    else
        return 4 * d_fold_rows64.row[j];
}

template <int NP, int R>
struct FoldSmem
{
    static constexpr int LD = NP + 4; // NP entries, then up to 4 right-hand sides
    static constexpr size_t m_bytes = (size_t)make_fold_rows<NP>().chunks * 16;
    static constexpr size_t lin_off = m_bytes;
    static constexpr size_t x_off = (lin_off + NP * sizeof(int) + 15) / 16 * 16;
    static constexpr size_t raw = x_off + (size_t)R * NP * sizeof(double);
    // Systems sharing a warp sit 4 G bytes apart modulo 128, so the G words each
    // writes per step, and the rows they broadcast, fall on disjoint banks.
    static constexpr size_t bytes = raw + (size_t)((4 * (NP / 2) - (int)(raw % 128) + 128) % 128);
};

// The step loops of the folded kernels: unrolled by the compiler up to 32
// rows; at 64, where its unroller gives up (and the rows would go to local
// memory), instantiated step by step.
template <int NP, typename F>
__device__ __forceinline__ void fold_steps(F &&f)
{
    if constexpr (NP > 32)
        static_for<0, NP>([&](auto JC) { f(decltype(JC)::value); });
    else
    {
#pragma unroll
        for (int j = 0; j < NP; ++j) f(j);
    }
}

template <int G>
struct FoldGrp
{
    unsigned mask; // the system's lanes
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    template <typename T>
    __device__ __forceinline__ T bcast(T v, int src) const
    {
        return __shfl_sync(mask, v, src, G);
    }
    template <typename T>
    __device__ __forceinline__ T sum(T v) const
    {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    template <typename T>
    __device__ __forceinline__ T max(T v) const
    {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o, G));
        return v;
    }
};

// Back substitution L^T x = y for both rows of the lane; row r of M holds
// column r of L times sqrt(d_r), read with 16-byte loads of the lane's rows.
template <int NP, int Q>
__device__ __forceinline__ void fold_back(const FoldGrp<NP / 2> &fg, const float *M, int t, const float (&ya)[Q],
                                          const float (&yb)[Q], float inv_a, float inv_b, float (&xa)[Q],
                                          float (&xb)[Q])
{
    constexpr int G = NP / 2;
    const int rb = NP - 1 - t;
    float acc_a[Q], acc_b[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        acc_a[q] = ya[q];
        acc_b[q] = yb[q];
        xa[q] = 0.0f;
        xb[q] = 0.0f;
    }
    const float4 *Ma = reinterpret_cast<const float4 *>(M + fold_row<NP>(t));
    const float4 *Mb = reinterpret_cast<const float4 *>(M + fold_row<NP>(rb));
    float4 ma = make_float4(0, 0, 0, 0), mb = ma;
    fold_steps<NP>([&](const int ic) {
        const int i = NP - 1 - ic;
        if (i % 4 == 3)
        {
            ma = Ma[i / 4];
            mb = Mb[i / 4];
        }
        const float ea = (i % 4 == 0) ? ma.x : (i % 4 == 1) ? ma.y : (i % 4 == 2) ? ma.z : ma.w;
        const float eb = (i % 4 == 0) ? mb.x : (i % 4 == 1) ? mb.y : (i % 4 == 2) ? mb.z : mb.w;
        float xi[Q];
        if (i < G)
        {
            if (t == i)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q) xa[q] = acc_a[q] * inv_a;
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) xi[q] = fg.bcast(xa[q], i);
        }
        else
        {
            if (rb == i)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q) xb[q] = acc_b[q] * inv_b;
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) xi[q] = fg.bcast(xb[q], NP - 1 - i);
        }
        if (t < i)
        {
            const float l = ea * inv_a;
#pragma unroll
            for (int q = 0; q < Q; ++q) acc_a[q] -= l * xi[q];
        }
        if (rb < i)
        {
            const float l = eb * inv_b;
#pragma unroll
            for (int q = 0; q < Q; ++q) acc_b[q] -= l * xi[q];
        }
    });
}

// Forward substitution L y = rhs from the factor kept in M (the refinement
// fallback): L[r][j] = M[j][r] / sqrt(M[j][j]).
template <int NP, int Q>
__device__ __forceinline__ void fold_forward(const FoldGrp<NP / 2> &fg, const float *M, int t, const float (&ra)[Q],
                                             const float (&rb_rhs)[Q], float (&ya)[Q], float (&yb)[Q])
{
    constexpr int G = NP / 2;
    const int rb = NP - 1 - t;
    float acc_a[Q], acc_b[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        acc_a[q] = ra[q];
        acc_b[q] = rb_rhs[q];
        ya[q] = 0.0f;
        yb[q] = 0.0f;
    }
    fold_steps<NP>([&](const int j) {
        const float *Mj = M + fold_row<NP>(j);
        const float inv_j = rsqrtf(Mj[j]);
        float yj[Q];
        if (j < G)
        {
            if (t == j)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q) ya[q] = acc_a[q] * inv_j;
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) yj[q] = fg.bcast(ya[q], j);
        }
        else
        {
            if (rb == j)
            {
#pragma unroll
                for (int q = 0; q < Q; ++q) yb[q] = acc_b[q] * inv_j;
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) yj[q] = fg.bcast(yb[q], NP - 1 - j);
        }
        if (j < G && t > j)
        {
            const float l = Mj[t] * inv_j;
#pragma unroll
            for (int q = 0; q < Q; ++q) acc_a[q] -= l * yj[q];
        }
        if (rb > j)
        {
            const float l = Mj[rb] * inv_j;
#pragma unroll
            for (int q = 0; q < Q; ++q) acc_b[q] -= l * yj[q];
        }
    });
}

// FP64 residuals of both rows: res = rhs - A64 x, A64 rows gathered from the
// double pair table, X the solutions of all rows.
template <int NP, int Q>
__device__ __forceinline__ void fold_residuals(const FoldGrp<NP / 2> &fg, const double *__restrict__ pair64,
                                               long long pc, const int *LIN, double *X, int n, int t, int lin_a,
                                               int lin_b, bool live_a, bool live_b, const double (&xa)[Q],
                                               const double (&xb)[Q], const double (&rhs_a)[Q],
                                               const double (&rhs_b)[Q], double (&res_a)[Q], double (&res_b)[Q])
{
    const int rb = NP - 1 - t;
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        X[q * NP + t] = xa[q];
        X[q * NP + rb] = xb[q];
        res_a[q] = rhs_a[q];
        res_b[q] = rhs_b[q];
    }
    fg.sync();
    const double *base_a = pair64 + pc + lin_a, *base_b = pair64 + pc + lin_b;
#pragma unroll
    for (int c = 0; c < NP; ++c)
    {
        if (c < n)
        {
            const int l = LIN[c];
            double xc[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) xc[q] = X[q * NP + c];
            if (live_a)
            {
                const double a = __ldg(base_a - l);
#pragma unroll
                for (int q = 0; q < Q; ++q) res_a[q] -= a * xc[q];
            }
            if (live_b)
            {
                const double b = __ldg(base_b - l);
#pragma unroll
                for (int q = 0; q < Q; ++q) res_b[q] -= b * xc[q];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
    {
        if (!live_a) res_a[q] = -xa[q];
        if (!live_b) res_b[q] = -xb[q];
    }
    fg.sync();
}

// The bilinear forms x_u^T A64 x_w of the dual-weighted correction, from the
// lower triangle only: for symmetric A,
//   x_u^T A x_w = sum_r ( A_rr u_r w_r + u_r P_w(r) + w_r P_u(r) ),
//   P_w(r) = sum_{c<r} A_rc w_c,
// so each lane gathers the entries of its two rows left of the diagonal (P)
// and the diagonal (D) from the double pair table: one gather per entry of the
// triangle instead of one per entry of the matrix. X receives the R solution
// vectors of all rows.
template <int NP, int R>
__device__ __forceinline__ void fold_bilinear(const FoldGrp<NP / 2> &fg, const double *__restrict__ pair64,
                                              long long pc, const int *LIN, double *X, int n, int t, int lin_a,
                                              int lin_b, bool live_a, bool live_b, const double (&xa)[R],
                                              const double (&xb)[R], double (&Pa)[R], double (&Pb)[R], double &Da,
                                              double &Db)
{
    constexpr int G = NP / 2;
    const int rb = NP - 1 - t;
#pragma unroll
    for (int q = 0; q < R; ++q)
    {
        X[q * NP + t] = xa[q];
        X[q * NP + rb] = xb[q];
        Pa[q] = 0.0;
        Pb[q] = 0.0;
    }
    Da = 0.0;
    Db = 0.0;
    fg.sync();
    const double *base_a = pair64 + pc + lin_a, *base_b = pair64 + pc + lin_b;
#pragma unroll
    for (int c = 0; c < NP; ++c)
    {
        if (c < n)
        {
            const int l = LIN[c];
            double xc[R];
#pragma unroll
            for (int q = 0; q < R; ++q) xc[q] = X[q * NP + c];
            if (c < G && live_a && c <= t)
            {
                const double p = __ldg(base_a - l);
                if (c < t)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) Pa[q] += p * xc[q];
                }
                else
                    Da = p;
            }
            if (live_b && c <= rb)
            {
                const double p = __ldg(base_b - l);
                if (c < rb)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) Pb[q] += p * xc[q];
                }
                else
                    Db = p;
            }
        }
    }
    fg.sync();
}

// Threads per block of the folded kernel (one block per SM): 512 (registers
// capped at 128), so all the systems in flight on an SM come from one run of
// neighbouring cells; the narrow variant (kVariantFoldNarrow) runs 256 with up
// to 255 registers. Systems of 33 to 64 neighbours fold onto one warp each (two
// rows of up to 64 entries per lane): 256-thread blocks.
template <int NP>
constexpr int fold_threads()
{
    return NP <= 32 ? 512 : 256;
}

template <int NP, bool ORDINARY, int TH>
__global__ void __launch_bounds__(TH, 1)
    k_solve_fold(const Geom g, const int2 *__restrict__ cells, const int *__restrict__ n_items_ptr,
                 const int2 *__restrict__ nb_rec, int ind_value, const float *__restrict__ pair32, SolveParams P)
{
    constexpr int G = NP / 2;   // lanes per system
    constexpr int SPW = 32 / G; // systems per warp
    constexpr int QB = ORDINARY ? 2 : 1;
    constexpr int R = QB + 1;
    typedef FoldSmem<NP, R> SM;
    constexpr int LD = SM::LD;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int h = lane / G; // the warp's system slot
    const int t = lane % G;
    const int rb = NP - 1 - t;
    FoldGrp<G> fg;
    fg.mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (h * G));
    unsigned char *gb = smem + SM::bytes * (warp * SPW + h);
    float *M = reinterpret_cast<float *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + SM::lin_off);
    double *X = reinterpret_cast<double *>(gb + SM::x_off);
    const long long pc = P.pc;
    const double *pair64 = P.pair64;

    // The block's contiguous run of items; the warps take SPW consecutive items
    // at a time, so every lane of a warp runs the same number of iterations (a
    // slot past the end solves an empty system and writes nothing).
    const int n_items = *n_items_ptr;
    const int per_block = (n_items + gridDim.x - 1) / gridDim.x;
    const int run_first = blockIdx.x * per_block;
    const int run_end = min(n_items, run_first + per_block);
    const int wstride = nwarps * SPW;
    int base = run_first + warp * SPW;
    int2 w_cur = base + h < run_end ? cells[base + h] : make_int2(0, 0);
    int2 w_nxt = base + wstride + h < run_end ? cells[base + wstride + h] : make_int2(0, 0);
    int2 rec_a = t < w_cur.y ? nb_rec[(long long)w_cur.x * g.k + t] : make_int2(0, 0);
    int2 rec_b = rb < w_cur.y ? nb_rec[(long long)w_cur.x * g.k + rb] : make_int2(0, 0);
    for (; base < run_end; base += wstride)
    {
        const bool valid = base + h < run_end;
        const int my_cell = w_cur.x, my_n = w_cur.y;
        const bool live_a = t < my_n, live_b = rb < my_n;
        const int lin_a = rec_a.x, lin_b = rec_b.x;
        const double vc_a = centred_value(live_a, __int_as_float(rec_a.y), ind_value, P.mf);
        const double vc_b = centred_value(live_b, __int_as_float(rec_b.y), ind_value, P.mf);
        // records of the next iteration
        rec_a = t < w_nxt.y ? nb_rec[(long long)w_nxt.x * g.k + t] : make_int2(0, 0);
        rec_b = rb < w_nxt.y ? nb_rec[(long long)w_nxt.x * g.k + rb] : make_int2(0, 0);
        w_cur = w_nxt;
        w_nxt = base + 2 * wstride + h < run_end ? cells[base + 2 * wstride + h] : make_int2(0, 0);
        LIN[t] = live_a ? lin_a : 0;
        LIN[rb] = live_b ? lin_b : 0;
        fg.sync();

        // ---- assembly: lower triangles of rows a and b; padding rows are identity
        float ra[G], rbv[NP];
#pragma unroll
        for (int c = 0; c < G; ++c)
        {
            float a = 0.0f;
            if (live_a && c <= t) a = __ldg(pair32 + pc + lin_a - LIN[c]);
            if (!live_a && c == t) a = 1.0f;
            ra[c] = a;
        }
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            float a = 0.0f;
            if (live_b && c <= rb) a = __ldg(pair32 + pc + lin_b - LIN[c]);
            if (!live_b && c == rb) a = 1.0f;
            rbv[c] = a;
        }
        const double b64_a = live_a ? __ldg(pair64 + pc + lin_a) : 0.0;
        const double b64_b = live_b ? __ldg(pair64 + pc + lin_b) : 0.0;

        // ---- factorisation with the forward substitution of b, 1 and v - mean
        float rhs_a[R], rhs_b[R], ya[R], yb[R];
        rhs_a[0] = (float)b64_a;
        rhs_b[0] = (float)b64_b;
        if constexpr (ORDINARY)
        {
            rhs_a[1] = live_a ? 1.0f : 0.0f;
            rhs_b[1] = live_b ? 1.0f : 0.0f;
        }
        rhs_a[R - 1] = (float)vc_a;
        rhs_b[R - 1] = (float)vc_b;
#pragma unroll
        for (int q = 0; q < R; ++q)
        {
            ya[q] = 0.0f;
            yb[q] = 0.0f;
        }
        bool fail = false;
        float inv_a = 0.0f, inv_b = 0.0f;
        fold_steps<NP>([&](const int j) {
            // row j of the packed matrix holds columns 4*(j/4) on
            float *Mj = M + fold_row<NP>(j);
            if (j < G)
            {
                if (t >= (j & ~3)) Mj[t] = ra[j];
                if (t == j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) Mj[NP + q] = rhs_a[q];
                }
            }
            if (rb >= (j & ~3)) Mj[rb] = rbv[j];
            if (j >= G && rb == j)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) Mj[NP + q] = rhs_b[q];
            }
            fg.sync();
            float mj[LD];
            const float4 *mv = reinterpret_cast<const float4 *>(Mj);
#pragma unroll
            for (int q = j / 4; q < LD / 4; ++q)
            {
                const float4 v4 = mv[q];
                mj[4 * q] = v4.x;
                mj[4 * q + 1] = v4.y;
                mj[4 * q + 2] = v4.z;
                mj[4 * q + 3] = v4.w;
            }
            const float d = mj[j];
            fail |= !(d > 0.0f);
            const float inv_s = rsqrtf(d);
            const float inv2 = inv_s * inv_s;
            if (j < G)
            {
                const float s = ra[j] * inv2;
#pragma unroll
                for (int c = j + 1; c < G; ++c) ra[c] -= s * mj[c];
                if (t > j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) rhs_a[q] -= s * mj[NP + q];
                }
                ra[j] *= inv_s;
                if (t == j)
                {
                    inv_a = inv_s;
#pragma unroll
                    for (int q = 0; q < R; ++q) ya[q] = rhs_a[q] * inv_s;
                }
            }
            {
                const float s = rbv[j] * inv2;
#pragma unroll
                for (int c = j + 1; c < NP; ++c) rbv[c] -= s * mj[c];
                if (rb > j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) rhs_b[q] -= s * mj[NP + q];
                }
                rbv[j] *= inv_s;
                if (rb == j)
                {
                    inv_b = inv_s;
#pragma unroll
                    for (int q = 0; q < R; ++q) yb[q] = rhs_b[q] * inv_s;
                }
            }
        });

        // ---- back substitution and the dual-weighted FP64 correction of the forms
        float xsa[R], xsb[R];
        fold_back<NP, R>(fg, M, t, ya, yb, inv_a, inv_b, xsa, xsb);
        double xa[R], xb[R];
#pragma unroll
        for (int q = 0; q < R; ++q)
        {
            xa[q] = (double)xsa[q];
            xb[q] = (double)xsb[q];
        }
        const double one_a = live_a ? 1.0 : 0.0, one_b = live_b ? 1.0 : 0.0;
        double r64a[QB], r64b[QB], resa[QB], resb[QB], xqa[QB], xqb[QB];
#pragma unroll
        for (int q = 0; q < QB; ++q)
        {
            r64a[q] = q == 0 ? b64_a : one_a;
            r64b[q] = q == 0 ? b64_b : one_b;
            xqa[q] = xa[q];
            xqb[q] = xb[q];
        }
        // u^T A^-1 w = u^T x_w + x_u^T w - x_u^T A64 x_w + O(|e_u| |e_w|); solution
        // q: 0 = x_b, 1 = x_1 (OK), R-1 = x_v
        double Pa[R], Pb[R], Da, Db;
        fold_bilinear<NP, R>(fg, pair64, pc, LIN, X, my_n, t, lin_a, lin_b, live_a, live_b, xa, xb, Pa, Pb, Da, Db);
        auto bil = [&](int u, int w) {
            return Da * xa[u] * xa[w] + xa[u] * Pa[w] + xa[w] * Pa[u] + Db * xb[u] * xb[w] + xb[u] * Pb[w] +
                   xb[w] * Pb[u];
        };
        constexpr int V = R - 1;
        const double corr_vb = xa[V] * b64_a + xb[V] * b64_b - bil(V, 0);
        const double corr_bb = xa[0] * b64_a + xb[0] * b64_b - bil(0, 0);
        double f_vb = vc_a * xa[0] + vc_b * xb[0] + corr_vb;
        double f_bb = b64_a * xa[0] + b64_b * xb[0] + corr_bb;
        double f_1b = 0.0, f_v1 = 0.0, f_11 = 0.0;
        if constexpr (ORDINARY)
        {
            f_1b = one_a * xa[0] + one_b * xb[0] + xa[1] * b64_a + xb[1] * b64_b - bil(1, 0);
            f_v1 = vc_a * xa[1] + vc_b * xb[1] + xa[V] * one_a + xb[V] * one_b - bil(V, 1);
            f_11 = one_a * xa[1] + one_b * xb[1] + xa[1] * one_a + xb[1] * one_b - bil(1, 1);
        }
        double s_vb = fg.sum(f_vb), s_bb = fg.sum(f_bb);
        double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
        if constexpr (ORDINARY)
        {
            s_1b = fg.sum(f_1b);
            s_v1 = fg.sum(f_v1);
            s_11 = fg.sum(f_11);
        }
        // a-posteriori check: the first-order correction of each form relative
        // to the form's scale; what remains after it is about its square
        const double abs_vb = fg.sum(fabs(vc_a * xa[0]) + fabs(vc_b * xb[0])) + 1e-300;
        const double abs_bb = fg.sum(fabs(b64_a * xa[0]) + fabs(b64_b * xb[0])) + 1e-300;
        const double c1 = fabs(fg.sum(corr_vb)) / abs_vb;
        const double c2 = fabs(fg.sum(corr_bb)) / abs_bb;
        const double dd = fmax(c1, c2);
        bool escalate = fail || !(dd * dd <= P.tol) || !(s_vb == s_vb) || !(s_bb == s_bb);
        if (escalate && P.steps > 0 && !fail)
        {
            // classic refinement x += A32^-1 (b - A64 x) of b (and 1), then the forms uncorrected
            double prev = 0.0;
            bool done = false;
            for (int it = 0; it < P.steps && !done; ++it)
            {
#pragma unroll
                for (int q = 0; q < QB; ++q)
                {
                    xqa[q] = xa[q];
                    xqb[q] = xb[q];
                }
                fold_residuals<NP, QB>(fg, pair64, pc, LIN, X, my_n, t, lin_a, lin_b, live_a, live_b, xqa, xqb, r64a,
                                       r64b, resa, resb);
                float rfa[QB], rfb[QB], yya[QB], yyb[QB], dda[QB], ddb[QB];
#pragma unroll
                for (int q = 0; q < QB; ++q)
                {
                    rfa[q] = (float)resa[q];
                    rfb[q] = (float)resb[q];
                }
                fold_forward<NP, QB>(fg, M, t, rfa, rfb, yya, yyb);
                fold_back<NP, QB>(fg, M, t, yya, yyb, inv_a, inv_b, dda, ddb);
                double dmax = 0.0, xmax = 0.0;
#pragma unroll
                for (int q = 0; q < QB; ++q)
                {
                    xa[q] += (double)dda[q];
                    xb[q] += (double)ddb[q];
                    dmax = fmax(dmax, fmax(fabs((double)dda[q]), fabs((double)ddb[q])));
                    xmax = fmax(xmax, fmax(fabs(xa[q]), fabs(xb[q])));
                }
                dmax = fg.max(dmax);
                xmax = fg.max(xmax);
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
                done = err <= P.tol;
            }
            if (done)
            {
                escalate = false;
                s_vb = fg.sum(vc_a * xa[0] + vc_b * xb[0]);
                s_bb = fg.sum(b64_a * xa[0] + b64_b * xb[0]);
                if constexpr (ORDINARY)
                {
                    s_1b = fg.sum(one_a * xa[0] + one_b * xb[0]);
                    s_v1 = fg.sum(vc_a * xa[1] + vc_b * xb[1]);
                    s_11 = fg.sum(one_a * xa[1] + one_b * xb[1]);
                }
            }
        }
        if (valid && t == 0)
        {
            const SolveOut &out = P.out;
            if (escalate)
            {
                int slot = atomicAdd(P.esc_count, 1);
                P.esc_cells[slot] = make_int2(my_cell, my_n);
                if (out.status) out.status[my_cell] = 4;
            }
            else
            {
                // forms -> estimate and variance (my_kriging_weights.h:312-357)
                double est, var;
                bool bad = fail;
                if constexpr (ORDINARY)
                {
                    if (fabs(s_11) < 1e-15) bad = true;
                    const double mu = (s_1b - 1.0) / s_11;
                    est = s_vb - mu * s_v1;
                    var = P.c0 - s_bb + mu * s_1b - mu;
                }
                else
                {
                    est = (double)(out.cell_mean ? out.cell_mean[my_cell] : P.mf) + s_vb;
                    var = P.c0 - s_bb;
                }
                if (var < 0) var = 0;
                if (!bad)
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
        }
        fg.sync();
    }
}

// FP64-plain systems of up to 64 neighbours, folded like k_solve_fold (G = NP/2
// lanes per system, lane t owning rows t and NP-1-t). FP64 plain needs only the
// forward substitution: every kriging quantity is a bilinear form
// u^T A^-1 w = (L^-1 u) . (L^-1 w) of b, (OK) the ones vector and v - mean, so the
// forward solutions that ride in the factorisation's broadcast rows are summed
// directly; there is no back substitution and no residual.
template <int NP>
struct Fold64Smem
{
    static constexpr int LD = NP + 4; // doubles: NP entries, then up to 4 right-hand sides
    // Row j is read only at step j (no back substitution), so two rows in turn
    // suffice: the step's warp synchronisation orders the writes of row j + 2
    // after every lane's reads of row j.
    static constexpr size_t m_bytes = (size_t)2 * LD * sizeof(double);
    static constexpr size_t lin_off = m_bytes;
    // systems sharing a warp 16 bytes apart modulo 128: their broadcast rows on different banks
    static constexpr size_t bytes = (lin_off + NP * sizeof(int) + 127) / 128 * 128 + 16;
};

// Threads per block of the FP64 folded kernel (one block per SM): 384 threads
// cap registers at 168, which the step's row read 16 bytes at a time fits with
// almost no spills, and give each scheduler three warps to cover the FP64
// dependency latency (256 threads: 198M cells/s; 320: 173M; 512, spilling: 196M;
// 384: 211M on the 256x256x128 benchmark); the narrow variant runs 256. Systems
// of 33 to 64 neighbours fold onto one warp each (rows t and 63 - t: 96
// doubles a lane), in 256-thread blocks with up to 255 registers.
template <int NP>
constexpr int fold64_threads()
{
    return NP <= 32 ? 384 : 256;
}

template <int NP, bool ORDINARY, int TH>
__global__ void __launch_bounds__(TH, 1)
    k_solve_fold64(const Geom g, const int2 *__restrict__ cells, const int *__restrict__ n_items_ptr,
                   const int2 *__restrict__ nb_rec, int ind_value, SolveParams P)
{
    constexpr int G = NP / 2;
    constexpr int SPW = 32 / G;
    constexpr int QB = ORDINARY ? 2 : 1;
    constexpr int R = QB + 1;
    typedef Fold64Smem<NP> SM;
    constexpr int LD = SM::LD;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int h = lane / G;
    const int t = lane % G;
    const int rb = NP - 1 - t;
    FoldGrp<G> fg;
    fg.mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (h * G));
    unsigned char *gb = smem + SM::bytes * (warp * SPW + h);
    double *M = reinterpret_cast<double *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + SM::lin_off);
    const long long pc = P.pc;
    const double *pair64 = P.pair64;

    const int n_items = *n_items_ptr;
    const int per_block = (n_items + gridDim.x - 1) / gridDim.x;
    const int run_first = blockIdx.x * per_block;
    const int run_end = min(n_items, run_first + per_block);
    const int wstride = nwarps * SPW;
    int base = run_first + warp * SPW;
    int2 w_cur = base + h < run_end ? cells[base + h] : make_int2(0, 0);
    int2 w_nxt = base + wstride + h < run_end ? cells[base + wstride + h] : make_int2(0, 0);
    int2 rec_a = t < w_cur.y ? nb_rec[(long long)w_cur.x * g.k + t] : make_int2(0, 0);
    int2 rec_b = rb < w_cur.y ? nb_rec[(long long)w_cur.x * g.k + rb] : make_int2(0, 0);
    for (; base < run_end; base += wstride)
    {
        const bool valid = base + h < run_end;
        const int my_cell = w_cur.x, my_n = w_cur.y;
        const bool live_a = t < my_n, live_b = rb < my_n;
        const int lin_a = rec_a.x, lin_b = rec_b.x;
        const double vc_a = centred_value(live_a, __int_as_float(rec_a.y), ind_value, P.mf);
        const double vc_b = centred_value(live_b, __int_as_float(rec_b.y), ind_value, P.mf);
        rec_a = t < w_nxt.y ? nb_rec[(long long)w_nxt.x * g.k + t] : make_int2(0, 0);
        rec_b = rb < w_nxt.y ? nb_rec[(long long)w_nxt.x * g.k + rb] : make_int2(0, 0);
        w_cur = w_nxt;
        w_nxt = base + 2 * wstride + h < run_end ? cells[base + 2 * wstride + h] : make_int2(0, 0);
        LIN[t] = live_a ? lin_a : 0;
        LIN[rb] = live_b ? lin_b : 0;
        fg.sync();

        // ---- assembly (lower triangles of rows a and b; padding rows identity)
        double ra[G], rbv[NP];
        const double *base_a = pair64 + pc + lin_a, *base_b = pair64 + pc + lin_b;
#pragma unroll
        for (int c = 0; c < G; ++c)
        {
            double a = 0.0;
            if (live_a && c <= t) a = __ldg(base_a - LIN[c]);
            if (!live_a && c == t) a = 1.0;
            ra[c] = a;
        }
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            double a = 0.0;
            if (live_b && c <= rb) a = __ldg(base_b - LIN[c]);
            if (!live_b && c == rb) a = 1.0;
            rbv[c] = a;
        }
        const double b64_a = live_a ? __ldg(base_a) : 0.0;
        const double b64_b = live_b ? __ldg(base_b) : 0.0;

        // ---- factorisation with the forward substitution of b, 1 and v - mean
        double rhs_a[R], rhs_b[R], ya[R], yb[R];
        rhs_a[0] = b64_a;
        rhs_b[0] = b64_b;
        if constexpr (ORDINARY)
        {
            rhs_a[1] = live_a ? 1.0 : 0.0;
            rhs_b[1] = live_b ? 1.0 : 0.0;
        }
        rhs_a[R - 1] = vc_a;
        rhs_b[R - 1] = vc_b;
#pragma unroll
        for (int q = 0; q < R; ++q)
        {
            ya[q] = 0.0;
            yb[q] = 0.0;
        }
        bool fail = false;
        fold_steps<NP>([&](const int j) {
            double *Mj = M + (j & 1) * LD;
            if (j < G)
            {
                Mj[t] = ra[j];
                if (t == j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) Mj[NP + q] = rhs_a[q];
                }
            }
            Mj[rb] = rbv[j];
            if (j >= G && rb == j)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) Mj[NP + q] = rhs_b[q];
            }
            fg.sync();
            // row j is applied as it is read, 16 bytes at a time, so it never
            // sits in registers whole
            const double d = Mj[j];
            fail |= !(d > 0.0);
            const double inv_s = rsqrt(d);
            const double inv2 = inv_s * inv_s;
            const double s_a = j < G ? ra[j] * inv2 : 0.0;
            const double s_b = rbv[j] * inv2;
            const double2 *mv = reinterpret_cast<const double2 *>(Mj);
#pragma unroll
            for (int q2 = j / 2; q2 < LD / 2; ++q2)
            {
                const double2 v2 = mv[q2];
#pragma unroll
                for (int e = 0; e < 2; ++e)
                {
                    const int c = 2 * q2 + e;
                    const double m = e == 0 ? v2.x : v2.y;
                    if (c > j && c < NP)
                    {
                        if (j < G && c < G) ra[c] -= s_a * m;
                        rbv[c] -= s_b * m;
                    }
                    else if (c >= NP && c < NP + R)
                    {
                        if (j < G && t > j) rhs_a[c - NP] -= s_a * m;
                        if (rb > j) rhs_b[c - NP] -= s_b * m;
                    }
                }
            }
            if (j < G)
            {
                ra[j] *= inv_s;
                if (t == j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) ya[q] = rhs_a[q] * inv_s;
                }
            }
            rbv[j] *= inv_s;
            if (rb == j)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) yb[q] = rhs_b[q] * inv_s;
            }
        });

        // ---- forms (L^-1 u) . (L^-1 w); q: 0 = b, 1 = ones (OK), R-1 = v - mean
        constexpr int V = R - 1;
        const double s_vb = fg.sum(ya[V] * ya[0] + yb[V] * yb[0]);
        const double s_bb = fg.sum(ya[0] * ya[0] + yb[0] * yb[0]);
        double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
        if constexpr (ORDINARY)
        {
            s_1b = fg.sum(ya[1] * ya[0] + yb[1] * yb[0]);
            s_v1 = fg.sum(ya[V] * ya[1] + yb[V] * yb[1]);
            s_11 = fg.sum(ya[1] * ya[1] + yb[1] * yb[1]);
        }
        if (valid && t == 0)
        {
            // forms -> estimate and variance (my_kriging_weights.h:312-357)
            const SolveOut &out = P.out;
            double est, var;
            bool bad = fail;
            if constexpr (ORDINARY)
            {
                if (fabs(s_11) < 1e-15) bad = true;
                const double mu = (s_1b - 1.0) / s_11;
                est = s_vb - mu * s_v1;
                var = P.c0 - s_bb + mu * s_1b - mu;
            }
            else
            {
                est = (double)(out.cell_mean ? out.cell_mean[my_cell] : P.mf) + s_vb;
                var = P.c0 - s_bb;
            }
            if (var < 0) var = 0;
            if (!bad)
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
        fg.sync();
    }
}

template <int NP, typename TF, bool ORD, bool REF, int TH>
static cudaError_t launch_one(const Geom &g, const int2 *cells, const int *n_items, int max_items, const int2 *nb_rec,
                              int ind_value, const float *pair32, const SolveParams &P, int n_sm, cudaStream_t st)
{
    int blocks = 0;
    if constexpr (REF)
    {
        constexpr int fthreads = TH;
        constexpr int spb = fthreads / (NP / 2); // systems per block
        const size_t smem = FoldSmem<NP, ORD ? 3 : 2>::bytes * spb;
        auto kern = k_solve_fold<NP, ORD, TH>;
        cudaError_t e = launch_kernel(kern, fthreads, smem, max_items, spb, n_sm, blocks);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)blocks, fthreads, smem, st>>>(g, cells, n_items, nb_rec, ind_value, pair32, P);
    }
    else
    {
        constexpr int fthreads = TH;
        constexpr int spb = fthreads / (NP / 2); // systems per block
        const size_t smem = Fold64Smem<NP>::bytes * spb;
        auto kern = k_solve_fold64<NP, ORD, TH>;
        cudaError_t e = launch_kernel(kern, fthreads, smem, max_items, spb, n_sm, blocks);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)blocks, fthreads, smem, st>>>(g, cells, n_items, nb_rec, ind_value, P);
    }
    return cudaGetLastError();
}

template <int NP>
static cudaError_t launch_np(int precision, int variant, bool ordinary, const Geom &g, const int2 *cells,
                             const int *n_items, int max_items, const int2 *nb_rec, int ind_value, const float *pair32,
                             const SolveParams &P, int n_sm, cudaStream_t st)
{
#define HB_ARGS g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st
    if constexpr (NP <= 32)
    {
        if (precision == 0)
        {
            if (variant == kVariantFoldNarrow)
                return ordinary ? launch_one<NP, double, true, false, 256>(HB_ARGS)
                                : launch_one<NP, double, false, false, 256>(HB_ARGS);
            return ordinary ? launch_one<NP, double, true, false, 384>(HB_ARGS)
                            : launch_one<NP, double, false, false, 384>(HB_ARGS);
        }
        if constexpr (NP == 32)
        {
            if (variant == kVariantTile || variant == kVariantTileNarrow)
                return launch_solve_tile(NP, ordinary, variant == kVariantTile ? 384 : 192, HB_ARGS);
        }
        if (variant == kVariantQuad || variant == kVariantQuadNarrow || variant == kVariantDefault)
            return launch_solve_quad(NP, ordinary, variant == kVariantQuadNarrow ? 256 : 384, HB_ARGS);
        if (variant == kVariantFoldNarrow)
            return ordinary ? launch_one<NP, float, true, true, 256>(HB_ARGS)
                            : launch_one<NP, float, false, true, 256>(HB_ARGS);
        return ordinary ? launch_one<NP, float, true, true, 512>(HB_ARGS)
                        : launch_one<NP, float, false, true, 512>(HB_ARGS);
    }
    else
    {
        if (variant != kVariantFold) return launch_solve_wide(precision, ordinary, HB_ARGS);
        if (precision == 0)
            return ordinary ? launch_one<NP, double, true, false, 256>(HB_ARGS)
                            : launch_one<NP, double, false, false, 256>(HB_ARGS);
        return ordinary ? launch_one<NP, float, true, true, 256>(HB_ARGS)
                        : launch_one<NP, float, false, true, 256>(HB_ARGS);
    }
#undef HB_ARGS
}

bool solve_variant_valid(int np, int precision, int variant)
{
    if (variant == kVariantDefault) return true;
    if (np > 32) return variant == kVariantFold || variant == kVariantWide;
    if (precision == 1)
        return (variant >= kVariantFold && variant <= kVariantQuadNarrow) ||
               ((variant == kVariantTile || variant == kVariantTileNarrow) && np == 32);
    return variant == kVariantFold || variant == kVariantFoldNarrow;
}

cudaError_t launch_solve_bucket(int np, int precision, int variant, bool ordinary, const Geom &g, const int2 *cells,
                                const int *n_items, int max_items, const int2 *nb_rec, const int *nb_n, int ind_value,
                                const double *pair64, const float *pair32, double mean, double c0, int steps,
                                double tol, const SolveOut &out, int2 *esc_cells, int *esc_count, int n_sm,
                                cudaStream_t st)
{
    (void)nb_n;
    SolveParams P;
    P.pair64 = pair64;
    P.pc = g.pair_center;
    P.mf = (float)mean; // mean_t is float (typedefs.h:122)
    P.c0 = c0;
    P.steps = steps;
    P.tol = tol;
    P.out = out;
    P.esc_cells = esc_cells;
    P.esc_count = esc_count;
#define HB_NARGS precision, variant, ordinary, g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st
    switch (np)
    {
    case 8:
        return launch_np<8>(HB_NARGS);
    case 16:
        return launch_np<16>(HB_NARGS);
    case 32:
        return launch_np<32>(HB_NARGS);
    case 64:
        return launch_np<64>(HB_NARGS);
    default:
        return cudaErrorInvalidValue;
    }
#undef HB_NARGS
}
} // namespace hb
