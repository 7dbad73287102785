// Batched kriging solves of 33 to 64 neighbours, one warp per system (S1/S2/K2
// of the hot path for the largest bucket: the dpotrf / dpotrs calls of
// sk_kriging_weights_3 and ok_kriging_weights_3, my_kriging_weights.h:147-165
// and :284-303, and the combine of combiner.h:10-25).
//
// Lane t owns rows a = t and b = 63 - t of the system (the fold of the smaller
// kernels). The factorisation is right-looking, with every row held in
// registers SHIFTED: before step j, ra[k] holds A(a, j + k) and rbv[k] holds
// A(b, j + k), so the entries a step reads and writes sit at the same register
// indices whatever j is. Column j is broadcast through shared memory shifted
// the same way (W[k] = A(j + 1 + k, j), the diagonal at W[63], the right-hand
// sides after it), the update is
//     rbv[k] = rbv[k + 1] - (A(b, j) / A(j, j)) W[k]
// (likewise ra), and the steps of a phase of eight run as a rolled loop over
// one code body whose array lengths (64 - 8p, 32 - 8p) are fixed for the
// phase. Compared with a fully unrolled triangular factorisation this does
// about 15 % more FMAs, but its code is about 1/20 the size: unrolled, the
// FP32 kernel's 64 steps plus its back substitution and correction did not fit
// the instruction caches, and its warps waited on instruction fetch ten times
// as long as on anything else.
//
// k_solve_wide64: FP64 plain, forward substitution only (the forms are
// (L^-1 u) . (L^-1 w)). k_solve_wide32: FP32 factorisation (two steps a body
// as a rank-2 update, the rows as float2 pairs shifted by two, so that the
// update runs as packed FP32x2 FMAs) and substitutions,
// the bilinear forms corrected with the FP64 dual-weighted residual from the
// lower triangle (as the other FP32-refined kernels do); a system whose check
// fails is queued for the FP64 kernel.
#include "engine.cuh"
#include "kernels.h"
#include "solve_common.cuh"
#include "solve_quad.cuh" // static_for

#include <cstdint>

namespace hb
{
constexpr int kWideNP = 64;
constexpr int kWidePhase = 8; // factorisation steps per rolled phase

// Broadcast buffer: 63 column entries, the diagonal at [63], R right-hand
// sides from [64]; padded to 16 bytes.
template <typename T, int R>
__host__ __device__ constexpr int wide_ldw()
{
    return ((kWideNP + R) * (int)sizeof(T) + 15) / 16 * 16 / (int)sizeof(T);
}

// Start of column j in the packed column-major lower triangle
__host__ __device__ constexpr int wide_col(int j)
{
    return kWideNP * j - j * (j - 1) / 2;
}

template <typename T, int R, bool BACK>
struct WideSmem
{
    static constexpr int LDW = wide_ldw<T, R>();
    // two broadcast buffers in turn; FP32 (BACK) broadcasts two columns a body
    static constexpr size_t w_bytes = (size_t)(BACK ? 4 : 2) * LDW * sizeof(T);
    static constexpr size_t lin_off = w_bytes;
    // (FP32) the factor's columns before scaling, for the back substitution
    static constexpr size_t lc_off = lin_off + kWideNP * sizeof(int);
    static constexpr size_t lc_bytes = BACK ? (size_t)kWideNP * (kWideNP + 1) / 2 * sizeof(float) : 0;
    // (FP32) the R solution vectors in double, for the correction's row sums
    static constexpr size_t x_off = (lc_off + lc_bytes + 15) / 16 * 16;
    static constexpr size_t raw = x_off + (BACK ? (size_t)R * kWideNP * sizeof(double) : 0);
    static constexpr size_t bytes = (raw + 15) / 16 * 16;
};

__device__ __forceinline__ float wide_rsqrt(float d) { return rsqrtf(d); }
__device__ __forceinline__ double wide_rsqrt(double d) { return rsqrt(d); }

// One shift-update of the lane's rows by column j (entries in W):
// r[k] = r[k + 1] - s W[k] for k < L - 1 (L <= N), read 16 bytes at a time.
template <int L, typename T, int N>
__device__ __forceinline__ void wide_shift(T (&r)[N], T s, const T *W)
{
    if constexpr (L > 1)
    {
        constexpr int V = 16 / (int)sizeof(T);
        static_for<0, (L - 1 + V - 1) / V>([&](auto CC) {
            constexpr int c = decltype(CC)::value;
            T w[V];
            if constexpr (V == 4)
            {
                const float4 v = reinterpret_cast<const float4 *>(W)[c];
                w[0] = v.x;
                w[1] = v.y;
                w[2] = v.z;
                w[3] = v.w;
            }
            else
            {
                const double2 v = reinterpret_cast<const double2 *>(W)[c];
                w[0] = v.x;
                w[1] = v.y;
            }
#pragma unroll
            for (int e = 0; e < V; ++e)
            {
                const int k = V * c + e;
                if (k < L - 1) r[k] = r[k + 1] - s * w[e];
            }
        });
    }
}

// Right-looking Cholesky of the warp's system with the forward substitution
// of R right-hand sides riding in the broadcast rows. On return ya / yb hold
// the forward solutions of rows a and b, inv_a / inv_b their 1 / L(r, r);
// with KEEP the factor's columns before scaling are left in LC
// (LC[wide_col(j) + r - j] = L(r, j) sqrt(A(j, j)) for r >= j).
template <typename T, int R, bool KEEP>
__device__ __forceinline__ bool wide_factor(T (&ra)[32], T (&rbv)[kWideNP], T (&rhs_a)[R], T (&rhs_b)[R],
                                            T (&ya)[R], T (&yb)[R], T &inv_a, T &inv_b, int t, T *Wbuf, float *LC)
{
    constexpr int NP = kWideNP;
    constexpr int LDW = wide_ldw<T, R>();
    const int b = NP - 1 - t;
    bool fail = false;
    static_for<0, NP / kWidePhase>([&](auto PC) {
        constexpr int p = decltype(PC)::value;
        constexpr int LA = 32 - kWidePhase * p > 0 ? 32 - kWidePhase * p : 0;
        constexpr int LB = NP - kWidePhase * p;
#pragma unroll 1
        for (int jj = 0; jj < kWidePhase; ++jj)
        {
            const int j = kWidePhase * p + jj;
            T *W = Wbuf + (j & 1) * LDW;
            if constexpr (LA > 0)
            {
                if (t > j) W[t - j - 1] = ra[0];
                if (t == j)
                {
                    W[NP - 1] = ra[0];
#pragma unroll
                    for (int q = 0; q < R; ++q) W[NP + q] = rhs_a[q];
                }
                if constexpr (KEEP)
                {
                    if (t >= j) LC[wide_col(j) + t - j] = (float)ra[0];
                }
            }
            if (b > j) W[b - j - 1] = rbv[0];
            if (b == j)
            {
                W[NP - 1] = rbv[0];
#pragma unroll
                for (int q = 0; q < R; ++q) W[NP + q] = rhs_b[q];
            }
            if constexpr (KEEP)
            {
                if (b >= j) LC[wide_col(j) + b - j] = (float)rbv[0];
            }
            __syncwarp();
            const T d = W[NP - 1];
            fail |= !(d > T(0));
            const T inv_s = wide_rsqrt(d);
            const T inv2 = inv_s * inv_s;
            const T s_b = rbv[0] * inv2;
            T wr[R];
#pragma unroll
            for (int q = 0; q < R; ++q) wr[q] = W[NP + q];
            if constexpr (LA > 0)
            {
                const T s_a = ra[0] * inv2;
                wide_shift<LA>(ra, s_a, W);
                if (t > j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) rhs_a[q] -= s_a * wr[q];
                }
                if (t == j)
                {
                    inv_a = inv_s;
#pragma unroll
                    for (int q = 0; q < R; ++q) ya[q] = rhs_a[q] * inv_s;
                }
            }
            wide_shift<LB>(rbv, s_b, W);
            if (b > j)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) rhs_b[q] -= s_b * wr[q];
            }
            if (b == j)
            {
                inv_b = inv_s;
#pragma unroll
                for (int q = 0; q < R; ++q) yb[q] = rhs_b[q] * inv_s;
            }
        }
    });
    return fail;
}

// FP32: r[m] = r[m + 1] - s0 (V[2m + 2], V[2m + 3]) - s1 (U[2m + 2], U[2m + 3])
// for pairs m < L - 1 (L <= N): two steps' updates of the lane's row, shifted
// by two entries, as packed FP32x2 FMAs on aligned register pairs.
template <int L, int N>
__device__ __forceinline__ void wide_shift2(float2 (&r)[N], float s0, float s1, const float *V, const float *U)
{
    if constexpr (L > 1)
    {
        const float2 n0 = make_float2(-s0, -s0), n1 = make_float2(-s1, -s1);
        static_for<0, L / 2 + 1>([&](auto KC) {
            constexpr int k = decltype(KC)::value; // 16-byte chunk k holds pairs 2k, 2k + 1
            constexpr bool lo = 2 * k - 1 >= 0 && 2 * k - 1 < L - 1, hi = 2 * k < L - 1;
            if constexpr (lo || hi)
            {
                const float4 v = reinterpret_cast<const float4 *>(V)[k];
                const float4 u = reinterpret_cast<const float4 *>(U)[k];
                if constexpr (lo)
                {
                    constexpr int m = 2 * k - 1;
                    r[m] = __ffma2_rn(n1, make_float2(u.x, u.y), __ffma2_rn(n0, make_float2(v.x, v.y), r[m + 1]));
                }
                if constexpr (hi)
                {
                    constexpr int m = 2 * k;
                    r[m] = __ffma2_rn(n1, make_float2(u.z, u.w), __ffma2_rn(n0, make_float2(v.z, v.w), r[m + 1]));
                }
            }
        });
    }
}

// The FP32 factorisation two steps at a time (a rank-2 update), rows held as
// float2 pairs shifted by two per body, so both updates run as packed FP32x2
// FMAs on aligned pairs. Column j is broadcast from row j on (V[i] = A(j + i,
// j), the diagonal at V[0]) and column j + 1, after step j's update, from row
// j on as well (U[i] = A'(j + i, j + 1), its diagonal at U[1]): the entries a
// pair of rows needs then sit in aligned pairs of both buffers. Results,
// outputs and the kept columns in LC are those of wide_factor<float, R, true>
// (the same FMAs in the same order).
template <int R, int PH>
__device__ __forceinline__ bool wide_factor2(float2 (&ra)[16], float2 (&rb)[32], float (&rhs_a)[R],
                                             float (&rhs_b)[R], float (&ya)[R], float (&yb)[R], float &inv_a,
                                             float &inv_b, int t, float *Wbuf, float *LC)
{
    constexpr int NP = kWideNP;
    constexpr int LDW = wide_ldw<float, R>();
    const int b = NP - 1 - t;
    bool fail = false;
    static_for<0, NP / PH>([&](auto PC) {
        constexpr int p = decltype(PC)::value;
        constexpr int LA = 32 - PH * p > 0 ? (32 - PH * p) / 2 : 0; // pairs
        constexpr int LB = (NP - PH * p) / 2;
#pragma unroll 1
        for (int jj = 0; jj < PH; jj += 2)
        {
            const int j = PH * p + jj;
            float *V = Wbuf + ((j >> 1) & 1) * 2 * LDW;
            float *U = V + LDW;
            // ---- step j
            if constexpr (LA > 0)
            {
                if (t >= j)
                {
                    V[t - j] = ra[0].x;
                    LC[wide_col(j) + t - j] = ra[0].x;
                }
                if (t == j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) V[NP + q] = rhs_a[q];
                }
            }
            if (b >= j)
            {
                V[b - j] = rb[0].x;
                LC[wide_col(j) + b - j] = rb[0].x;
            }
            if (b == j)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) V[NP + q] = rhs_b[q];
            }
            __syncwarp();
            const float d0 = V[0];
            fail |= !(d0 > 0.0f);
            const float i0 = rsqrtf(d0);
            const float i0s = i0 * i0;
            const float v1 = V[1];
            float vr[R];
#pragma unroll
            for (int q = 0; q < R; ++q) vr[q] = V[NP + q];
            const float sb0 = rb[0].x * i0s;
            const float cb = rb[0].y - sb0 * v1; // A'(b, j + 1)
            if (b > j)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) rhs_b[q] -= sb0 * vr[q];
            }
            if (b == j)
            {
                inv_b = i0;
#pragma unroll
                for (int q = 0; q < R; ++q) yb[q] = rhs_b[q] * i0;
            }
            float sa0 = 0.0f, ca = 0.0f;
            if constexpr (LA > 0)
            {
                sa0 = ra[0].x * i0s;
                ca = ra[0].y - sa0 * v1;
                if (t > j)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) rhs_a[q] -= sa0 * vr[q];
                }
                if (t == j)
                {
                    inv_a = i0;
#pragma unroll
                    for (int q = 0; q < R; ++q) ya[q] = rhs_a[q] * i0;
                }
            }
            // ---- step j + 1: column j + 1 after step j
            if constexpr (LA > 0)
            {
                if (t > j)
                {
                    U[t - j] = ca;
                    LC[wide_col(j + 1) + t - j - 1] = ca;
                }
                if (t == j + 1)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) U[NP + q] = rhs_a[q];
                }
            }
            if (b > j)
            {
                U[b - j] = cb;
                LC[wide_col(j + 1) + b - j - 1] = cb;
            }
            if (b == j + 1)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) U[NP + q] = rhs_b[q];
            }
            __syncwarp();
            const float d1 = U[1];
            fail |= !(d1 > 0.0f);
            const float i1 = rsqrtf(d1);
            const float i1s = i1 * i1;
            float ur[R];
#pragma unroll
            for (int q = 0; q < R; ++q) ur[q] = U[NP + q];
            const float sb1 = cb * i1s;
            if (b > j + 1)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) rhs_b[q] -= sb1 * ur[q];
            }
            if (b == j + 1)
            {
                inv_b = i1;
#pragma unroll
                for (int q = 0; q < R; ++q) yb[q] = rhs_b[q] * i1;
            }
            float sa1 = 0.0f;
            if constexpr (LA > 0)
            {
                sa1 = ca * i1s;
                if (t > j + 1)
                {
#pragma unroll
                    for (int q = 0; q < R; ++q) rhs_a[q] -= sa1 * ur[q];
                }
                if (t == j + 1)
                {
                    inv_a = i1;
#pragma unroll
                    for (int q = 0; q < R; ++q) ya[q] = rhs_a[q] * i1;
                }
            }
            // ---- both updates, the rows shifted by two
            wide_shift2<LB>(rb, sb0, sb1, V, U);
            if constexpr (LA > 0) wide_shift2<LA>(ra, sa0, sa1, V, U);
        }
    });
    return fail;
}

__device__ __forceinline__ double wide_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The item loop shared by both kernels: each warp takes items run_first +
// warp, + warps, ... of the block's contiguous run, with the next item's
// records loaded during the current solve.
struct WideItems
{
    int item, end, stride;
    int2 w;
    int2 rec_a, rec_b;
    __device__ __forceinline__ void load(const Geom &g, const int2 *__restrict__ cells,
                                         const int2 *__restrict__ nb_rec, int t)
    {
        w = item < end ? cells[item] : make_int2(0, 0);
        const int b = kWideNP - 1 - t;
        rec_a = t < w.y ? nb_rec[(long long)w.x * g.k + t] : make_int2(0, 0);
        rec_b = b < w.y ? nb_rec[(long long)w.x * g.k + b] : make_int2(0, 0);
    }
};

// FP64 plain, forward substitution only.
template <bool ORDINARY, int TH>
__global__ void __launch_bounds__(TH, 1)
    k_solve_wide64(const Geom g, const int2 *__restrict__ cells, const int *__restrict__ n_items_ptr,
                   const int2 *__restrict__ nb_rec, int ind_value, SolveParams P)
{
    constexpr int NP = kWideNP;
    constexpr int QB = ORDINARY ? 2 : 1;
    constexpr int R = QB + 1;
    constexpr int V = R - 1;
    typedef WideSmem<double, R, false> SM;
    extern __shared__ __align__(16) unsigned char smem[];
    const int t = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = NP - 1 - t;
    unsigned char *gb = smem + SM::bytes * warp;
    double *Wbuf = reinterpret_cast<double *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + SM::lin_off);
    const double *p64c = P.pair64 + P.pc;

    const int n_items = *n_items_ptr;
    const int per_block = (n_items + gridDim.x - 1) / gridDim.x;
    WideItems it;
    it.item = blockIdx.x * per_block + warp;
    it.end = min(n_items, blockIdx.x * per_block + per_block);
    it.stride = TH / 32;
    it.load(g, cells, nb_rec, t);
    while (it.item < it.end)
    {
        const int my_cell = it.w.x, my_n = it.w.y;
        const bool live_a = t < my_n, live_b = b < my_n;
        const int lin_a = it.rec_a.x, lin_b = it.rec_b.x;
        const double vc_a = centred_value(live_a, __int_as_float(it.rec_a.y), ind_value, P.mf);
        const double vc_b = centred_value(live_b, __int_as_float(it.rec_b.y), ind_value, P.mf);
        it.item += it.stride;
        it.load(g, cells, nb_rec, t);
        LIN[t] = live_a ? lin_a : 0;
        LIN[b] = live_b ? lin_b : 0;
        __syncwarp();

        // ---- assembly (lower triangles of rows a and b; padding rows identity)
        double ra[32], rbv[NP];
        const double *base_a = p64c + lin_a, *base_b = p64c + lin_b;
#pragma unroll
        for (int c = 0; c < 32; ++c)
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
            if (live_b && c <= b) a = __ldg(base_b - LIN[c]);
            if (!live_b && c == b) a = 1.0;
            rbv[c] = a;
        }
        double rhs_a[R], rhs_b[R], ya[R], yb[R];
        rhs_a[0] = live_a ? __ldg(base_a) : 0.0;
        rhs_b[0] = live_b ? __ldg(base_b) : 0.0;
        if constexpr (ORDINARY)
        {
            rhs_a[1] = live_a ? 1.0 : 0.0;
            rhs_b[1] = live_b ? 1.0 : 0.0;
        }
        rhs_a[V] = vc_a;
        rhs_b[V] = vc_b;
#pragma unroll
        for (int q = 0; q < R; ++q) ya[q] = yb[q] = 0.0;
        double inv_a = 0.0, inv_b = 0.0;
        const bool fail = wide_factor<double, R, false>(ra, rbv, rhs_a, rhs_b, ya, yb, inv_a, inv_b, t, Wbuf,
                                                         nullptr);

        // ---- forms (L^-1 u) . (L^-1 w); q: 0 = b, 1 = ones (OK), V = v - mean
        const double s_vb = wide_sum(ya[V] * ya[0] + yb[V] * yb[0]);
        const double s_bb = wide_sum(ya[0] * ya[0] + yb[0] * yb[0]);
        double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
        if constexpr (ORDINARY)
        {
            s_1b = wide_sum(ya[1] * ya[0] + yb[1] * yb[0]);
            s_v1 = wide_sum(ya[V] * ya[1] + yb[V] * yb[1]);
            s_11 = wide_sum(ya[1] * ya[1] + yb[1] * yb[1]);
        }
        if (t == 0) write_solution<ORDINARY>(P, my_cell, fail, s_vb, s_bb, s_1b, s_v1, s_11);
        __syncwarp();
    }
}

// FP32 factorisation and substitutions, bilinear forms corrected in FP64.
template <bool ORDINARY, int TH>
__global__ void __launch_bounds__(TH, 1)
    k_solve_wide32(const Geom g, const int2 *__restrict__ cells, const int *__restrict__ n_items_ptr,
                   const int2 *__restrict__ nb_rec, int ind_value, const float *__restrict__ pair32, SolveParams P)
{
    constexpr int NP = kWideNP;
    constexpr int QB = ORDINARY ? 2 : 1;
    constexpr int R = QB + 1;
    constexpr int V = R - 1;
    typedef WideSmem<float, R, true> SM;
    extern __shared__ __align__(16) unsigned char smem[];
    const int t = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = NP - 1 - t;
    unsigned char *gb = smem + SM::bytes * warp;
    float *Wbuf = reinterpret_cast<float *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + SM::lin_off);
    float *LC = reinterpret_cast<float *>(gb + SM::lc_off);
    double *X = reinterpret_cast<double *>(gb + SM::x_off);
    const double *p64c = P.pair64 + P.pc;
    const float *p32c = pair32 + P.pc;
    const double d64 = __ldg(p64c);

    const int n_items = *n_items_ptr;
    const int per_block = (n_items + gridDim.x - 1) / gridDim.x;
    WideItems it;
    it.item = blockIdx.x * per_block + warp;
    it.end = min(n_items, blockIdx.x * per_block + per_block);
    it.stride = TH / 32;
    it.load(g, cells, nb_rec, t);
    while (it.item < it.end)
    {
        const int my_cell = it.w.x, my_n = it.w.y;
        const bool live_a = t < my_n, live_b = b < my_n;
        const int lin_a = it.rec_a.x, lin_b = it.rec_b.x;
        const double vc_a = centred_value(live_a, __int_as_float(it.rec_a.y), ind_value, P.mf);
        const double vc_b = centred_value(live_b, __int_as_float(it.rec_b.y), ind_value, P.mf);
        it.item += it.stride;
        it.load(g, cells, nb_rec, t);
        LIN[t] = live_a ? lin_a : 0;
        LIN[b] = live_b ? lin_b : 0;
        __syncwarp();

        // ---- assembly from the float pair table
        float2 ra[16], rbv[NP / 2];
#pragma unroll
        for (int c = 0; c < 32; ++c)
        {
            float a = 0.0f;
            if (live_a && c <= t) a = __ldg(p32c + lin_a - LIN[c]);
            if (!live_a && c == t) a = 1.0f;
            if (c & 1)
                ra[c >> 1].y = a;
            else
                ra[c >> 1].x = a;
        }
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            float a = 0.0f;
            if (live_b && c <= b) a = __ldg(p32c + lin_b - LIN[c]);
            if (!live_b && c == b) a = 1.0f;
            if (c & 1)
                rbv[c >> 1].y = a;
            else
                rbv[c >> 1].x = a;
        }
        const double b64_a = live_a ? __ldg(p64c + lin_a) : 0.0;
        const double b64_b = live_b ? __ldg(p64c + lin_b) : 0.0;
        float rhs_a[R], rhs_b[R], ya[R], yb[R];
        rhs_a[0] = (float)b64_a;
        rhs_b[0] = (float)b64_b;
        if constexpr (ORDINARY)
        {
            rhs_a[1] = live_a ? 1.0f : 0.0f;
            rhs_b[1] = live_b ? 1.0f : 0.0f;
        }
        rhs_a[V] = (float)vc_a;
        rhs_b[V] = (float)vc_b;
#pragma unroll
        for (int q = 0; q < R; ++q) ya[q] = yb[q] = 0.0f;
        float inv_a = 0.0f, inv_b = 0.0f;
        const bool fail = wide_factor2<R, kWidePhase>(ra, rbv, rhs_a, rhs_b, ya, yb, inv_a, inv_b, t, Wbuf, LC);
        __syncwarp();

        // ---- back substitution L^T x = y from the kept columns: lane t reads
        // column t (and b) of the factor, L(i, t) = LC[wide_col(t) + i - t] inv_t
        float acc_a[R], acc_b[R], xa[R], xb[R];
#pragma unroll
        for (int q = 0; q < R; ++q)
        {
            acc_a[q] = ya[q];
            acc_b[q] = yb[q];
            xa[q] = xb[q] = 0.0f;
        }
        const float *La = LC + wide_col(t) - t;
        const float *Lb = LC + wide_col(b) - b;
#pragma unroll 1
        for (int i = NP - 1; i >= 32; --i)
        {
            if (b == i)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) xb[q] = acc_b[q] * inv_b;
            }
            float xi[R];
#pragma unroll
            for (int q = 0; q < R; ++q) xi[q] = __shfl_sync(0xffffffffu, xb[q], NP - 1 - i);
            const float la = La[i] * inv_a;
#pragma unroll
            for (int q = 0; q < R; ++q) acc_a[q] -= la * xi[q];
            if (b < i)
            {
                const float lb = Lb[i] * inv_b;
#pragma unroll
                for (int q = 0; q < R; ++q) acc_b[q] -= lb * xi[q];
            }
        }
#pragma unroll 1
        for (int i = 31; i >= 0; --i)
        {
            if (t == i)
            {
#pragma unroll
                for (int q = 0; q < R; ++q) xa[q] = acc_a[q] * inv_a;
            }
            float xi[R];
#pragma unroll
            for (int q = 0; q < R; ++q) xi[q] = __shfl_sync(0xffffffffu, xa[q], i);
            if (t < i)
            {
                const float la = La[i] * inv_a;
#pragma unroll
                for (int q = 0; q < R; ++q) acc_a[q] -= la * xi[q];
            }
        }

        // ---- the dual-weighted FP64 correction of the forms:
        // u^T A^-1 w = u^T x_w + x_u^T w - x_u^T A64 x_w + O(|e_u| |e_w|), the
        // quadratic term from the lower triangle: sum_r A_rr u_r w_r + u_r P_w(r)
        // + w_r P_u(r), P_w(r) = sum_{c<r} A_rc w_c (one FP64 gather per entry)
        double x_a[R], x_b[R];
#pragma unroll
        for (int q = 0; q < R; ++q)
        {
            x_a[q] = (double)xa[q];
            x_b[q] = (double)xb[q];
            X[q * NP + t] = x_a[q];
            X[q * NP + b] = x_b[q];
        }
        __syncwarp();
        double Pa[R], Pb[R];
#pragma unroll
        for (int q = 0; q < R; ++q) Pa[q] = Pb[q] = 0.0;
        const double *base_a = p64c + lin_a, *base_b = p64c + lin_b;
        // (eight columns a batch: the batch's sixteen gathers in flight together;
        // every LIN and X entry of the 64 rows is set, padding rows to zero)
        constexpr int PB = 8;
#pragma unroll 1
        for (int c0 = 0; c0 < my_n; c0 += PB)
        {
            double pa[PB], pb[PB];
#pragma unroll
            for (int e = 0; e < PB; ++e)
            {
                const int c = c0 + e;
                const int l = LIN[c];
                pa[e] = live_a && c < t ? __ldg(base_a - l) : 0.0;
                pb[e] = live_b && c < b ? __ldg(base_b - l) : 0.0;
            }
#pragma unroll
            for (int e = 0; e < PB; ++e)
            {
#pragma unroll
                for (int q = 0; q < R; ++q)
                {
                    const double xc = X[q * NP + c0 + e];
                    Pa[q] = fma(pa[e], xc, Pa[q]);
                    Pb[q] = fma(pb[e], xc, Pb[q]);
                }
            }
        }
        const double one_a = live_a ? 1.0 : 0.0, one_b = live_b ? 1.0 : 0.0;
        const double da = one_a * d64, db = one_b * d64;
        auto bil = [&](int u, int w) {
            return da * x_a[u] * x_a[w] + x_a[u] * Pa[w] + x_a[w] * Pa[u] + db * x_b[u] * x_b[w] + x_b[u] * Pb[w] +
                   x_b[w] * Pb[u];
        };
        const double corr_vb = x_a[V] * b64_a + x_b[V] * b64_b - bil(V, 0);
        const double corr_bb = x_a[0] * b64_a + x_b[0] * b64_b - bil(0, 0);
        const double s_vb = wide_sum(vc_a * x_a[0] + vc_b * x_b[0] + corr_vb);
        const double s_bb = wide_sum(b64_a * x_a[0] + b64_b * x_b[0] + corr_bb);
        double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
        if constexpr (ORDINARY)
        {
            s_1b = wide_sum(one_a * x_a[0] + one_b * x_b[0] + x_a[1] * b64_a + x_b[1] * b64_b - bil(1, 0));
            s_v1 = wide_sum(vc_a * x_a[1] + vc_b * x_b[1] + x_a[V] * one_a + x_b[V] * one_b - bil(V, 1));
            s_11 = wide_sum(2.0 * (one_a * x_a[1] + one_b * x_b[1]) - bil(1, 1));
        }
        // a-posteriori check: the first-order correction of each form relative
        // to the form's scale; what remains after it is about its square
        const double abs_vb = wide_sum(fabs(vc_a * x_a[0]) + fabs(vc_b * x_b[0])) + 1e-300;
        const double abs_bb = wide_sum(fabs(b64_a * x_a[0]) + fabs(b64_b * x_b[0])) + 1e-300;
        const double c1 = fabs(wide_sum(corr_vb)) / abs_vb;
        const double c2 = fabs(wide_sum(corr_bb)) / abs_bb;
        const double dd = fmax(c1, c2);
        const bool escalate = fail || !(dd * dd <= P.tol) || !(s_vb == s_vb) || !(s_bb == s_bb);
        if (t == 0)
        {
            if (escalate)
            {
                const int slot = atomicAdd(P.esc_count, 1);
                P.esc_cells[slot] = make_int2(my_cell, my_n);
                if (P.out.status) P.out.status[my_cell] = 4;
            }
            else
                write_solution<ORDINARY>(P, my_cell, fail, s_vb, s_bb, s_1b, s_v1, s_11);
        }
        __syncwarp();
    }
}

// Threads per block: 256 (up to 255 registers; the FP64 rows take 192). FP32
// in 384-thread blocks (168 registers) spilled in the factorisation's body and
// ran 6 % slower (213 against 200 ms on the clustered 512x512x64 grid).
template <bool ORD, bool F64>
static cudaError_t launch_wide_one(const Geom &g, const int2 *cells, const int *n_items, int max_items,
                                   const int2 *nb_rec, int ind_value, const float *pair32, const SolveParams &P,
                                   int n_sm, cudaStream_t st)
{
    constexpr int R = ORD ? 3 : 2;
    constexpr int TH = 256;
    const size_t smem = (F64 ? WideSmem<double, R, false>::bytes : WideSmem<float, R, true>::bytes) * (TH / 32);
    int blocks = 0;
    if constexpr (F64)
    {
        auto kern = k_solve_wide64<ORD, TH>;
        cudaError_t e = launch_kernel(kern, TH, smem, max_items, TH / 32, n_sm, blocks);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)blocks, TH, smem, st>>>(g, cells, n_items, nb_rec, ind_value, P);
    }
    else
    {
        auto kern = k_solve_wide32<ORD, TH>;
        cudaError_t e = launch_kernel(kern, TH, smem, max_items, TH / 32, n_sm, blocks);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)blocks, TH, smem, st>>>(g, cells, n_items, nb_rec, ind_value, pair32, P);
    }
    return cudaGetLastError();
}

cudaError_t launch_solve_wide(int precision, bool ordinary, const Geom &g, const int2 *cells, const int *n_items,
                              int max_items, const int2 *nb_rec, int ind_value, const float *pair32,
                              const SolveParams &P, int n_sm, cudaStream_t st)
{
#define HB_ARGS g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st
    if (precision == 0)
        return ordinary ? launch_wide_one<true, true>(HB_ARGS) : launch_wide_one<false, true>(HB_ARGS);
    return ordinary ? launch_wide_one<true, false>(HB_ARGS) : launch_wide_one<false, false>(HB_ARGS);
#undef HB_ARGS
}
} // namespace hb
