// A folded FP64 solve of up to 32 symmetric positive definite systems per
// warp pair (shared by the simulation and cokriging kernels).
//
// Sixteen lanes hold one system: lane t owns rows t and 31 - t of the lower
// triangle (rows of a system with n < 32 unknowns are padded with the
// identity). The right-looking Cholesky factorisation broadcasts column j of
// the updated matrix through shared-memory row j, and carries the forward
// substitution of QB right-hand sides in the same rows; the back substitution
// reads column i of L back from the lane's own rows (row r of M holds column r
// of L times sqrt(d_r)). The matrix entries are covariances read from a pair
// table: A[r][c] = pair_c[lin_r - lin_c] with lin the pair-table offsets of the
// unknowns relative to the target.
#pragma once
#include <cuda_runtime.h>

namespace hb
{
constexpr int kFold32NP = 32, kFold32G = 16;
constexpr int kFold32LD = kFold32NP + 2; // 32 entries, then up to two right-hand sides

// M is stored packed: row j is read and written only from column 2*(j/2) on
// (its first 16-byte pair holding a column >= j), so it keeps LD - 2*(j/2)
// doubles. Row j's column c sits at double row[j] + c; the rows follow one
// another, each start moved forward until row[j] is even (16-byte pairs) and
// its residue modulo 16 is used by at most one earlier row of its group of 16
// (rows t and 31 - t of the lanes), so the back substitution's 8-byte column
// reads keep the two-way bank conflicts of the square layout at 74% of its
// footprint; the L1 cache gets what the shared memory gives up.
struct Fold32Rows
{
    int row[kFold32NP];
    int doubles;
};
constexpr Fold32Rows make_fold32_rows()
{
    Fold32Rows f{};
    int end = 0;
    int cnt[2][16] = {};
    for (int j = 0; j < kFold32NP; ++j)
    {
        const int a = 2 * (j / 2), grp = j / 16;
        int p = end;
        while ((p - a) % 2 != 0 || cnt[grp][(p - a) % 16] >= 2) ++p;
        cnt[grp][(p - a) % 16] += 1;
        f.row[j] = p - a;
        end = p + kFold32LD - a;
    }
    f.doubles = end;
    return f;
}
__device__ constexpr Fold32Rows d_fold32_rows = make_fold32_rows();
constexpr size_t kFold32MBytes = (size_t)make_fold32_rows().doubles * 8;
// per system: packed M, then LIN (32 ints); systems sharing a warp 16 bytes
// apart modulo 128 so that their broadcast rows fall on different banks
constexpr size_t kFold32SysBytes = (kFold32MBytes + kFold32NP * 4 + 127) / 128 * 128 + 16;

// Solves A [x] = [rhs] for the lane's rows t and 31 - t (QB <= 2 right-hand
// sides; rows of non-live unknowns carry zeros). `gm` is the system's lane
// mask; LIN must hold the 32 offsets (0 for non-live rows) and be visible to
// the system's lanes. load_rhs(rhs_a, rhs_b) fills the lane's right-hand sides
// once the matrix loads are issued (their loads then queue behind those);
// after_assembly() and after_factor() run at those points (the callers issue
// prefetches there). Returns true when a pivot is not
// positive (or NaN), or, with EPS_PIVOT, below machine epsilon (the test of
// the reference's Gaussian elimination, gauss_solver.cpp:37-41). With SCALE,
// A[r][c] = pair * (sig_r * sig_c), SIG holding the 32 row scales (visible to
// the system's lanes) and sig_a / sig_b the lane's own. nmax, the same on every
// lane of the warp, bounds the live unknowns of both its systems: the steps of
// the padding rows beyond it change no live row and are skipped (a uniform
// bound keeps the warp's two systems in step; rows of M beyond it are never
// written nor read).
template <int QB, bool EPS_PIVOT = false, bool SCALE = false, typename F0, typename F1, typename F2>
__device__ __forceinline__ bool fold32_solve(const double *pair_c, const int *LIN, double *M, unsigned gm, int t,
                                             bool live_a, bool live_b, int lin_a, int lin_b, F0 load_rhs,
                                             double (&xa)[QB], double (&xb)[QB], F1 after_assembly,
                                             F2 after_factor, const double *SIG = nullptr, double sig_a = 1.0,
                                             double sig_b = 1.0, int nmax = kFold32NP)
{
    constexpr int NP = kFold32NP, G = kFold32G, LD = kFold32LD;
    const int rb = NP - 1 - t;
    const int row_a = d_fold32_rows.row[t], row_b = d_fold32_rows.row[rb]; // the lane's rows in M
    // ---- assembly (lower triangles of rows t and 31 - t; padding rows identity)
    double ra[G], rbv[NP];
    const double *base_a = pair_c + lin_a, *base_b = pair_c + lin_b;
#pragma unroll
    for (int c = 0; c < G; ++c)
    {
        double e = 0.0;
        if (live_a && c <= t)
        {
            e = __ldg(base_a - LIN[c]);
            if (SCALE) e = __dmul_rn(e, __dmul_rn(sig_a, SIG[c]));
        }
        if (!live_a && c == t) e = 1.0;
        ra[c] = e;
    }
#pragma unroll
    for (int c = 0; c < NP; ++c)
    {
        double e = 0.0;
        if (live_b && c <= rb)
        {
            e = __ldg(base_b - LIN[c]);
            if (SCALE) e = __dmul_rn(e, __dmul_rn(sig_b, SIG[c]));
        }
        if (!live_b && c == rb) e = 1.0;
        rbv[c] = e;
    }
    double rhs_a[QB], rhs_b[QB], ya[QB], yb[QB];
    load_rhs(rhs_a, rhs_b);
    after_assembly();

    // ---- factorisation with the forward substitution of the right-hand sides
#pragma unroll
    for (int q = 0; q < QB; ++q)
    {
        ya[q] = 0.0;
        yb[q] = 0.0;
    }
    bool fail = false;
    double inv_a = 0.0, inv_b = 0.0;
#pragma unroll
    for (int j = 0; j < NP; ++j)
    {
        if (j >= nmax) break;
        // row j of the packed matrix holds columns 2*(j/2) on
        double *Mj = M + d_fold32_rows.row[j];
        if (j < G)
        {
            if (t >= (j & ~1)) Mj[t] = ra[j];
            if (t == j)
            {
#pragma unroll
                for (int q = 0; q < QB; ++q) Mj[NP + q] = rhs_a[q];
            }
        }
        if (rb >= (j & ~1)) Mj[rb] = rbv[j];
        if (j >= G && rb == j)
        {
#pragma unroll
            for (int q = 0; q < QB; ++q) Mj[NP + q] = rhs_b[q];
        }
        __syncwarp(gm);
        double mj[LD];
        const double2 *mv = reinterpret_cast<const double2 *>(Mj);
#pragma unroll
        for (int q = j / 2; q < LD / 2; ++q)
        {
            const double2 v2 = mv[q];
            mj[2 * q] = v2.x;
            mj[2 * q + 1] = v2.y;
        }
        const double d = mj[j];
        fail |= EPS_PIVOT ? !(d >= 2.220446049250313080847e-16) : !(d > 0.0);
        const double inv_s = rsqrt(d);
        const double inv2 = inv_s * inv_s;
        if (j < G)
        {
            const double sc = ra[j] * inv2;
#pragma unroll
            for (int c = j + 1; c < G; ++c) ra[c] -= sc * mj[c];
            if (t > j)
            {
#pragma unroll
                for (int q = 0; q < QB; ++q) rhs_a[q] -= sc * mj[NP + q];
            }
            ra[j] *= inv_s;
            if (t == j)
            {
                inv_a = inv_s;
#pragma unroll
                for (int q = 0; q < QB; ++q) ya[q] = rhs_a[q] * inv_s;
            }
        }
        {
            const double sc = rbv[j] * inv2;
#pragma unroll
            for (int c = j + 1; c < NP; ++c) rbv[c] -= sc * mj[c];
            if (rb > j)
            {
#pragma unroll
                for (int q = 0; q < QB; ++q) rhs_b[q] -= sc * mj[NP + q];
            }
            rbv[j] *= inv_s;
            if (rb == j)
            {
                inv_b = inv_s;
#pragma unroll
                for (int q = 0; q < QB; ++q) yb[q] = rhs_b[q] * inv_s;
            }
        }
    }

    after_factor();

    // ---- back substitution L^T x = y; L[i][row] = M[row][i] / sqrt(d_row)
#pragma unroll
    for (int q = 0; q < QB; ++q)
    {
        xa[q] = 0.0;
        xb[q] = 0.0;
    }
#pragma unroll
    for (int i = NP - 1; i >= 0; --i)
    {
        if (i >= nmax) continue;
        double xi[QB];
        if (i >= G)
        {
            if (rb == i)
            {
#pragma unroll
                for (int q = 0; q < QB; ++q) xb[q] = yb[q] * inv_b;
            }
#pragma unroll
            for (int q = 0; q < QB; ++q) xi[q] = __shfl_sync(gm, xb[q], NP - 1 - i, G);
        }
        else
        {
            if (t == i)
            {
#pragma unroll
                for (int q = 0; q < QB; ++q) xa[q] = ya[q] * inv_a;
            }
#pragma unroll
            for (int q = 0; q < QB; ++q) xi[q] = __shfl_sync(gm, xa[q], i, G);
        }
        if (t < i)
        {
            const double l = M[row_a + i] * inv_a;
#pragma unroll
            for (int q = 0; q < QB; ++q) ya[q] -= l * xi[q];
        }
        if (rb < i)
        {
            const double l = M[row_b + i] * inv_b;
#pragma unroll
            for (int q = 0; q < QB; ++q) yb[q] -= l * xi[q];
        }
    }

    return fail;
}
} // namespace hb
