// FP32-refined batched kriging solves with four rows per lane ("quad fold"),
// for systems of up to 32 neighbours (S1/S2/K2 of the hot path: the
// dpotrf / dpotrs calls of sk_kriging_weights_3 and ok_kriging_weights_3,
// my_kriging_weights.h:147-165 and :284-303, and the combine of
// combiner.h:10-25).
//
// Layout. A system of NP (padded) unknowns is solved by G = NP / 4 lanes, so a
// warp holds 32 / G systems. Lane t owns the four rows
//   r0 = t, r1 = NP/2 - 1 - t, r2 = NP/2 + t, r3 = NP - 1 - t,
// whose lower-triangle lengths add up to 2 NP + 2 for every lane. Slot k keeps
// its row in a register array of len(k) = NP/4, NP/2, 3NP/4, NP floats (every
// row of slot k is shorter than len(k)); entries past a row's diagonal are
// never read. Padding rows (neighbour count n <= r < NP) are identity rows
// with zero right-hand sides.
//
// Factorisation: right-looking Cholesky with the forward substitution of the
// right-hand sides b, (OK) the ones vector and v - mean fused in. Step j: each
// lane writes A[r][j] of its rows into a broadcast row of the system's shared
// buffer and the owner of row j appends its right-hand sides; after a warp
// barrier every lane reads the row 16 bytes at a time and applies it as it
// reads (A[r][c] -= A[r][j] A[c][j] / A[j][j], paired columns through the
// packed FP32x2 fused multiply-add). Two broadcast rows are used in turn.
// The factor stays in registers: after step j, A[r][j] holds L[r][j].
//
// Back substitution L^T x = y from registers: for i = NP-1 down to 0 the
// owner of row i publishes L[i][0..i-1] through the same two-row buffer and
// its x_i (shuffled), and every lane subtracts L[i][r] x_i from the rows r < i
// it owns. Shared memory per system is two rows, the neighbours' pair-table
// offsets and the FP64 solutions of the correction (about 1.2 KB for
// NP = 32), so the SM's L1 stays available for the pair-table gathers.
//
// Precision: every kriging quantity is a bilinear form u^T A^-1 w; with the
// float solutions x_u = A32^-1 u and x_w it is corrected by one FP64 residual
//   u^T A^-1 w = u^T x_w + x_u^T w - x_u^T A64 x_w + O(|e_u| |e_w|),
// where x_u^T A64 x_w is formed from the lower triangle of the double pair
// table (one gather per entry). The relative size of the first-order
// correction bounds what remains; a system above `tol`, or whose float factor
// breaks down, is queued (status 4) for the two-rows-per-lane FP32 kernel of
// solve.cu, which runs classic refinement (x += A32^-1 (b - A64 x), FP64
// residuals) and hands what still does not converge to the FP64 kernel.
#include "engine.cuh"
#include "kernels.h"
#include "solve_common.cuh"
#include "solve_quad.cuh"

#include <cstdint>
#include <type_traits>

namespace hb
{
template <int NP, int R>
struct QuadSmem
{
    static constexpr int G = NP / 4;
    static constexpr int LDB = NP + 4; // floats per broadcast row: NP entries, then 4 right-hand sides
    static constexpr size_t lin_off = (size_t)2 * LDB * sizeof(float);
    static constexpr size_t rec_off = (lin_off + NP * sizeof(int) + 15) / 16 * 16;
    static constexpr size_t raw = rec_off + (size_t)2 * NP * sizeof(int2);
    // Systems of one warp sit 4 G bytes (at least 16) apart modulo 128, so the
    // rows their lanes write at each step fall on distinct banks.
    static constexpr int shift = 4 * G < 16 ? 16 : 4 * G;
    static constexpr size_t bytes = raw + (size_t)((shift - (int)(raw % 128) + 128) % 128);
};

// Threads per block TH: 384 (168 registers, twelve warps) or 256 (255
// registers, eight warps), one block per SM.
template <int NP, bool ORDINARY, int TH>
__global__ void __launch_bounds__(TH, 1)
    k_solve_quad(const Geom g, const int2 *__restrict__ cells, const int *__restrict__ n_items_ptr,
                 const int2 *__restrict__ nb_rec, int ind_value, const float *__restrict__ pair32, SolveParams P)
{
    constexpr int G = NP / 4;   // lanes per system
    constexpr int H = NP / 2;
    constexpr int SPW = 32 / G; // systems per warp
    constexpr int QB = ORDINARY ? 2 : 1;
    constexpr int R = QB + 1;   // b, (OK) 1, v - mean
    constexpr int V = R - 1;
    typedef QuadSmem<NP, R> SM;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int h = lane / G; // the warp's system slot
    const int t = lane % G;
    unsigned char *sb = smem + SM::bytes * (warp * SPW + h);
    float *B = reinterpret_cast<float *>(sb);
    int *LIN = reinterpret_cast<int *>(sb + SM::lin_off);
    int2 *REC = reinterpret_cast<int2 *>(sb + SM::rec_off); // two sets of NP records, in turn
    const int rows[4] = {t, H - 1 - t, H + t, NP - 1 - t};
    const long long pc = P.pc;
    const double *pair64 = P.pair64;
    const float *p32c = pair32 + pc;
    const double *p64c = pair64 + pc;
    const double d64 = __ldg(p64c); // cov(p, p) of the pair table: every live diagonal entry

    // The block's contiguous run of items; the warps take SPW consecutive
    // items at a time (a slot past the end solves an empty system and writes
    // nothing), so every lane of a warp runs the same iterations. Each lane
    // copies the records of its own rows for the next iteration into shared
    // memory while the current one is solved.
    const int n_items = *n_items_ptr;
    const int per_block = (n_items + gridDim.x - 1) / gridDim.x;
    const int run_first = blockIdx.x * per_block;
    const int run_end = min(n_items, run_first + per_block);
    const int wstride = nwarps * SPW;
    int base = run_first + warp * SPW;
    int2 w_cur = base + h < run_end ? cells[base + h] : make_int2(0, 0);
    int2 w_nxt = base + wstride + h < run_end ? cells[base + wstride + h] : make_int2(0, 0);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (rows[k] < w_cur.y) q_cp_async8(REC + rows[k], nb_rec + (long long)w_cur.x * g.k + rows[k]);
    q_cp_async_commit();
    int par = 0;
    for (; base < run_end; base += wstride, par ^= 1)
    {
        const bool valid = base + h < run_end;
        const int my_cell = w_cur.x, my_n = w_cur.y;
        const int2 *rec = REC + par * NP;
        q_cp_async_wait_all();
#pragma unroll
        for (int k = 0; k < 4; ++k) LIN[rows[k]] = rows[k] < my_n ? rec[rows[k]].x : 0;
        // records of the next iteration
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (rows[k] < w_nxt.y)
                q_cp_async8(REC + (par ^ 1) * NP + rows[k], nb_rec + (long long)w_nxt.x * g.k + rows[k]);
        q_cp_async_commit();
        w_cur = w_nxt;
        w_nxt = base + 2 * wstride + h < run_end ? cells[base + 2 * wstride + h] : make_int2(0, 0);
        __syncwarp();

        // ---- assembly and factorisation with the forward substitution of b, 1 and v - mean
        float2 A[5 * NP / 4];
        q_assemble<NP>(A, LIN, p32c, rows, my_n);
        float rhs[4][R]; // right-hand sides, then forward solutions, then float solutions
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            const bool live = rows[k] < my_n;
            rhs[k][0] = live ? __ldg(p32c + LIN[rows[k]]) : 0.0f;
            if constexpr (ORDINARY) rhs[k][1] = live ? 1.0f : 0.0f;
            rhs[k][V] = (float)centred_value(live, __int_as_float(rec[rows[k]].y), ind_value, P.mf);
        }
        float inv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        const bool fail = q_factor<NP, R>(A, rhs, inv, rows, t, B);
        __syncwarp();
        // ---- back substitution with the correction's FP64 row sums
        // x_u^T A x_w = sum_r ( A_rr u_r w_r + u_r P_w(r) + w_r P_u(r) ), P_w(r) = sum_{c<r} A_rc w_c
        bool live[4];
        int lin[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            live[k] = rows[k] < my_n;
            lin[k] = LIN[rows[k]];
        }
        double Pk[4][R];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int q = 0; q < R; ++q) Pk[k][q] = 0.0;
        q_back_p<NP, R, 2>(A, rows, inv, t, B, rhs, p64c, lin, LIN, live, Pk);

        // ---- the dual-weighted FP64 correction of the bilinear forms
        double b64[4], vc[4], one[4], x[4][R];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            b64[k] = live[k] ? __ldg(p64c + lin[k]) : 0.0;
            vc[k] = centred_value(live[k], __int_as_float(rec[rows[k]].y), ind_value, P.mf);
            one[k] = live[k] ? 1.0 : 0.0;
#pragma unroll
            for (int q = 0; q < R; ++q) x[k][q] = (double)rhs[k][q];
        }
        auto bil = [&](int u, int w) {
            double sacc = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                sacc += one[k] * d64 * x[k][u] * x[k][w] + x[k][u] * Pk[k][w] + x[k][w] * Pk[k][u];
            return sacc;
        };
        auto dot = [&](const double (&a)[4], int w) {
            double sacc = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) sacc += a[k] * x[k][w];
            return sacc;
        };
        // u^T A^-1 w = u^T x_w + x_u^T w - x_u^T A64 x_w; solution q: 0 = x_b, 1 = x_1 (OK), V = x_v
        const double corr_vb = dot(b64, V) - bil(V, 0);
        const double corr_bb = dot(b64, 0) - bil(0, 0);
        double s_vb = q_sum<G>(dot(vc, 0) + corr_vb);
        double s_bb = q_sum<G>(dot(b64, 0) + corr_bb);
        double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
        if constexpr (ORDINARY)
        {
            s_1b = q_sum<G>(dot(one, 0) + dot(b64, 1) - bil(1, 0));
            s_v1 = q_sum<G>(dot(vc, 1) + dot(one, V) - bil(V, 1));
            s_11 = q_sum<G>(2.0 * dot(one, 1) - bil(1, 1));
        }
        // a-posteriori check: the first-order correction of each form relative
        // to the form's scale; what remains after it is about its square
        double abs_vb = 0.0, abs_bb = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            abs_vb += fabs(vc[k] * x[k][0]);
            abs_bb += fabs(b64[k] * x[k][0]);
        }
        abs_vb = q_sum<G>(abs_vb) + 1e-300;
        abs_bb = q_sum<G>(abs_bb) + 1e-300;
        const double c1 = fabs(q_sum<G>(corr_vb)) / abs_vb;
        const double c2 = fabs(q_sum<G>(corr_bb)) / abs_bb;
        const double dd = fmax(c1, c2);
        const bool escalate = fail || !(dd * dd <= P.tol) || !(s_vb == s_vb) || !(s_bb == s_bb);
        if (valid && t == 0)
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
    q_cp_async_wait_all();
}

template <int NP, bool ORD, int TH>
static cudaError_t launch_quad_one(const Geom &g, const int2 *cells, const int *n_items, int max_items,
                                   const int2 *nb_rec, int ind_value, const float *pair32, const SolveParams &P,
                                   int n_sm, cudaStream_t st)
{
    constexpr int spb = TH / 32 * (32 / (NP / 4));
    const size_t smem = QuadSmem<NP, ORD ? 3 : 2>::bytes * spb;
    auto kern = k_solve_quad<NP, ORD, TH>;
    int blocks = 0;
    cudaError_t e = launch_kernel(kern, TH, smem, max_items, spb, n_sm, blocks);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)blocks, TH, smem, st>>>(g, cells, n_items, nb_rec, ind_value, pair32, P);
    return cudaGetLastError();
}

template <int NP, bool ORD>
static cudaError_t launch_quad_th(int threads, const Geom &g, const int2 *cells, const int *n_items, int max_items,
                                  const int2 *nb_rec, int ind_value, const float *pair32, const SolveParams &P,
                                  int n_sm, cudaStream_t st)
{
    if (threads == 256)
        return launch_quad_one<NP, ORD, 256>(g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st);
    return launch_quad_one<NP, ORD, 384>(g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st);
}

cudaError_t launch_solve_quad(int np, bool ordinary, int threads, const Geom &g, const int2 *cells,
                              const int *n_items, int max_items, const int2 *nb_rec, int ind_value,
                              const float *pair32, const SolveParams &P, int n_sm, cudaStream_t st)
{
#define HB_QARGS threads, g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st
    switch (np)
    {
    case 8:
        return ordinary ? launch_quad_th<8, true>(HB_QARGS) : launch_quad_th<8, false>(HB_QARGS);
    case 16:
        return ordinary ? launch_quad_th<16, true>(HB_QARGS) : launch_quad_th<16, false>(HB_QARGS);
    case 32:
        return ordinary ? launch_quad_th<32, true>(HB_QARGS) : launch_quad_th<32, false>(HB_QARGS);
    default:
        return cudaErrorInvalidValue;
    }
#undef HB_QARGS
}
} // namespace hb
