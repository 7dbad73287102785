// Pieces shared by the batched kriging solve kernels (solve.cu, solve_quad.cu):
// the launch parameters, the centring of neighbour values, the conversion of
// the bilinear forms into estimate and variance with the per-cell outputs,
// and the persistent launch shape.
#pragma once
#include "engine.cuh"
#include "kernels.h"

namespace hb
{
struct SolveParams
{
    const double *pair64;
    long long pc;
    float mf;
    double c0;
    int steps;
    double tol;
    SolveOut out;
    int2 *esc_cells;
    int *esc_count;
};

// neighbour value centred on the (float) mean as combine() does (combiner.h:19-24)
__device__ __forceinline__ double centred_value(bool live, float vraw, int ind_value, float mf)
{
    float v = 0.0f;
    if (live) v = ind_value >= 0 ? (vraw == (float)ind_value ? 1.0f : 0.0f) : vraw;
    return live ? (double)(v - mf) : 0.0;
}

// The bilinear forms of one system -> estimate and variance
// (my_kriging_weights.h:312-357 for OK, :175-194 for SK) and the per-cell
// outputs. s_vb = (v - m)^T A^-1 b, s_bb = b^T A^-1 b and, for OK,
// s_1b = 1^T A^-1 b, s_v1 = (v - m)^T A^-1 1, s_11 = 1^T A^-1 1.
template <bool ORDINARY>
__device__ __forceinline__ void write_solution(const SolveParams &P, int cell, bool fail, double s_vb, double s_bb,
                                               double s_1b, double s_v1, double s_11)
{
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
        est = (double)(out.cell_mean ? out.cell_mean[cell] : P.mf) + s_vb;
        var = P.c0 - s_bb;
    }
    if (var < 0) var = 0;
    if (!bad)
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

// Persistent launch shape: as many blocks as the SMs keep resident at `smem`
// bytes each (never more than the items need), with the smallest carveout.
template <typename K>
static cudaError_t launch_kernel(K kern, int threads, size_t smem, int max_items, int gpb, int n_sm, int &blocks_out)
{
    int per_sm = 0;
    cudaError_t e = set_smem_min_carveout(kern, threads, smem, per_sm);
    if (e != cudaSuccess) return e;
    long long want = ((long long)max_items + gpb - 1) / gpb;
    long long blocks = (long long)n_sm * per_sm;
    if (want < blocks) blocks = want;
    if (blocks < 1) blocks = 1;
    blocks_out = (int)blocks;
    return cudaSuccess;
}
} // namespace hb

namespace hb
{
// FP32-refined solves of up to 32 neighbours, four rows per lane (solve_quad.cu)
// FP32-refined solves of 17 to 32 neighbours from a union matrix shared by
// the block (solve_tile.cu; threads per block: 384 or 192)
cudaError_t launch_solve_tile(int np, bool ordinary, int threads, const Geom &g, const int2 *cells, const int *n_items,
                              int max_items, const int2 *nb_rec, int ind_value, const float *pair32,
                              const SolveParams &P, int n_sm, cudaStream_t st);
// FP32-refined (precision 1) and FP64-plain solves of 33 to 64 neighbours,
// one warp per system (solve_wide.cu)
cudaError_t launch_solve_wide(int precision, bool ordinary, const Geom &g, const int2 *cells, const int *n_items,
                              int max_items, const int2 *nb_rec, int ind_value, const float *pair32,
                              const SolveParams &P, int n_sm, cudaStream_t st);
// (threads per block: 384 or 256)
cudaError_t launch_solve_quad(int np, bool ordinary, int threads, const Geom &g, const int2 *cells,
                              const int *n_items, int max_items, const int2 *nb_rec, int ind_value,
                              const float *pair32, const SolveParams &P, int n_sm, cudaStream_t st);
} // namespace hb
