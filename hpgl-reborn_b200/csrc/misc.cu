// Supporting kernels of the kriging pipeline: pair-covariance tables, work
// buckets, failure handling, indicator order relations, and the solver for
// neighbour counts above 64.
#include "engine.cuh"
#include "kernels.h"
#include "sk_single.cuh"

#include <cstdint>

namespace hb
{
// ------------------------------------------------------------- pair tables
// Device evaluation of the covariance model for displacements outside the
// exactly tabulated search block: same formulas as cov_model.h:146-183, the
// transform sum without contraction (explicit round-to-nearest ops).
__device__ double cov_model_dev(const DevModel &m, int dx, int dy, int dz)
{
    double v0 = (double)dx, v1 = (double)dy, v2 = (double)dz;
    double acc = 0.0;
    for (int i = 0; i < 3; ++i)
    {
        double d = 0.0;
        d = __dadd_rn(d, __dmul_rn(v0, m.T[3 * i + 0]));
        d = __dadd_rn(d, __dmul_rn(v1, m.T[3 * i + 1]));
        d = __dadd_rn(d, __dmul_rn(v2, m.T[3 * i + 2]));
        acc = __dadd_rn(acc, __dmul_rn(d, d));
    }
    double h = sqrt(acc);
    if (h < 0.0001) return m.sill;
    double u = h / m.r0;
    if (m.type == 2) return (m.sill - m.nugget) * exp(-3.0 * (u * u));
    if (m.type == 1) return (m.sill - m.nugget) * exp((-3.0 * h) / m.r0);
    if (h > m.r0) return 0.0;
    return (m.sill - m.nugget) * (1.0 - (1.5 * h) / m.r0 + 0.5 * (u * u * u));
}

// pair[i] for displacement d: the host's exact value inside the search
// block, else (analytic flavour) the device model, else (truncated) 0.
__global__ void k_build_pair(const Geom g, DevModel m, int truncated, const double *__restrict__ search_vals,
                             double *__restrict__ pair64, float *__restrict__ pair32)
{
    long long total = (long long)g.pnx * g.pny * (2 * g.phz + 1);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
    {
        int ix = (int)(i % g.pnx);
        int iy = (int)((i / g.pnx) % g.pny);
        int iz = (int)(i / ((long long)g.pnx * g.pny));
        int dx = ix - g.phx, dy = iy - g.phy, dz = iz - g.phz;
        double v;
        if (key_in_block(g, dx, dy, dz))
            v = search_vals[key_index(g, dx, dy, dz)];
        else if (truncated)
            v = 0.0;
        else
            v = cov_model_dev(m, dx, dy, dz);
        pair64[i] = v;
        pair32[i] = (float)v;
    }
}

void launch_build_pair(const Geom &g, const DevModel &m, int truncated, const double *search_vals, double *pair64,
                       float *pair32, cudaStream_t st)
{
    k_build_pair<<<2368, 256, 0, st>>>(g, m, truncated, search_vals, pair64, pair32);
}

// ------------------------------------------------------------- buckets
__device__ __forceinline__ int bucket_of(int n)
{
    if (n <= 0) return -1;
    if (n <= 8) return 0;
    if (n <= 16) return 1;
    if (n <= 32) return 2;
    if (n <= 64) return 3;
    return 4;
}

// Per-cell status before the solve: -1 informed (continuous kriging only),
// 1 no neighbours, 3 pending (to be solved).
// Per-cell status and the solve work lists, as a stable partition by bucket:
// the list of every bucket holds its cells in ascending cell order, so the
// solver's blocks, which take contiguous runs of a list, work on neighbouring
// cells. Three passes over tiles of kTile cells: counts (and the moments of n
// per bucket, for the flop count), a one-block scan, and the ordered fill.
constexpr int kTileThreads = 256, kTileIters = 8, kTile = kTileThreads * kTileIters;

long long prepare_tiles(long long n_cells) { return (n_cells + kTile - 1) / kTile; }

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// status: -1 informed (not kriged), 1 no neighbours, 3 queued for a solve.
// tile_cnt[q * T + tile] = cells of bucket q in the tile; tile_mom[(3q + e) * T + tile]
// = sum of n^(e+1) over them.
__global__ void __launch_bounds__(kTileThreads) k_prepare(const Geom g, const uint8_t *__restrict__ mask, int all_cells,
                                                          const int *__restrict__ nb_n, signed char *__restrict__ status,
                                                          int *__restrict__ tile_cnt,
                                                          unsigned long long *__restrict__ tile_mom)
{
    const int T = gridDim.x;
    const long long base = (long long)blockIdx.x * kTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int cnt[kBuckets];
    unsigned long long mom[kBuckets * 3];
#pragma unroll
    for (int q = 0; q < kBuckets; ++q) cnt[q] = 0;
#pragma unroll
    for (int q = 0; q < kBuckets * 3; ++q) mom[q] = 0;
    for (int it = 0; it < kTileIters; ++it)
    {
        const long long c = base + it * kTileThreads + threadIdx.x;
        int b = -1, n = 0;
        if (c < g.n_cells)
        {
            if (!all_cells && mask[c])
                status[c] = -1;
            else
            {
                n = nb_n[c];
                b = bucket_of(n);
                status[c] = b < 0 ? 1 : 3;
            }
        }
        const unsigned long long nn = (unsigned long long)n;
#pragma unroll
        for (int q = 0; q < kBuckets; ++q)
        {
            cnt[q] += __popc(__ballot_sync(0xffffffffu, b == q));
            if (b == q)
            {
                mom[3 * q] += nn;
                mom[3 * q + 1] += nn * nn;
                mom[3 * q + 2] += nn * nn * nn;
            }
        }
    }
    __shared__ int s_cnt[kTileThreads / 32][kBuckets];
    __shared__ unsigned long long s_mom[kTileThreads / 32][kBuckets * 3];
#pragma unroll
    for (int q = 0; q < kBuckets * 3; ++q)
    {
        const unsigned long long v = warp_sum_u64(mom[q]);
        if (lane == 0) s_mom[warp][q] = v;
    }
    if (lane == 0)
    {
#pragma unroll
        for (int q = 0; q < kBuckets; ++q) s_cnt[warp][q] = cnt[q];
    }
    __syncthreads();
    if (threadIdx.x < kBuckets)
    {
        int v = 0;
        for (int w = 0; w < kTileThreads / 32; ++w) v += s_cnt[w][threadIdx.x];
        tile_cnt[threadIdx.x * T + blockIdx.x] = v;
    }
    else if (threadIdx.x >= 32 && threadIdx.x < 32 + kBuckets * 3)
    {
        const int q = threadIdx.x - 32;
        unsigned long long v = 0;
        for (int w = 0; w < kTileThreads / 32; ++w) v += s_mom[w][q];
        tile_mom[q * T + blockIdx.x] = v;
    }
}

// One block: exclusive scan of every bucket's tile counts (in place, as offsets
// into the whole list), bucket totals and offsets, and the moments.
__global__ void __launch_bounds__(1024) k_prepare_scan(int T, int *__restrict__ tile_cnt,
                                                       const unsigned long long *__restrict__ tile_mom,
                                                       int *__restrict__ bucket_cnt, int *__restrict__ bucket_off,
                                                       unsigned long long *__restrict__ moments)
{
    __shared__ int s_part[1024];
    __shared__ int s_total[kBuckets];
    const int per = (T + blockDim.x - 1) / blockDim.x;
    const int t0 = threadIdx.x * per, t1 = min(T, t0 + per);
    for (int q = 0; q < kBuckets; ++q)
    {
        int *tc = tile_cnt + (long long)q * T;
        int local = 0;
        for (int t = t0; t < t1; ++t) local += tc[t];
        s_part[threadIdx.x] = local;
        __syncthreads();
        // Hillis-Steele inclusive scan of the per-thread sums
        for (int o = 1; o < (int)blockDim.x; o <<= 1)
        {
            const int v = threadIdx.x >= o ? s_part[threadIdx.x - o] : 0;
            __syncthreads();
            s_part[threadIdx.x] += v;
            __syncthreads();
        }
        int run = s_part[threadIdx.x] - local;
        for (int t = t0; t < t1; ++t)
        {
            const int c = tc[t];
            tc[t] = run;
            run += c;
        }
        if (threadIdx.x == blockDim.x - 1) s_total[q] = s_part[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        int run = 0;
        for (int q = 0; q < kBuckets; ++q)
        {
            bucket_cnt[q] = s_total[q];
            bucket_off[q] = run;
            run += s_total[q];
        }
        bucket_off[kBuckets] = run;
    }
    // moments: every thread sums a strided share of each of the 3 kBuckets rows
    __shared__ unsigned long long s_m[32];
    for (int q = 0; q < kBuckets * 3; ++q)
    {
        unsigned long long v = 0;
        for (int t = threadIdx.x; t < T; t += blockDim.x) v += tile_mom[(long long)q * T + t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x < 32)
        {
            unsigned long long w = threadIdx.x < (blockDim.x >> 5) ? s_m[threadIdx.x] : 0ULL;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if (threadIdx.x == 0) moments[q] = w;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kTileThreads) k_bucket_fill(const Geom g, const signed char *__restrict__ status,
                                                              const int *__restrict__ nb_n,
                                                              const int *__restrict__ tile_off,
                                                              const int *__restrict__ bucket_off,
                                                              int2 *__restrict__ cells)
{
    const int T = gridDim.x;
    const long long base = (long long)blockIdx.x * kTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int W = kTileThreads / 32;
    __shared__ int s_wc[W][kBuckets];
    __shared__ int s_run[kBuckets];
    if (threadIdx.x < kBuckets) s_run[threadIdx.x] = bucket_off[threadIdx.x] + tile_off[threadIdx.x * T + blockIdx.x];
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    for (int it = 0; it < kTileIters; ++it)
    {
        const long long c = base + it * kTileThreads + threadIdx.x;
        int b = -1, n = 0;
        if (c < g.n_cells && status[c] == 3)
        {
            n = nb_n[c];
            b = bucket_of(n);
        }
        unsigned my_bl = 0;
#pragma unroll
        for (int q = 0; q < kBuckets; ++q)
        {
            const unsigned bl = __ballot_sync(0xffffffffu, b == q);
            if (b == q) my_bl = bl;
            if (lane == 0) s_wc[warp][q] = __popc(bl);
        }
        __syncthreads();
        if (b >= 0)
        {
            int off = s_run[b];
            for (int w = 0; w < warp; ++w) off += s_wc[w][b];
            cells[off + __popc(my_bl & lt)] = make_int2((int)c, n);
        }
        __syncthreads();
        if (threadIdx.x < kBuckets)
        {
            int v = 0;
            for (int w = 0; w < W; ++w) v += s_wc[w][threadIdx.x];
            s_run[threadIdx.x] += v;
        }
        __syncthreads();
    }
}

void launch_prepare(const Geom &g, const uint8_t *mask, int all_cells, const int *nb_n, signed char *status,
                    int *bucket_cnt, int *bucket_off, int *tile_cnt, unsigned long long *tile_mom, int2 *cells,
                    unsigned long long *moments, cudaStream_t st)
{
    const int T = (int)prepare_tiles(g.n_cells);
    k_prepare<<<T, kTileThreads, 0, st>>>(g, mask, all_cells, nb_n, status, tile_cnt, tile_mom);
    k_prepare_scan<<<1, 1024, 0, st>>>(T, tile_cnt, tile_mom, bucket_cnt, bucket_off, moments);
    k_bucket_fill<<<T, kTileThreads, 0, st>>>(g, status, nb_n, tile_cnt, bucket_off, cells);
}

// ------------------------------------------------------------- finalize
// Continuous kriging outputs for cells the solver did not write
// (cont_kriging.h:80-110): informed cells are copied, failures of SK get the
// mean (LVM: the cell's own mean, lvm_kriging.cpp:33), failures of OK are left
// alone.
__global__ void k_finalize_cont(const Geom g, const float *__restrict__ in_data, signed char *__restrict__ status,
                                int simple, float mean_f, const float *__restrict__ cell_mean,
                                float *__restrict__ out_data, uint8_t *__restrict__ out_mask,
                                double *__restrict__ est64, double *__restrict__ var)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < g.n_cells;
         c += (long long)gridDim.x * blockDim.x)
    {
        signed char s = status[c];
        if (s == -1)
        {
            out_data[c] = in_data[c];
            out_mask[c] = 1;
            if (est64) est64[c] = (double)in_data[c];
            if (var) var[c] = 0.0;
        }
        else if (s >= 1)
        {
            if (s >= 3) status[c] = 2; // not written by any solver: treat as singular
            if (simple)
            {
                out_data[c] = cell_mean ? cell_mean[c] : mean_f;
                out_mask[c] = 1;
            }
            if (est64) est64[c] = __longlong_as_double(0x7ff8000000000000LL);
            if (var) var[c] = -1.0;
        }
    }
}

void launch_finalize_cont(const Geom &g, const float *in_data, signed char *status, int simple, float mean_f,
                          const float *cell_mean, float *out_data, uint8_t *out_mask, double *est64, double *var,
                          cudaStream_t st)
{
    k_finalize_cont<<<1184, 256, 0, st>>>(g, in_data, status, simple, mean_f, cell_mean, out_data, out_mask, est64,
                                          var);
}

// Indicator category c: cells whose solve failed (or had no neighbours) take
// the marginal probability (indicator_kriging.h:137-140).
__global__ void k_ik_fail_fill(const Geom g, const signed char *__restrict__ status, float marginal, int c, int m,
                               float *__restrict__ probs)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.n_cells;
         i += (long long)gridDim.x * blockDim.x)
        if (status[i] != 0) probs[i * m + c] = marginal;
}

void launch_ik_fail_fill(const Geom &g, const signed char *status, float marginal, int c, int m, float *probs,
                         cudaStream_t st)
{
    k_ik_fail_fill<<<1184, 256, 0, st>>>(g, status, marginal, c, m, probs);
}

// Order relations (indicator_kriging.h:34-59) and the first-maximum argmax
// (cdf_utils.cpp:11-27).
__global__ void k_ik_finalize(long long n_cells, int m, float *__restrict__ probs, uint8_t *__restrict__ out_data,
                              uint8_t *__restrict__ out_mask)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_cells;
         i += (long long)gridDim.x * blockDim.x)
    {
        float *p = probs + i * m;
        for (int c = 0; c < m; ++c)
        {
            float v = p[c];
            if (v < 0.0f) v = 0.0f;
            else if (v > 1.0f) v = 1.0f;
            p[c] = v;
        }
        for (int c = 0; c + 1 < m; ++c)
            if (p[c] > p[c + 1])
            {
                float s = __fadd_rn(p[c], p[c + 1]);
                float avg = (float)((double)s / 2.0);
                p[c] = avg;
                p[c + 1] = avg;
            }
        double best = p[0];
        int arg = 0;
        for (int c = 1; c < m; ++c)
            if ((double)p[c] > best)
            {
                best = p[c];
                arg = c;
            }
        out_data[i] = (uint8_t)arg;
        out_mask[i] = 1;
    }
}

void launch_ik_finalize(long long n_cells, int m, float *probs, uint8_t *out_data, uint8_t *out_mask, cudaStream_t st)
{
    k_ik_finalize<<<1184, 256, 0, st>>>(n_cells, m, probs, out_data, out_mask);
}

// Median IK decision (median_ik.cpp:15-21 through a float); failures use the
// marginal (the reference leaves this case undefined).
__global__ void k_mik_finalize(long long n_cells, const signed char *__restrict__ status,
                               const double *__restrict__ est64, double marginal1, uint8_t *__restrict__ out_data,
                               uint8_t *__restrict__ out_mask, float *__restrict__ prob_out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_cells;
         i += (long long)gridDim.x * blockDim.x)
    {
        double p = status[i] == 0 ? est64[i] : (double)(float)marginal1;
        float pf = (float)p;
        out_data[i] = pf <= 0.5f ? 0 : 1;
        out_mask[i] = 1;
        if (prob_out) prob_out[i] = pf;
    }
}

void launch_mik_finalize(long long n_cells, const signed char *status, const double *est64, double marginal1,
                         uint8_t *out_data, uint8_t *out_mask, float *prob_out, cudaStream_t st)
{
    k_mik_finalize<<<1184, 256, 0, st>>>(n_cells, status, est64, marginal1, out_data, out_mask, prob_out);
}

// ------------------------------------------------------------- large systems
// Neighbour counts above 64: one CTA per system, matrix in global scratch,
// double precision, right-looking Cholesky with block barriers.
__global__ void __launch_bounds__(256) k_solve_large(const Geom g, const int2 *__restrict__ cells,
                                                     const int *__restrict__ n_items_ptr, const int2 *__restrict__ nb_rec,
                                                     const int *__restrict__ nb_n, int ind_value,
                                                     const double *__restrict__ pair64, int ordinary, double mean,
                                                     double c0, double *__restrict__ scratch, SolveOut out)
{
    const int n_items = *n_items_ptr;
    const int kmax = g.k;
    double *A = scratch + (size_t)blockIdx.x * ((size_t)kmax * kmax + 4 * kmax);
    double *rhs = A + (size_t)kmax * kmax; // b, ones, x(b), x(1)
    const long long pc = g.pair_center;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x)
    {
        const int cell = cells[item].x;
        const int n = cells[item].y;
        const int2 *rec = nb_rec + (long long)cell * kmax;
        for (int e = threadIdx.x; e < n * n; e += blockDim.x)
        {
            int i = e / n, j = e % n;
            A[(size_t)i * n + j] = pair64[pc + rec[i].x - rec[j].x];
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            rhs[i] = pair64[pc + rec[i].x];
            rhs[kmax + i] = 1.0;
        }
        __syncthreads();
        bool fail = false;
        for (int j = 0; j < n; ++j)
        {
            double d = A[(size_t)j * n + j];
            if (!(d > 0.0)) fail = true;
            double ljj = sqrt(d);
            __syncthreads();
            for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + j] /= ljj;
            if (threadIdx.x == 0) A[(size_t)j * n + j] = ljj;
            __syncthreads();
            int span = n - j - 1;
            for (int e = threadIdx.x; e < span * span; e += blockDim.x)
            {
                int i = j + 1 + e / span, c = j + 1 + e % span;
                if (c <= i) A[(size_t)i * n + c] -= A[(size_t)i * n + j] * A[(size_t)c * n + j];
            }
            __syncthreads();
        }
        if (threadIdx.x < 2)
        {
            double *x = rhs + (threadIdx.x == 0 ? 2 * kmax : 3 * kmax);
            const double *src = rhs + (threadIdx.x == 0 ? 0 : kmax);
            for (int i = 0; i < n; ++i)
            {
                double s = src[i];
                for (int c = 0; c < i; ++c) s -= A[(size_t)i * n + c] * x[c];
                x[i] = s / A[(size_t)i * n + i];
            }
            for (int i = n - 1; i >= 0; --i)
            {
                double s = x[i];
                for (int c = i + 1; c < n; ++c) s -= A[(size_t)c * n + i] * x[c];
                x[i] = s / A[(size_t)i * n + i];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            const double *x = rhs + 2 * kmax, *y = rhs + 3 * kmax;
            double mu = 0.0, sx = 0, sy = 0;
            for (int i = 0; i < n; ++i)
            {
                sx += x[i];
                sy += y[i];
            }
            if (ordinary)
            {
                if (fabs(sy) < 1e-15) fail = true;
                mu = (sx - 1.0) / sy;
            }
            const float mf = (float)mean;
            double est = out.cell_mean ? (double)out.cell_mean[cell] : (double)mf, var = c0 - mu;
            for (int i = 0; i < n; ++i)
            {
                double w = ordinary ? x[i] - mu * y[i] : x[i];
                float vr = __int_as_float(rec[i].y);
                double v = ind_value >= 0 ? (vr == (float)ind_value ? 1.0 : 0.0) : (double)vr;
                est += w * (double)((float)v - mf);
                var -= w * rhs[i];
            }
            if (var < 0) var = 0;
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
        __syncthreads();
    }
}

size_t large_scratch_doubles(int k, int blocks) { return (size_t)blocks * ((size_t)k * k + 4 * (size_t)k); }

cudaError_t launch_solve_large(const Geom &g, const int2 *cells, const int *n_items, int blocks, const int2 *nb_rec,
                               const int *nb_n, int ind_value, const double *pair64, bool ordinary, double mean,
                               double c0, double *scratch, const SolveOut &out, cudaStream_t st)
{
    k_solve_large<<<blocks, 256, 0, st>>>(g, cells, n_items, nb_rec, nb_n, ind_value, pair64, ordinary ? 1 : 0, mean,
                                          c0, scratch, out);
    return cudaGetLastError();
}
} // namespace hb

namespace hb
{
// ------------------------------------------------------------- single system
// SK weights for arbitrary real coordinates (sk_single.cuh); status[0] = 1 on success.
__global__ void k_sk_weights(DevModel m, const double *__restrict__ pts, int n, double *__restrict__ A,
                             double *__restrict__ w, int *__restrict__ status)
{
    const bool fail = sk_single_solve(m, pts, n, A, w);
    if (threadIdx.x == 0) status[0] = fail ? 0 : 1;
}

void launch_sk_weights(const DevModel &m, const double *pts, int n, double *A, double *w, int *status,
                       cudaStream_t st)
{
    k_sk_weights<<<1, 256, 0, st>>>(m, pts, n, A, w, status);
}
} // namespace hb
