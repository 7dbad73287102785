// Sequential Gaussian simulation on the GPU (sequential_simulation.h:51-118,
// sequential_gaussian_simulation.cpp:18-131).
//
// The reference visits every node in the order of a linear congruential walk
// and kriges each one that is not yet informed from the first max_nb informed
// cells of its search template, so the neighbour set of a node depends only on
// which cells are informed when it is visited: the conditioning cells and the
// nodes earlier in the walk. With rank(j) = the node's position among the
// simulated nodes (-1 for conditioning cells, INT_MAX for cells never
// simulated), "informed when j is visited" is rank(q) < rank(j). Every
// neighbour set is therefore known before any value is drawn:
//
//   k_sgs_path     walk positions -> nodes (the LCG in closed form per chunk)
//   k_sgs_index    ranks of the simulated nodes (after a scan over the walk)
//   k_sgs_search   each simulated node's neighbours: the template scanned in
//                  order with the rank predicate, one warp per node
//   k_sgs_levels   dependency levels: level(j) = 1 + max level of its simulated
//                  neighbours; a single pass over the ranks in ticket order
//   k_sgs_solve_*  one launch per level: every node of a level depends only on
//                  lower levels, so a level is kriged and drawn in parallel
//                  (FP64: two nodes per warp for up to 32 neighbours, one
//                  block per node beyond)
//
// The draws are the reference's: one std::uniform_real_distribution<double>
// draw of a std::mt19937 per simulated node, in walk order (generated on the
// host), pushed through the inverse Gaussian CDF with the reference's float
// mean and double variance.
#include "engine.cuh"
#include "fold32.cuh"
#include "kernels.h"

#include <cuda/atomic>

#include <algorithm>
#include <climits>

namespace hb
{
// ------------------------------------------------------------------ scalar maths
// gaussian_cdf_t (gaussian_distribution.h): Abramowitz & Stegun 26.2.17 and the
// Odeh & Evans inverse, every operation rounded as the reference's double code
// rounds it (no contraction); exp and log are CUDA's (within 1 ulp of glibc's).
__device__ double sgs_gauss_inverse(double pr, double mean, double var)
{
    if (pr <= 0.0 || pr >= 1.0) return mean;
    double p2 = pr > 0.5 ? __dsub_rn(1.0, pr) : pr;
    if (p2 < 1e-150) p2 = 1e-150;
    const double y = __dsqrt_rn(log(__ddiv_rn(1.0, __dmul_rn(p2, p2))));
    double num = __dadd_rn(__dmul_rn(-0.453642210148e-4, y), -0.0204231210245);
    num = __dadd_rn(__dmul_rn(num, y), -0.342242088547);
    num = __dadd_rn(__dmul_rn(num, y), -1.0);
    num = __dadd_rn(__dmul_rn(num, y), -0.322232431088);
    double den = __dadd_rn(__dmul_rn(0.38560700634e-2, y), 0.103537752850);
    den = __dadd_rn(__dmul_rn(den, y), 0.531103462366);
    den = __dadd_rn(__dmul_rn(den, y), 0.588581570495);
    den = __dadd_rn(__dmul_rn(den, y), 0.0993484626060);
    double xp = __dadd_rn(y, __ddiv_rn(num, den));
    if (pr < 0.5) xp = -xp;
    return __dadd_rn(__dmul_rn(xp, __dsqrt_rn(var)), mean);
}

// standard normal CDF (mean 0, variance 1: sx = x exactly)
__device__ double sgs_gauss_cdf(double x)
{
    double sx = x;
    const bool neg = sx < 0;
    if (neg) sx = -sx;
    const double t = __ddiv_rn(1.0, __dadd_rn(1.0, __dmul_rn(0.2316419, sx)));
    const double c = __ddiv_rn(1.0, __dsqrt_rn(__dmul_rn(2.0, 3.14159265358)));
    const double zx = __dmul_rn(c, exp(__ddiv_rn(__dmul_rn(-sx, sx), 2.0)));
    double q = __dadd_rn(__dmul_rn(1.330274429, t), -1.821255978);
    q = __dadd_rn(__dmul_rn(q, t), 1.781477937);
    q = __dadd_rn(__dmul_rn(q, t), -0.356563782);
    q = __dadd_rn(__dmul_rn(q, t), 0.319381530);
    double r = __dsub_rn(1.0, __dmul_rn(__dmul_rn(zx, q), t));
    if (neg) r = __dsub_rn(1.0, r);
    return r;
}

// first index whose value is not less than x (std::lower_bound)
__device__ __forceinline__ long long lower_bound_f(const float *a, long long n, float x)
{
    long long lo = 0, hi = n;
    while (lo < hi)
    {
        const long long mid = lo + (hi - lo) / 2;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// non_parametric_cdf_2_t::operator() and ::inverse (non_parametric_cdf.h:215-270)
__device__ float sgs_np_prob(const float *v, const float *p, long long n, float x)
{
    const long long i2 = lower_bound_f(v, n, x);
    if (i2 == n) return p[n - 1];
    if (i2 == 0) return p[0];
    const float x1 = v[i2 - 1], x2 = v[i2], y1 = p[i2 - 1], y2 = p[i2];
    return __fadd_rn(y1, __fmul_rn(__fdiv_rn(__fsub_rn(y2, y1), __fsub_rn(x2, x1)), __fsub_rn(x, x1)));
}

__device__ float sgs_np_inverse(const float *v, const float *p, long long n, float q)
{
    if (n <= 0) return 0.0f;
    const long long i2 = lower_bound_f(p, n, q);
    if (i2 == 0) return v[0];
    if (i2 == n) return v[n - 1];
    const float x1 = v[i2 - 1], x2 = v[i2], y1 = p[i2 - 1], y2 = p[i2];
    return __fadd_rn(x1, __fmul_rn(__fdiv_rn(__fsub_rn(x2, x1), __fsub_rn(y2, y1)), __fsub_rn(q, y1)));
}

// ------------------------------------------------------------------ transforms
// transform_cdf_p (cdf_utils.h:14-25) into the Gaussian space: informed cells
// only; LVM means (transform_cdf_ptr) for every cell.
__global__ void k_sgs_forward(long long n, float *__restrict__ data, const uint8_t *__restrict__ mask,
                              const float *__restrict__ means_in, float *__restrict__ means_out,
                              const float *__restrict__ cv, const float *__restrict__ cp, long long cn)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        if (cv && mask[i])
            data[i] = __double2float_rn(sgs_gauss_inverse((double)sgs_np_prob(cv, cp, cn, data[i]), 0.0, 1.0));
        if (means_out)
            means_out[i] = cv ? __double2float_rn(sgs_gauss_inverse((double)sgs_np_prob(cv, cp, cn, means_in[i]), 0.0,
                                                                    1.0))
                              : means_in[i];
    }
}

// Marks the simulated cells informed and maps every informed cell back
// (transform_cdf_p(output, gaussian_cdf_t(), cdf)).
__global__ void k_sgs_finalize(long long n, float *__restrict__ data, uint8_t *__restrict__ mask,
                               const int *__restrict__ rank_of, int n_sim, const signed char *__restrict__ st_in,
                               signed char *__restrict__ status, const float *__restrict__ cv,
                               const float *__restrict__ cp, long long cn)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int r = rank_of[i];
        const bool sim = r >= 0 && r < n_sim;
        if (sim) mask[i] = 1;
        if (status) status[i] = sim ? st_in[r] : (signed char)(r < 0 ? -1 : 3);
        if (cv && mask[i]) data[i] = sgs_np_inverse(cv, cp, cn, __double2float_rn(sgs_gauss_cdf((double)data[i])));
    }
}

// ------------------------------------------------------------------ the walk
// R_{p+1} = (A R_p + C) mod M from R_0; f^m(x) = a_m x + c_m (mod M) by squaring.
struct AffineMod
{
    long long a, c;
};
__device__ __forceinline__ AffineMod affine_then(AffineMod first, AffineMod second, long long M)
{
    // second(first(x)) = a2 (a1 x + c1) + c2
    return {(second.a * first.a) % M, (second.a * first.c + second.c) % M};
}

constexpr int kWalkChunk = 64;

// walk position p -> node; flag[p] = 1 when the node is simulated (not
// informed, simulation mask 1). Requires a full-period walk (a permutation).
__global__ void k_sgs_path(SgsWalk w, const uint8_t *__restrict__ mask, const uint8_t *__restrict__ sim_mask,
                           int *__restrict__ path_cell, int *__restrict__ flag)
{
    const long long chunks = (w.M + kWalkChunk - 1) / kWalkChunk;
    for (long long ch = (long long)blockIdx.x * blockDim.x + threadIdx.x; ch < chunks;
         ch += (long long)gridDim.x * blockDim.x)
    {
        const long long p0 = ch * kWalkChunk;
        // R_{p0} = f^{p0}(R_0)
        AffineMod acc = {1, 0}, base = {w.A % w.M, w.C % w.M};
        for (long long e = p0; e > 0; e >>= 1)
        {
            if (e & 1) acc = affine_then(acc, base, w.M);
            base = affine_then(base, base, w.M);
        }
        long long R = (acc.a * w.R0 + acc.c) % w.M;
        const long long p1 = p0 + kWalkChunk < w.M ? p0 + kWalkChunk : w.M;
        for (long long p = p0; p < p1; ++p)
        {
            const int cell = (int)R;
            path_cell[p] = cell;
            flag[p] = (!mask[cell] && (!sim_mask || sim_mask[cell] == 1)) ? 1 : 0;
            R = (w.A * R + w.C) % w.M;
        }
    }
}

// rank_of[cell]: the rank of a simulated cell, -1 for informed cells, INT_MAX
// for cells never simulated; sim_cells[rank] = cell. `scan` holds the exclusive
// scan of the flags; `path_cell` and the flags come from k_sgs_path.
__global__ void k_sgs_index(long long n, const int *__restrict__ path_cell, const int *__restrict__ flag,
                            const int *__restrict__ scan, const uint8_t *__restrict__ mask, int *__restrict__ rank_of,
                            int *__restrict__ sim_cells)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
    {
        const int cell = path_cell[p];
        if (flag[p])
        {
            rank_of[cell] = scan[p];
            sim_cells[scan[p]] = cell;
        }
        else
            rank_of[cell] = mask[cell] ? -1 : INT_MAX;
    }
}

// ------------------------------------------------------------------ search
// neighbour_lookup_t::find (sugarbox_neighbour_lookup.h:39-63) with the rank
// predicate: the first k template offsets, in template order, whose cell lies
// in the grid and was informed before the node. One warp per node, 32 offsets
// per step. nb_rank receives each neighbour's rank (-1 for a conditioning
// cell), which the level pass reads instead of gathering rank_of again. With
// fixed_rank >= 0 every node compares against fixed_rank instead of its own
// rank (cokriging: every target sees the same informed cells).
__global__ void __launch_bounds__(256) k_sgs_search(const Geom g, const int4 *__restrict__ tmpl, int n_tmpl,
                                                    const int *__restrict__ sim_cells, int n_sim,
                                                    const int *__restrict__ rank_of, int k, int fixed_rank,
                                                    int *__restrict__ nb, int *__restrict__ nb_rank, int rank_stride,
                                                    int *__restrict__ nb_cnt)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n_sim; r += warps)
    {
        const int cell = sim_cells[r];
        const int x = cell % g.nx, y = (int)((cell / g.nx) % g.ny), z = (int)(cell / ((long long)g.nx * g.ny));
        int found = 0;
        int *out = nb + r * (long long)k;
        int *out_rank = nb_rank ? nb_rank + r * (long long)rank_stride : nullptr;
        const int thr = fixed_rank >= 0 ? fixed_rank : (int)r;
        for (int base = 0; base < n_tmpl && found < k; base += 32)
        {
            const int t = base + lane;
            bool hit = false;
            int q = 0, rq = 0;
            if (t < n_tmpl)
            {
                const int4 o = tmpl[t];
                const int X = x + o.x, Y = y + o.y, Z = z + o.z;
                if ((unsigned)X < (unsigned)g.nx && (unsigned)Y < (unsigned)g.ny && (unsigned)Z < (unsigned)g.nz)
                {
                    q = (int)(((long long)Z * g.ny + Y) * g.nx + X);
                    rq = rank_of[q];
                    hit = rq < thr;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            const int slot = found + __popc(m & ((1u << lane) - 1u));
            if (hit && slot < k)
            {
                out[slot] = q;
                if (out_rank) out_rank[slot] = rq;
            }
            found += __popc(m);
        }
        if (lane == 0) nb_cnt[r] = found < k ? found : k;
    }
}

// ------------------------------------------------------------------ levels
__device__ __forceinline__ int ld_relaxed_gpu(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(int *p, int v)
{
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned long long kLevelWaitNs = 2000000000ull; // a wait that lasts 2 s is an error

// levp1[r] = level(r) + 1 (0 = not yet known). Warps take batches of 32
// consecutive ranks in ticket order and every lane publishes its own level as
// soon as its dependencies are known, so a chain of dependencies advances one
// node at a time rather than one batch at a time. A rank waits only on lower
// ranks: those of earlier tickets, whose warps are running, and those of lower
// lanes of its own batch, which independent thread scheduling keeps running
// while it waits. So every wait ends; each still gives up after kLevelWaitNs
// (err = 1), and once err is set every wait ends at once. The spin reads the
// timer and the error flag every 64 polls and does not sleep (sleeping between
// polls doubled the pass).
__device__ __forceinline__ int sgs_wait_level(const int *levp1, int tq, int *err)
{
    int v = ld_relaxed_gpu(&levp1[tq]);
    if (v != 0) return v;
    const unsigned long long t0 = global_ns();
    unsigned polls = 0;
    while ((v = ld_relaxed_gpu(&levp1[tq])) == 0)
    {
        if ((++polls & 63u) == 0 && (ld_relaxed_gpu(err) != 0 || global_ns() - t0 > kLevelWaitNs))
        {
            atomicExch(err, 1);
            return 1;
        }
    }
    return v;
}

__global__ void __launch_bounds__(256) k_sgs_levels(const int *__restrict__ nb_rank, const int *__restrict__ nb_cnt,
                                                    int k, int n_sim, int *levp1, int *ticket, int level_cap,
                                                    int *max_level, int *err)
{
    const int lane = threadIdx.x & 31;
    for (;;)
    {
        int b = 0;
        if (lane == 0) b = atomicAdd(ticket, 1);
        b = __shfl_sync(0xffffffffu, b, 0);
        const long long base = (long long)b * 32;
        if (base >= n_sim) break;
        const long long r = base + lane;
        int L = 0;
        if (r < n_sim)
        {
            const int n = nb_cnt ? nb_cnt[r] : k; // without counts: k slots, -1 where empty
            const int *row = nb_rank + r * (long long)k;
            // sixteen neighbours at a time: their ranks, then every published level
            // at once; waits only for the missing ones
            for (int i0 = 0; i0 < n; i0 += 16)
            {
                int tq[16], v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) tq[j] = i0 + j < n ? row[i0 + j] : -1;
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = tq[j] >= 0 ? ld_relaxed_gpu(&levp1[tq[j]]) : -1;
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    if (v[j] == 0) v[j] = sgs_wait_level(levp1, tq[j], err);
                    L = max(L, v[j]); // level(dep) + 1
                }
            }
            if (L >= level_cap) atomicExch(err, 2);
            st_relaxed_gpu(&levp1[r], L + 1);
        }
        __syncwarp();
        int m = L;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) atomicMax(max_level, m);
    }
}

// level_count[l] = number of ranks of level l (a shared-memory histogram of the
// first kSgsHistLevels levels, global atomics beyond)
constexpr int kSgsHistLevels = 4096;
__global__ void __launch_bounds__(256) k_sgs_level_count(int n_sim, const int *__restrict__ levp1, int level_cap,
                                                         int *__restrict__ level_count)
{
    __shared__ int h[kSgsHistLevels];
    for (int i = threadIdx.x; i < kSgsHistLevels; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_sim; r += gridDim.x * blockDim.x)
    {
        const int l = levp1[r] - 1;
        if (l < 0 || l >= level_cap) continue; // only after an error, which the host reports
        if (l < kSgsHistLevels)
            atomicAdd(&h[l], 1);
        else
            atomicAdd(&level_count[l], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSgsHistLevels; i += blockDim.x)
        if (h[i]) atomicAdd(&level_count[i], h[i]);
}

// sums of n, n^2, n^3 over the neighbour counts (the solve's algorithmic flops)
__global__ void __launch_bounds__(256) k_sgs_moments(int n_sim, const int *__restrict__ nb_cnt, double *__restrict__ mom)
{
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_sim; r += gridDim.x * blockDim.x)
    {
        const double n = (double)nb_cnt[r];
        s1 += n;
        s2 += n * n;
        s3 += n * n * n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        s3 += __shfl_xor_sync(0xffffffffu, s3, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        atomicAdd(&mom[0], s1);
        atomicAdd(&mom[1], s2);
        atomicAdd(&mom[2], s3);
    }
}

// order[level_off[l] + i]: the ranks of level l (any order inside a level)
__global__ void k_sgs_level_fill(int n_sim, const int *__restrict__ levp1, const int *__restrict__ level_off,
                                 int *__restrict__ level_fill, int *__restrict__ order)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_sim; r += gridDim.x * blockDim.x)
    {
        const int l = levp1[r] - 1;
        const int pos = atomicAdd(&level_fill[l], 1);
        order[level_off[l] + pos] = r;
    }
}

// ------------------------------------------------------------------ solve + draw
struct SgsNode
{
    int status; // 0 kriged, 1 no neighbours, 2 singular
    float mean; // combine()'s float estimate
    double var;
};

struct SgsSolveArgs
{
    Geom g;
    const int *order;
    int n_items;
    const int *sim_cells;
    const int *nb;
    const int *nb_cnt;
    int k;
    const double *pair64;
    float *data;
    const float *means; // LVM (Gaussian-space means) or null
    const double *uniforms;
    signed char *st_rank; // status per rank
    int ordinary;
};

// n <= 32: two nodes per warp, sixteen lanes each, lane t holding rows t and
// 31 - t of A (the folded lower triangle, as the kriging solves lay it out).
// The right-looking factorisation broadcasts column j through shared memory
// row j and carries the forward substitution of b (and, for ordinary kriging,
// of the ones vector); the back substitution reads column i of L from the
// lane's own shared rows. The weights then go through combine() one by one.
constexpr int kSgsNP = kFold32NP, kSgsG = kFold32G;
constexpr int kSgsLD = kFold32LD;
constexpr int kSgsFoldThreads = 256;

constexpr size_t kSgsSysBytes = kFold32SysBytes;

// BOUND (k < 32): the factorisation stops at the warp's largest system
template <bool ORD, bool BOUND>
__global__ void __launch_bounds__(kSgsFoldThreads, 1) k_sgs_solve_fold(const SgsSolveArgs a)
{
    constexpr int NP = kSgsNP, G = kSgsG, LD = kSgsLD, QB = ORD ? 2 : 1;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int h = lane / G, t = lane % G, rb = NP - 1 - t;
    const unsigned gm = 0xFFFFu << (h * G);
    unsigned char *gb = smem + kSgsSysBytes * (warp * 2 + h);
    double *M = reinterpret_cast<double *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + kFold32MBytes);
    const int row_a = d_fold32_rows.row[t], row_b = d_fold32_rows.row[rb]; // the lane's rows in M
    const Geom &g = a.g;
    const long long pc = g.pair_center;
    const double *pair64 = a.pair64;
    // The next item's chain of dependent loads (rank, cell and count; its
    // neighbours; their values) is issued in three stages during the current
    // item's solve. Its neighbours belong to lower levels, already final.
    const int stride = gridDim.x * nwarps * 2;
    int nr = 0, ncell = 0, nn = 0, nqa = 0, nqb = 0;
    float nva = 0.0f, nvb = 0.0f, nma = 0.0f, nmb = 0.0f;
    auto stage_a = [&](int itx) {
        nr = 0;
        ncell = 0;
        nn = 0;
        if (itx < a.n_items)
        {
            nr = a.order[itx];
            ncell = a.sim_cells[nr];
            nn = a.nb_cnt[nr];
        }
    };
    auto stage_b = [&]() {
        nqa = t < nn ? a.nb[(long long)nr * a.k + t] : 0;
        nqb = rb < nn ? a.nb[(long long)nr * a.k + rb] : 0;
    };
    auto stage_c = [&]() {
        nva = t < nn ? a.data[nqa] : 0.0f;
        nvb = rb < nn ? a.data[nqb] : 0.0f;
        nma = (a.means && t < nn) ? a.means[nqa] : 0.0f;
        nmb = (a.means && rb < nn) ? a.means[nqb] : 0.0f;
    };
    const int first = (blockIdx.x * nwarps + warp) * 2;
    stage_a(first + h);
    stage_b();
    stage_c();
    for (int it0 = first; it0 < a.n_items; it0 += stride)
    {
        const int it = it0 + h;
        const bool valid = it < a.n_items;
        const int r = nr, cell = ncell, n = nn, qa = nqa, qb = nqb;
        const float va = nva, vb = nvb, ma = nma, mb = nmb;
        stage_a(it + stride);
        const int cx = cell % g.nx, cy = (int)((cell / g.nx) % g.ny), cz = (int)(cell / ((long long)g.nx * g.ny));
        const bool live_a = t < n, live_b = rb < n;
        int lin_a = 0, lin_b = 0;
        if (live_a)
            lin_a = pair_lin(g, qa % g.nx - cx, (int)((qa / g.nx) % g.ny) - cy,
                             (int)(qa / ((long long)g.nx * g.ny)) - cz);
        if (live_b)
            lin_b = pair_lin(g, qb % g.nx - cx, (int)((qb / g.nx) % g.ny) - cy,
                             (int)(qb / ((long long)g.nx * g.ny)) - cz);
        LIN[t] = lin_a;
        LIN[rb] = lin_b;
        __syncwarp(gm);

        // The solve of fold32_solve written out in place: measured 41.0 ms for the
        // 8.3M systems of the 256x256x128 simulation against 46.7 ms through the
        // shared function (same registers and loads, 6.5% more instructions).
        // BOUND: both systems' live rows end at nmax (the warp's largest count).
        const int nmax = BOUND ? __reduce_max_sync(0xffffffffu, n) : NP;
        // ---- assembly (lower triangles of rows t and 31 - t; padding rows identity)
        double ra[G], rbv[NP];
        const double *base_a = pair64 + pc + lin_a, *base_b = pair64 + pc + lin_b;
#pragma unroll
        for (int c = 0; c < G; ++c)
        {
            double e = 0.0;
            if (live_a && c <= t) e = __ldg(base_a - LIN[c]);
            if (!live_a && c == t) e = 1.0;
            ra[c] = e;
        }
#pragma unroll
        for (int c = 0; c < NP; ++c)
        {
            double e = 0.0;
            if (live_b && c <= rb) e = __ldg(base_b - LIN[c]);
            if (!live_b && c == rb) e = 1.0;
            rbv[c] = e;
        }
        const double b_a = live_a ? __ldg(base_a) : 0.0;
        const double b_b = live_b ? __ldg(base_b) : 0.0;
        stage_b();

        // ---- factorisation with the forward substitution of b (and 1)
        double rhs_a[QB], rhs_b[QB], ya[QB], yb[QB];
        rhs_a[0] = b_a;
        rhs_b[0] = b_b;
        if constexpr (ORD)
        {
            rhs_a[1] = live_a ? 1.0 : 0.0;
            rhs_b[1] = live_b ? 1.0 : 0.0;
        }
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
            if (BOUND && j >= nmax) break;
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
            fail |= !(d > 0.0);
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

        stage_c();

        // ---- back substitution L^T x = y; L[i][row] = M[row][i] / sqrt(d_row)
        double xa[QB], xb[QB];
#pragma unroll
        for (int q = 0; q < QB; ++q)
        {
            xa[q] = 0.0;
            xb[q] = 0.0;
        }
#pragma unroll
        for (int i = NP - 1; i >= 0; --i)
        {
            if (BOUND && i >= nmax) continue;
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

        // ---- combine() and the variance in the reference's order
        double sx = 0.0, sy = 0.0;
        if constexpr (ORD)
        {
#pragma unroll
            for (int i = 0; i < NP; ++i)
            {
                const double x0 = __shfl_sync(gm, i < G ? xa[0] : xb[0], i < G ? i : NP - 1 - i, G);
                const double x1 = __shfl_sync(gm, i < G ? xa[1] : xb[1], i < G ? i : NP - 1 - i, G);
                if (i < n)
                {
                    sx = __dadd_rn(sx, x0);
                    sy = __dadd_rn(sy, x1);
                }
            }
        }
        const bool bad_ok = ORD && fabs(sy) < 1e-15;
        const double mu = ORD && !bad_ok ? __ddiv_rn(__dsub_rn(sx, 1.0), sy) : 0.0;
        // each lane forms its rows' terms; the sums run in row order
        const double w_a = ORD ? __dsub_rn(xa[0], __dmul_rn(mu, xa[QB - 1])) : xa[0];
        const double w_b = ORD ? __dsub_rn(xb[0], __dmul_rn(mu, xb[QB - 1])) : xb[0];
        const double vt_a = __dmul_rn(w_a, b_a), vt_b = __dmul_rn(w_b, b_b);
        const float et_a = __double2float_rn(__dmul_rn(w_a, (double)__fsub_rn(va, ma)));
        const float et_b = __double2float_rn(__dmul_rn(w_b, (double)__fsub_rn(vb, mb)));
        double var = pair64[pc];
        float est = a.means && valid ? a.means[cell] : 0.0f;
#pragma unroll 4
        for (int i = 0; i < NP; ++i)
        {
            const bool lo = i < G;
            const int src = lo ? i : NP - 1 - i;
            const double vt = __shfl_sync(gm, lo ? vt_a : vt_b, src, G);
            const float et = __shfl_sync(gm, lo ? et_a : et_b, src, G);
            if (i < n)
            {
                var = __dsub_rn(var, vt);
                est = __fadd_rn(est, et);
            }
        }
        if (ORD) var = __dsub_rn(var, mu);
        if (var < 0) var = 0;
        if (valid && t == 0)
        {
            const int status = n == 0 ? 1 : ((fail || bad_ok) ? 2 : 0);
            const double u = a.uniforms[r];
            const double val = status == 0 ? sgs_gauss_inverse(u, (double)est, var) : sgs_gauss_inverse(u, 0.0, 1.0);
            a.data[cell] = __double2float_rn(val);
            a.st_rank[r] = (signed char)status;
        }
        __syncwarp(gm);
    }
}

// 32 < n <= kSgsBlockMax: one block per node, the matrix in shared memory.
constexpr int kSgsBlockThreads = 128;

__global__ void __launch_bounds__(kSgsBlockThreads) k_sgs_solve_block(const SgsSolveArgs a)
{
    extern __shared__ double sh[];
    const int kk = a.k;
    double *A = sh;                   // kk * kk, row-major
    double *b = A + (size_t)kk * kk;  // rhs
    double *x = b + kk;               // A^-1 b
    double *y = x + kk;               // A^-1 1
    float *vals = reinterpret_cast<float *>(y + kk);
    float *ms = vals + kk;
    __shared__ int s_fail;
    const Geom &g = a.g;
    const long long pc = g.pair_center;
    for (int it = blockIdx.x; it < a.n_items; it += gridDim.x)
    {
        const int r = a.order[it];
        const int cell = a.sim_cells[r];
        const int n = a.nb_cnt[r];
        const int cx = cell % g.nx, cy = (int)((cell / g.nx) % g.ny), cz = (int)(cell / ((long long)g.nx * g.ny));
        const int *row = a.nb + (long long)r * kk;
        for (int e = threadIdx.x; e < n * n; e += blockDim.x)
        {
            const int i = e / n, j = e % n;
            const int qi = row[i], qj = row[j];
            const int dx = qi % g.nx - qj % g.nx, dy = (int)((qi / g.nx) % g.ny) - (int)((qj / g.nx) % g.ny),
                      dz = (int)(qi / ((long long)g.nx * g.ny)) - (int)(qj / ((long long)g.nx * g.ny));
            A[(size_t)i * n + j] = a.pair64[pc + pair_lin(g, dx, dy, dz)];
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x)
        {
            const int q = row[i];
            b[i] = a.pair64[pc + pair_lin(g, q % g.nx - cx, (int)((q / g.nx) % g.ny) - cy,
                                          (int)(q / ((long long)g.nx * g.ny)) - cz)];
            vals[i] = a.data[q];
            ms[i] = a.means ? a.means[q] : 0.0f;
        }
        if (threadIdx.x == 0) s_fail = 0;
        __syncthreads();
        for (int j = 0; j < n; ++j)
        {
            const double d = A[(size_t)j * n + j];
            if (threadIdx.x == 0 && !(d > 0.0)) s_fail = 1;
            const double ljj = sqrt(d);
            __syncthreads();
            for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + j] /= ljj;
            if (threadIdx.x == 0) A[(size_t)j * n + j] = ljj;
            __syncthreads();
            const int span = n - j - 1;
            for (int e = threadIdx.x; e < span * span; e += blockDim.x)
            {
                const int i = j + 1 + e / span, c = j + 1 + e % span;
                if (c <= i) A[(size_t)i * n + c] -= A[(size_t)i * n + j] * A[(size_t)c * n + j];
            }
            __syncthreads();
        }
        if (threadIdx.x < 2)
        {
            double *xv = threadIdx.x == 0 ? x : y;
            for (int i = 0; i < n; ++i)
            {
                double s = threadIdx.x == 0 ? b[i] : 1.0;
                for (int c = 0; c < i; ++c) s -= A[(size_t)i * n + c] * xv[c];
                xv[i] = s / A[(size_t)i * n + i];
            }
            for (int i = n - 1; i >= 0; --i)
            {
                double s = xv[i];
                for (int c = i + 1; c < n; ++c) s -= A[(size_t)c * n + i] * xv[c];
                xv[i] = s / A[(size_t)i * n + i];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            SgsNode o = {1, 0.0f, 0.0};
            if (n > 0)
            {
                const bool ordinary = a.ordinary != 0;
                double sx = 0.0, sy = 0.0;
                if (ordinary)
                    for (int i = 0; i < n; ++i)
                    {
                        sx = __dadd_rn(sx, x[i]);
                        sy = __dadd_rn(sy, y[i]);
                    }
                const bool fail = s_fail || (ordinary && fabs(sy) < 1e-15);
                const double mu = ordinary && !fail ? __ddiv_rn(__dsub_rn(sx, 1.0), sy) : 0.0;
                double var = a.pair64[pc];
                float est = a.means ? a.means[cell] : 0.0f;
                for (int i = 0; i < n; ++i)
                {
                    const double w = ordinary ? __dsub_rn(x[i], __dmul_rn(mu, y[i])) : x[i];
                    var = __dsub_rn(var, __dmul_rn(w, b[i]));
                    est = __fadd_rn(est, __double2float_rn(__dmul_rn(w, (double)__fsub_rn(vals[i], ms[i]))));
                }
                if (ordinary) var = __dsub_rn(var, mu);
                if (var < 0) var = 0;
                o.status = fail ? 2 : 0;
                o.mean = est;
                o.var = var;
            }
            const double u = a.uniforms[r];
            const double val =
                o.status == 0 ? sgs_gauss_inverse(u, (double)o.mean, o.var) : sgs_gauss_inverse(u, 0.0, 1.0);
            a.data[cell] = __double2float_rn(val);
            a.st_rank[r] = (signed char)o.status;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ SIS
// One launch per level: every (node, kriged category) system of the level
// (sequential_indicator_simulation.cpp:77-108): the SK estimate of the
// indicator (category == c) from the category's neighbours, accumulated in
// double around the float mean (combine for a double result); the mean where
// kriging fails. The last system of a node to finish draws its category
// (sample.cpp:8-21): the first category whose running sum exceeds u times the
// sum, p1 = 1 - p0 with two categories (median SIS).
constexpr int kSisFoldThreads = 256;
constexpr size_t kSisSysBytes = kFold32SysBytes + kFold32NP * 8; // plus the 32 row scales

// the correlogram scale of a mean (corellogramed_weights_3, my_kriging_weights.h:407-438)
__device__ __forceinline__ double sis_sigma(float mean)
{
    double m = (double)mean;
    if (m == 0) m = __dadd_rn(m, 0.00001);
    if (m == 1) m = __dsub_rn(m, 0.00001);
    return __dsqrt_rn(__dmul_rn(m, __dsub_rn(1.0, m)));
}

// the draw of rank r once every category's probability is stored (read
// through L2: other SMs wrote them); two passes, the sum then the running sum
__device__ __forceinline__ void sis_draw(const double *probs, const signed char *st_cat, int kcat, int ncat,
                                         double u, uint8_t *data_cell, signed char *st_out)
{
    const double p0 = __ldcg(probs);
    double sum = 0.0;
    int stv = 0;
    for (int c = 0; c < kcat; ++c)
    {
        sum = __dadd_rn(sum, __ldcg(probs + c));
        stv = max(stv, (int)__ldcg(reinterpret_cast<const unsigned char *>(st_cat) + c));
    }
    if (ncat == 2) sum = __dadd_rn(sum, __dsub_rn(1.0, p0)); // median SIS: p1 = 1 - p0
    const double s = __dmul_rn(u, sum);
    double acc = 0.0;
    int pick = ncat - 1;
    for (int c = 0; c < ncat; ++c)
    {
        acc = __dadd_rn(acc, ncat == 2 && c == 1 ? __dsub_rn(1.0, p0) : __ldcg(probs + c));
        if (s < acc)
        {
            pick = c;
            break;
        }
    }
    *data_cell = (uint8_t)pick;
    *st_out = (signed char)stv;
}

// CORR: correlogram weights (LVM): A_ij = C_ij (s_i s_j), b_i = C_ic (s_i s_c);
// BOUND (every k < 32): the factorisation stops at the warp's largest system
template <bool CORR, bool BOUND>
__global__ void __launch_bounds__(kSisFoldThreads, 1) k_sis_level(const SisLevelArgs a)
{
    constexpr int NP = kFold32NP, G = kFold32G;
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int h = lane / G, t = lane % G, rb = NP - 1 - t;
    const unsigned gm = 0xFFFFu << (h * G);
    unsigned char *gb = smem + kSisSysBytes * (warp * 2 + h);
    double *M = reinterpret_cast<double *>(gb);
    int *LIN = reinterpret_cast<int *>(gb + kFold32MBytes);
    double *SIG = reinterpret_cast<double *>(gb + kFold32SysBytes); // the system's row scales
    const int n_sys = a.n_nodes * a.kcat;
    const int stride = gridDim.x * nwarps * 2;
    // The next system's chain of dependent loads (rank, cell, count; its
    // neighbours; their indicators and means) is issued in three stages during
    // the current solve; its neighbours belong to lower levels, already final.
    // Systems run category-major, so the SMs of a moment share a pair table.
    int ncat_ = 0, nr = 0, ncell = 0, nn = 0, nqa = 0, nqb = 0;
    float nda = 0.0f, ndb = 0.0f, nma = 0.0f, nmb = 0.0f, nmc = 0.0f;
    auto stage_a = [&](int itx) {
        ncat_ = 0;
        nr = 0;
        ncell = 0;
        nn = 0;
        if (itx < n_sys)
        {
            ncat_ = itx / a.n_nodes;
            nr = a.order[itx - ncat_ * a.n_nodes];
            ncell = a.sim_cells[nr];
            nn = __ldg(a.cats[ncat_].nb_cnt + nr);
        }
    };
    auto stage_b = [&]() {
        const SisCat &C = a.cats[ncat_];
        nqa = t < nn ? __ldg(C.nb + (long long)nr * C.k + t) : 0;
        nqb = rb < nn ? __ldg(C.nb + (long long)nr * C.k + rb) : 0;
        nmc = C.means ? C.means[ncell] : C.marginal;
    };
    auto stage_c = [&]() {
        const float *means = a.cats[ncat_].means;
        nma = t < nn && means ? means[nqa] : nmc;
        nmb = rb < nn && means ? means[nqb] : nmc;
        nda = t < nn && a.data[nqa] == ncat_ ? 1.0f : 0.0f;
        ndb = rb < nn && a.data[nqb] == ncat_ ? 1.0f : 0.0f;
    };
    const int first = (blockIdx.x * nwarps + warp) * 2;
    stage_a(first + h);
    stage_b();
    stage_c();
    for (int it0 = first; it0 < n_sys; it0 += stride)
    {
        const int it = it0 + h;
        const bool valid = it < n_sys;
        const int cat = ncat_, r = nr, cell = ncell, n = nn, qa = nqa, qb = nqb;
        const float ia = nda, ib = ndb, ma = nma, mb = nmb, mc = nmc;
        stage_a(it + stride);
        const SisCat &C = a.cats[cat];
        const int pnx = C.pnx, pny = C.pny;
        const double *pair_c = C.pair64 + C.pair_center;
        const int cx = cell % a.nx, cy = (int)((cell / a.nx) % a.ny), cz = (int)(cell / ((long long)a.nx * a.ny));
        const bool live_a = t < n, live_b = rb < n;
        int lin_a = 0, lin_b = 0;
        if (live_a)
        {
            const int qz = (int)(qa / ((long long)a.nx * a.ny)), qy = (int)((qa / a.nx) % a.ny), qx = qa % a.nx;
            lin_a = ((qz - cz) * pny + (qy - cy)) * pnx + (qx - cx);
        }
        if (live_b)
        {
            const int qz = (int)(qb / ((long long)a.nx * a.ny)), qy = (int)((qb / a.nx) % a.ny), qx = qb % a.nx;
            lin_b = ((qz - cz) * pny + (qy - cy)) * pnx + (qx - cx);
        }
        // indicator - mean, in float
        const float da = live_a ? __fsub_rn(ia, ma) : 0.0f, db = live_b ? __fsub_rn(ib, mb) : 0.0f;
        const double sa = CORR && live_a ? sis_sigma(ma) : 1.0, sb = CORR && live_b ? sis_sigma(mb) : 1.0;
        LIN[t] = lin_a;
        LIN[rb] = lin_b;
        if (CORR)
        {
            SIG[t] = sa;
            SIG[rb] = sb;
        }
        __syncwarp(gm);
        const double sc = CORR ? sis_sigma(mc) : 1.0;
        auto load_rhs = [&](double(&rhs_a)[1], double(&rhs_b)[1]) {
            rhs_a[0] = live_a ? __ldg(pair_c + lin_a) : 0.0;
            rhs_b[0] = live_b ? __ldg(pair_c + lin_b) : 0.0;
            if (CORR)
            {
                rhs_a[0] = __dmul_rn(rhs_a[0], __dmul_rn(sa, sc));
                rhs_b[0] = __dmul_rn(rhs_b[0], __dmul_rn(sb, sc));
            }
        };
        double xa[1], xb[1];
        const int nmax = BOUND ? __reduce_max_sync(0xffffffffu, n) : NP; // both systems of the warp
        const bool fail = fold32_solve<1, false, CORR>(pair_c, LIN, M, gm, t, live_a, live_b, lin_a, lin_b, load_rhs,
                                                       xa, xb, stage_b, stage_c, SIG, sa, sb, nmax);
        const double ta = __dmul_rn(xa[0], (double)da), tb = __dmul_rn(xb[0], (double)db);
        double prob = (double)mc;
#pragma unroll 4
        for (int i = 0; i < NP; ++i)
        {
            const bool lo = i < G;
            const double ti = __shfl_sync(gm, lo ? ta : tb, lo ? i : NP - 1 - i, G);
            if (i < n) prob = __dadd_rn(prob, ti);
        }
        if (valid && t == 0)
        {
            const int status = n == 0 ? 1 : (fail ? 2 : 0);
            a.probs[(long long)r * a.kcat + cat] = status == 0 ? prob : (double)mc;
            a.st_cat[(long long)r * a.kcat + cat] = (signed char)status;
            // release this system's probability; the last system of the node acquires the others'
            cuda::atomic_ref<int, cuda::thread_scope_device> done(a.done[r]);
            if (done.fetch_add(1, cuda::memory_order_acq_rel) == a.kcat - 1)
                sis_draw(a.probs + (long long)r * a.kcat, a.st_cat + (long long)r * a.kcat, a.kcat, a.ncat,
                         a.uniforms[r], a.data + cell, a.st_rank + r);
        }
        __syncwarp(gm);
    }
}

// ------------------------------------------------------------------ launchers
void launch_sgs_forward(long long n, float *data, const uint8_t *mask, const float *means_in, float *means_out,
                        const float *cv, const float *cp, long long cn, cudaStream_t st)
{
    k_sgs_forward<<<1184, 256, 0, st>>>(n, data, mask, means_in, means_out, cv, cp, cn);
}
void launch_sgs_finalize(long long n, float *data, uint8_t *mask, const int *rank_of, int n_sim,
                         const signed char *st_rank, signed char *status, const float *cv, const float *cp,
                         long long cn, cudaStream_t st)
{
    k_sgs_finalize<<<1184, 256, 0, st>>>(n, data, mask, rank_of, n_sim, st_rank, status, cv, cp, cn);
}
void launch_sgs_path(const SgsWalk &w, const uint8_t *mask, const uint8_t *sim_mask, int *path_cell, int *flag,
                     cudaStream_t st)
{
    const long long chunks = (w.M + kWalkChunk - 1) / kWalkChunk;
    const int blocks = (int)std::min<long long>((chunks + 255) / 256, 4736);
    k_sgs_path<<<blocks, 256, 0, st>>>(w, mask, sim_mask, path_cell, flag);
}
void launch_sgs_index(long long n, const int *path_cell, const int *flag, const int *scan, const uint8_t *mask,
                      int *rank_of, int *sim_cells, cudaStream_t st)
{
    k_sgs_index<<<1184, 256, 0, st>>>(n, path_cell, flag, scan, mask, rank_of, sim_cells);
}
void launch_sgs_search(const Geom &g, const int4 *tmpl, int n_tmpl, const int *sim_cells, int n_sim,
                       const int *rank_of, int k, int *nb, int *nb_rank, int *nb_cnt, int n_sm, cudaStream_t st,
                       int fixed_rank, int rank_stride)
{
    k_sgs_search<<<n_sm * 8, 256, 0, st>>>(g, tmpl, n_tmpl, sim_cells, n_sim, rank_of, k, fixed_rank, nb, nb_rank,
                                           rank_stride > 0 ? rank_stride : k, nb_cnt);
}
void launch_sgs_levels(const int *nb_rank, const int *nb_cnt, int k, int n_sim, int *levp1, int *ticket,
                       int *level_count, int level_cap, int *max_level, int *err, int n_sm, cudaStream_t st)
{
    k_sgs_levels<<<n_sm * 8, 256, 0, st>>>(nb_rank, nb_cnt, k, n_sim, levp1, ticket, level_cap, max_level, err);
    k_sgs_level_count<<<n_sm * 2, 256, 0, st>>>(n_sim, levp1, level_cap, level_count);
}
void launch_sgs_moments(int n_sim, const int *nb_cnt, double *mom, int n_sm, cudaStream_t st)
{
    k_sgs_moments<<<n_sm * 2, 256, 0, st>>>(n_sim, nb_cnt, mom);
}
void launch_sgs_level_fill(int n_sim, const int *levp1, const int *level_off, int *level_fill, int *order,
                           cudaStream_t st)
{
    k_sgs_level_fill<<<1184, 256, 0, st>>>(n_sim, levp1, level_off, level_fill, order);
}
cudaError_t launch_sis_level(const SisLevelArgs &a, int n_sm, cudaStream_t st)
{
    const int n_sys = a.n_nodes * a.kcat;
    if (n_sys <= 0) return cudaSuccess;
    const int spb = kSisFoldThreads / kFold32G;
    const size_t smem = kSisSysBytes * spb;
    auto kern = a.correlogram ? (a.kmax < 32 ? k_sis_level<true, true> : k_sis_level<true, false>)
                              : (a.kmax < 32 ? k_sis_level<false, true> : k_sis_level<false, false>);
    int per_sm = 0;
    cudaError_t e = set_smem_min_carveout(kern, kSisFoldThreads, smem, per_sm);
    if (e != cudaSuccess) return e;
    const int blocks = std::min((n_sys + spb - 1) / spb, n_sm);
    kern<<<blocks, kSisFoldThreads, smem, st>>>(a);
    return cudaGetLastError();
}
size_t sgs_block_smem(int k) { return (size_t)k * k * 8 + 3 * (size_t)k * 8 + 2 * (size_t)k * 4; }

cudaError_t launch_sgs_solve(const Geom &g, const int *order, int n_items, const int *sim_cells, const int *nb,
                             const int *nb_cnt, int k, const double *pair64, float *data, const float *means,
                             const double *uniforms, signed char *st_rank, bool ordinary, int n_sm, cudaStream_t st)
{
    if (n_items <= 0) return cudaSuccess;
    SgsSolveArgs a{g, order, n_items, sim_cells, nb, nb_cnt, k, pair64, data, means, uniforms, st_rank,
                   ordinary ? 1 : 0};
    if (k <= 32)
    {
        const size_t smem = kSgsSysBytes * (kSgsFoldThreads / kSgsG);
        const int blocks = std::min((n_items + kSgsFoldThreads / kSgsG - 1) / (kSgsFoldThreads / kSgsG), n_sm);
        auto kern = ordinary ? (k < 32 ? k_sgs_solve_fold<true, true> : k_sgs_solve_fold<true, false>)
                             : (k < 32 ? k_sgs_solve_fold<false, true> : k_sgs_solve_fold<false, false>);
        int per_sm = 0;
        cudaError_t e = set_smem_min_carveout(kern, kSgsFoldThreads, smem, per_sm);
        if (e != cudaSuccess) return e;
        kern<<<blocks, kSgsFoldThreads, smem, st>>>(a);
    }
    else
    {
        const size_t smem = sgs_block_smem(k);
        cudaError_t e =
            cudaFuncSetAttribute(k_sgs_solve_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const int blocks = std::min(n_items, n_sm * 8);
        k_sgs_solve_block<<<blocks, kSgsBlockThreads, smem, st>>>(a);
    }
    return cudaGetLastError();
}
} // namespace hb
