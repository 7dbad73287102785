// Neighbour search on the GPU, bit-exact with the reference's
// indexed_neighbour_lookup_t::find (sugarbox_indexed_neighbour_lookup.h:67-124).
//
// Stages (all on one stream, no host round trip in between):
//   1. compact the informed cells into points, ascending node order;
//   2. bin the points (clusterizer.cpp:74-188): per-bin counts, offsets and
//      ascending-node lists; a bin holding more than `limit` points is exceeded;
//   3. per bin, decide the path of its cells: template scan when any of the 27
//      surrounding bins is exceeded (clusterizer.cpp:169-188), else the bins;
//   4. k_search: one CTA per bin. Cluster path: the CTA stages the candidate
//      list of the 27 bins (z, y, x nested, ascending nodes inside a bin) in
//      shared memory; each warp takes one cell, looks up every candidate's
//      selection key (dense covariance rank, host-built with the reference's
//      own double arithmetic), finds the k-th smallest key by radix select,
//      and keeps the k best. If a run of equal keys straddles the k-th slot the
//      reference's choice depends on std::sort's permutation; such cells are
//      queued for stage 5. Template path: one warp per cell walks the sorted
//      template 32 offsets at a time with a ballot on the mask.
//   5. k_resolve_ties: one thread per queued cell rebuilds the filtered
//      candidate list and runs the introsort restatement (gnu_introsort.h),
//      which reproduces std::sort's permutation, then takes the first k.
#include <algorithm>

#include "engine.cuh"
#include "gnu_introsort.h"
#include "kernels.h"

#include <cstdint>

namespace hb
{
// ------------------------------------------------------------------ scan
// Exclusive scan of n ints in place, in three passes; tile = 1024 per block.
constexpr int kScanTile = 1024;

__global__ void k_scan_tiles(int *v, long long n, int *tile_sums)
{
    __shared__ int warp_sums[32];
    long long base = (long long)blockIdx.x * kScanTile;
    int t = threadIdx.x; // 256 threads, 4 items each
    int a[4];
    int s = 0;
    for (int i = 0; i < 4; ++i)
    {
        long long idx = base + t * 4 + i;
        a[i] = idx < n ? v[idx] : 0;
        s += a[i];
    }
    int lane = t & 31, w = t >> 5;
    int incl = s;
    for (int o = 1; o < 32; o <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        int ws = lane < 8 ? warp_sums[lane] : 0;
        int wi = ws;
        for (int o = 1; o < 8; o <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < 8) warp_sums[lane] = wi - ws;
        if (lane == 7) tile_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    int run = warp_sums[w] + incl - s;
    for (int i = 0; i < 4; ++i)
    {
        long long idx = base + t * 4 + i;
        if (idx < n) v[idx] = run;
        run += a[i];
    }
}

__global__ void k_scan_add(int *v, long long n, const int *tile_offsets)
{
    long long idx = (long long)blockIdx.x * kScanTile + threadIdx.x;
    int add = tile_offsets[blockIdx.x];
    for (int i = 0; i < kScanTile; i += blockDim.x)
        if (idx + i < n) v[idx + i] += add;
}

// Exclusive scan; `total` (device int) receives the sum. `tmp` needs
// scan_tmp_ints(n) ints.
long long scan_tmp_ints(long long n)
{
    long long t = (n + kScanTile - 1) / kScanTile;
    long long need = t + 1;
    if (t > 1) need += scan_tmp_ints(t);
    return need;
}

int scan_kernels(long long n)
{
    const long long tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles <= 0) return 0;
    if (tiles == 1) return 1;
    return 2 + scan_kernels(tiles);
}

void exclusive_scan(int *v, long long n, int *tmp, int *total, cudaStream_t st)
{
    long long tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles <= 0)
    {
        cudaMemsetAsync(total, 0, sizeof(int), st);
        return;
    }
    int *sums = tmp;
    k_scan_tiles<<<(unsigned)tiles, 256, 0, st>>>(v, n, sums);
    if (tiles == 1)
    {
        cudaMemcpyAsync(total, sums, sizeof(int), cudaMemcpyDeviceToDevice, st);
        return;
    }
    exclusive_scan(sums, tiles, tmp + tiles + 1, total, st);
    k_scan_add<<<(unsigned)tiles, 256, 0, st>>>(v, n, sums);
}

// ------------------------------------------------------------------ points
// flag[i] = 1 for informed cells (mask != 0, property_array.h:53-58)
__global__ void k_flag_informed(const uint8_t *__restrict__ mask, long long n, int *__restrict__ flag)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        flag[i] = mask[i] != 0;
}

// after the exclusive scan, pos[i] is the point id of informed cell i
__global__ void k_emit_points(const uint8_t *__restrict__ mask, const int *__restrict__ pos, Geom g,
                              const float *__restrict__ val_f, const float *__restrict__ mean_f,
                              const uint8_t *__restrict__ val_u8,
                              int *__restrict__ pts_node, unsigned long long *__restrict__ pts_xyz,
                              float *__restrict__ pts_val, uint8_t *__restrict__ pts_cat,
                              int *__restrict__ pid_of_node)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.n_cells;
         i += (long long)gridDim.x * blockDim.x)
    {
        if (!mask[i])
        {
            if (pid_of_node) pid_of_node[i] = -1;
            continue;
        }
        int p = pos[i];
        int node = (int)i;
        int x = node % g.nx, y = node % (g.nx * g.ny) / g.nx, z = node / (g.nx * g.ny);
        pts_node[p] = node;
        pts_xyz[p] = pack_xyz(x, y, z);
        // continuous value (LVM: minus its cell's mean, the float subtraction of
        // combiner.h:19-24), or the category as a float (indicator kriging)
        pts_val[p] = val_f ? (mean_f ? val_f[i] - mean_f[i] : val_f[i]) : (val_u8 ? (float)val_u8[i] : 0.0f);
        if (val_u8 && pts_cat) pts_cat[p] = val_u8[i];
        if (pid_of_node) pid_of_node[i] = p;
    }
}

// ------------------------------------------------------------------ bins
__device__ __forceinline__ int bin_of(const Geom &g, int x, int y, int z)
{
    int cx = x / g.rx, cy = y / g.ry, cz = z / g.rz;
    return (cz * g.by + cy) * g.bx + cx;
}

__global__ void k_bin_count(const unsigned long long *__restrict__ pts_xyz, const int *__restrict__ n_pts,
                            Geom g, int *__restrict__ bin_cnt)
{
    int m = *n_pts;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x)
    {
        int x, y, z;
        unpack_xyz(pts_xyz[p], x, y, z);
        atomicAdd(&bin_cnt[bin_of(g, x, y, z)], 1);
    }
}

__global__ void k_bin_fill(const unsigned long long *__restrict__ pts_xyz, const int *__restrict__ n_pts,
                           Geom g, const int *__restrict__ bin_start, int *__restrict__ bin_fill,
                           int *__restrict__ bin_pts)
{
    int m = *n_pts;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x)
    {
        int x, y, z;
        unpack_xyz(pts_xyz[p], x, y, z);
        int b = bin_of(g, x, y, z);
        int s = atomicAdd(&bin_fill[b], 1);
        bin_pts[bin_start[b] + s] = p;
    }
}

// Restores ascending point order inside each non-exceeded bin (insertion sort;
// bins hold at most `limit` points) and records per-bin flags:
//   bit 0: exceeded (count > limit)
__global__ void k_bin_sort(Geom g, const int *__restrict__ bin_start, const int *__restrict__ bin_cnt,
                           int *__restrict__ bin_pts, uint8_t *__restrict__ bin_flag)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.n_bins; b += gridDim.x * blockDim.x)
    {
        int c = bin_cnt[b];
        bool exceeded = c > g.limit;
        bin_flag[b] = exceeded ? 1 : 0;
        if (exceeded) continue;
        int *a = bin_pts + bin_start[b];
        for (int i = 1; i < c; ++i)
        {
            int v = a[i];
            int j = i - 1;
            while (j >= 0 && a[j] > v)
            {
                a[j + 1] = a[j];
                --j;
            }
            a[j + 1] = v;
        }
    }
}

// bit 1: the cells of this bin take the template path
__global__ void k_bin_region(Geom g, uint8_t *__restrict__ bin_flag, const int *__restrict__ bin_cnt,
                             int *__restrict__ max_cand, int *__restrict__ n_template_bins,
                             int *__restrict__ template_bins, int *__restrict__ max_cand_tmpl)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.n_bins; b += gridDim.x * blockDim.x)
    {
        int cx = b % g.bx, cy = (b / g.bx) % g.by, cz = b / (g.bx * g.by);
        bool tmpl = false;
        int cand = 0;
        for (int k = cz - 1; k <= cz + 1; ++k)
            for (int j = cy - 1; j <= cy + 1; ++j)
                for (int i = cx - 1; i <= cx + 1; ++i)
                {
                    if (i < 0 || j < 0 || k < 0 || i >= g.bx || j >= g.by || k >= g.bz) continue;
                    int nb = (k * g.by + j) * g.bx + i;
                    if (bin_flag[nb] & 1) tmpl = true;
                    cand += bin_cnt[nb];
                }
        if (tmpl)
        {
            bin_flag[b] |= 2;
            template_bins[atomicAdd(n_template_bins, 1)] = b;
            atomicMax(max_cand_tmpl, cand);
        }
        else
            atomicMax(max_cand, cand);
    }
}

// ------------------------------------------------------------------ search
struct SearchSmem
{
    // layout computed at launch: [cand_x | cand_y | cand_z | cand_pid] (C_cap ints each),
    // then per warp: keys[C_cap] u32, hist[256] u32, sel[k_cap] u64
};

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Selects, for the cell at (x, y, z), the up-to-k candidates with the
// smallest keys. Returns the number selected (written to `out` as point ids,
// keys ascending, ties in candidate order) or -1 when a run of equal keys
// straddles the k-th slot.
__device__ int select_cell(const Geom &g, int x, int y, int z, int C, const int *cx, const int *cy,
                           const int *cz, const int *cpid, const float *cval,
                           const uint32_t *__restrict__ keytab, uint32_t *keys, uint32_t *hist,
                           unsigned long long *sel, int rank_bits, int lane, int *out_pid, int2 *out_rec)
{
    const int k = g.k;
    int kept = 0;
    for (int i = lane; i < C; i += 32)
    {
        int dx = cx[i] - x, dy = cy[i] - y, dz = cz[i] - z;
        uint32_t key = keytab[key_index(g, dx, dy, dz)];
        keys[i] = key;
        kept += key != kKeyExcluded;
    }
    for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
    __syncwarp();

    uint32_t kstar = kKeyExcluded; // select every kept candidate when kept <= k
    if (kept > k)
    {
        // radix select of the k-th smallest key, 8 bits per pass from the top
        int passes = (rank_bits + 7) / 8;
        uint32_t prefix = 0;
        int remaining = k; // 1-based rank still to locate inside the prefix class
        for (int p = passes - 1; p >= 0; --p)
        {
            int shift = 8 * p;
            for (int b = lane; b < 256; b += 32) hist[b] = 0;
            __syncwarp();
            for (int i = lane; i < C; i += 32)
            {
                uint32_t key = keys[i];
                if (key == kKeyExcluded) continue;
                if (p + 1 < passes && (key >> (shift + 8)) != prefix) continue;
                atomicAdd(&hist[(key >> shift) & 255u], 1u);
            }
            __syncwarp();
            // locate the digit holding the remaining-th key
            uint32_t h[8];
            uint32_t s = 0;
            for (int q = 0; q < 8; ++q)
            {
                h[q] = hist[lane * 8 + q];
                s += h[q];
            }
            uint32_t incl = s;
            for (int o = 1; o < 32; o <<= 1)
            {
                uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            uint32_t excl = incl - s;
            int digit = -1;
            uint32_t below = 0;
            if ((int)excl < remaining && (int)incl >= remaining)
            {
                uint32_t run = excl;
                for (int q = 0; q < 8; ++q)
                {
                    if ((int)(run + h[q]) >= remaining)
                    {
                        digit = lane * 8 + q;
                        below = run;
                        break;
                    }
                    run += h[q];
                }
            }
            unsigned who = __ballot_sync(0xffffffffu, digit >= 0);
            int src = __ffs(who) - 1;
            digit = __shfl_sync(0xffffffffu, digit, src);
            below = __shfl_sync(0xffffffffu, below, src);
            prefix = (prefix << 8) | (uint32_t)digit;
            remaining -= (int)below;
            __syncwarp();
        }
        kstar = prefix;
    }

    // compact the selection in candidate order: keys < kstar, then keys == kstar
    int n_less = 0, n_eq = 0;
    for (int base = 0; base < C; base += 32)
    {
        int i = base + lane;
        uint32_t key = i < C ? keys[i] : kKeyExcluded;
        bool less = (kept > k) ? key < kstar : key != kKeyExcluded;
        bool eq = (kept > k) && key == kstar;
        unsigned bl = __ballot_sync(0xffffffffu, less);
        unsigned be = __ballot_sync(0xffffffffu, eq);
        if (less)
        {
            int slot = n_less + __popc(bl & lanemask_lt());
            if (slot < k) sel[slot] = ((unsigned long long)key << 32) | (unsigned)i;
        }
        n_less += __popc(bl);
        n_eq += __popc(be);
    }
    int n_sel;
    if (kept <= k)
        n_sel = kept;
    else
    {
        int need = k - n_less;
        if (n_eq != need) return -1; // tie group straddles the k-th slot
        // append the whole tie group (it fits exactly)
        int w = n_less;
        for (int base = 0; base < C; base += 32)
        {
            int i = base + lane;
            bool eq = i < C && keys[i] == kstar;
            unsigned be = __ballot_sync(0xffffffffu, eq);
            if (eq) sel[w + __popc(be & lanemask_lt())] = ((unsigned long long)kstar << 32) | (unsigned)i;
            w += __popc(be);
        }
        n_sel = k;
    }
    __syncwarp();
    // order by (key, candidate position): rank of each entry among the selection
    for (int e = lane; e < n_sel; e += 32)
    {
        unsigned long long me = sel[e];
        int rank = 0;
        for (int f = 0; f < n_sel; ++f) rank += sel[f] < me;
        const int pos = (int)(me & 0xFFFFFFFFu);
        if (out_pid) out_pid[rank] = cpid[pos];
        if (out_rec) out_rec[rank] = make_int2(pair_lin(g, cx[pos] - x, cy[pos] - y, cz[pos] - z), __float_as_int(cval[pos]));
    }
    __syncwarp();
    return n_sel;
}

// Template path (sugarbox_neighbour_lookup.h:171-197): one warp per cell walks the
// sorted template 32 offsets at a time and keeps the first k informed nodes.
// The informed cells as a bitmap over the grid padded by (hx, hy, hz) cells on
// every side (padding bits 0): bit (q & 31) of word q >> 5 for the padded index
// q = ((z + hz) PY + (y + hy)) PX + (x + hx), PX = nx + 2 hx, PY = ny + 2 hy.
__global__ void k_mask_bits_padded(const Geom g, const uint8_t *__restrict__ mask, int hx, int hy, int hz,
                                   long long n_padded, uint32_t *__restrict__ bits)
{
    const int lane = threadIdx.x & 31;
    const long long PX = g.nx + 2LL * hx, PY = g.ny + 2LL * hy;
    for (long long base = ((long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31LL; base < n_padded;
         base += (long long)gridDim.x * blockDim.x)
    {
        const long long q = base + lane;
        bool inf = false;
        if (q < n_padded)
        {
            const long long x = q % PX - hx, y = (q / PX) % PY - hy, z = q / (PX * PY) - hz;
            if (x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz)
                inf = mask[(z * g.ny + y) * g.nx + x] != 0;
        }
        const unsigned w = __ballot_sync(0xffffffffu, inf);
        if (lane == 0) bits[base >> 5] = w;
    }
}

// Template path (sugarbox_neighbour_lookup.h:171-197): walk the sorted template
// and take the first k informed nodes. Template entries are {dx, dy, dz, padded
// linear offset}; with the padded bitmap a probe needs no bounds check (offsets
// reaching out of the grid land on padding). A warp tests 4 x 32 offsets per
// round: the entries and bits of all four steps are loaded before the first is
// consumed, then the steps are taken in order (the same first-k as the serial walk).
__device__ void template_cells(const Geom &g, const uint32_t *__restrict__ bits, int hx, int hy, int hz,
                               const uint8_t *__restrict__ mask, int all_cells, int x0, int y0, int z0, int wx,
                               int wy, int n_cells_bin, int warp, int nwarps, int lane,
                               const float *__restrict__ pts_vf, const int4 *__restrict__ tmpl, int n_tmpl,
                               const int *__restrict__ pid_of_node, int *__restrict__ nb_pid,
                               int2 *__restrict__ nb_rec, int *__restrict__ nb_n, int *__restrict__ n_template_cells)
{
    constexpr int U = 4;
    const int k = g.k;
    const long long PX = g.nx + 2LL * hx, PY = g.ny + 2LL * hy;
    int counted = 0;
    for (int c = warp; c < n_cells_bin; c += nwarps)
    {
        int x = x0 + c % wx, y = y0 + (c / wx) % wy, z = z0 + c / (wx * wy);
        long long cell = ((long long)z * g.ny + y) * g.nx + x;
        if (!all_cells && mask[cell]) continue;
        ++counted;
        const long long qc = ((long long)(z + hz) * PY + (y + hy)) * PX + (x + hx);
        int found = 0;
        for (int base = 0; base < n_tmpl && found < k; base += 32 * U)
        {
            bool ok[U];
            int t_of[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const int t = base + 32 * u + lane;
                t_of[u] = t;
                ok[u] = false;
                if (t < n_tmpl)
                {
                    const long long q = qc + tmpl[t].w;
                    ok[u] = (bits[q >> 5] >> (q & 31)) & 1u;
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                if (found >= k) break; // warp-uniform
                const unsigned bl = __ballot_sync(0xffffffffu, ok[u]);
                const int slot = found + __popc(bl & lanemask_lt());
                if (ok[u] && slot < k)
                {
                    const int4 o = tmpl[t_of[u]];
                    const long long node = ((long long)(z + o.z) * g.ny + (y + o.y)) * g.nx + (x + o.x);
                    const int p = pid_of_node[node];
                    if (nb_pid) nb_pid[cell * k + slot] = p;
                    if (nb_rec) nb_rec[cell * k + slot] = make_int2(pair_lin(g, o.x, o.y, o.z), __float_as_int(pts_vf[p]));
                }
                found += __popc(bl);
            }
        }
        if (lane == 0) nb_n[cell] = min(found, k);
    }
    if (lane == 0 && counted) atomicAdd(n_template_cells, counted);
}

__global__ void __launch_bounds__(256) k_search(
    const Geom g, const uint8_t *__restrict__ mask, int all_cells, const int *__restrict__ bin_start,
    const int *__restrict__ bin_cnt, const uint8_t *__restrict__ bin_flag, const int *__restrict__ bin_pts,
    const unsigned long long *__restrict__ pts_xyz, const float *__restrict__ pts_vf, const uint32_t *__restrict__ keytab,
    int rank_bits, const int4 *__restrict__ tmpl, int n_tmpl, const int *__restrict__ pid_of_node, int cand_cap,
    int *__restrict__ nb_pid, int2 *__restrict__ nb_rec, int *__restrict__ nb_n, int *__restrict__ tie_cells,
    int *__restrict__ tie_count, int *__restrict__ n_template_cells)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int b = blockIdx.x;
    const int bxi = b % g.bx, byi = (b / g.bx) % g.by, bzi = b / (g.bx * g.by);
    const int x0 = bxi * g.rx, y0 = byi * g.ry, z0 = bzi * g.rz;
    if (x0 >= g.nx || y0 >= g.ny || z0 >= g.nz) return; // bin past the grid: no cells
    const int x1 = min(x0 + g.rx, g.nx), y1 = min(y0 + g.ry, g.ny), z1 = min(z0 + g.rz, g.nz);
    const int wx = x1 - x0, wy = y1 - y0, wz = z1 - z0;
    const int n_cells_bin = wx * wy * wz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int k = g.k;

    if (bin_flag[b] & 2) return; // k_search_template

    // ---------------- cluster path
    int *cx = reinterpret_cast<int *>(smem);
    int *cy = cx + cand_cap;
    int *cz = cy + cand_cap;
    int *cpid = cz + cand_cap;
    float *cval = reinterpret_cast<float *>(cpid + cand_cap);
    unsigned char *wbase = reinterpret_cast<unsigned char *>(cval + cand_cap);
    const size_t per_warp = (size_t)cand_cap * 4 + 256 * 4 + (size_t)k * 8;
    uint32_t *keys = reinterpret_cast<uint32_t *>(wbase + per_warp * warp);
    uint32_t *hist = keys + cand_cap;
    unsigned long long *sel = reinterpret_cast<unsigned long long *>(hist + 256);

    // stage the 27-bin candidate list in the reference's order
    __shared__ int s_off[28];
    if (threadIdx.x == 0)
    {
        int run = 0, q = 0;
        for (int kk = bzi - 1; kk <= bzi + 1; ++kk)
            for (int jj = byi - 1; jj <= byi + 1; ++jj)
                for (int ii = bxi - 1; ii <= bxi + 1; ++ii)
                {
                    s_off[q] = run;
                    if (ii >= 0 && jj >= 0 && kk >= 0 && ii < g.bx && jj < g.by && kk < g.bz)
                        run += bin_cnt[(kk * g.by + jj) * g.bx + ii];
                    ++q;
                }
        s_off[27] = run;
    }
    __syncthreads();
    const int C = s_off[27];
    for (int q = 0; q < 27; ++q)
    {
        int kk = bzi - 1 + q / 9, jj = byi - 1 + (q / 3) % 3, ii = bxi - 1 + q % 3;
        if (ii < 0 || jj < 0 || kk < 0 || ii >= g.bx || jj >= g.by || kk >= g.bz) continue;
        int nb = (kk * g.by + jj) * g.bx + ii;
        int s = bin_start[nb], cnt = s_off[q + 1] - s_off[q];
        for (int i = threadIdx.x; i < cnt; i += blockDim.x)
        {
            int p = bin_pts[s + i];
            int px, py, pz;
            unpack_xyz(pts_xyz[p], px, py, pz);
            int d = s_off[q] + i;
            cx[d] = px;
            cy[d] = py;
            cz[d] = pz;
            cpid[d] = p;
            cval[d] = pts_vf[p];
        }
    }
    __syncthreads();

    for (int c = warp; c < n_cells_bin; c += nwarps)
    {
        int x = x0 + c % wx, y = y0 + (c / wx) % wy, z = z0 + c / (wx * wy);
        long long cell = ((long long)z * g.ny + y) * g.nx + x;
        if (!all_cells && mask[cell]) continue;
        int n = select_cell(g, x, y, z, C, cx, cy, cz, cpid, cval, keytab, keys, hist, sel, rank_bits, lane,
                            nb_pid ? nb_pid + cell * k : nullptr, nb_rec ? nb_rec + cell * k : nullptr);
        if (lane == 0)
        {
            if (n < 0)
            {
                nb_n[cell] = k; // list filled by k_resolve_ties
                int slot = atomicAdd(tie_count, 1);
                tie_cells[slot] = (int)cell;
            }
            else
                nb_n[cell] = n;
        }
    }
}

// ---------------------------------------------------------------- fast path
// Cluster-path selection for k <= 64 with 16-bit ranks: each candidate's key
// is (rank << 16) | candidate position (unique, ordered like (covariance desc,
// position)). A count-based search for a rank threshold T with
// k <= #(rank <= T) <= CAP (seeded by the k-th rank of this warp's previous
// cell) leaves at most CAP survivors, which are compacted in candidate order
// and sorted in registers (bitonic network over the warp). The k-th key then
// decides exactness: if the (k+1)-th survivor has the same rank the tie group
// straddles the k-th slot and the cell goes to k_resolve_ties.
template <int E>
__device__ __forceinline__ void warp_bitonic_sort(uint32_t (&v)[E], int lane)
{
    // element index i = e * 32 + lane; ascending over 32 * E elements
#pragma unroll
    for (int size = 2; size <= 32 * E; size <<= 1)
    {
#pragma unroll
        for (int j = size >> 1; j > 0; j >>= 1)
        {
            if (j >= 32)
            {
#pragma unroll
                for (int e = 0; e < E; ++e)
                {
                    const int pe = e ^ (j >> 5);
                    if (pe > e)
                    {
                        const bool up = (((e * 32 + lane) & size) == 0);
                        const uint32_t a = v[e], b = v[pe];
                        const bool sw = up ? (a > b) : (a < b);
                        v[e] = sw ? b : a;
                        v[pe] = sw ? a : b;
                    }
                }
            }
            else
            {
#pragma unroll
                for (int e = 0; e < E; ++e)
                {
                    const bool up = (((e * 32 + lane) & size) == 0);
                    const uint32_t p = __shfl_xor_sync(0xffffffffu, v[e], j);
                    const bool lower = (lane & j) == 0;
                    v[e] = (lower == up) ? min(v[e], p) : max(v[e], p);
                }
            }
        }
    }
}

__device__ __forceinline__ int warp_count_le(const uint32_t *keys, int C, uint32_t rank_t, int lane)
{
    int c = 0;
    for (int i = lane; i < C; i += 32) c += (keys[i] >> 16) <= rank_t;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
}

template <int E>
__device__ __forceinline__ int select_fast(const Geom &g, int C, const int *cklin, const int *cplin, const int *cpid,
                           const float *cval, int kc0, int klin_c, int plin_c,
                           const uint16_t *__restrict__ keytab, uint32_t *keys, uint32_t *sel, int lane,
                           int &kguess, int *out_pid, int2 *out_rec)
{
    constexpr int CAP = 32 * E;
    const int k = g.k;
    int kept = 0;
    for (int i = lane; i < C; i += 32)
    {
        const uint32_t r16 = keytab[kc0 + cklin[i] - klin_c];
        const uint32_t comp = r16 == 0xFFFFu ? 0xFFFFFFFFu : ((r16 << 16) | (uint32_t)i);
        keys[i] = comp;
        kept += r16 != 0xFFFFu;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
    __syncwarp();

    uint32_t T = 0xFFFEu; // keep every kept candidate
    if (kept > CAP)
    {
        // invariant: #(rank <= tlo) < k (tlo = -1 means none), #(rank <= thi) >= k
        int tlo = -1, thi = 0xFFFE;
        bool thi_tight = false; // thi known to give more than CAP survivors
        int t = kguess >= 0 ? min(kguess + (kguess >> 2) + 8, 0xFFFE) : 64;
        for (int it = 0; it < 40; ++it)
        {
            const int c = warp_count_le(keys, C, (uint32_t)t, lane);
            if (c < k)
            {
                tlo = t;
                t = thi_tight ? tlo + (thi - tlo + 1) / 2 : min(2 * t + 16, thi);
                if (t <= tlo) t = tlo + 1;
            }
            else if (c > CAP)
            {
                thi = t;
                thi_tight = true;
                if (t == tlo + 1)
                {
                    // the tie group at rank t holds more than CAP - #(rank < t) keys:
                    // it straddles the k-th slot
                    kguess = t;
                    return -1;
                }
                t = tlo + (t - tlo) / 2;
            }
            else
            {
                T = (uint32_t)t;
                break;
            }
        }
        if (T == 0xFFFEu) return -1; // no threshold found: leave the cell to the exact resolver
    }
    // compact survivors (rank <= T) in candidate order
    int cnt = 0;
    for (int base = 0; base < C; base += 32)
    {
        const int i = base + lane;
        const uint32_t key = i < C ? keys[i] : 0xFFFFFFFFu;
        const bool in = (key >> 16) <= T && key != 0xFFFFFFFFu;
        const unsigned bl = __ballot_sync(0xffffffffu, in);
        if (in)
        {
            const int slot = cnt + __popc(bl & lanemask_lt());
            if (slot < CAP) sel[slot] = key;
        }
        cnt += __popc(bl);
    }
    __syncwarp();
    if (cnt > CAP) cnt = CAP; // cannot happen: T bounds the survivors
    uint32_t v[E];
#pragma unroll
    for (int e = 0; e < E; ++e)
    {
        const int i = e * 32 + lane;
        v[e] = i < cnt ? sel[i] : 0xFFFFFFFFu;
    }
    warp_bitonic_sort<E>(v, lane);
    // sorted element i sits in v[i / 32] of lane i % 32
    const int n_sel = cnt < k ? cnt : k;
    if (n_sel <= 0) return 0;
    const uint32_t kth = __shfl_sync(0xffffffffu, v[(n_sel - 1) >> 5], (n_sel - 1) & 31);
    if (cnt > k)
    {
        const uint32_t nxt = __shfl_sync(0xffffffffu, v[k >> 5], k & 31);
        if ((nxt >> 16) == (kth >> 16))
        {
            kguess = (int)(kth >> 16);
            return -1;
        }
    }
    kguess = (int)(kth >> 16);
#pragma unroll
    for (int e = 0; e < E; ++e)
    {
        const int i = e * 32 + lane;
        if (i < n_sel)
        {
            const int pos = (int)(v[e] & 0xFFFFu);
            if (out_pid) out_pid[i] = cpid[pos];
            if (out_rec) out_rec[i] = make_int2(cplin[pos] - plin_c, __float_as_int(cval[pos]));
        }
    }
    return n_sel;
}

// Float prefilter of select_fast. One sweep forms every candidate's squared
// transformed distance h2f in float (no table reads) and keeps those with
// h2f <= Tg; only these (at most CAP) read their exact ranks, which are sorted
// as in select_fast. A candidate left out has h2f > Tg, so its true h2 exceeds
// lo = (sqrt(Tg / (1 + 4u)) - e3)^2 (three roundings in h2f, e3 the bound on the
// coordinate error). With the ranks non-decreasing in h2, lo above the largest
// h2 carrying the k-th kept rank (or above every kept offset's h2 when fewer
// than k are kept) means every candidate left out ranks strictly after the
// k-th, so the outcome equals the exact path's. Returns n_sel, -1 for a tie group straddling
// the k-th slot, or -2 when the prefilter cannot decide (the caller then runs
// select_fast). On success or -1, H receives that bound.
template <int E>
__device__ __forceinline__ int select_surr(const Geom &g, const SurrDev &sd, int C, const float4 *ctp, const int *cklin,
                           const int *cplin, const int *cpid, const float *cval, int kc0, int klin_c, int plin_c,
                           const uint16_t *__restrict__ keytab, uint32_t *sel, int lane, float tcx, float tcy,
                           float tcz, float Tg, const uint32_t *sub, int n_sub, double &H, int &kguess,
                           int *out_pid, int2 *out_rec)
{
    constexpr int CAP = 32 * E;
    const int k = g.k;
    int cnt = 0;
    __syncwarp(); // the previous cell's reads of sel are done
    // candidates scanned: the sublist `sub` (n_sub entries) when given, else all C
    const int n_scan = sub ? n_sub : C;
    for (int base = 0; base < n_scan; base += 32)
    {
        const int j = base + lane;
        bool in = false;
        int i = 0;
        if (j < n_scan)
        {
            i = sub ? (int)sub[j] : j;
            const float4 t = ctp[i];
            const float qx = t.x - tcx, qy = t.y - tcy, qz = t.z - tcz;
            in = fmaf(qz, qz, fmaf(qy, qy, qx * qx)) <= Tg;
        }
        const unsigned bl = __ballot_sync(0xffffffffu, in);
        if (in)
        {
            const int slot = cnt + __popc(bl & lanemask_lt());
            if (slot < CAP) sel[slot] = (uint32_t)i;
        }
        cnt += __popc(bl);
        if (cnt > CAP) return -2;
    }
    __syncwarp();
    uint32_t v[E];
#pragma unroll
    for (int e = 0; e < E; ++e)
    {
        const int i = e * 32 + lane;
        v[e] = 0xFFFFFFFFu;
        if (i < cnt)
        {
            const uint32_t pos = sel[i];
            const uint32_t r16 = keytab[kc0 + cklin[pos] - klin_c];
            if (r16 != 0xFFFFu) v[e] = (r16 << 16) | pos;
        }
    }
    __syncwarp();
    warp_bitonic_sort<E>(v, lane);
    int nk = 0;
#pragma unroll
    for (int e = 0; e < E; ++e) nk += __popc(__ballot_sync(0xffffffffu, v[e] != 0xFFFFFFFFu));
    uint32_t kth = 0;
    if (nk >= k)
    {
        kth = __shfl_sync(0xffffffffu, v[(k - 1) >> 5], (k - 1) & 31);
        H = sd.h2_rank[kth >> 16];
    }
    else
        H = sd.h2_cut;
    const double s = sqrt((double)Tg / (1.0 + 4.0 / 16777216.0)) - sd.e3;
    const double lo = s > 0.0 ? s * s * (1.0 - 1e-12) : 0.0;
    if (!(lo > H)) return -2;
    const int n_sel = nk < k ? nk : k;
    if (nk > k)
    {
        const uint32_t nxt = __shfl_sync(0xffffffffu, v[k >> 5], k & 31);
        if ((nxt >> 16) == (kth >> 16))
        {
            kguess = (int)(kth >> 16);
            return -1;
        }
    }
    if (n_sel > 0) kguess = (int)(__shfl_sync(0xffffffffu, v[(n_sel - 1) >> 5], (n_sel - 1) & 31) >> 16);
#pragma unroll
    for (int e = 0; e < E; ++e)
    {
        const int i = e * 32 + lane;
        if (i < n_sel)
        {
            const int pos = (int)(v[e] & 0xFFFFu);
            if (out_pid) out_pid[i] = cpid[pos];
            if (out_rec) out_rec[i] = make_int2(cplin[pos] - plin_c, __float_as_int(cval[pos]));
        }
    }
    return n_sel;
}

// transformed coordinates of an offset from the bin corner, in float
__device__ __forceinline__ float4 surr_coords(const SurrDev &sd, int x, int y, int z)
{
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    return make_float4(fmaf(sd.T[2], fz, fmaf(sd.T[1], fy, sd.T[0] * fx)),
                       fmaf(sd.T[5], fz, fmaf(sd.T[4], fy, sd.T[3] * fx)),
                       fmaf(sd.T[8], fz, fmaf(sd.T[7], fy, sd.T[6] * fx)), 0.0f);
}

template <int E>
__global__ void __launch_bounds__(256) k_search_fast(
    const Geom g, const uint8_t *__restrict__ mask, int all_cells, const int *__restrict__ bin_start,
    const int *__restrict__ bin_cnt, const uint8_t *__restrict__ bin_flag, const int *__restrict__ bin_pts,
    const unsigned long long *__restrict__ pts_xyz, const float *__restrict__ pts_vf,
    const uint16_t *__restrict__ keytab16, const SurrDev sd, int template_bins,
    const int *__restrict__ pid_of_node, int cand_cap, int *__restrict__ nb_pid, int2 *__restrict__ nb_rec,
    int *__restrict__ nb_n, int *__restrict__ tie_cells, int *__restrict__ tie_count,
    int *__restrict__ n_template_cells, int *__restrict__ exact_cells)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int b = blockIdx.x;
    const int bxi = b % g.bx, byi = (b / g.bx) % g.by, bzi = b / (g.bx * g.by);
    const int x0 = bxi * g.rx, y0 = byi * g.ry, z0 = bzi * g.rz;
    if (x0 >= g.nx || y0 >= g.ny || z0 >= g.nz) return;
    const int x1 = min(x0 + g.rx, g.nx), y1 = min(y0 + g.ry, g.ny), z1 = min(z0 + g.rz, g.nz);
    const int wx = x1 - x0, wy = y1 - y0, wz = z1 - z0;
    const int n_cells_bin = wx * wy * wz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int k = g.k;

    // the cluster-path bins, or (template_bins) the template-path bins with
    // template positions as keys
    if (((bin_flag[b] >> 1) & 1) != template_bins) return;

    float4 *ctp = reinterpret_cast<float4 *>(smem);
    int *cklin = reinterpret_cast<int *>(ctp + cand_cap);
    int *cplin = cklin + cand_cap;
    int *cpid = cplin + cand_cap;
    float *cval = reinterpret_cast<float *>(cpid + cand_cap);
    uint32_t *wbase = reinterpret_cast<uint32_t *>(cval + cand_cap);
    uint32_t *keys = wbase + (size_t)warp * (cand_cap + 32 * E);
    uint32_t *sel = keys + cand_cap;

    __shared__ int s_off[28];
    if (threadIdx.x == 0)
    {
        int run = 0, q = 0;
        for (int kk = bzi - 1; kk <= bzi + 1; ++kk)
            for (int jj = byi - 1; jj <= byi + 1; ++jj)
                for (int ii = bxi - 1; ii <= bxi + 1; ++ii)
                {
                    s_off[q] = run;
                    if (ii >= 0 && jj >= 0 && kk >= 0 && ii < g.bx && jj < g.by && kk < g.bz)
                        run += bin_cnt[(kk * g.by + jj) * g.bx + ii];
                    ++q;
                }
        s_off[27] = run;
    }
    __syncthreads();
    const int C = s_off[27];
    for (int q = 0; q < 27; ++q)
    {
        int kk = bzi - 1 + q / 9, jj = byi - 1 + (q / 3) % 3, ii = bxi - 1 + q % 3;
        if (ii < 0 || jj < 0 || kk < 0 || ii >= g.bx || jj >= g.by || kk >= g.bz) continue;
        int nb = (kk * g.by + jj) * g.bx + ii;
        int s = bin_start[nb], cnt = s_off[q + 1] - s_off[q];
        for (int i = threadIdx.x; i < cnt; i += blockDim.x)
        {
            int p = bin_pts[s + i];
            int px, py, pz;
            unpack_xyz(pts_xyz[p], px, py, pz);
            int d = s_off[q] + i;
            // linear offsets relative to the bin corner: key and pair table indices
            // of a displacement are differences of these
            cklin[d] = ((pz - z0) * g.kny + (py - y0)) * g.knx + (px - x0);
            cplin[d] = ((pz - z0) * g.pny + (py - y0)) * g.pnx + (px - x0);
            cpid[d] = p;
            cval[d] = pts_vf[p];
            ctp[d] = surr_coords(sd, px - x0, py - y0, pz - z0);
        }
    }
    __syncthreads();
    const int kc0 = (g.khz * g.kny + g.khy) * g.knx + g.khx;
    // Each warp walks a contiguous run of the bin's cells in snake order (x
    // alternating direction per row, y per layer), so consecutive cells are
    // unit steps apart and the k-th distance moves by at most the step norm.
    const int run_len = (n_cells_bin + nwarps - 1) / nwarps;
    const int c0 = warp * run_len, c1 = min(c0 + run_len, n_cells_bin);
    int kguess = -1;
    bool have_h = false;
    double h_prev = 0.0;
    float path = 0.0f;
    int n_exact = 0, n_done = 0;
    // Chunks of kChunk consecutive cells share a sublist of the candidates within
    // R of the chunk's centre (transformed coordinates), kept in `keys`. A cell scans
    // it instead of all C when sqrt(Tg) + |cell - centre| + slack <= R: every
    // candidate left out of the sublist is then farther than sqrt(Tg) from the cell
    // (true distance), so it lies beyond the prefilter's threshold like any other
    // candidate the prefilter drops. select_fast reuses `keys`, invalidating the sublist.
    // (Search stage on the 256x256x128 benchmark by chunk length: 4: 9.38 ms, 6: 9.12,
    // 8: 9.14-9.20, 12: 9.66, 16: 10.31, 24: 11.57.)
    constexpr int kChunk = 8;
    int ch_left = 0, n_sub = 0;
    bool sl_ok = false;
    float ccx = 0.f, ccy = 0.f, ccz = 0.f, Rcov = 0.f;
    const float slack = (float)(2.0 * sd.e3) + 1e-3f;
    auto snake = [&](int cc, int &sx, int &sy, int &sz) {
        const int row = cc / wx;
        sx = cc - row * wx;
        if (row & 1) sx = wx - 1 - sx;
        sz = row / wy;
        sy = row - sz * wy;
        if (sz & 1) sy = wy - 1 - sy;
    };
    for (int c = c0; c < c1; ++c)
    {
        if (c > c0) path += (c % wx) ? sd.step[0] : ((c / wx) % wy ? sd.step[1] : sd.step[2]);
        int cxr, cyr, czr;
        snake(c, cxr, cyr, czr);
        if (ch_left == 0)
        {
            ch_left = min(kChunk, c1 - c);
            sl_ok = false;
            if (sd.on && have_h)
            {
                // centre and radius of the chunk's cells in transformed coordinates
                int sx, sy, sz;
                snake(c + min(lane, ch_left - 1), sx, sy, sz);
                const float4 q = surr_coords(sd, sx, sy, sz);
                float lo_x = q.x, hi_x = q.x, lo_y = q.y, hi_y = q.y, lo_z = q.z, hi_z = q.z;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                {
                    lo_x = fminf(lo_x, __shfl_xor_sync(0xffffffffu, lo_x, o));
                    hi_x = fmaxf(hi_x, __shfl_xor_sync(0xffffffffu, hi_x, o));
                    lo_y = fminf(lo_y, __shfl_xor_sync(0xffffffffu, lo_y, o));
                    hi_y = fmaxf(hi_y, __shfl_xor_sync(0xffffffffu, hi_y, o));
                    lo_z = fminf(lo_z, __shfl_xor_sync(0xffffffffu, lo_z, o));
                    hi_z = fmaxf(hi_z, __shfl_xor_sync(0xffffffffu, hi_z, o));
                }
                ccx = 0.5f * (lo_x + hi_x);
                ccy = 0.5f * (lo_y + hi_y);
                ccz = 0.5f * (lo_z + hi_z);
                const float ex = hi_x - ccx, ey = hi_y - ccy, ez = hi_z - ccz;
                const float rho = sqrtf(ex * ex + ey * ey + ez * ez);
                Rcov = (float)sqrt(h_prev) + 2.0f * rho + 1.5f;
                const float R2 = Rcov * Rcov;
                __syncwarp();
                n_sub = 0;
                for (int base = 0; base < C; base += 32)
                {
                    const int i = base + lane;
                    bool in = false;
                    if (i < C)
                    {
                        const float4 t = ctp[i];
                        const float dx = t.x - ccx, dy = t.y - ccy, dz = t.z - ccz;
                        in = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) <= R2;
                    }
                    const unsigned bl = __ballot_sync(0xffffffffu, in);
                    if (in) keys[n_sub + __popc(bl & lanemask_lt())] = (uint32_t)i;
                    n_sub += __popc(bl);
                }
                __syncwarp();
                sl_ok = true;
            }
        }
        --ch_left;
        const long long cell = ((long long)(z0 + czr) * g.ny + (y0 + cyr)) * g.nx + (x0 + cxr);
        if (!all_cells && mask[cell]) continue;
        const int klin_c = (czr * g.kny + cyr) * g.knx + cxr;
        const int plin_c = (czr * g.pny + cyr) * g.pnx + cxr;
        int *o_pid = nb_pid ? nb_pid + cell * k : nullptr;
        int2 *o_rec = nb_rec ? nb_rec + cell * k : nullptr;
        int n = -2;
        double h = 0.0;
        if (sd.on && have_h)
        {
            const double rt = sqrt(h_prev) + (double)path + 2.0 * sd.e3;
            const float Tg = __double2float_ru(rt * rt * (1.0 + 1e-6));
            const float4 tc = surr_coords(sd, cxr, cyr, czr);
            bool use_sub = false;
            if (sl_ok)
            {
                const float dx = tc.x - ccx, dy = tc.y - ccy, dz = tc.z - ccz;
                const float dc = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
                // R excludes candidates at float distance > R from the centre: true
                // distance > R - e3 - rounding; the cell is within dc + e3 of the
                // centre; slack covers both errors and the roundings of dc and sqrt(Tg)
                use_sub = sqrtf(Tg) * (1.0f + 1e-6f) + dc * (1.0f + 1e-6f) + slack + 1e-5f * Rcov <= Rcov;
            }
            n = select_surr<E>(g, sd, C, ctp, cklin, cplin, cpid, cval, kc0, klin_c, plin_c, keytab16, sel, lane,
                               tc.x, tc.y, tc.z, Tg, use_sub ? keys : nullptr, n_sub, h, kguess, o_pid, o_rec);
        }
        if (n == -2)
        {
            n = select_fast<E>(g, C, cklin, cplin, cpid, cval, kc0, klin_c, plin_c, keytab16, keys, sel, lane,
                               kguess, o_pid, o_rec);
            sl_ok = false; // keys[] now holds select_fast's keys
            n_exact += sd.on;
            h = (sd.on && kguess >= 0) ? sd.h2_rank[kguess] : 0.0;
            have_h = sd.on && kguess >= 0 && n != 0;
        }
        else
            have_h = n != 0;
        h_prev = h;
        path = 0.0f;
        ++n_done;
        if (lane == 0)
        {
            if (n < 0)
            {
                nb_n[cell] = k;
                int slot = atomicAdd(tie_count, 1);
                tie_cells[slot] = (int)cell;
            }
            else
                nb_n[cell] = n;
        }
    }
    if (exact_cells && lane == 0 && n_exact) atomicAdd(exact_cells, n_exact);
    if (template_bins && n_template_cells && lane == 0 && n_done) atomicAdd(n_template_cells, n_done);
}

size_t search_fast_smem_bytes(int cand_cap, int k, int warps)
{
    const int E = k <= 32 ? 2 : 4;
    return (size_t)cand_cap * 32 + (size_t)warps * ((size_t)cand_cap + 32 * E) * 4;
}

cudaError_t launch_search_fast(const Geom &g, const uint8_t *mask, int all_cells, const int *bin_start,
                               const int *bin_cnt, const uint8_t *bin_flag, const int *bin_pts,
                               const unsigned long long *pts_xyz, const float *pts_vf, const uint16_t *keytab16,
                               const SurrDev &sd, int template_bins, const int *pid_of_node, int cand_cap,
                               int warps, int *nb_pid, int2 *nb_rec, int *nb_n, int *tie_cells, int *tie_count,
                               int *n_template_cells, int *exact_cells, cudaStream_t st)
{
    size_t smem = search_fast_smem_bytes(cand_cap, g.k, warps);
    if (g.k <= 32)
    {
        cudaError_t e = cudaFuncSetAttribute(k_search_fast<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_search_fast<2><<<g.n_bins, warps * 32, smem, st>>>(g, mask, all_cells, bin_start, bin_cnt, bin_flag, bin_pts,
                                                            pts_xyz, pts_vf, keytab16, sd, template_bins, pid_of_node,
                                                            cand_cap, nb_pid, nb_rec, nb_n, tie_cells, tie_count,
                                                            n_template_cells, exact_cells);
    }
    else
    {
        cudaError_t e = cudaFuncSetAttribute(k_search_fast<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_search_fast<4><<<g.n_bins, warps * 32, smem, st>>>(g, mask, all_cells, bin_start, bin_cnt, bin_flag, bin_pts,
                                                            pts_xyz, pts_vf, keytab16, sd, template_bins, pid_of_node,
                                                            cand_cap, nb_pid, nb_rec, nb_n, tie_cells, tie_count,
                                                            n_template_cells, exact_cells);
    }
    return cudaGetLastError();
}

// One thread per tie-straddling cell: rebuild the threshold-filtered candidate
// list in the reference's order, sort it with the std::sort restatement and
// keep the first k. `scratch` holds cap entries per thread.
struct KeyPid
{
    uint32_t key;
    int pid;
};
struct KeyLess
{
    __device__ bool operator()(const KeyPid &a, const KeyPid &b) const { return a.key < b.key; }
};

__global__ void k_resolve_ties(const Geom g, const int *__restrict__ tie_cells, const int *__restrict__ tie_count,
                               int first, int chunk, const int *__restrict__ bin_start,
                               const int *__restrict__ bin_cnt, const int *__restrict__ bin_pts,
                               const unsigned long long *__restrict__ pts_xyz,
                               const float *__restrict__ pts_vf, const uint32_t *__restrict__ keytab,
                               KeyPid *__restrict__ scratch, int cap, int *__restrict__ nb_pid,
                               int2 *__restrict__ nb_rec)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int idx = first + t;
    if (t >= chunk || idx >= *tie_count) return;
    int cell = tie_cells[idx];
    int x = cell % g.nx, y = cell % (g.nx * g.ny) / g.nx, z = cell / (g.nx * g.ny);
    int bxi = x / g.rx, byi = y / g.ry, bzi = z / g.rz;
    KeyPid *a = scratch + (size_t)t * cap;
    int n = 0;
    for (int kk = bzi - 1; kk <= bzi + 1; ++kk)
        for (int jj = byi - 1; jj <= byi + 1; ++jj)
            for (int ii = bxi - 1; ii <= bxi + 1; ++ii)
            {
                if (ii < 0 || jj < 0 || kk < 0 || ii >= g.bx || jj >= g.by || kk >= g.bz) continue;
                int nb = (kk * g.by + jj) * g.bx + ii;
                int s = bin_start[nb], cnt = bin_cnt[nb];
                for (int i = 0; i < cnt; ++i)
                {
                    int p = bin_pts[s + i];
                    int px, py, pz;
                    unpack_xyz(pts_xyz[p], px, py, pz);
                    uint32_t key = keytab[key_index(g, px - x, py - y, pz - z)];
                    if (key != kKeyExcluded && n < cap) a[n++] = KeyPid{key, p};
                }
            }
    gis::sort(a, (long)n, KeyLess());
    const long long base = (long long)cell * g.k;
    int m = n < g.k ? n : g.k;
    for (int i = 0; i < m; ++i)
    {
        const int p = a[i].pid;
        if (nb_pid) nb_pid[base + i] = p;
        if (nb_rec)
        {
            int px, py, pz;
            unpack_xyz(pts_xyz[p], px, py, pz);
            nb_rec[base + i] = make_int2(pair_lin(g, px - x, py - y, pz - z), __float_as_int(pts_vf[p]));
        }
    }
}

// One warp per tie-straddling cell, 16-bit ranks: the warp rebuilds the
// threshold-filtered candidate list in the reference's order in shared memory,
// replays introsort's partitions along the k-th slot (warp_select_first_k, the
// same set std::sort leaves in front), and the warp
// orders the selected k by (rank, position) for output.
struct RankLess
{
    __device__ bool operator()(uint32_t a, uint32_t b) const { return (a >> 16) < (b >> 16); }
};

// partition_around_front (libstdc++'s unguarded partition with the pivot at lo)
// by a warp. On the array as it stands, let L be the positions in (lo, hi) that
// stop the left scan (not less than the pivot), ascending, and R those in
// [lo, hi) that stop the right scan (pivot not less than them), descending.
// The serial loop swaps a[L[m]] and a[R[m]] while L[m] < R[m]; every such L
// lies below every such R, so the swaps are disjoint and independent, and the
// loop returns min(L[M], R[M-1]) for the first M with L[M] >= R[M] (an exhausted
// L counts as +inf, R[-1] as +inf). lstop / rstop hold hi - lo positions each
// (16-bit: candidate lists stay below 65,536 entries).
template <typename Less>
__device__ int warp_partition_around_front(uint32_t *a, int lo, int hi, Less less, uint16_t *lstop, uint16_t *rstop,
                                           int lane)
{
    const uint32_t pivot = a[lo];
    int nr = 0;
    for (int top = hi - 1; top >= lo; top -= 32)
    {
        const int j = top - lane;
        const bool st = j >= lo && !less(pivot, a[j]);
        const unsigned bl = __ballot_sync(0xffffffffu, st);
        if (st) rstop[nr + __popc(bl & lanemask_lt())] = (uint16_t)j;
        nr += __popc(bl);
    }
    __syncwarp();
    int nl = 0, M = -1, LM = 0x7fffffff;
    for (int base = lo + 1; base < hi; base += 32)
    {
        const int i = base + lane;
        const bool st = i < hi && !less(a[i], pivot);
        const unsigned bl = __ballot_sync(0xffffffffu, st);
        const int m = nl + __popc(bl & lanemask_lt());
        const bool cross = st && (m >= nr || i >= rstop[m]);
        if (st && !cross) lstop[m] = (uint16_t)i;
        const unsigned cb = __ballot_sync(0xffffffffu, cross);
        if (cb)
        {
            const int src = __ffs(cb) - 1;
            M = __shfl_sync(0xffffffffu, m, src);
            LM = __shfl_sync(0xffffffffu, i, src);
            break;
        }
        nl += __popc(bl);
    }
    if (M < 0) M = nl;
    __syncwarp();
    for (int m = lane; m < M; m += 32)
    {
        const int x = lstop[m], y = rstop[m];
        const uint32_t t = a[x];
        a[x] = a[y];
        a[y] = t;
    }
    __syncwarp();
    const int rm1 = M > 0 ? rstop[M - 1] : 0x7fffffff;
    return LM < rm1 ? LM : rm1;
}

// gis::select_first_k with the partitions done by the warp (median choice,
// heapsort fallback and the final short insertion sort by lane 0): the same
// first-k set std::sort leaves in front.
template <typename Less>
__device__ void warp_select_first_k(uint32_t *a, int n, int k, Less less, uint16_t *lstop, uint16_t *rstop,
                                    int lane)
{
    const int kThreshold = 16;
    if (n <= 0 || k <= 0 || k >= n) return;
    int lo = 0, hi = n;
    int depth = 2 * gis::floor_log2(n);
    while (hi - lo > kThreshold)
    {
        if (depth == 0)
        {
            if (lane == 0) gis::heap_sort_range(a, (long)lo, (long)hi, less);
            __syncwarp();
            return;
        }
        --depth;
        const int mid = lo + (hi - lo) / 2;
        if (lane == 0) gis::median_to_front(a, (long)lo, (long)lo + 1, (long)mid, (long)hi - 1, less);
        __syncwarp();
        const int cut = warp_partition_around_front(a, lo, hi, less, lstop, rstop, lane);
        if (cut == k) return;
        if (cut > k)
            hi = cut;
        else
            lo = cut;
    }
    if (lane == 0) gis::insertion_sort_guarded(a, (long)lo, (long)hi, less);
    __syncwarp();
}

// shared memory of one warp: the 27 bins' list offsets and starts, the list
// (key and slot), the point ids, the two stop lists
__host__ __device__ inline size_t ties_warp_bytes(int cap) { return 256 + ((size_t)cap * 12 + 15) / 16 * 16; }

// chunks of 32 candidates whose loads a warp has in flight at once while it
// builds a cell's list
constexpr int kTieChunks = 4;

template <int E>
__global__ void __launch_bounds__(128) k_resolve_ties_fast(
    const Geom g, const int *__restrict__ tie_cells, const int *__restrict__ tie_count,
    const int *__restrict__ bin_start, const int *__restrict__ bin_cnt, const int *__restrict__ bin_pts,
    const unsigned long long *__restrict__ pts_xyz, const float *__restrict__ pts_vf,
    const uint16_t *__restrict__ keytab, int cap, int *__restrict__ nb_pid, int2 *__restrict__ nb_rec)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int *bpre = reinterpret_cast<int *>(smem + (size_t)warp * ties_warp_bytes(cap)); // 28: list offsets
    int *bst = bpre + 32;                                                                // 27: bin starts
    uint32_t *arr = reinterpret_cast<uint32_t *>(bpre + 64);
    int *pid = reinterpret_cast<int *>(arr + cap);
    uint16_t *lstop = reinterpret_cast<uint16_t *>(pid + cap), *rstop = lstop + cap;
    const int n_ties = *tie_count;
    for (int t = blockIdx.x * nwarps + warp; t < n_ties; t += gridDim.x * nwarps)
    {
        const int cell = tie_cells[t];
        const int x = cell % g.nx, y = cell % (g.nx * g.ny) / g.nx, z = cell / (g.nx * g.ny);
        const int bxi = x / g.rx, byi = y / g.ry, bzi = z / g.rz;
        // the 27 bins (z, y, x nested) as one list: lane q < 27 holds bin q's
        // start and count, the prefix sums give each bin's offset in the list
        int bs = 0, bc = 0;
        if (lane < 27)
        {
            const int kk = bzi - 1 + lane / 9, jj = byi - 1 + (lane / 3) % 3, ii = bxi - 1 + lane % 3;
            if (ii >= 0 && jj >= 0 && kk >= 0 && ii < g.bx && jj < g.by && kk < g.bz)
            {
                const int nb = (kk * g.by + jj) * g.bx + ii;
                bs = bin_start[nb];
                bc = bin_cnt[nb];
            }
        }
        int incl = bc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int tv = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += tv;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 26);
        __syncwarp(); // the previous cell's reads of bpre / bst are done
        if (lane < 27)
        {
            bpre[lane] = incl - bc;
            bst[lane] = bs;
        }
        __syncwarp();
        // kTieChunks chunks of 32 list entries at a time: their three dependent
        // loads (point, coordinates, key) in flight together, then the chunks
        // compacted in list order
        int n = 0;
        for (int base = 0; base < total; base += 32 * kTieChunks)
        {
            int p[kTieChunks];
            unsigned long long q[kTieChunks];
            uint32_t key[kTieChunks];
#pragma unroll
            for (int u = 0; u < kTieChunks; ++u)
            {
                const int gi = base + 32 * u + lane;
                p[u] = -1;
                if (gi < total)
                {
                    int b = 0; // the last bin whose offset is <= gi
#pragma unroll
                    for (int st = 16; st > 0; st >>= 1)
                        if (b + st <= 26 && bpre[b + st] <= gi) b += st;
                    p[u] = bin_pts[bst[b] + gi - bpre[b]];
                }
            }
#pragma unroll
            for (int u = 0; u < kTieChunks; ++u) q[u] = p[u] >= 0 ? pts_xyz[p[u]] : 0ull;
#pragma unroll
            for (int u = 0; u < kTieChunks; ++u)
            {
                key[u] = 0xFFFFu;
                if (p[u] >= 0)
                {
                    int px, py, pz;
                    unpack_xyz(q[u], px, py, pz);
                    key[u] = keytab[key_index(g, px - x, py - y, pz - z)];
                }
            }
#pragma unroll
            for (int u = 0; u < kTieChunks; ++u)
            {
                const bool keep = key[u] != 0xFFFFu;
                const unsigned bl = __ballot_sync(0xffffffffu, keep);
                const int slot = n + __popc(bl & lanemask_lt());
                if (keep && slot < cap)
                {
                    arr[slot] = (key[u] << 16) | (uint32_t)slot;
                    pid[slot] = p[u];
                }
                n += __popc(bl);
            }
        }
        if (n > cap) n = cap; // cannot happen: cap bounds every candidate list
        __syncwarp();
        warp_select_first_k(arr, n, g.k, RankLess(), lstop, rstop, lane);
        const int m = n < g.k ? n : g.k;
        uint32_t v[E];
#pragma unroll
        for (int e = 0; e < E; ++e)
        {
            const int i = e * 32 + lane;
            v[e] = i < m ? arr[i] : 0xFFFFFFFFu;
        }
        warp_bitonic_sort<E>(v, lane);
        const long long base = (long long)cell * g.k;
#pragma unroll
        for (int e = 0; e < E; ++e)
        {
            const int i = e * 32 + lane;
            if (i < m)
            {
                const int j = (int)(v[e] & 0xFFFFu);
                const int p = pid[j];
                if (nb_pid) nb_pid[base + i] = p;
                if (nb_rec)
                {
                    int px, py, pz;
                    unpack_xyz(pts_xyz[p], px, py, pz);
                    nb_rec[base + i] = make_int2(pair_lin(g, px - x, py - y, pz - z), __float_as_int(pts_vf[p]));
                }
            }
        }
        __syncwarp();
    }
}

size_t resolve_ties_fast_smem(int cap, int warps) { return (size_t)warps * ties_warp_bytes(cap); }

cudaError_t launch_resolve_ties_fast(const Geom &g, const int *tie_cells, const int *tie_count, int n_ties,
                                     const int *bin_start, const int *bin_cnt, const int *bin_pts,
                                     const unsigned long long *pts_xyz, const float *pts_vf, const uint16_t *keytab16,
                                     int cap, int *nb_pid, int2 *nb_rec, int n_sm, cudaStream_t st)
{
    // Four warps a block while that keeps as many warps resident as one-warp
    // blocks would (the candidate lists of clustered data fill shared memory:
    // 31 KB a warp at 2,580 candidates, seven warps an SM in one-warp blocks,
    // four in four-warp blocks).
    constexpr size_t kSmemSM = 227u * 1024u;
    const size_t pw = ties_warp_bytes(cap);
    const long r1 = std::min<long>(32, (long)(kSmemSM / pw));
    const long r4 = 4 * (long)(kSmemSM / (4 * pw));
    const int warps = r4 >= r1 ? 4 : 1;
    const size_t smem = resolve_ties_fast_smem(cap, warps);
    int blocks = (n_ties + warps - 1) / warps;
    if (blocks > n_sm * 64 / warps) blocks = n_sm * 64 / warps;
    if (blocks < 1) blocks = 1;
    if (g.k <= 32)
    {
        cudaError_t e = cudaFuncSetAttribute(k_resolve_ties_fast<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_resolve_ties_fast<2><<<blocks, warps * 32, smem, st>>>(g, tie_cells, tie_count, bin_start, bin_cnt, bin_pts,
                                                                 pts_xyz, pts_vf, keytab16, cap, nb_pid, nb_rec);
    }
    else
    {
        cudaError_t e = cudaFuncSetAttribute(k_resolve_ties_fast<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_resolve_ties_fast<4><<<blocks, warps * 32, smem, st>>>(g, tie_cells, tie_count, bin_start, bin_cnt, bin_pts,
                                                                 pts_xyz, pts_vf, keytab16, cap, nb_pid, nb_rec);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------ launchers
void launch_flag_informed(const uint8_t *mask, long long n, int *flag, cudaStream_t st)
{
    k_flag_informed<<<1184, 256, 0, st>>>(mask, n, flag);
}
void launch_emit_points(const uint8_t *mask, const int *pos, const Geom &g, const float *val_f,
                        const float *mean_f, const uint8_t *val_u8, int *pts_node, unsigned long long *pts_xyz,
                        float *pts_val, uint8_t *pts_cat, int *pid_of_node, cudaStream_t st)
{
    k_emit_points<<<1184, 256, 0, st>>>(mask, pos, g, val_f, mean_f, val_u8, pts_node, pts_xyz, pts_val, pts_cat,
                                        pid_of_node);
}
void launch_bin_count(const unsigned long long *pts_xyz, const int *n_pts, const Geom &g, int *bin_cnt,
                      cudaStream_t st)
{
    k_bin_count<<<592, 256, 0, st>>>(pts_xyz, n_pts, g, bin_cnt);
}
void launch_bin_fill(const unsigned long long *pts_xyz, const int *n_pts, const Geom &g, const int *bin_start,
                     int *bin_fill, int *bin_pts, cudaStream_t st)
{
    k_bin_fill<<<592, 256, 0, st>>>(pts_xyz, n_pts, g, bin_start, bin_fill, bin_pts);
}
void launch_bin_sort(const Geom &g, const int *bin_start, const int *bin_cnt, int *bin_pts, uint8_t *bin_flag,
                     cudaStream_t st)
{
    int blocks = (g.n_bins + 255) / 256;
    k_bin_sort<<<blocks, 256, 0, st>>>(g, bin_start, bin_cnt, bin_pts, bin_flag);
}
void launch_bin_region(const Geom &g, uint8_t *bin_flag, const int *bin_cnt, int *max_cand, int *n_tmpl_bins,
                       int *tmpl_bins, int *max_cand_tmpl, cudaStream_t st)
{
    int blocks = (g.n_bins + 255) / 256;
    k_bin_region<<<blocks, 256, 0, st>>>(g, bin_flag, bin_cnt, max_cand, n_tmpl_bins, tmpl_bins, max_cand_tmpl);
}

// Template-path cells (k_search and k_search_fast leave their bins alone): a
// grid of (template bins) x (slices), each warp scanning the sorted template
// for one cell at a time, so the few bins that take this path (those around an
// overflowing bin) are spread over the whole GPU.
__global__ void __launch_bounds__(256) k_search_template(
    const Geom g, const uint32_t *__restrict__ bits, int hx, int hy, int hz, const uint8_t *__restrict__ mask,
    int all_cells, const int *__restrict__ template_bins,
    const float *__restrict__ pts_vf, const int4 *__restrict__ tmpl, int n_tmpl, const int *__restrict__ pid_of_node,
    int *__restrict__ nb_pid, int2 *__restrict__ nb_rec, int *__restrict__ nb_n, int *__restrict__ n_template_cells)
{
    const int b = template_bins[blockIdx.x];
    const int bxi = b % g.bx, byi = (b / g.bx) % g.by, bzi = b / (g.bx * g.by);
    const int x0 = bxi * g.rx, y0 = byi * g.ry, z0 = bzi * g.rz;
    if (x0 >= g.nx || y0 >= g.ny || z0 >= g.nz) return;
    const int wx = min(x0 + g.rx, g.nx) - x0, wy = min(y0 + g.ry, g.ny) - y0, wz = min(z0 + g.rz, g.nz) - z0;
    const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int warp = blockIdx.y * nwarps + (threadIdx.x >> 5);
    template_cells(g, bits, hx, hy, hz, mask, all_cells, x0, y0, z0, wx, wy, wx * wy * wz, warp, nwarps * gridDim.y, lane,
                   pts_vf, tmpl,
                   n_tmpl, pid_of_node, nb_pid, nb_rec, nb_n, n_template_cells);
}

long long template_padded_cells(const Geom &g)
{
    return ((long long)g.nx + 2LL * g.rx) * ((long long)g.ny + 2LL * g.ry) * ((long long)g.nz + 2LL * g.rz);
}

int template_padded_offset(const Geom &g, int dx, int dy, int dz)
{
    const long long PX = g.nx + 2LL * g.rx, PY = g.ny + 2LL * g.ry;
    return (int)(((long long)dz * PY + dy) * PX + dx);
}

cudaError_t launch_search_template(const Geom &g, const uint8_t *mask, uint32_t *bits, int all_cells,
                                   const int *tmpl_bins, int n_tmpl_bins, const float *pts_vf, const int4 *tmpl,
                                   int n_tmpl, const int *pid_of_node, int *nb_pid, int2 *nb_rec, int *nb_n,
                                   int *n_template_cells, int n_sm, cudaStream_t st)
{
    if (n_tmpl_bins <= 0) return cudaSuccess;
    {
        const long long n_padded = template_padded_cells(g);
        const int blocks = (int)std::min<long long>((n_padded + 255) / 256, (long long)n_sm * 16);
        k_mask_bits_padded<<<blocks, 256, 0, st>>>(g, mask, g.rx, g.ry, g.rz, n_padded, bits);
    }
    // about four waves of 256-thread blocks, at most one warp per 32 cells of a bin
    const long long cells = (long long)g.rx * g.ry * g.rz;
    long long split = ((long long)4 * n_sm * 8 + n_tmpl_bins - 1) / n_tmpl_bins;
    split = std::min(split, std::max(1LL, cells / (8 * 32)));
    split = std::max(1LL, std::min(split, 65535LL));
    dim3 grid((unsigned)n_tmpl_bins, (unsigned)split);
    k_search_template<<<grid, 256, 0, st>>>(g, bits, g.rx, g.ry, g.rz, mask, all_cells, tmpl_bins, pts_vf, tmpl,
                                            n_tmpl, pid_of_node, nb_pid, nb_rec, nb_n, n_template_cells);
    return cudaGetLastError();
}

size_t search_smem_bytes(int cand_cap, int k, int warps)
{
    return (size_t)cand_cap * 20 + (size_t)warps * ((size_t)cand_cap * 4 + 256 * 4 + (size_t)k * 8);
}

cudaError_t launch_search(const Geom &g, const uint8_t *mask, int all_cells, const int *bin_start,
                          const int *bin_cnt, const uint8_t *bin_flag, const int *bin_pts,
                          const unsigned long long *pts_xyz, const float *pts_vf, const uint32_t *keytab,
                          int rank_bits, const int4 *tmpl, int n_tmpl, const int *pid_of_node, int cand_cap,
                          int warps, int *nb_pid, int2 *nb_rec, int *nb_n, int *tie_cells, int *tie_count,
                          int *n_template_cells, cudaStream_t st)
{
    size_t smem = search_smem_bytes(cand_cap, g.k, warps);
    cudaError_t e = cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_search<<<g.n_bins, warps * 32, smem, st>>>(g, mask, all_cells, bin_start, bin_cnt, bin_flag, bin_pts,
                                                  pts_xyz, pts_vf, keytab, rank_bits, tmpl, n_tmpl, pid_of_node,
                                                  cand_cap, nb_pid, nb_rec, nb_n, tie_cells, tie_count,
                                                  n_template_cells);
    return cudaGetLastError();
}

void launch_resolve_ties(const Geom &g, const int *tie_cells, const int *tie_count, int first, int chunk,
                         const int *bin_start, const int *bin_cnt, const int *bin_pts,
                         const unsigned long long *pts_xyz, const float *pts_vf, const uint32_t *keytab,
                         void *scratch, int cap, int *nb_pid, int2 *nb_rec, cudaStream_t st)
{
    int threads = 64;
    int blocks = (chunk + threads - 1) / threads;
    k_resolve_ties<<<blocks, threads, 0, st>>>(g, tie_cells, tie_count, first, chunk, bin_start, bin_cnt,
                                               bin_pts, pts_xyz, pts_vf, keytab,
                                               reinterpret_cast<KeyPid *>(scratch), cap, nb_pid, nb_rec);
}
size_t tie_entry_bytes() { return sizeof(KeyPid); }
} // namespace hb
