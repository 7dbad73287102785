// Device-side data layout shared by the search and solve kernels.
//
// Grid: node = x + nx*y + nx*ny*z (Fortran order of the caller's arrays,
// sugarbox_grid.cpp:70-74). Conditioning ("informed") cells are compacted in
// ascending node order into points; point p has node pts_node[p], packed
// coordinates pts_xyz[p] and value pts_val[p] (or category pts_cat[p]).
//
// Bins (the reference's clusterizer, clusterizer.cpp:74-188): bin size = the
// search radius per axis, (g / r + 2) bins per axis; a bin lists its points in
// ascending node order; a bin with more than `limit` points is "exceeded" and
// every cell whose 27 surrounding bins include an exceeded one uses the
// template scan instead of the bins.
//
// Neighbour lists: per kriged cell slot, up to `k` point ids (int32) in
// covariance-descending order plus a count (uint8/int16 -> int32 here).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hb
{
constexpr uint32_t kKeyExcluded = 0xFFFFFFFFu;

// Packs (x, y, z) grid coordinates (each < 2^21) into 64 bits.
__host__ __device__ __forceinline__ unsigned long long pack_xyz(int x, int y, int z)
{
    return (unsigned long long)(unsigned)x | ((unsigned long long)(unsigned)y << 21) |
           ((unsigned long long)(unsigned)z << 42);
}
__host__ __device__ __forceinline__ void unpack_xyz(unsigned long long p, int &x, int &y, int &z)
{
    x = (int)(p & 0x1FFFFF);
    y = (int)((p >> 21) & 0x1FFFFF);
    z = (int)((p >> 42) & 0x1FFFFF);
}

struct Geom
{
    int nx, ny, nz;          // grid
    long long n_cells;
    int rx, ry, rz;          // search radiuses (bin sizes)
    int bx, by, bz;          // bins per axis
    int n_bins;
    int limit;               // clusterizer limit = |template| / 250
    int k;                   // max neighbours
    // selection-key block (|d_a| <= kh_a), x fastest
    int khx, khy, khz, knx, kny;
    // pair-covariance block (|d_a| <= ph_a), x fastest
    int phx, phy, phz, pnx, pny;
    long long pair_center;   // index of offset (0,0,0) in the pair block
};

__host__ __device__ __forceinline__ long long key_index(const Geom &g, int dx, int dy, int dz)
{
    return ((long long)(dz + g.khz) * g.kny + (dy + g.khy)) * g.knx + (dx + g.khx);
}
__host__ __device__ __forceinline__ bool key_in_block(const Geom &g, int dx, int dy, int dz)
{
    return dx >= -g.khx && dx <= g.khx && dy >= -g.khy && dy <= g.khy && dz >= -g.khz && dz <= g.khz;
}
// linear pair-table offset of a displacement: pair index = pair_center + lin(d)
__host__ __device__ __forceinline__ int pair_lin(const Geom &g, int dx, int dy, int dz)
{
    return (dz * g.pny + dy) * g.pnx + dx;
}
// Dynamic shared memory of `smem` bytes per block for `kern`, then the
// smallest shared-memory carveout that holds the blocks an SM keeps resident
// at that size (per_sm, returned): the rest of the SM's unified L1 / shared
// storage stays L1 for the kernels' pair-table gathers.
template <typename K>
inline cudaError_t set_smem_min_carveout(K kern, int threads, size_t smem, int &per_sm)
{
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int dev = 0, smem_sm = 0, reserved = 0;
    cudaFuncAttributes fa{};
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess &&
        cudaFuncGetAttributes(&fa, kern) == cudaSuccess && smem_sm > 0)
    {
        const long long need = (long long)per_sm * ((long long)smem + (long long)fa.sharedSizeBytes + reserved);
        int pct = (int)((need * 100 + smem_sm - 1) / smem_sm);
        pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
} // namespace hb
