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
} // namespace hb
