// FP32-refined batched kriging solves of up to 32 neighbours that read their
// covariances from a union matrix shared by the block (S1/S2/K2 of the hot
// path: the dpotrf / dpotrs calls of sk_kriging_weights_3 and
// ok_kriging_weights_3, my_kriging_weights.h:147-165 and :284-303, and the
// combine of combiner.h:10-25).
//
// Work items (cells) are consecutive in grid order, so the neighbour sets of
// the items a block solves at once overlap heavily: on the 256x256x128
// benchmark 48 consecutive items of 32 neighbours name about 113 distinct
// conditioning points and about 3,000 distinct point pairs, against 25,000
// (lower-triangle) matrix entries their systems hold. Each round of the block
// therefore
//   1. decodes the items' neighbour records into grid nodes, gathers the
//      distinct ones in a shared hash table (the union, at most 144 or 112 by block size) and
//      numbers them by grid index (deterministic whatever the hash contention);
//   2. fills the lower triangle of the union's FP64 covariance matrix in
//      shared memory from the double pair table (one gather per distinct pair,
//      spread over the block's threads);
//   3. renumbers each system's rows in increasing union index, so that entry
//      (r, c), c <= r, of a system sits at tri(u_r) + u_c of the union matrix;
//   4. solves each system as the four-rows-per-lane kernel does (solve_quad.cu:
//      FP32 factorisation with the fused forward substitution, back
//      substitution through published rows, FP64 dual-weighted correction),
//      with the matrix read from the union matrix instead of the pair tables
//      and the correction's FP64 row sums accumulated inside the back
//      substitution as each solution component becomes known.
// A round whose union exceeds that is split into parts of fewer warps
// (12, 6, 3, 1), each with its own union; a single warp's four systems always
// fit. Row order does not change the solution; the forms differ from the
// other kernels' only by rounding.
#include "engine.cuh"
#include "kernels.h"
#include "solve_common.cuh"
#include "solve_quad.cuh"

#include <cstdint>

namespace hb
{
constexpr int kTileHash = 512; // hash slots (a power of two, above 4 * 32 * 4 live records per warp part)

// Union points per part of a round: 144 for 384-thread blocks (48 items, one
// block per SM), 112 for 192-thread blocks (24 items, two blocks per SM).
template <int TH>
constexpr int tile_umax()
{
    return TH >= 384 ? 144 : 112;
}

template <int NP, int R>
struct TileSys
{
    static constexpr int G = NP / 4;
    static constexpr int LDB = NP + 4;
    static constexpr size_t srec_off = (size_t)2 * LDB * sizeof(float);     // NP sorted records {lin, value}
    static constexpr size_t ui_off = srec_off + (size_t)NP * sizeof(int2);   // NP union indices (bytes)
    static constexpr size_t bits_off = ui_off + NP;                          // 5 words: the system's union bitmap
    static constexpr size_t rec_off = (bits_off + 5 * sizeof(unsigned) + 15) / 16 * 16; // 2 x NP staged records
    static constexpr size_t raw = rec_off + (size_t)2 * NP * sizeof(int2);
    static constexpr int shift = 4 * G < 16 ? 16 : 4 * G;
    static constexpr size_t bytes = raw + (size_t)((shift - (int)(raw % 128) + 128) % 128);
};

// block-level shared layout after the per-system areas
template <int UMAX>
struct TileBlock
{
    static constexpr int tri = UMAX * (UMAX + 1) / 2;
    static constexpr size_t um_off = 0;                                          // tri doubles
    static constexpr size_t hkey_off = um_off + (size_t)tri * sizeof(double);    // kTileHash ints
    static constexpr size_t hidx_off = hkey_off + (size_t)kTileHash * sizeof(int); // kTileHash ints
    static constexpr size_t hxyz_off = hidx_off + (size_t)kTileHash * sizeof(int); // kTileHash packed coords
    static constexpr size_t up_off = hxyz_off + (size_t)kTileHash * sizeof(unsigned long long); // UMAX coords
    static constexpr size_t ut_off = up_off + (size_t)UMAX * sizeof(unsigned long long); // coords, slot order
    static constexpr size_t uk_off = ut_off + (size_t)UMAX * sizeof(unsigned long long); // keys, slot order
    static constexpr size_t ur_off = uk_off + (size_t)UMAX * sizeof(int);  // slot order -> key rank
    static constexpr size_t gcnt_off = ur_off + (size_t)UMAX * sizeof(int); // 16 group counts
    static constexpr size_t misc_off = gcnt_off + 16 * sizeof(int);             // [0] union size
    static constexpr size_t bytes = misc_off + 16;
};

__device__ __forceinline__ unsigned tile_hash(int key)
{
    return ((unsigned)key * 2654435761u) >> (32 - 9);
}

// d = (dx, dy, dz) of a pair-table offset lin = (dz pny + dy) pnx + dx, |d_a| <= ph_a
__device__ __forceinline__ void decode_lin(const Geom &g, int lin, int &dx, int &dy, int &dz)
{
    const int P = g.pnx * g.pny;
    int z = __float2int_rn((float)lin * (1.0f / (float)P));
    int rem = lin - z * P;
    if (2 * rem > P) ++z, rem -= P;
    if (2 * rem < -P) --z, rem += P;
    int y = __float2int_rn((float)rem * (1.0f / (float)g.pnx));
    int x = rem - y * g.pnx;
    if (2 * x > g.pnx) ++y, x -= g.pnx;
    if (2 * x < -g.pnx) --y, x += g.pnx;
    dx = x;
    dy = y;
    dz = z;
}

// Back substitution L^T x = y (q_back_p of solve_quad.cuh) with the correction's
// FP64 row sums P_k = sum_{c < r_k} A64[r_k][c] x_c accumulated as each x_c
// is shuffled: A64[r_k][c] = um[rb[k] + u_c], u_c the union index of row c.
template <int NP, int Q>
__device__ __forceinline__ void t_back(const float2 (&A)[5 * NP / 4], const int (&rows)[4], const float (&inv)[4],
                                       int t, float *B, float (&acc)[4][Q], const double *__restrict__ um,
                                       const int (&rb)[4], const unsigned char *ui, const bool (&live)[4],
                                       double (&Pk)[4][Q])
{
    constexpr int G = NP / 4;
    constexpr int LDB = NP + 4;
    static_for<0, NP>([&](auto IC) {
        constexpr int i = NP - 1 - decltype(IC)::value;
        constexpr int ko = q_slot<NP>(i), to = q_owner<NP>(i);
        float *Bi = B + (i & 1) * LDB;
        if (t == to)
        {
#pragma unroll
            for (int q = 0; q < Q; ++q) acc[ko][q] *= inv[ko];
            float4 *bo = reinterpret_cast<float4 *>(Bi);
#pragma unroll
            for (int c4 = 0; c4 < (i + 3) / 4; ++c4)
            {
                const int e = (q_off<NP>(ko) + 4 * c4) >> 1;
                bo[c4] = make_float4(A[e].x, A[e].y, A[e + 1].x, A[e + 1].y);
            }
        }
        float xi[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) xi[q] = __shfl_sync(0xffffffffu, acc[ko][q], to, G);
        const int ui_i = ui[i];
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            if (q_lo<NP>(k) < i)
            {
                if (rows[k] < i)
                {
                    const float l = Bi[rows[k]];
#pragma unroll
                    for (int q = 0; q < Q; ++q) acc[k][q] -= l * xi[q];
                }
            }
            if (q_hi<NP>(k) > i)
            {
                if (rows[k] > i && live[k])
                {
                    const double a = um[rb[k] + ui_i];
#pragma unroll
                    for (int q = 0; q < Q; ++q) Pk[k][q] = fma(a, (double)xi[q], Pk[k][q]);
                }
            }
        }
    });
}

template <int NP, bool ORDINARY, int TH>
__global__ void __launch_bounds__(TH, TH >= 384 ? 1 : 2)
    k_solve_tile(const Geom g, const int2 *__restrict__ cells, const int *__restrict__ n_items_ptr,
                 const int2 *__restrict__ nb_rec, int ind_value, const float *__restrict__ pair32, SolveParams P)
{
    constexpr int G = NP / 4;   // lanes per system
    constexpr int H = NP / 2;
    constexpr int SPW = 32 / G; // systems per warp
    constexpr int NW = TH / 32;
    constexpr int UMAX = tile_umax<TH>();
    typedef TileBlock<UMAX> TB;
    constexpr int QB = ORDINARY ? 2 : 1;
    constexpr int R = QB + 1;
    constexpr int V = R - 1;
    typedef TileSys<NP, R> SM;
    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int h = lane / G;
    const int t = lane % G;
    unsigned char *sb = smem + SM::bytes * (warp * SPW + h);
    float *B = reinterpret_cast<float *>(sb);
    int2 *SREC = reinterpret_cast<int2 *>(sb + SM::srec_off);
    unsigned char *UI = sb + SM::ui_off;
    unsigned *BITS = reinterpret_cast<unsigned *>(sb + SM::bits_off);
    int2 *REC = reinterpret_cast<int2 *>(sb + SM::rec_off);
    unsigned char *bb = smem + SM::bytes * (NW * SPW);
    double *UM = reinterpret_cast<double *>(bb + TB::um_off);
    int *HKEY = reinterpret_cast<int *>(bb + TB::hkey_off);
    int *HIDX = reinterpret_cast<int *>(bb + TB::hidx_off);
    unsigned long long *HXYZ = reinterpret_cast<unsigned long long *>(bb + TB::hxyz_off);
    unsigned long long *UP = reinterpret_cast<unsigned long long *>(bb + TB::up_off);
    unsigned long long *UT = reinterpret_cast<unsigned long long *>(bb + TB::ut_off);
    int *UK = reinterpret_cast<int *>(bb + TB::uk_off);
    int *UR = reinterpret_cast<int *>(bb + TB::ur_off);
    int *GCNT = reinterpret_cast<int *>(bb + TB::gcnt_off);
    int *MISC = reinterpret_cast<int *>(bb + TB::misc_off);
    const int rows[4] = {t, H - 1 - t, H + t, NP - 1 - t};
    const long long pc = P.pc;
    const double *p64c = P.pair64 + pc;
    const float *p32c = pair32 + pc;
    const double d64 = __ldg(p64c);

    for (int s = tid; s < kTileHash; s += TH) HKEY[s] = -1;

    const int n_items = *n_items_ptr;
    const int per_block = (n_items + gridDim.x - 1) / gridDim.x;
    const int run_first = blockIdx.x * per_block;
    const int run_end = min(n_items, run_first + per_block);
    constexpr int SPB = NW * SPW; // items per round
    int2 w_cur = run_first + warp * SPW + h < run_end ? cells[run_first + warp * SPW + h] : make_int2(0, 0);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (rows[k] < w_cur.y) q_cp_async8(REC + rows[k], nb_rec + (long long)w_cur.x * g.k + rows[k]);
    q_cp_async_commit();
    int par = 0;
    for (int rb0 = run_first; rb0 < run_end; rb0 += SPB, par ^= 1)
    {
        const int item = rb0 + warp * SPW + h;
        const bool valid = item < run_end;
        const int my_cell = w_cur.x, my_n = w_cur.y;
        const int2 *rec = REC + par * NP;
        const int nxt = item + SPB;
        const int2 w_nxt = nxt < run_end ? cells[nxt] : make_int2(0, 0);
        q_cp_async_wait_all();
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (rows[k] < w_nxt.y)
                q_cp_async8(REC + (par ^ 1) * NP + rows[k], nb_rec + (long long)w_nxt.x * g.k + rows[k]);
        q_cp_async_commit();
        __syncthreads(); // the hash is clear, the previous round's union matrix is no longer read

        // grid coordinates of this item's cell, and its records' nodes
        const int cz = my_cell / (g.nx * g.ny);
        const int cr = my_cell - cz * (g.nx * g.ny);
        const int cy = cr / g.nx;
        const int cx = cr - cy * g.nx;
        bool live[4];
        int key[4];
        unsigned long long xyz[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            live[k] = rows[k] < my_n;
            key[k] = -1;
            xyz[k] = 0;
            if (live[k])
            {
                int dx, dy, dz;
                decode_lin(g, rec[rows[k]].x, dx, dy, dz);
                const int px = cx + dx, py = cy + dy, pz = cz + dz;
                key[k] = px + g.nx * (py + g.ny * pz);
                xyz[k] = pack_xyz(px, py, pz);
            }
        }

        // parts of the round: all warps, then halves, ... until each part's union fits
        int pw = NW;
        int p_first = 0;
        while (p_first < NW)
        {
            const bool in_part = warp >= p_first && warp < p_first + pw;
            // ---- 1. the part's distinct nodes in the hash table
            int slot[4] = {-1, -1, -1, -1};
            if (in_part)
            {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    if (!live[k]) continue;
                    unsigned s = tile_hash(key[k]);
                    for (int probe = 0; probe < kTileHash; ++probe)
                    {
                        const int old = atomicCAS(&HKEY[s], -1, key[k]);
                        if (old == -1)
                        {
                            HXYZ[s] = xyz[k];
                            slot[k] = (int)s;
                            break;
                        }
                        if (old == key[k])
                        {
                            slot[k] = (int)s;
                            break;
                        }
                        s = (s + 1) & (kTileHash - 1);
                    }
                }
            }
            __syncthreads();
            // ---- 2. the distinct nodes compacted in slot order
            for (int gi = warp; gi < kTileHash / 32; gi += NW)
            {
                const bool occ = HKEY[gi * 32 + lane] != -1;
                const unsigned bal = __ballot_sync(0xffffffffu, occ);
                if (lane == 0) GCNT[gi] = __popc(bal);
            }
            __syncthreads();
            for (int gi = warp; gi < kTileHash / 32; gi += NW)
            {
                int before = 0;
                for (int j = 0; j < gi; ++j) before += GCNT[j];
                const int s = gi * 32 + lane;
                const bool occ = HKEY[s] != -1;
                const unsigned bal = __ballot_sync(0xffffffffu, occ);
                const int u = before + __popc(bal & ((1u << lane) - 1u));
                HIDX[s] = u;
                if (occ && u < UMAX)
                {
                    UK[u] = HKEY[s];
                    UT[u] = HXYZ[s];
                }
                if (gi == kTileHash / 32 - 1 && lane == 31)
                {
                    const int un = before + __popc(bal);
                    MISC[0] = un;
                    // keys padded to a multiple of four for the rank's vector reads
                    for (int v = un; v < ((un + 3) & ~3) && v < UMAX; ++v) UK[v] = 0x7fffffff;
                }
            }
            __syncthreads();
            const int U = MISC[0];
            if (U > UMAX && pw > 1)
            {
                // clear and retry the same warps in smaller parts
                for (int s = tid; s < kTileHash; s += TH) HKEY[s] = -1;
                __syncthreads();
                pw = pw > 3 ? pw / 2 : 1;
                continue;
            }
            // ---- 2b. union index = rank of the node's key among the union's keys, so
            //          that the numbering (and with it each system's row order) does
            //          not depend on which thread won a contended hash slot; TPN
            //          threads per node, each counting over its share of the keys
            constexpr int TPN = TH >= 2 * UMAX ? 2 : 1;
            if (warp * (32 / TPN) < U)
            {
                const int e = tid / TPN, part = tid % TPN;
                const int ke = e < U ? UK[e] : 0;
                const int U4 = (U + 3) & ~3;
                const int hb = TPN == 2 ? (U4 / 4 + 1) / 2 * 4 : U4;
                const int v0 = part ? hb : 0, v1 = part ? U4 : hb;
                const int4 *k4 = reinterpret_cast<const int4 *>(UK);
                int r = 0;
                for (int v = v0; v < v1; v += 4)
                {
                    const int4 q = k4[v >> 2];
                    r += (q.x < ke ? 1 : 0) + (q.y < ke ? 1 : 0) + (q.z < ke ? 1 : 0) + (q.w < ke ? 1 : 0);
                }
                if constexpr (TPN == 2) r += __shfl_xor_sync(0xffffffffu, r, 1);
                if (e < U && part == 0)
                {
                    UR[e] = r;
                    UP[r] = UT[e];
                }
            }
            __syncthreads();
            // ---- 3. each system's rows in increasing union index (warp-local)
            int ua[4] = {0, 0, 0, 0};
            if (in_part)
            {
                if (t < 5) BITS[t] = 0u;
                __syncwarp();
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (live[k])
                    {
                        ua[k] = UR[HIDX[slot[k]]];
                        atomicOr(&BITS[ua[k] >> 5], 1u << (ua[k] & 31));
                    }
                __syncwarp();
                unsigned bw[5];
#pragma unroll
                for (int w = 0; w < 5; ++w) bw[w] = BITS[w];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (live[k])
                    {
                        const int wi = ua[k] >> 5;
                        int rank = __popc(bw[0] & (wi == 0 ? ((1u << (ua[k] & 31)) - 1u) : 0xffffffffu));
#pragma unroll
                        for (int w = 1; w < 5; ++w)
                            if (w <= wi)
                                rank += __popc(bw[w] & (w == wi ? ((1u << (ua[k] & 31)) - 1u) : 0xffffffffu));
                        SREC[rank] = rec[rows[k]];
                        UI[rank] = (unsigned char)ua[k];
                    }
            }
            // ---- 4. the union's lower triangle from the double pair table
            // (FB entries a thread at a time, their gathers in flight together)
            const int T = U * (U + 1) / 2;
            constexpr int FB = 8;
            for (int e0 = tid; e0 < T; e0 += FB * TH)
            {
                double v[FB];
#pragma unroll
                for (int f = 0; f < FB; ++f)
                {
                    const int e = e0 + f * TH;
                    v[f] = 0.0;
                    if (e < T)
                    {
                        int a = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
                        if (a * (a + 1) / 2 > e) --a;
                        if ((a + 1) * (a + 2) / 2 <= e) ++a;
                        const int b = e - a * (a + 1) / 2;
                        int ax, ay, az, bx, by, bz;
                        unpack_xyz(UP[a], ax, ay, az);
                        unpack_xyz(UP[b], bx, by, bz);
                        const int dx = ax - bx, dy = ay - by, dz = az - bz;
                        if (dx >= -g.phx && dx <= g.phx && dy >= -g.phy && dy <= g.phy && dz >= -g.phz &&
                            dz <= g.phz)
                            v[f] = __ldg(p64c + pair_lin(g, dx, dy, dz));
                    }
                }
#pragma unroll
                for (int f = 0; f < FB; ++f)
                    if (e0 + f * TH < T) UM[e0 + f * TH] = v[f];
            }
            __syncthreads();
            // the hash is read no more in this part: clear it for the next part or round
            for (int s = tid; s < kTileHash; s += TH) HKEY[s] = -1;

            if (in_part)
            {
                // ---- 5. the systems of the part, rows in union order
                const unsigned char *ui = UI;
                int lin[4], rbase[4];
                float vcf[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    const int2 sr = live[k] ? SREC[rows[k]] : make_int2(0, 0);
                    lin[k] = sr.x;
                    vcf[k] = (float)centred_value(live[k], __int_as_float(sr.y), ind_value, P.mf);
                    const int u = live[k] ? ui[rows[k]] : 0;
                    rbase[k] = u * (u + 1) / 2;
                }
                float2 A[5 * NP / 4];
#pragma unroll
                for (int c = 0; c < NP; ++c)
                {
                    const int uc = ui[c];
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                    {
                        if (c < q_len<NP>(k))
                        {
                            float a = 0.0f;
                            if (live[k] && c <= rows[k]) a = (float)UM[rbase[k] + uc];
                            if (!live[k] && c == rows[k]) a = 1.0f;
                            q_set<NP>(A, k, c, a);
                        }
                    }
                }
                float rhs[4][R];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    rhs[k][0] = live[k] ? __ldg(p32c + lin[k]) : 0.0f;
                    if constexpr (ORDINARY) rhs[k][1] = live[k] ? 1.0f : 0.0f;
                    rhs[k][V] = vcf[k];
                }
                float inv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                const bool fail = q_factor<NP, R>(A, rhs, inv, rows, t, B);
                __syncwarp();
                double Pk[4][R];
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int q = 0; q < R; ++q) Pk[k][q] = 0.0;
                t_back<NP, R>(A, rows, inv, t, B, rhs, UM, rbase, ui, live, Pk);

                // ---- the dual-weighted FP64 correction of the bilinear forms
                double b64[4], vc[4], one[4], x[4][R];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    b64[k] = live[k] ? __ldg(p64c + lin[k]) : 0.0;
                    vc[k] = (double)vcf[k];
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
                const double corr_vb = dot(b64, V) - bil(V, 0);
                const double corr_bb = dot(b64, 0) - bil(0, 0);
                const double s_vb = q_sum<G>(dot(vc, 0) + corr_vb);
                const double s_bb = q_sum<G>(dot(b64, 0) + corr_bb);
                double s_1b = 0.0, s_v1 = 0.0, s_11 = 0.0;
                if constexpr (ORDINARY)
                {
                    s_1b = q_sum<G>(dot(one, 0) + dot(b64, 1) - bil(1, 0));
                    s_v1 = q_sum<G>(dot(vc, 1) + dot(one, V) - bil(V, 1));
                    s_11 = q_sum<G>(2.0 * dot(one, 1) - bil(1, 1));
                }
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
                        const int slot_e = atomicAdd(P.esc_count, 1);
                        P.esc_cells[slot_e] = make_int2(my_cell, my_n);
                        if (P.out.status) P.out.status[my_cell] = 4;
                    }
                    else
                        write_solution<ORDINARY>(P, my_cell, fail, s_vb, s_bb, s_1b, s_v1, s_11);
                }
                __syncwarp();
            }
            p_first += pw;
            __syncthreads(); // the part's union matrix is read no more
        }
        w_cur = w_nxt;
    }
    q_cp_async_wait_all();
}

template <bool ORD, int TH>
static cudaError_t launch_tile_one(const Geom &g, const int2 *cells, const int *n_items, int max_items,
                                   const int2 *nb_rec, int ind_value, const float *pair32, const SolveParams &P,
                                   int n_sm, cudaStream_t st)
{
    constexpr int spb = TH / 32 * 4;
    const size_t smem = TileSys<32, ORD ? 3 : 2>::bytes * spb + TileBlock<tile_umax<TH>()>::bytes;
    auto kern = k_solve_tile<32, ORD, TH>;
    int blocks = 0;
    cudaError_t e = launch_kernel(kern, TH, smem, max_items, spb, n_sm, blocks);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)blocks, TH, smem, st>>>(g, cells, n_items, nb_rec, ind_value, pair32, P);
    return cudaGetLastError();
}

cudaError_t launch_solve_tile(int np, bool ordinary, int threads, const Geom &g, const int2 *cells,
                              const int *n_items, int max_items, const int2 *nb_rec, int ind_value,
                              const float *pair32, const SolveParams &P, int n_sm, cudaStream_t st)
{
    if (np != 32 || (threads != 384 && threads != 192)) return cudaErrorInvalidValue;
#define HB_ARGS g, cells, n_items, max_items, nb_rec, ind_value, pair32, P, n_sm, st
    if (threads == 384)
        return ordinary ? launch_tile_one<true, 384>(HB_ARGS) : launch_tile_one<false, 384>(HB_ARGS);
    return ordinary ? launch_tile_one<true, 192>(HB_ARGS) : launch_tile_one<false, 192>(HB_ARGS);
#undef HB_ARGS
}
} // namespace hb
