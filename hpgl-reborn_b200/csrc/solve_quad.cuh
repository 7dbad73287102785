// Device pieces of the four-rows-per-lane FP32 solves (solve_quad.cu,
// solve_tile.cu): the folded row layout, the compile-time step loop, the
// factorisation with the fused forward substitution, the back substitution
// through published rows, warp-segment sums and the asynchronous copies.
#pragma once
#include "engine.cuh"

#include <cstdint>
#include <type_traits>

namespace hb
{
// row array length and offset of slot k (floats; all even)
template <int NP>
__host__ __device__ constexpr int q_len(int k)
{
    return k == 0 ? NP / 4 : k == 1 ? NP / 2 : k == 2 ? 3 * NP / 4 : NP;
}
template <int NP>
__host__ __device__ constexpr int q_off(int k)
{
    return k == 0 ? 0 : k == 1 ? NP / 4 : k == 2 ? 3 * NP / 4 : 3 * NP / 2;
}
// slot and lane owning row j
template <int NP>
__host__ __device__ constexpr int q_slot(int j)
{
    return j < NP / 4 ? 0 : j < NP / 2 ? 1 : j < 3 * NP / 4 ? 2 : 3;
}
template <int NP>
__host__ __device__ constexpr int q_owner(int j)
{
    return j < NP / 4 ? j : j < NP / 2 ? NP / 2 - 1 - j : j < 3 * NP / 4 ? j - NP / 2 : NP - 1 - j;
}
// smallest and largest row slot k can hold
template <int NP>
__host__ __device__ constexpr int q_lo(int k)
{
    return k * NP / 4;
}
template <int NP>
__host__ __device__ constexpr int q_hi(int k)
{
    return (k + 1) * NP / 4 - 1;
}

// Calls f(std::integral_constant<int, I>) for I = B .. E-1 in order, so that
// every register-array index derived from I is a compile-time constant.
template <int B, int E, typename F>
__device__ __forceinline__ void static_for(F &&f)
{
    if constexpr (B < E)
    {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

template <int NP>
__device__ __forceinline__ float q_get(const float2 (&A)[5 * NP / 4], int k, int c)
{
    const int i = q_off<NP>(k) + c;
    return (i & 1) ? A[i >> 1].y : A[i >> 1].x;
}
template <int NP>
__device__ __forceinline__ void q_set(float2 (&A)[5 * NP / 4], int k, int c, float v)
{
    const int i = q_off<NP>(k) + c;
    if (i & 1)
        A[i >> 1].y = v;
    else
        A[i >> 1].x = v;
}

template <int G, typename T>
__device__ __forceinline__ T q_sum(T v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

// Back substitution L^T x = y through published rows: at step i the owner of
// row i finishes x_i, publishes its row of L (column i of L^T) to the broadcast
// buffer and shuffles x_i to the system's lanes, which subtract L(i, r) x_i
// from their rows r < i. The correction's FP64 row sums
// Pk[k][q] = sum_{c < rows[k]} A64[rows[k]][c] x_c[q] are accumulated at the
// same steps, each lane's A64 entries of column i gathered D steps ahead so
// that the gathers' latency hides behind the substitution (17 % off the
// benchmark's bucket-32 solve against row sums formed after the substitution:
// 27.2 against 32.8 ms). `acc` holds y on entry and x on exit; the caller
// synchronises the warp before the first use of B.
template <int NP, int Q, int D>
__device__ __forceinline__ void q_back_p(const float2 (&A)[5 * NP / 4], const int (&rows)[4], const float (&inv)[4],
                                         int t, float *B, float (&acc)[4][Q], const double *__restrict__ p64c,
                                         const int (&lin)[4], const int *LIN, const bool (&live)[4],
                                         double (&Pk)[4][Q])
{
    constexpr int G = NP / 4;
    constexpr int LDB = NP + 4;
    double pre[D][4];
    auto fetch = [&](auto SC) {
        constexpr int s = decltype(SC)::value;
        constexpr int c = NP - 1 - s;
        if constexpr (c >= 0)
        {
            const int l = LIN[c];
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                pre[s % D][k] = 0.0;
                if (q_hi<NP>(k) > c)
                {
                    if (live[k] && rows[k] > c) pre[s % D][k] = __ldg(p64c + lin[k] - l);
                }
            }
        }
    };
    static_for<0, D>([&](auto SC) { fetch(SC); });
    static_for<0, NP>([&](auto IC) {
        constexpr int s = decltype(IC)::value;
        constexpr int i = NP - 1 - s;
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
#pragma unroll
                for (int q = 0; q < Q; ++q) Pk[k][q] = fma(pre[s % D][k], (double)xi[q], Pk[k][q]);
            }
        }
        fetch(std::integral_constant<int, s + D>());
    });
}

// 8-byte global -> shared copy that does not occupy registers while in flight
__device__ __forceinline__ void q_cp_async8(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void q_cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void q_cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Assembly of the lane's four rows (lower triangles) from the float pair
// table: A[r][c] = pair32[pc + lin_r - lin_c] for c <= r < n; padding rows are
// identity rows.
template <int NP>
__device__ __forceinline__ void q_assemble(float2 (&A)[5 * NP / 4], const int *LIN, const float *__restrict__ p32c,
                                           const int (&rows)[4], int n)
{
    int lin[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) lin[k] = LIN[rows[k]];
#pragma unroll
    for (int c4 = 0; c4 < NP / 4; ++c4)
    {
        const int4 l4 = reinterpret_cast<const int4 *>(LIN)[c4];
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
            const int c = 4 * c4 + e;
            const int l = e == 0 ? l4.x : e == 1 ? l4.y : e == 2 ? l4.z : l4.w;
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                if (c < q_len<NP>(k))
                {
                    float a = 0.0f;
                    if (rows[k] < n && c <= rows[k]) a = __ldg(p32c + lin[k] - l);
                    if (rows[k] >= n && c == rows[k]) a = 1.0f;
                    q_set<NP>(A, k, c, a);
                }
            }
        }
    }
}

// Right-looking Cholesky of the lane's rows with the forward substitution of
// Q right-hand sides fused in; afterwards A holds L, rhs the forward
// solutions of the lane's rows and inv the reciprocals of their diagonal.
// Returns true when a pivot is not positive. B is the system's two-row
// buffer; the caller synchronises the warp before and after.
template <int NP, int Q>
__device__ __forceinline__ bool q_factor(float2 (&A)[5 * NP / 4], float (&rhs)[4][Q], float (&inv)[4],
                                         const int (&rows)[4], int t, float *B)
{
    constexpr int LDB = NP + 4;
    static_assert(Q <= 4, "at most four right-hand sides");
    bool fail = false;
    static_for<0, NP>([&](auto JC) {
        constexpr int j = decltype(JC)::value;
        constexpr int ko = q_slot<NP>(j), to = q_owner<NP>(j);
        float *Bj = B + (j & 1) * LDB;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (j < q_len<NP>(k)) Bj[rows[k]] = q_get<NP>(A, k, j);
        if (t == to)
            *reinterpret_cast<float4 *>(Bj + NP) = make_float4(rhs[ko][0], Q > 1 ? rhs[ko][1 % Q] : 0.0f,
                                                               Q > 2 ? rhs[ko][2 % Q] : 0.0f,
                                                               Q > 3 ? rhs[ko][3 % Q] : 0.0f);
        __syncwarp();
        const float d = Bj[j];
        fail |= !(d > 0.0f);
        const float inv_s = rsqrtf(d);
        const float inv2 = inv_s * inv_s;
        float s[4];
        float2 ns[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            s[k] = 0.0f;
            if (j + 1 < q_len<NP>(k) && rows[k] > j) s[k] = q_get<NP>(A, k, j) * inv2;
            ns[k] = make_float2(-s[k], -s[k]);
        }
        const float4 *bv = reinterpret_cast<const float4 *>(Bj);
#pragma unroll
        for (int q4 = j / 4; q4 < NP / 4; ++q4)
        {
            const float4 v = bv[q4];
#pragma unroll
            for (int p = 0; p < 2; ++p)
            {
                const int c = 4 * q4 + 2 * p;
                const float2 bp = p == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                {
                    if (c < q_len<NP>(k))
                    {
                        const int e = (q_off<NP>(k) + c) >> 1;
                        if (c > j)
                            A[e] = __ffma2_rn(ns[k], bp, A[e]);
                        else if (c == j && c + 1 < q_len<NP>(k))
                            A[e].y = fmaf(-s[k], bp.y, A[e].y);
                    }
                }
            }
        }
        const float4 vr = bv[NP / 4];
        const float rj[4] = {vr.x, vr.y, vr.z, vr.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            if (j + 1 < q_len<NP>(k))
            {
#pragma unroll
                for (int q = 0; q < Q; ++q) rhs[k][q] = fmaf(-s[k], rj[q], rhs[k][q]);
            }
            if (j < q_len<NP>(k)) q_set<NP>(A, k, j, q_get<NP>(A, k, j) * inv_s);
        }
        if (t == to)
        {
            inv[ko] = inv_s;
#pragma unroll
            for (int q = 0; q < Q; ++q) rhs[ko][q] *= inv_s;
        }
    });
    return fail;
}

} // namespace hb
