// The uniform draws of the simulation, generated on the host.
//
// The reference draws with std::mt19937 and std::uniform_real_distribution
// <double>(0, 1) (bs_random_generator.cpp:21-25). This file computes the same
// numbers faster than the standard library: the Mersenne Twister MT19937
// (Matsumoto & Nishimura, 1998: n = 624, m = 397, matrix 0x9908B0DF, the
// standard tempering and seeding), its state refreshed 624 words at a time in
// loops the compiler vectorises, and each double formed from two consecutive
// outputs as libstdc++'s generate_canonical<double, 53> forms it:
// RN(g1 + g2 * 2^32) / 2^64, with 1 replaced by the largest double below 1.
// The loops are built for AVX-512, AVX2 and the baseline instruction set and
// the loader picks the widest the host has; integer steps and one rounding per
// draw make every build give the same numbers.
#include "host_model.h"

#include <cstdint>

namespace hb
{
namespace
{
constexpr int kN = 624, kM = 397;
constexpr uint32_t kMatrix = 0x9908B0DFu, kUpper = 0x80000000u, kLower = 0x7FFFFFFFu;

inline uint32_t twist(uint32_t cur, uint32_t next, uint32_t far)
{
    const uint32_t y = (cur & kUpper) | (next & kLower);
    return far ^ (y >> 1) ^ ((0u - (y & 1u)) & kMatrix);
}

#if defined(__x86_64__) && defined(__GNUC__)
#define HB_DRAW_CLONES __attribute__((target_clones("avx512f", "avx2", "default")))
#else
#define HB_DRAW_CLONES
#endif

// `blocks` state refreshes with their tempered outputs in buf, then the doubles
// of the first m (<= 312 * blocks) draws they make into out
HB_DRAW_CLONES void refill_and_convert(uint32_t *x, uint32_t *buf, int blocks, long long m, double *out)
{
    for (int b = 0; b < blocks; ++b)
    {
        uint32_t *o = buf + b * kN;
        for (int k = 0; k < kN - kM; ++k) x[k] = twist(x[k], x[k + 1], x[k + kM]);
        for (int k = kN - kM; k < kN - 1; ++k) x[k] = twist(x[k], x[k + 1], x[k + kM - kN]);
        x[kN - 1] = twist(x[kN - 1], x[0], x[kM - 1]);
        for (int k = 0; k < kN; ++k)
        {
            uint32_t y = x[k];
            y ^= y >> 11;
            y ^= (y << 7) & 0x9D2C5680u;
            y ^= (y << 15) & 0xEFC60000u;
            y ^= y >> 18;
            o[k] = y;
        }
    }
    const double below_one = 0x1.fffffffffffffp-1;
    for (long long j = 0; j < m; ++j)
    {
        const double u = ((double)buf[2 * j] + (double)buf[2 * j + 1] * 4294967296.0) * 0x1p-64;
        out[j] = u >= 1.0 ? below_one : u;
    }
}

} // namespace

void sgs_draws(unsigned long long seed, long long n, double *out)
{
    uint32_t x[kN];
    x[0] = (uint32_t)seed;
    for (int i = 1; i < kN; ++i) x[i] = 1812433253u * (x[i - 1] ^ (x[i - 1] >> 30)) + (uint32_t)i;
    uint32_t buf[2 * kN];
    long long i = 0;
    while (i < n)
    {
        // two refills: 1248 outputs, 624 draws
        const long long m = n - i < kN ? n - i : kN;
        refill_and_convert(x, buf, 2, m, out + i);
        i += m;
    }
}
} // namespace hb
