// The solve-kernel tuning table: which launch shape runs each
// (neighbour-count bucket, covariance type, precision) key. Keys start at
// kVariantDefault, which resolves to the built-in pick; set_solve_variant
// overrides one key (the tuning cache and the tests use it).
#include "kernels.h"

#include <atomic>

namespace hb
{
namespace
{
constexpr int kCovTypes = 3;
std::atomic<int> g_table[2][4][kCovTypes];

int bucket_index(int np)
{
    switch (np)
    {
    case 8:
        return 0;
    case 16:
        return 1;
    case 32:
        return 2;
    case 64:
        return 3;
    default:
        return -1;
    }
}

// the built-in pick of each key
int builtin_variant(int np, int precision)
{
    if (precision == 1 && np <= 32) return kVariantQuad;
    return kVariantFold;
}
} // namespace

int solve_variant(int np, int cov_type, int precision)
{
    const int b = bucket_index(np);
    if (b < 0 || precision < 0 || precision > 1) return kVariantFold;
    const int c = cov_type >= 0 && cov_type < kCovTypes ? cov_type : 0;
    const int v = g_table[precision][b][c].load(std::memory_order_relaxed);
    return v == kVariantDefault ? builtin_variant(np, precision) : v;
}

// Returns the key's previous setting (kVariantDefault when it had none), or
// -1 when the key or the variant is invalid.
int set_solve_variant(int np, int cov_type, int precision, int variant)
{
    const int b = bucket_index(np);
    if (b < 0 || precision < 0 || precision > 1 || cov_type < 0 || cov_type >= kCovTypes) return -1;
    if (variant < 0 || variant >= kVariantCount || !solve_variant_valid(np, precision, variant)) return -1;
    return g_table[precision][b][cov_type].exchange(variant, std::memory_order_relaxed);
}
} // namespace hb
