// The solve-kernel tuning table: which launch shape runs each
// (neighbour-count bucket, covariance type, precision) key.
//
// A key starts at kVariantDefault, which resolves to the built-in pick. It is
// set by an explicit override (set_solve_variant), by a tuning cache read
// from a JSON file (tune_load: the file the offline tuner writes), or, in
// tuning mode, by timing every variant the key can run the first time the
// engine meets a large enough bucket of it (tune_record; engine.cu). tune_save
// writes the keys that have a setting, with the timings that chose them.
#include "engine_api.h"
#include "kernels.h"

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace hb
{
namespace
{
constexpr int kCovTypes = 3;
constexpr int kNpBuckets = 4;
std::atomic<int> g_table[2][kNpBuckets][kCovTypes];
std::atomic<int> g_mode{0};
std::mutex g_ms_mu;
double g_ms[2][kNpBuckets][kCovTypes][kVariantCount]; // timings behind a tuned pick (ms per 1M systems)
int g_source[2][kNpBuckets][kCovTypes];               // 0 none, 1 override, 2 cache file, 3 timed here

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
    if (np > 32) return kVariantWide;
    if (precision == 1) return kVariantQuad;
    return kVariantFold;
}

bool key_ok(int b, int cov_type, int precision)
{
    return b >= 0 && precision >= 0 && precision <= 1 && cov_type >= 0 && cov_type < kCovTypes;
}

const char *kVariantNames[kVariantCount] = {"default", "fold", "quad", "fold_narrow", "quad_narrow", "tile",
                                            "tile_narrow", "wide"};
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
    if (!key_ok(b, cov_type, precision)) return -1;
    if (variant < 0 || variant >= kVariantCount || !solve_variant_valid(np, precision, variant)) return -1;
    {
        std::lock_guard<std::mutex> lk(g_ms_mu);
        g_source[precision][b][cov_type] = variant == kVariantDefault ? 0 : 1;
    }
    return g_table[precision][b][cov_type].exchange(variant, std::memory_order_relaxed);
}

int tune_mode() { return g_mode.load(std::memory_order_relaxed); }
void set_tune_mode(int on) { g_mode.store(on ? 1 : 0, std::memory_order_relaxed); }

// whether the tuning mode should time this key now (no setting yet)
bool tune_wanted(int np, int cov_type, int precision)
{
    const int b = bucket_index(np);
    if (!tune_mode() || !key_ok(b, cov_type, precision)) return false;
    return g_table[precision][b][cov_type].load(std::memory_order_relaxed) == kVariantDefault;
}

// Records the timings of every variant of a key (ms per 1M systems, <= 0 for
// a variant that did not run) and sets the fastest.
void tune_record(int np, int cov_type, int precision, const double *ms_per_variant)
{
    const int b = bucket_index(np);
    if (!key_ok(b, cov_type, precision)) return;
    int best = kVariantDefault;
    double best_ms = 0.0;
    std::lock_guard<std::mutex> lk(g_ms_mu);
    for (int v = 1; v < kVariantCount; ++v)
    {
        g_ms[precision][b][cov_type][v] = ms_per_variant[v];
        if (ms_per_variant[v] > 0.0 && (best == kVariantDefault || ms_per_variant[v] < best_ms))
        {
            best = v;
            best_ms = ms_per_variant[v];
        }
    }
    if (best == kVariantDefault) return;
    g_source[precision][b][cov_type] = 3;
    g_table[precision][b][cov_type].store(best, std::memory_order_relaxed);
}

// The cache file: a JSON list of objects
//   {"np": 32, "cov_type": 1, "precision": 1, "variant": "quad",
//    "ms_per_million": {"fold": 4.81, "quad": 3.95}}
// Reading takes np, cov_type, precision and variant (a name or a number) of
// each object and ignores everything else.
namespace
{
bool json_int(const std::string &obj, const char *key, int &out)
{
    const std::string k = std::string("\"") + key + "\"";
    size_t p = obj.find(k);
    if (p == std::string::npos) return false;
    p = obj.find(':', p + k.size());
    if (p == std::string::npos) return false;
    ++p;
    while (p < obj.size() && (obj[p] == ' ' || obj[p] == '\t' || obj[p] == '\n' || obj[p] == '\r')) ++p;
    if (p < obj.size() && obj[p] == '"')
    {
        const size_t e = obj.find('"', p + 1);
        if (e == std::string::npos) return false;
        const std::string name = obj.substr(p + 1, e - p - 1);
        for (int v = 0; v < kVariantCount; ++v)
            if (name == kVariantNames[v])
            {
                out = v;
                return true;
            }
        return false;
    }
    char *end = nullptr;
    const long v = std::strtol(obj.c_str() + p, &end, 10);
    if (end == obj.c_str() + p) return false;
    out = (int)v;
    return true;
}
} // namespace

int tune_load(const char *path, std::string &err)
{
    FILE *f = std::fopen(path, "rb");
    if (!f)
    {
        err = std::string("cannot open ") + path;
        return -1;
    }
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    // every entry is checked before any is applied: a file that fails leaves
    // the table as it was
    struct Entry
    {
        int prec, b, cov, var;
    };
    std::vector<Entry> entries;
    size_t pos = 0;
    while (true)
    {
        // objects are the innermost {...} holding an "np" key
        const size_t open = text.find("\"np\"", pos);
        if (open == std::string::npos) break;
        const size_t lb = text.rfind('{', open);
        size_t rb = text.find('}', open);
        // skip a nested timing object: the entry closes at the brace after the
        // one that closes it (rb is then that inner brace, the first after open)
        const size_t nested = text.find('{', open);
        if (rb != std::string::npos && nested != std::string::npos && nested < rb) rb = text.find('}', rb + 1);
        if (lb == std::string::npos || rb == std::string::npos)
        {
            err = "malformed tuning cache";
            return -1;
        }
        const std::string obj = text.substr(lb, rb - lb + 1);
        pos = rb + 1;
        int np = 0, cov = 0, prec = 0, var = 0;
        if (!json_int(obj, "np", np) || !json_int(obj, "cov_type", cov) || !json_int(obj, "precision", prec) ||
            !json_int(obj, "variant", var))
        {
            err = "tuning cache entry without np, cov_type, precision and variant";
            return -1;
        }
        const int b = bucket_index(np);
        if (!key_ok(b, cov, prec) || var <= 0 || var >= kVariantCount || !solve_variant_valid(np, prec, var))
        {
            err = "tuning cache entry with an invalid key or variant";
            return -1;
        }
        entries.push_back({prec, b, cov, var});
    }
    std::lock_guard<std::mutex> lk(g_ms_mu);
    for (const Entry &e : entries)
    {
        g_table[e.prec][e.b][e.cov].store(e.var, std::memory_order_relaxed);
        g_source[e.prec][e.b][e.cov] = 2;
    }
    return (int)entries.size();
}

int tune_save(const char *path, std::string &err)
{
    static const int nps[kNpBuckets] = {8, 16, 32, 64};
    std::string out = "[\n";
    int n = 0;
    std::lock_guard<std::mutex> lk(g_ms_mu);
    for (int p = 0; p < 2; ++p)
        for (int b = 0; b < kNpBuckets; ++b)
            for (int c = 0; c < kCovTypes; ++c)
            {
                const int v = g_table[p][b][c].load(std::memory_order_relaxed);
                if (v == kVariantDefault) continue;
                char line[512];
                int len = std::snprintf(line, sizeof line,
                                        "%s  {\"np\": %d, \"cov_type\": %d, \"precision\": %d, \"variant\": \"%s\"",
                                        n ? ",\n" : "", nps[b], c, p, kVariantNames[v]);
                std::string entry(line, (size_t)len);
                std::string timings;
                for (int w = 1; w < kVariantCount; ++w)
                    if (g_ms[p][b][c][w] > 0.0)
                    {
                        len = std::snprintf(line, sizeof line, "%s\"%s\": %.4f", timings.empty() ? "" : ", ",
                                            kVariantNames[w], g_ms[p][b][c][w]);
                        timings.append(line, (size_t)len);
                    }
                if (!timings.empty()) entry += ", \"ms_per_million\": {" + timings + "}";
                entry += "}";
                out += entry;
                ++n;
            }
    out += n ? "\n]\n" : "]\n";
    FILE *f = std::fopen(path, "wb");
    if (!f)
    {
        err = std::string("cannot write ") + path;
        return -1;
    }
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    std::fclose(f);
    if (!ok)
    {
        err = std::string("short write to ") + path;
        return -1;
    }
    return n;
}

// Forgets every setting (all keys back to their built-in picks).
void tune_reset()
{
    std::lock_guard<std::mutex> lk(g_ms_mu);
    for (int p = 0; p < 2; ++p)
        for (int b = 0; b < kNpBuckets; ++b)
            for (int c = 0; c < kCovTypes; ++c)
            {
                g_table[p][b][c].store(kVariantDefault, std::memory_order_relaxed);
                g_source[p][b][c] = 0;
                for (int w = 0; w < kVariantCount; ++w) g_ms[p][b][c][w] = 0.0;
            }
}
} // namespace hb
