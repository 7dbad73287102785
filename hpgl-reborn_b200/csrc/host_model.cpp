// See host_model.h. Built with the host compiler at -O3 without -march,
// -mfma or -ffast-math (plain SSE2 double, no contraction).
#include "host_model.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

namespace hb
{
static double deg2rad(double deg) { return (deg * 3.14159265358979323846264338327950288419) / 180; }

// c = a * b for 3x3 row-major, summing k ascending from 0 (tnt_cmat.h:525-538)
static void mul3(const double *a, const double *b, double *c)
{
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k)
        {
            double s = 0;
            for (int j = 0; j < 3; ++j) s += a[3 * i + j] * b[3 * j + k];
            c[3 * i + k] = s;
        }
}

bool make_transform(const double *ranges, const double *angles, double *T)
{
    for (int i = 0; i < 3; ++i)
        if (ranges[i] == 0) return false;
    double S[9] = {0}, Z[9] = {0}, Y[9] = {0}, X[9] = {0};
    S[0] = 1.0;
    S[4] = ranges[0] / ranges[1];
    S[8] = ranges[0] / ranges[2];
    const double a0 = deg2rad(angles[0]), a1 = deg2rad(angles[1]), a2 = deg2rad(angles[2]);
    Z[0] = cos(a0); Z[4] = cos(a0); Z[1] = sin(a0); Z[3] = -sin(a0); Z[8] = 1;
    Y[0] = cos(a1); Y[8] = cos(a1); Y[2] = -sin(a1); Y[6] = sin(a1); Y[4] = 1;
    X[4] = cos(a2); X[8] = cos(a2); X[5] = sin(a2); X[7] = -sin(a2); X[0] = 1;
    double xy[9], xyz[9];
    mul3(X, Y, xy);
    mul3(xy, Z, xyz);
    mul3(S, xyz, T);
    return true;
}

double CovModel::h_of(double v0, double v1, double v2) const
{
    double acc = 0.0;
    for (int i = 0; i < 3; ++i)
    {
        double d = 0.0;
        d += v0 * T[3 * i + 0];
        d += v1 * T[3 * i + 1];
        d += v2 * T[3 * i + 2];
        acc += d * d;
    }
    return sqrt(acc);
}

double CovModel::of_h(double h) const
{
    const double r0 = ranges[0];
    if (h < 0.0001) return sill;
    switch (type)
    {
    case COV_GAUSSIAN:
        return (sill - nugget) * exp(-3 * pow(h / r0, 2));
    case COV_EXPONENTIAL:
        return (sill - nugget) * exp(-3 * h / r0);
    default:
        if (h > r0) return 0;
        return (sill - nugget) * (1 - 1.5 * h / r0 + 0.5 * pow(h / r0, 3));
    }
}

bool make_model(int type, const double *ranges, const double *angles, double sill, double nugget,
                CovModel &m, std::string &err)
{
    if (type < 0 || type > 2)
    {
        err = "unknown covariance type " + std::to_string(type);
        return false;
    }
    m.type = type;
    for (int i = 0; i < 3; ++i)
    {
        m.ranges[i] = ranges[i];
        m.angles[i] = angles[i];
    }
    m.sill = sill;
    m.nugget = nugget;
    if (!make_transform(ranges, angles, m.T))
    {
        err = "create_transform: All covariance ranges should be non-zero";
        return false;
    }
    return true;
}

double Flavour::at_offset(int dx, int dy, int dz) const
{
    if (truncated)
    {
        // precalculated_covariance.h:249-264: the table entry of offset
        // c2 - c1 = d, built as cov((0,0,0), d) from doubles (v = 0 - d)
        if (dx < -r[0] || dx > r[0] || dy < -r[1] || dy > r[1] || dz < -r[2] || dz > r[2]) return 0;
        return m.of_h(m.h_of(0.0 - (double)dx, 0.0 - (double)dy, 0.0 - (double)dz));
    }
    // cov_model_t on integer points: v = center - (center + d) in int
    return m.of_h(m.h_of((double)(0 - dx), (double)(0 - dy), (double)(0 - dz)));
}

std::vector<Offset> build_template(const Flavour &f)
{
    struct Ent
    {
        Offset o;
        double key;
    };
    std::vector<Ent> v;
    const double thr = f.threshold();
    for (int z = -f.r[2]; z <= f.r[2]; ++z)
        for (int y = -f.r[1]; y <= f.r[1]; ++y)
            for (int x = -f.r[0]; x <= f.r[0]; ++x)
            {
                if (f.at_offset(x, y, z) > thr)
                {
                    Offset o = {0 - x, 0 - y, 0 - z};
                    v.push_back({o, f.at_offset(o.dx, o.dy, o.dz)});
                }
            }
    // covariance descending, libstdc++ std::sort as in covariance_field.h:359
    std::sort(v.begin(), v.end(), [](const Ent &a, const Ent &b) { return a.key > b.key; });
    std::vector<Offset> out;
    out.reserve(v.size());
    for (const Ent &e : v) out.push_back(e.o);
    return out;
}

std::vector<Offset> build_template(const Flavour &f, const KeyTable &kt)
{
    // the same sequence of (offset, key) as build_template(f), read from the key
    // table (the +-r box lies inside the key block, and kt.vals holds at_offset)
    struct Ent
    {
        Offset o;
        double key;
    };
    auto val = [&](int dx, int dy, int dz) {
        return kt.vals[((long)(dz + kt.half[2]) * kt.n[1] + (dy + kt.half[1])) * kt.n[0] + (dx + kt.half[0])];
    };
    std::vector<Ent> v;
    const double thr = f.threshold();
    for (int z = -f.r[2]; z <= f.r[2]; ++z)
        for (int y = -f.r[1]; y <= f.r[1]; ++y)
            for (int x = -f.r[0]; x <= f.r[0]; ++x)
            {
                if (val(x, y, z) > thr)
                {
                    Offset o = {0 - x, 0 - y, 0 - z};
                    v.push_back({o, val(o.dx, o.dy, o.dz)});
                }
            }
    std::sort(v.begin(), v.end(), [](const Ent &a, const Ent &b) { return a.key > b.key; });
    std::vector<Offset> out;
    out.reserve(v.size());
    for (const Ent &e : v) out.push_back(e.o);
    return out;
}

int clamp_threads(int n)
{
    int hw = (int)std::thread::hardware_concurrency();
    if (hw <= 0) hw = 1;
    if (n <= 0) n = hw;
    return std::min(n, 64);
}

void build_key_table(const Flavour &f, KeyTable &kt, int n_threads)
{
    for (int a = 0; a < 3; ++a)
    {
        kt.half[a] = 2 * f.r[a] - 1;
        kt.n[a] = 2 * kt.half[a] + 1;
    }
    const long total = (long)kt.n[0] * kt.n[1] * kt.n[2];
    kt.vals.assign(total, 0.0);
    kt.rank.assign(total, KEY_EXCLUDED);
    const double thr = f.threshold();
    const int nt = clamp_threads(n_threads);
    const int nz = kt.n[2];
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t]() {
            for (int iz = t; iz < nz; iz += nt)
                for (int iy = 0; iy < kt.n[1]; ++iy)
                    for (int ix = 0; ix < kt.n[0]; ++ix)
                    {
                        long i = ((long)iz * kt.n[1] + iy) * kt.n[0] + ix;
                        kt.vals[i] = f.at_offset(ix - kt.half[0], iy - kt.half[1], iz - kt.half[2]);
                    }
        });
    for (auto &th : pool) th.join();
    // dense descending ranks of the kept values. The kept (value, index) pairs
    // are sorted by the value's bit pattern, which orders positive doubles like
    // their values (least-significant-digit radix sort, 11-bit digits, digits
    // that every key shares skipped), then ranked walking down from the top.
    // The block is symmetric (index total-1-i holds -d) and so are the values
    // (cov(-d) is formed from the same squares as cov(d)), so the first half and
    // the centre are ranked and the mirrors take their ranks.
    struct KI
    {
        uint64_t key;
        uint32_t idx;
    };
    std::vector<KI> a, b;
    a.reserve(total / 8 + 1);
    const long half = (total - 1) / 2; // the centre's index
    bool symmetric = true;
    for (long i = 0; i <= half && symmetric; ++i) symmetric = kt.vals[i] == kt.vals[total - 1 - i];
    const long last = symmetric ? half : total - 1;
    for (long i = 0; i <= last; ++i)
        if (kt.vals[i] > thr)
        {
            uint64_t bits;
            std::memcpy(&bits, &kt.vals[i], 8);
            a.push_back({bits, (uint32_t)i});
        }
    b.resize(a.size());
    for (int shift = 0; shift < 64; shift += 11)
    {
        size_t cnt[2048] = {0};
        for (const KI &e : a) ++cnt[(e.key >> shift) & 2047];
        if (!a.empty() && cnt[(a[0].key >> shift) & 2047] == a.size()) continue; // one digit value: order kept
        size_t pos = 0;
        for (int d = 0; d < 2048; ++d)
        {
            const size_t c = cnt[d];
            cnt[d] = pos;
            pos += c;
        }
        for (const KI &e : a) b[cnt[(e.key >> shift) & 2047]++] = e;
        a.swap(b);
    }
    uint32_t r = 0;
    for (size_t j = a.size(); j-- > 0;)
    {
        if (j + 1 < a.size() && a[j].key != a[j + 1].key) ++r;
        kt.rank[a[j].idx] = r;
        if (symmetric) kt.rank[total - 1 - a[j].idx] = r;
    }
    kt.n_ranks = a.empty() ? 0 : r + 1;
}

long template_size(const Flavour &f, const KeyTable &kt)
{
    const double thr = f.threshold();
    long n = 0;
    for (int z = -f.r[2]; z <= f.r[2]; ++z)
        for (int y = -f.r[1]; y <= f.r[1]; ++y)
        {
            const double *row = &kt.vals[((long)(z + kt.half[2]) * kt.n[1] + (y + kt.half[1])) * kt.n[0] + kt.half[0]];
            for (int x = -f.r[0]; x <= f.r[0]; ++x) n += row[x] > thr;
        }
    return n;
}

namespace
{
// h2 = ||T v||^2 in double, v the negated offset (as the key block stores it)
double offset_h2(const Flavour &f, int dx, int dy, int dz)
{
    const double v[3] = {(double)(0 - dx), (double)(0 - dy), (double)(0 - dz)};
    double acc = 0.0;
    for (int r = 0; r < 3; ++r)
    {
        double d = 0.0;
        d += v[0] * f.m.T[3 * r + 0];
        d += v[1] * f.m.T[3 * r + 1];
        d += v[2] * f.m.T[3 * r + 2];
        acc += d * d;
    }
    return acc;
}

// The bounds of the float evaluation, which do not depend on the keys.
void surrogate_geometry(const Flavour &f, Surrogate &sg)
{
    // A transformed coordinate is formed in float as fma(T2, z, fma(T1, y, T0 * x))
    // for the cell and for the candidate, both relative to the bin corner, then
    // subtracted: with |T' - T| <= u |T| and four roundings, each component is off
    // by at most 5.02 u sum_j |T_ij| (|p_j| + |c_j|), where |p_j| <= 2 r_j and
    // |c_j| < r_j. 16 u sum_j |T_ij| r_j bounds that with room to spare.
    const double u = 1.0 / 16777216.0;
    double E = 0.0;
    for (int r = 0; r < 3; ++r)
    {
        double s = 0.0;
        for (int c = 0; c < 3; ++c) s += std::fabs(f.m.T[3 * r + c]) * (double)f.r[c];
        E = std::max(E, 16.0 * u * s);
    }
    sg.e3 = 1.7320508075688774 * E + 1e-30;
    for (int a = 0; a < 3; ++a)
    {
        double s = 0.0;
        for (int r = 0; r < 3; ++r) s += f.m.T[3 * r + a] * f.m.T[3 * r + a];
        sg.step[a] = (float)(std::sqrt(s) * (1.0 + 1e-6));
    }
}
} // namespace

void build_surrogate(const Flavour &f, const KeyTable &kt, Surrogate &sg, bool running_max)
{
    sg.ok = false;
    sg.h2_rank.clear();
    for (int i = 0; i < 9; ++i) sg.T[i] = (float)f.m.T[i];
    if (kt.n_ranks == 0) return;
    // per rank the smallest and largest h2 carrying it (offsets whose h2 agree
    // mathematically can differ in the last bit and still share a covariance)
    std::vector<double> lo(kt.n_ranks, 1e308), hi(kt.n_ranks, -1.0);
    for (int iz = 0; iz < kt.n[2]; ++iz)
        for (int iy = 0; iy < kt.n[1]; ++iy)
            for (int ix = 0; ix < kt.n[0]; ++ix)
            {
                const long i = ((long)iz * kt.n[1] + iy) * kt.n[0] + ix;
                const uint32_t rk = kt.rank[i];
                if (rk == KEY_EXCLUDED) continue;
                const double acc = offset_h2(f, ix - kt.half[0], iy - kt.half[1], iz - kt.half[2]);
                lo[rk] = std::min(lo[rk], acc);
                hi[rk] = std::max(hi[rk], acc);
            }
    if (running_max)
    {
        for (uint32_t r = 1; r < kt.n_ranks; ++r) hi[r] = std::max(hi[r], hi[r - 1]);
    }
    else
    {
        // ranks increase with h2: every h2 of rank r lies below every h2 of rank r + 1
        for (uint32_t r = 0; r + 1 < kt.n_ranks; ++r)
            if (!(hi[r] < lo[r + 1])) return;
    }
    sg.h2_rank = hi;
    sg.h2_cut = hi[kt.n_ranks - 1];
    surrogate_geometry(f, sg);
    sg.ok = true;
}

void build_surrogate_template(const Flavour &f, const std::vector<Offset> &tmpl, Surrogate &sg)
{
    sg.ok = false;
    sg.h2_rank.clear();
    for (int i = 0; i < 9; ++i) sg.T[i] = (float)f.m.T[i];
    if (tmpl.empty()) return;
    sg.h2_rank.resize(tmpl.size());
    double run = -1.0;
    for (size_t i = 0; i < tmpl.size(); ++i)
    {
        run = std::max(run, offset_h2(f, tmpl[i].dx, tmpl[i].dy, tmpl[i].dz));
        sg.h2_rank[i] = run;
    }
    sg.h2_cut = run;
    surrogate_geometry(f, sg);
    sg.ok = true;
}
} // namespace hb
