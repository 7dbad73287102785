// See host_model.h. Built with the host compiler at -O3 without -march,
// -mfma or -ffast-math (plain SSE2 double, no contraction).
#include "host_model.h"

#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>

namespace hb
{
namespace
{
// Host worker threads kept between calls: starting a dozen threads costs more
// than the table work they share. run(n, body) runs body(0) .. body(n-1) at the
// same time, body(0) on the calling thread. One run at a time; a caller that
// finds the workers busy (another thread's run) starts threads of its own. The
// workers are never joined or destroyed (they wait on a condition variable when
// idle), and a forked child starts a set of its own.
class Workers
{
  public:
    static Workers &get()
    {
        static std::mutex guard;
        static Workers *w = nullptr;
        std::lock_guard<std::mutex> lk(guard);
        if (!w || w->pid_ != getpid()) w = new Workers(); // the parent's set stays with the parent
        return *w;
    }
    void run(int n, const std::function<void(int)> &body)
    {
        if (n <= 1)
        {
            body(0);
            return;
        }
        std::unique_lock<std::mutex> mine(busy_, std::try_to_lock);
        if (!mine.owns_lock())
        {
            std::vector<std::thread> th;
            th.reserve(n - 1);
            for (int t = 1; t < n; ++t) th.emplace_back(body, t);
            body(0);
            for (auto &x : th) x.join();
            return;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            for (; started_ < n - 1; ++started_) std::thread(&Workers::loop, this, started_ + 1).detach();
            fn_ = &body;
            n_ = n;
            done_ = 0;
            ++job_;
        }
        wake_.notify_all();
        body(0);
        std::unique_lock<std::mutex> lk(m_);
        finished_.wait(lk, [&] { return done_ == n - 1; });
        fn_ = nullptr;
    }

  private:
    Workers() : pid_(getpid()) {}
    void loop(int w)
    {
        unsigned long seen = 0;
        for (;;)
        {
            const std::function<void(int)> *fn;
            {
                std::unique_lock<std::mutex> lk(m_);
                wake_.wait(lk, [&] { return job_ != seen; });
                seen = job_;
                if (w >= n_) continue;
                fn = fn_;
            }
            (*fn)(w);
            std::lock_guard<std::mutex> lk(m_);
            if (++done_ == n_ - 1) finished_.notify_one();
        }
    }
    pid_t pid_;
    std::mutex busy_, m_;
    std::condition_variable wake_, finished_;
    int started_ = 0, n_ = 0, done_ = 0;
    unsigned long job_ = 0;
    const std::function<void(int)> *fn_ = nullptr;
};

// A team of n host threads running one body (on the workers above). sync() is
// a reusable barrier for the whole team (spin, then yield: the phases between
// barriers are tens of microseconds, so sleeping would cost more than the
// work). Every member must reach every sync() of the body, in the same order,
// and the body must not throw (a member that left would hold the others at
// their next barrier): it allocates nothing.
class Team
{
  public:
    explicit Team(int n) : n_(n) {}
    int size() const { return n_; }
    void run(const std::function<void(int)> &body) { Workers::get().run(n_, body); }
    void sync()
    {
        const unsigned g = gen_.load(std::memory_order_acquire);
        if (count_.fetch_add(1, std::memory_order_acq_rel) == n_ - 1)
        {
            count_.store(0, std::memory_order_relaxed);
            gen_.store(g + 1, std::memory_order_release);
            return;
        }
        for (int spin = 0; gen_.load(std::memory_order_acquire) == g; ++spin)
            if (spin >= 512) std::this_thread::yield();
    }

  private:
    int n_;
    std::atomic<int> count_{0};
    std::atomic<unsigned> gen_{0};
};

// [lo, hi) of n items for member t of a team of nt
inline void share(long n, int t, int nt, long &lo, long &hi)
{
    lo = n * t / nt;
    hi = n * (t + 1) / nt;
}

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
} // namespace

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

// Keys a sorting member takes at least (a member more costs a barrier wait and
// a pass over its bucket counts), and the buckets of the pass that orders them.
constexpr long kMinSortPiece = 2048;
constexpr int kKeyBucketBits = 13;
constexpr int kKeyBuckets = 1 << kKeyBucketBits;

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
    kt.h2_lo.clear();
    kt.h2_hi.clear();
    const double thr = f.threshold();
    // The block is symmetric: index total-1-i holds -d, and cov(-d) equals
    // cov(d) bit for bit (negating v negates every product and partial sum of
    // T v exactly under round-to-nearest, so the squares are the same). The
    // first half and the centre are evaluated and ranked; the mirrors take
    // their values and ranks.
    const long n_half = (total - 1) / 2 + 1; // total is odd: the first half and the centre
    // Dense descending ranks of the kept values. A positive double's bit
    // pattern orders like its value, so the kept (pattern, index) pairs are
    // ordered by pattern: one bucket pass on the pattern's offset from the
    // smallest (its top 13 significant bits), then a sort inside each bucket.
    // Equal patterns may land in any order (they share a rank). The ranks are
    // then counted walking down from the top, and each rank's h2 range is taken
    // from its run of entries on the way.
    struct KI
    {
        uint64_t key;
        uint32_t idx;
    };
    struct Edge // a rank's h2 range over the entries at one end of a member's piece
    {
        long rank = -1;
        double lo = 0, hi = 0;
    };
    std::unique_ptr<KI[]> buf_a(new KI[n_half]), buf_b(new KI[n_half]);
    Team team(clamp_threads(n_threads));
    const int nt = team.size();
    std::vector<long> per(nt);                             // kept entries, then key changes, per member
    std::vector<uint64_t> kmin(nt), kmax(nt);              // pattern range per member
    std::vector<uint32_t *> hist(nt);                      // bucket counts, then scatter offsets, per member
    std::vector<uint32_t> bstart(kKeyBuckets + 1);        // bucket starts in the scattered list
    std::vector<uint32_t> part(nt);                        // keys per member's bucket range
    std::vector<Edge> edges(2 * (size_t)nt);
    kt.h2_lo.reserve(n_half); // at most one rank per kept entry: sized in the body without allocating
    kt.h2_hi.reserve(n_half);
    long n_kept = 0, n_changes = 0;
    team.run([&](int t) {
        uint32_t own_hist[kKeyBuckets], acc[kKeyBuckets];
        hist[t] = own_hist;
        // 1. values of this member's piece of the first half, and their mirrors
        long lo, hi;
        share(n_half, t, nt, lo, hi);
        int ix = (int)(lo % kt.n[0]), iy = (int)(lo / kt.n[0] % kt.n[1]), iz = (int)(lo / kt.n[0] / kt.n[1]);
        long kept = 0;
        for (long i = lo; i < hi; ++i)
        {
            const double v = f.at_offset(ix - kt.half[0], iy - kt.half[1], iz - kt.half[2]);
            kt.vals[i] = v;
            kt.vals[total - 1 - i] = v;
            kept += v > thr;
            if (++ix == kt.n[0])
            {
                ix = 0;
                if (++iy == kt.n[1])
                {
                    iy = 0;
                    ++iz;
                }
            }
        }
        per[t] = kept;
        team.sync();
        // 2. the kept pairs in index order, and the range of their patterns
        long pos = 0, m = 0;
        for (int s = 0; s < nt; ++s)
        {
            if (s < t) pos += per[s];
            m += per[s];
        }
        uint64_t mn = ~0ull, mx = 0;
        for (long i = lo; i < hi; ++i)
            if (kt.vals[i] > thr)
            {
                uint64_t bits;
                std::memcpy(&bits, &kt.vals[i], 8);
                buf_a[pos++] = {bits, (uint32_t)i};
                mn = std::min(mn, bits);
                mx = std::max(mx, bits);
            }
        kmin[t] = mn;
        kmax[t] = mx;
        team.sync();
        // 3. bucket pass over contiguous pieces, one per sorting member
        const int ns = (int)std::max(1L, std::min((long)nt, m / kMinSortPiece));
        const bool sorter = t < ns;
        long slo = 0, shi = 0, b0 = 0, b1 = 0;
        if (sorter)
        {
            share(m, t, ns, slo, shi);
            share(kKeyBuckets, t, ns, b0, b1);
        }
        for (int s = 0; s < nt; ++s)
        {
            mn = std::min(mn, kmin[s]);
            mx = std::max(mx, kmax[s]);
        }
        if (m == 0) mn = mx = 0;
        int width = 0; // significant bits of the largest offset
        while (width < 64 && ((mx - mn) >> width) != 0) ++width;
        const int shift = std::max(0, width - kKeyBucketBits);
        uint32_t *h = own_hist;
        if (sorter)
        {
            std::fill(h, h + kKeyBuckets, 0u);
            for (long j = slo; j < shi; ++j) ++h[(buf_a[j].key - mn) >> shift];
        }
        team.sync();
        // offsets: each member turns its range of buckets into running counts over
        // the pieces (bucket b of piece s starts after the earlier pieces' keys of
        // b), then adds the keys of all smaller buckets
        if (sorter)
        {
            std::fill(acc + b0, acc + b1, 0u);
            for (int s = 0; s < ns; ++s)
            {
                uint32_t *row = hist[s];
                for (long d = b0; d < b1; ++d)
                {
                    const uint32_t c = row[d];
                    row[d] = acc[d];
                    acc[d] += c;
                }
            }
            uint32_t sum = 0;
            for (long d = b0; d < b1; ++d) sum += acc[d];
            part[t] = sum;
        }
        team.sync();
        if (sorter)
        {
            uint32_t base = 0;
            for (int s = 0; s < t; ++s) base += part[s];
            for (long d = b0; d < b1; ++d)
            {
                bstart[d] = base;
                for (int s = 0; s < ns; ++s) hist[s][d] += base;
                base += acc[d];
            }
            if (t == ns - 1) bstart[kKeyBuckets] = base;
        }
        team.sync();
        if (sorter)
            for (long j = slo; j < shi; ++j)
            {
                const KI e = buf_a[j];
                buf_b[h[(e.key - mn) >> shift]++] = e;
            }
        team.sync();
        // 4. each sorting member orders its range of buckets
        KI *const sorted = buf_b.get();
        for (long d = b0; d < b1; ++d)
        {
            KI *first = sorted + bstart[d], *last = sorted + bstart[d + 1];
            if (last - first > 1) std::sort(first, last, [](const KI &x, const KI &y) { return x.key < y.key; });
        }
        team.sync();
        // 5. rank(j) = key changes between positions j and the top; each sorting
        // member counts the changes in its piece, then walks it down starting
        // from the changes above it
        long changes = 0;
        for (long j = slo; j < shi; ++j) changes += j + 1 < m && sorted[j].key != sorted[j + 1].key;
        per[t] = changes;
        team.sync();
        if (t == 0)
        {
            n_kept = m;
            for (int s = 0; s < ns; ++s) n_changes += per[s];
            if (m)
            {
                kt.h2_lo.assign(n_changes + 1, 1e308);
                kt.h2_hi.assign(n_changes + 1, -1.0);
            }
        }
        team.sync();
        // the walk: ranks and mirrors, and per rank the h2 range of its run of
        // entries; the runs at the two ends of the piece can continue into the
        // neighbouring pieces and are merged afterwards
        uint32_t r = 0;
        for (int s = t + 1; s < ns; ++s) r += (uint32_t)per[s];
        Edge run, &top = edges[2 * t], &bottom = edges[2 * t + 1];
        top.rank = bottom.rank = -1;
        for (long j = shi; j-- > slo;)
        {
            if (j + 1 < m && sorted[j].key != sorted[j + 1].key) ++r;
            const uint32_t idx = sorted[j].idx;
            kt.rank[idx] = r;
            kt.rank[total - 1 - idx] = r;
            const long q = idx / kt.n[0];
            const double h2 = offset_h2(f, (int)(idx - q * kt.n[0]) - kt.half[0], (int)(q % kt.n[1]) - kt.half[1],
                                        (int)(q / kt.n[1]) - kt.half[2]);
            if (run.rank != (long)r)
            {
                if (run.rank >= 0)
                {
                    if (top.rank < 0)
                        top = run;
                    else
                        kt.h2_lo[run.rank] = run.lo, kt.h2_hi[run.rank] = run.hi;
                }
                run.rank = r;
                run.lo = run.hi = h2;
            }
            run.lo = std::min(run.lo, h2);
            run.hi = std::max(run.hi, h2);
        }
        bottom = run;
        team.sync();
        if (t == 0)
            for (const Edge &e : edges)
                if (e.rank >= 0)
                {
                    kt.h2_lo[e.rank] = std::min(kt.h2_lo[e.rank], e.lo);
                    kt.h2_hi[e.rank] = std::max(kt.h2_hi[e.rank], e.hi);
                }
    });
    kt.n_ranks = n_kept ? (uint32_t)n_changes + 1 : 0;
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
    // mathematically can differ in the last bit and still share a covariance):
    // gathered by build_key_table for its ranks, else (ranks assigned since,
    // not symmetric in general) taken over the whole block
    std::vector<double> lo, hi;
    if (kt.h2_lo.size() == kt.n_ranks && kt.h2_hi.size() == kt.n_ranks)
    {
        lo = kt.h2_lo;
        hi = kt.h2_hi;
    }
    else
    {
        lo.assign(kt.n_ranks, 1e308);
        hi.assign(kt.n_ranks, -1.0);
        for (int iz = 0; iz < kt.n[2]; ++iz)
            for (int iy = 0; iy < kt.n[1]; ++iy)
                for (int ix = 0; ix < kt.n[0]; ++ix)
                {
                    const uint32_t rk = kt.rank[((long)iz * kt.n[1] + iy) * kt.n[0] + ix];
                    if (rk == KEY_EXCLUDED) continue;
                    const double acc = offset_h2(f, ix - kt.half[0], iy - kt.half[1], iz - kt.half[2]);
                    lo[rk] = std::min(lo[rk], acc);
                    hi[rk] = std::max(hi[rk], acc);
                }
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
