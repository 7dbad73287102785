// TEST INFRASTRUCTURE ONLY — the oracle. Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load this library, and only as the
// checker; the product path never calls it.
//
// A CPU restatement, in this project's own code, of the reference's kriging
// path (itohnobue/hpgl-reborn, src/geo_bsd/hpgl/). Each function cites the
// reference lines it follows. Parity of this restatement is pinned against
// the reference itself (oracle/_ref/libref_harness.so, built from the
// reference sources by oracle/Makefile) through tests/golden/ fixtures.
//
// Arithmetic is plain IEEE double without contraction (compiled without
// -march/-mfma/-ffast-math), the same as the reference build, so covariance
// values and neighbour ordering keys are bit-identical; orderings use the same
// libstdc++ std::sort the reference uses. The Cholesky solver is this file's
// own (the reference calls LAPACK dpotrf/dpotrs), so weights agree to
// rounding, not bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>
#include <omp.h>

#include "../hpgl-reborn_b200/csrc/gnu_introsort.h"

namespace ko
{
// ---------------------------------------------------------------- covariance
// cov_model.h:9-14
static double deg2rad(double deg) { return (deg * 3.14159265358979323846264338327950288419) / 180; }

// 3x3 product with the accumulation order of TNT's matmult (tnt_cmat.h:525-538):
// c[i][k] = ((0 + a[i][0]*b[0][k]) + a[i][1]*b[1][k]) + a[i][2]*b[2][k]
static void mat3_mul(const double *a, const double *b, double *c)
{
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k)
        {
            double s = 0;
            for (int j = 0; j < 3; ++j) s += a[3 * i + j] * b[3 * j + k];
            c[3 * i + k] = s;
        }
}

// T = S * ((Rx * Ry) * Rz), cov_model.h:16-61. Returns false on a zero range.
static bool make_transform(const double *ranges, const double *angles, double *T)
{
    for (int i = 0; i < 3; ++i)
        if (ranges[i] == 0) return false;
    double S[9] = {0}, Rz[9] = {0}, Ry[9] = {0}, Rx[9] = {0};
    S[0] = 1.0;
    S[4] = ranges[0] / ranges[1];
    S[8] = ranges[0] / ranges[2];
    Rz[0] = cos(deg2rad(angles[0]));
    Rz[4] = cos(deg2rad(angles[0]));
    Rz[1] = sin(deg2rad(angles[0]));
    Rz[3] = -sin(deg2rad(angles[0]));
    Rz[8] = 1;
    Ry[0] = cos(deg2rad(angles[1]));
    Ry[8] = cos(deg2rad(angles[1]));
    Ry[2] = -sin(deg2rad(angles[1]));
    Ry[6] = sin(deg2rad(angles[1]));
    Ry[4] = 1;
    Rx[4] = cos(deg2rad(angles[2]));
    Rx[8] = cos(deg2rad(angles[2]));
    Rx[5] = sin(deg2rad(angles[2]));
    Rx[7] = -sin(deg2rad(angles[2]));
    Rx[0] = 1;
    double xy[9], xyz[9];
    mat3_mul(Rx, Ry, xy);
    mat3_mul(xy, Rz, xyz);
    mat3_mul(S, xyz, T);
    return true;
}

struct Model
{
    int type; // 0 spherical, 1 exponential, 2 gaussian (covariance_type.h:6)
    double r0, sill, nugget;
    double T[9];

    // transfrom_and_norm, cov_model.h:63-77
    double h_of(double v0, double v1, double v2) const
    {
        double r = 0.0;
        for (int i = 0; i < 3; ++i)
        {
            double d = 0.0;
            d += v0 * T[3 * i + 0];
            d += v1 * T[3 * i + 1];
            d += v2 * T[3 * i + 2];
            r += d * d;
        }
        return sqrt(r);
    }
    // cov_model.h:146-183 (same expression shapes, so the same roundings)
    double of_h(double h) const
    {
        if (h < 0.0001) return sill;
        if (type == 2) return (sill - nugget) * exp(-3 * pow(h / r0, 2));
        if (type == 1) return (sill - nugget) * exp(-3 * h / r0);
        if (h > r0) return 0;
        return (sill - nugget) * (1 - 1.5 * h / r0 + 0.5 * pow(h / r0, 3));
    }
    // cov_model_t::operator()(c1, c2) on integer points: v = c1 - c2 in int, then double
    double at_int(int ax, int ay, int az, int bx, int by, int bz) const
    {
        return of_h(h_of((double)(ax - bx), (double)(ay - by), (double)(az - bz)));
    }
};

// A covariance "flavour" as the drivers instantiate it.
//  analytic  (OK, ordinary_kriging.cpp:29-33): cov_model_t on the two points;
//  truncated (SK / IK / median IK: precalculated_covariance.h:30-60,
//             covariance_field.h:108-169): the model on the integer offset
//             when it lies inside the +-radius box, else 0.
struct Flavour
{
    Model m;
    bool truncated;
    int rx, ry, rz;
    double at(int ax, int ay, int az, int bx, int by, int bz) const
    {
        if (truncated)
        {
            int dx = bx - ax, dy = by - ay, dz = bz - az;
            if (dx < -rx || dx > rx || dy < -ry || dy > ry || dz < -rz || dz > rz) return 0;
            // table entry for offset o holds cov((0,0,0), o) computed from doubles:
            // v = 0 - o (precalculated_covariance.h:240-243)
            return m.of_h(m.h_of(0.0 - (double)dx, 0.0 - (double)dy, 0.0 - (double)dz));
        }
        return m.at_int(ax, ay, az, bx, by, bz);
    }
};

static bool make_flavour(Flavour &f, bool truncated, int cov_type, const double *ranges,
                         const double *angles, double sill, double nugget, const int *radiuses)
{
    if (cov_type < 0 || cov_type > 2) return false;
    f.truncated = truncated;
    f.m.type = cov_type;
    f.m.r0 = ranges[0];
    f.m.sill = sill;
    f.m.nugget = nugget;
    f.rx = radiuses[0];
    f.ry = radiuses[1];
    f.rz = radiuses[2];
    return make_transform(ranges, angles, f.m.T);
}

// ---------------------------------------------------------------- grid
struct Grid
{
    int nx, ny, nz;
    long size() const { return (long)nx * ny * nz; }
    // sugarbox_grid.cpp:70-74
    void coord(int idx, int &x, int &y, int &z) const
    {
        x = idx % nx;
        y = idx % (nx * ny) / nx;
        z = idx / (nx * ny);
    }
    // sugarbox_grid.h:40-58 (out of grid -> -1)
    int index(int x, int y, int z) const
    {
        if ((unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz)
            return z * nx * ny + y * nx + x;
        return -1;
    }
};

// ---------------------------------------------------------------- search
struct Off
{
    int dx, dy, dz;
};

// calc_cov_field, covariance_field.h:62-106: offsets -(x,y,z) over the box in
// z,y,x ascending order whose covariance exceeds C(0)/100, sorted by
// covariance descending with std::sort (unstable).
static std::vector<Off> build_template(const Flavour &f)
{
    struct Ent
    {
        Off o;
        double key;
    };
    std::vector<Ent> v;
    double thr = f.at(0, 0, 0, 0, 0, 0) / 100;
    for (int z = -f.rz; z <= f.rz; ++z)
        for (int y = -f.ry; y <= f.ry; ++y)
            for (int x = -f.rx; x <= f.rx; ++x)
            {
                double c = f.at(0, 0, 0, x, y, z);
                if (c > thr)
                {
                    Off o = {0 - x, 0 - y, 0 - z};
                    // the sort key is the value stored for the offset itself
                    v.push_back({o, f.at(0, 0, 0, o.dx, o.dy, o.dz)});
                }
            }
    std::sort(v.begin(), v.end(), [](const Ent &a, const Ent &b) { return a.key > b.key; });
    std::vector<Off> out;
    out.reserve(v.size());
    for (auto &e : v)
    {
        if (e.key < thr) break; // second cut, covariance_field.h:93-103 (never triggers)
        out.push_back(e.o);
    }
    return out;
}

// clusterizer.cpp:74-188: bins of size radius, (g / r + 2) per axis; a bin keeps
// its first `limit` nodes (ascending node order) and is marked exceeded on the
// next one.
struct Bins
{
    int bx, by, bz, rx, ry, rz;
    size_t limit;
    std::vector<std::vector<int>> nodes;
    std::vector<char> exceeded;

    void init(const Grid &g, int rx_, int ry_, int rz_, size_t limit_)
    {
        rx = rx_;
        ry = ry_;
        rz = rz_;
        limit = limit_;
        bx = (int)(g.nx / (double)rx + 2);
        by = (int)(g.ny / (double)ry + 2);
        bz = (int)(g.nz / (double)rz + 2);
        nodes.assign((size_t)bx * by * bz, std::vector<int>());
        exceeded.assign((size_t)bx * by * bz, 0);
    }
    int bin_index(int cx, int cy, int cz) const
    {
        if (cx < 0 || cx > bx || cy < 0 || cy > by || cz < 0 || cz > bz) return -1;
        return cz * bx * by + cy * bx + cx;
    }
    void add(int node, int x, int y, int z)
    {
        int b = bin_index(x / rx, y / ry, z / rz);
        if (exceeded[b]) return;
        if (nodes[b].size() >= limit)
        {
            exceeded[b] = 1;
            nodes[b].clear();
            return;
        }
        nodes[b].push_back(node);
    }
    bool any_exceeded(int x, int y, int z) const
    {
        int cx = x / rx, cy = y / ry, cz = z / rz;
        for (int k = cz - 1; k <= cz + 1; ++k)
            for (int j = cy - 1; j <= cy + 1; ++j)
                for (int i = cx - 1; i <= cx + 1; ++i)
                {
                    int b = bin_index(i, j, k);
                    if (b >= 0 && exceeded[b]) return true;
                }
        return false;
    }
    void candidates(int x, int y, int z, std::vector<int> &out) const
    {
        out.clear();
        int cx = x / rx, cy = y / ry, cz = z / rz;
        for (int k = cz - 1; k <= cz + 1; ++k)
            for (int j = cy - 1; j <= cy + 1; ++j)
                for (int i = cx - 1; i <= cx + 1; ++i)
                {
                    int b = bin_index(i, j, k);
                    if (b >= 0) out.insert(out.end(), nodes[b].begin(), nodes[b].end());
                }
    }
};

struct Search
{
    Grid g;
    Flavour f;
    int max_nb;
    std::vector<Off> tmpl;
    Bins bins;
    const unsigned char *mask;

    bool informed(int idx) const { return idx >= 0 && idx < g.size() && mask[idx] != 0; }

    // sugarbox_indexed_neighbour_lookup.h:53-64 then add_node for informed nodes
    void init(const Grid &g_, const Flavour &f_, int max_nb_, const unsigned char *mask_)
    {
        g = g_;
        f = f_;
        max_nb = max_nb_;
        mask = mask_;
        tmpl = build_template(f);
        bins.init(g, f.rx, f.ry, f.rz, tmpl.size() / 250);
        for (long n = 0; n < g.size(); ++n)
            if (mask[n])
            {
                int x, y, z;
                g.coord((int)n, x, y, z);
                bins.add((int)n, x, y, z);
            }
    }

    // indexed_neighbour_lookup_t::find, sugarbox_indexed_neighbour_lookup.h:67-124
    // (template path: sugarbox_neighbour_lookup.h:171-197). Returns 1 when the
    // template path ran.
    int find(int node, std::vector<int> &idx) const
    {
        idx.clear();
        int x, y, z;
        g.coord(node, x, y, z);
        if (bins.any_exceeded(x, y, z))
        {
            for (size_t t = 0; t < tmpl.size() && (int)idx.size() < max_nb; ++t)
            {
                int n = g.index(x + tmpl[t].dx, y + tmpl[t].dy, z + tmpl[t].dz);
                if (informed(n)) idx.push_back(n);
            }
            return 1;
        }
        std::vector<int> cand;
        bins.candidates(x, y, z, cand);
        struct Ent
        {
            int index;
            double cov;
        };
        std::vector<Ent> e;
        double thr = f.at(x, y, z, x, y, z) / 100;
        for (int c : cand)
        {
            int cx, cy, cz;
            g.coord(c, cx, cy, cz);
            double v = f.at(x, y, z, cx, cy, cz);
            if (v > thr) e.push_back({c, v});
        }
        std::sort(e.begin(), e.end(), [](const Ent &a, const Ent &b) { return a.cov > b.cov; });
        for (size_t i = 0; i < e.size() && (int)i < max_nb; ++i) idx.push_back(e[i].index);
        return 0;
    }
};

// ---------------------------------------------------------------- solve
// Cholesky A = L L^T of a dense SPD matrix (this file's own algorithm; the
// reference calls LAPACK dpotrf('U')). Fails, as dpotrf does, on a pivot that
// is not > 0 (or is NaN).
template <typename R>
static bool cholesky(std::vector<R> &A, int n)
{
    for (int j = 0; j < n; ++j)
    {
        R d = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        if (!(d > 0)) return false;
        R ljj = std::sqrt(d);
        A[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i)
        {
            R s = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = s / ljj;
        }
    }
    return true;
}

template <typename R>
static void chol_solve(const std::vector<R> &L, int n, std::vector<R> &x)
{
    for (int i = 0; i < n; ++i)
    {
        R s = x[i];
        for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * x[k];
        x[i] = s / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i)
    {
        R s = x[i];
        for (int k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * x[k];
        x[i] = s / L[(size_t)i * n + i];
    }
}

// sk_kriging_weights_3 (my_kriging_weights.h:60-196) when ordinary == false,
// ok_kriging_weights_3 (my_kriging_weights.h:198-361) when true. Weights and
// variance in double; `R` is the precision of the factorisation.
template <typename R>
static bool weights(const Flavour &f, bool ordinary, int cx, int cy, int cz,
                    const std::vector<int> &xs, const std::vector<int> &ys,
                    const std::vector<int> &zs, std::vector<double> &w, double &var)
{
    int n = (int)xs.size();
    if (n <= 0) return false;
    std::vector<R> A((size_t)n * n);
    std::vector<double> b(n);
    for (int i = 0; i < n; ++i)
    {
        for (int j = i; j < n; ++j)
        {
            double c = f.at(xs[i], ys[i], zs[i], xs[j], ys[j], zs[j]);
            A[(size_t)i * n + j] = c;
            A[(size_t)j * n + i] = c;
        }
        b[i] = f.at(xs[i], ys[i], zs[i], cx, cy, cz);
    }
    if (!cholesky(A, n)) return false;
    double cr0 = f.at(cx, cy, cz, cx, cy, cz);
    w.assign(n, 0.0);
    if (!ordinary)
    {
        std::vector<R> x(b.begin(), b.end());
        chol_solve(A, n, x);
        var = cr0;
        for (int i = 0; i < n; ++i)
        {
            w[i] = (double)x[i];
            var -= w[i] * b[i];
        }
        if (var < 0) var = 0;
        return true;
    }
    std::vector<R> x(b.begin(), b.end()), y(n, (R)1);
    chol_solve(A, n, x);
    chol_solve(A, n, y);
    double sum_x = 0, sum_y = 0;
    for (int k = 0; k < n; ++k)
    {
        sum_x += (double)x[k];
        sum_y += (double)y[k];
    }
    if (std::abs(sum_y) < 1e-15) return false;
    double mu = (sum_x - 1) / sum_y;
    for (int k = 0; k < n; ++k) w[k] = (double)x[k] - mu * (double)y[k];
    var = cr0;
    for (int i = 0; i < n; ++i) var -= w[i] * b[i];
    var -= mu;
    if (var < 0) var = 0;
    return true;
}

// ---------------------------------------------------------------- per node
enum
{
    KI_SUCCESS = 0,
    KI_NO_NEIGHBOURS = 1,
    KI_SINGULARITY = 2
};

// kriging_interpolation (kriging_interpolation.h:230-315) + combine
// (combiner.h:10-25). `value_of(i)` gives the neighbour value as the float the
// reference subtracts the (float) mean from. est_d accumulates in double,
// est_f in float exactly as cont_kriging's float result does. `means` (LVM,
// lvm_kriging.cpp:16-39) gives a mean per node instead of the single `mean`.
template <typename R, typename ValueOf>
static int krige_node(const Search &s, bool ordinary, double mean, const float *means, int node,
                      ValueOf value_of, std::vector<int> &idx, int &path, double &est_d, double &var,
                      float &est_f)
{
    path = s.find(node, idx);
    if (idx.empty()) return KI_NO_NEIGHBOURS;
    int n = (int)idx.size();
    std::vector<int> xs(n), ys(n), zs(n);
    for (int i = 0; i < n; ++i) s.g.coord(idx[i], xs[i], ys[i], zs[i]);
    int cx, cy, cz;
    s.g.coord(node, cx, cy, cz);
    std::vector<double> w;
    if (!weights<R>(s.f, ordinary, cx, cy, cz, xs, ys, zs, w, var)) return KI_SINGULARITY;
    float m = means ? means[node] : (float)mean; // mean_t is float (typedefs.h:122)
    est_d = (double)m;
    est_f = m;
    for (int i = 0; i < n; ++i)
    {
        float d = value_of(idx[i]) - (means ? means[idx[i]] : m);
        est_d += w[i] * (double)d;
        est_f += (float)(w[i] * d);
    }
    return KI_SUCCESS;
}

// correct_order_relations (indicator_kriging.h:34-59)
static void order_relations(std::vector<float> &p)
{
    for (auto &v : p)
    {
        if (v < 0.0) v = 0.0f;
        else if (v > 1.0) v = 1.0f;
    }
    for (size_t i = 0; i + 1 < p.size(); ++i)
        if (p[i] > p[i + 1])
        {
            double avg = (p[i] + p[i + 1]) / 2.0;
            p[i] = (float)avg;
            p[i + 1] = (float)avg;
        }
}

// most_probable_category (cdf_utils.cpp:11-27): first maximum wins
static int argmax_first(const std::vector<float> &p)
{
    double best = p[0];
    int k = 0;
    for (size_t i = 1; i < p.size(); ++i)
        if (p[i] > best)
        {
            best = p[i];
            k = (int)i;
        }
    return k;
}

// ---------------------------------------------------------------- SGS
// path_random_generator.cpp:24-67. A linear congruential walk R <- (A R + C)
// mod size over every node, started at seed % size: A = 1 + the product of the
// primes dividing size (doubled when 4 divides size), C = the largest prime not
// above size / 3 that does not divide size (2 when there is none). The primes
// are walked in ascending order as the reference walks its prime table.
struct PathLcg
{
    long long A = 1, C = 2, M = 1, R = 0;
    bool init(long long size, long long seed)
    {
        if (size <= 0 || size > 10000000) return false;
        std::vector<int> primes; // ascending, up to the first prime above size
        {
            long long lim = size + 64;
            std::vector<char> comp((size_t)lim + 1, 0);
            for (long long i = 2; i <= lim; ++i)
            {
                if (comp[(size_t)i]) continue;
                primes.push_back((int)i);
                if (i > size) break;
                for (long long j = i * i; j <= lim; j += i) comp[(size_t)j] = 1;
            }
        }
        M = size;
        A = 1;
        size_t idx = 0;
        for (; idx < primes.size(); ++idx)
        {
            if (primes[idx] > size) break;
            if (size % primes[idx] == 0) A *= primes[idx];
        }
        if (M % 4 == 0) A *= 2;
        A += 1;
        idx = 0;
        while (idx + 1 < primes.size() && primes[idx + 1] <= size / 3) ++idx;
        for (long long k = (long long)idx; k >= 0; --k)
        {
            C = primes[(size_t)k];
            if (std::floor(double(size) / double(C)) != double(size) / double(C)) break;
        }
        R = seed % size;
        return R >= 0;
    }
    int next()
    {
        int r = (int)R;
        R = (A * R + C) % M;
        return r;
    }
};

// gaussian_cdf_t (gaussian_distribution.h): the cumulative distribution by
// Abramowitz & Stegun 26.2.17 and its inverse by the Odeh & Evans rational
// approximation, with the reference's expression shapes and guards.
static double gauss_cdf(double x, double mean, double var)
{
    const double p = 0.2316419;
    const double b[] = {0.319381530, -0.356563782, 1.781477937, -1.821255978, 1.330274429};
    double sx = (x - mean) / sqrt(var);
    bool neg = sx < 0;
    if (neg) sx = -sx;
    double t = 1 / (1 + p * sx);
    double zx = 1 / sqrt(2 * 3.14159265358) * exp(-sx * sx / 2);
    double r = 1 - zx * ((((b[4] * t + b[3]) * t + b[2]) * t + b[1]) * t + b[0]) * t;
    if (neg) r = 1 - r;
    return r;
}

static double gauss_inverse(double pr, double mean, double var)
{
    if (pr <= 0.0 || pr >= 1.0) return mean;
    const double ps[] = {-0.322232431088, -1.0, -0.342242088547, -0.0204231210245, -0.453642210148e-4};
    const double qs[] = {0.0993484626060, 0.588581570495, 0.531103462366, 0.103537752850, 0.38560700634e-2};
    double p2 = pr > 0.5 ? 1 - pr : pr;
    if (p2 < 1e-150) p2 = 1e-150;
    double y = sqrt(log(1 / (p2 * p2)));
    double xp = y + ((((ps[4] * y + ps[3]) * y + ps[2]) * y + ps[1]) * y + ps[0]) /
                        ((((qs[4] * y + qs[3]) * y + qs[2]) * y + qs[1]) * y + qs[0]);
    if (pr < 0.5) xp = -xp;
    return xp * sqrt(var) + mean;
}

// non_parametric_cdf_2_t (non_parametric_cdf.h:189-270): piecewise-linear in
// float between the table's points, clamped at both ends.
struct NpCdf
{
    const float *v = nullptr, *p = nullptr;
    long long n = 0;
    float prob(float x) const
    {
        const float *it = std::lower_bound(v, v + n, x);
        if (it == v + n) return p[n - 1];
        if (it == v) return p[0];
        long long i2 = it - v, i1 = i2 - 1;
        float x1 = v[i1], x2 = v[i2], y1 = p[i1], y2 = p[i2];
        return y1 + (y2 - y1) / (x2 - x1) * (x - x1);
    }
    float inverse(float q) const
    {
        if (n <= 0) return 0;
        const float *it = std::lower_bound(p, p + n, q);
        if (it == p) return v[0];
        if (it == p + n) return v[n - 1];
        long long i2 = it - p, i1 = i2 - 1;
        float x1 = v[i1], x2 = v[i2], y1 = p[i1], y2 = p[i2];
        return x1 + (x2 - x1) / (y2 - y1) * (q - y1);
    }
};

// ---------------------------------------------------------------- cokriging
// gauss_solve (gauss_solver.cpp:8-70): for column i the first unused row with a
// non-zero entry is normalised and subtracted from every other unused row; it
// fails when no row is found or the pivot is below machine epsilon.
static bool gauss_solve_ref(std::vector<double> &A, std::vector<double> &B, std::vector<double> &X, int size)
{
    std::vector<int> flags(size, 0), order(size, 0);
    for (int i = 0; i < size; ++i)
    {
        int row = -1;
        for (int j = 0; j < size; ++j)
            if (flags[j] == 0 && A[(size_t)j * size + i] != 0)
            {
                row = j;
                flags[j] = 1;
                order[i] = j;
                break;
            }
        if (row < 0) return false;
        double coef = A[(size_t)row * size + i];
        if (std::abs(coef) < std::numeric_limits<double>::epsilon()) return false;
        for (int j = i; j < size; ++j) A[(size_t)row * size + j] /= coef;
        B[row] /= coef;
        for (int j = 0; j < size; ++j)
            if (flags[j] == 0)
            {
                double c = A[(size_t)j * size + i];
                for (int k = i; k < size; ++k) A[(size_t)j * size + k] -= c * A[(size_t)row * size + k];
                B[j] -= c * B[row];
            }
    }
    X.assign(size, 0.0);
    for (int i = size - 1; i >= 0; --i)
    {
        int row = order[i];
        X[i] = B[row];
        for (int j = size - 1; j > i; --j) X[i] -= A[(size_t)row * size + j] * X[j];
    }
    return true;
}
} // namespace ko

using namespace ko;

extern "C" {

int ko_transform(const double *ranges, const double *angles, double *out9)
{
    return make_transform(ranges, angles, out9) ? 0 : -1;
}

// kind 0: analytic (OK); kind 1/2: box-truncated (SK, IK, median IK)
double ko_cov(int kind, int cov_type, const double *ranges, const double *angles, double sill,
              double nugget, const int *radiuses, const int *a, const int *b)
{
    Flavour f;
    if (!make_flavour(f, kind != 0, cov_type, ranges, angles, sill, nugget, radiuses)) return NAN;
    return f.at(a[0], a[1], a[2], b[0], b[1], b[2]);
}

int ko_template(int kind, int cov_type, const double *ranges, const double *angles, double sill,
                double nugget, const int *radiuses, int *out, int cap, int *out_limit)
{
    Flavour f;
    if (!make_flavour(f, kind != 0, cov_type, ranges, angles, sill, nugget, radiuses)) return -1;
    std::vector<Off> t = build_template(f);
    for (int i = 0; i < (int)t.size() && i < cap; ++i)
    {
        out[3 * i] = t[i].dx;
        out[3 * i + 1] = t[i].dy;
        out[3 * i + 2] = t[i].dz;
    }
    if (out_limit) *out_limit = (int)(t.size() / 250);
    return (int)t.size();
}

// Per-node kriging at the listed nodes. kind 0 = OK (analytic, ordinary
// system), 1 = SK (truncated, simple system). cont: values from `data`;
// indicator (ind_value >= 0): values are (data_u8 == ind_value). precision 0 =
// double factorisation, 1 = long double (x87 80-bit) for a sharper truth on
// ill-conditioned systems. Any output pointer may be null.
static int krige_nodes(int kind, const int *dims, const float *data_f, const unsigned char *data_u8,
                       int ind_value, const unsigned char *mask, int cov_type,
                       const double *ranges, const double *angles, double sill, double nugget,
                       const int *radiuses, int max_nb, double mean, const float *means,
                       const int *nodes, int n_nodes, int *out_idx, int *out_count,
                       unsigned char *out_path, double *out_est, double *out_var, float *out_est_f,
                       int *out_status, int precision, int n_threads)
{
    Grid g = {dims[0], dims[1], dims[2]};
    Flavour f;
    if (!make_flavour(f, kind != 0, cov_type, ranges, angles, sill, nugget, radiuses)) return -1;
    if (radiuses[0] <= 0 || radiuses[1] <= 0 || radiuses[2] <= 0) return -1;
    Search s;
    s.init(g, f, max_nb, mask);
    bool ordinary = (kind == 0);
    if (ordinary) mean = 0.0; // OK combines with no_mean_t (ordinary_kriging.cpp:31, mean_provider.h:8-15)
    if (ordinary) means = nullptr;
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int t = 0; t < n_nodes; ++t)
    {
        std::vector<int> idx;
        int path = 0;
        double est = 0, var = -1;
        float est_f = 0;
        int st;
        if (data_u8)
        {
            auto vo = [&](int i) -> float { return data_u8[i] == ind_value ? 1.0f : 0.0f; };
            st = precision ? krige_node<long double>(s, ordinary, mean, means, nodes[t], vo, idx, path, est, var, est_f)
                           : krige_node<double>(s, ordinary, mean, means, nodes[t], vo, idx, path, est, var, est_f);
        }
        else
        {
            auto vo = [&](int i) -> float { return data_f[i]; };
            st = precision ? krige_node<long double>(s, ordinary, mean, means, nodes[t], vo, idx, path, est, var, est_f)
                           : krige_node<double>(s, ordinary, mean, means, nodes[t], vo, idx, path, est, var, est_f);
        }
        if (out_idx)
            for (int i = 0; i < max_nb; ++i)
                out_idx[(size_t)t * max_nb + i] = i < (int)idx.size() ? idx[i] : -1;
        if (out_count) out_count[t] = (int)idx.size();
        if (out_path) out_path[t] = (unsigned char)path;
        if (out_est) out_est[t] = est;
        if (out_var) out_var[t] = var;
        if (out_est_f) out_est_f[t] = est_f;
        if (out_status) out_status[t] = st;
    }
    return 0;
}

int ko_krige_cont(int kind, const int *dims, const float *data, const unsigned char *mask,
                  int cov_type, const double *ranges, const double *angles, double sill,
                  double nugget, const int *radiuses, int max_nb, double mean, const int *nodes,
                  int n_nodes, int *out_idx, int *out_count, unsigned char *out_path,
                  double *out_est, double *out_var, float *out_est_f, int *out_status,
                  int precision, int n_threads)
{
    return krige_nodes(kind, dims, data, nullptr, -1, mask, cov_type, ranges, angles, sill, nugget,
                       radiuses, max_nb, mean, nullptr, nodes, n_nodes, out_idx, out_count, out_path,
                       out_est, out_var, out_est_f, out_status, precision, n_threads);
}

// LVM at the listed nodes: the SK flavour with a mean per node (lvm_kriging.cpp:28-34).
int ko_krige_lvm(const int *dims, const float *data, const unsigned char *mask, const float *means,
                 int cov_type, const double *ranges, const double *angles, double sill, double nugget,
                 const int *radiuses, int max_nb, const int *nodes, int n_nodes, int *out_idx,
                 int *out_count, unsigned char *out_path, double *out_est, double *out_var,
                 float *out_est_f, int *out_status, int precision, int n_threads)
{
    return krige_nodes(1, dims, data, nullptr, -1, mask, cov_type, ranges, angles, sill, nugget, radiuses,
                       max_nb, 0.0, means, nodes, n_nodes, out_idx, out_count, out_path, out_est, out_var,
                       out_est_f, out_status, precision, n_threads);
}

int ko_krige_ind(int kind, const int *dims, const unsigned char *data, const unsigned char *mask,
                 int ind_value, int cov_type, const double *ranges, const double *angles,
                 double sill, double nugget, const int *radiuses, int max_nb, double mean,
                 const int *nodes, int n_nodes, int *out_idx, int *out_count,
                 unsigned char *out_path, double *out_est, double *out_var, float *out_est_f,
                 int *out_status, int precision, int n_threads)
{
    return krige_nodes(kind, dims, nullptr, data, ind_value, mask, cov_type, ranges, angles, sill,
                       nugget, radiuses, max_nb, mean, nullptr, nodes, n_nodes, out_idx, out_count,
                       out_path, out_est, out_var, out_est_f, out_status, precision, n_threads);
}

// Whole-grid drivers with the reference's output semantics.
//
// cont_kriging (cont_kriging.h:63-117): informed cells are copied (mask 1);
// kriged cells get the float estimate (mask 1); on NO_NEIGHBOURS / SINGULARITY
// OK leaves the cell as the caller's clone of the input (undefined_on_failure,
// ordinary_kriging.cpp:31-33), SK writes the mean (mean_on_failure,
// simple_kriging.cpp:117-119). SK's automatic mean is calc_mean
// (calc_mean.cpp:6-30). `out_data`/`out_mask` must hold a copy of the input.
int ko_cont_grid(int kind, const int *dims, const float *data, const unsigned char *mask,
                 int cov_type, const double *ranges, const double *angles, double sill,
                 double nugget, const int *radiuses, int max_nb, int auto_mean, double mean,
                 float *out_data, unsigned char *out_mask, double *out_est, double *out_var,
                 int *out_status, int n_threads)
{
    long size = (long)dims[0] * dims[1] * dims[2];
    if (kind == 1 && auto_mean)
    {
        double sum = 0;
        long cnt = 0;
        for (long i = 0; i < size; ++i)
            if (mask[i])
            {
                sum += data[i];
                cnt += 1;
            }
        mean = cnt ? sum / cnt : 0.0;
    }
    std::vector<int> nodes;
    for (long i = 0; i < size; ++i)
        if (!mask[i]) nodes.push_back((int)i);
    std::vector<float> ef(nodes.size());
    std::vector<double> ed(nodes.size()), vd(nodes.size());
    std::vector<int> st(nodes.size());
    int rc = ko_krige_cont(kind, dims, data, mask, cov_type, ranges, angles, sill, nugget, radiuses,
                           max_nb, mean, nodes.data(), (int)nodes.size(), nullptr, nullptr, nullptr,
                           ed.data(), vd.data(), ef.data(), st.data(), 0, n_threads);
    if (rc) return rc;
    for (long i = 0; i < size; ++i)
        if (mask[i])
        {
            out_data[i] = data[i];
            out_mask[i] = 1;
            if (out_est) out_est[i] = data[i];
            if (out_var) out_var[i] = 0;
            if (out_status) out_status[i] = -1;
        }
    for (size_t t = 0; t < nodes.size(); ++t)
    {
        int i = nodes[t];
        if (out_est) out_est[i] = ed[t];
        if (out_var) out_var[i] = vd[t];
        if (out_status) out_status[i] = st[t];
        if (st[t] == KI_SUCCESS)
        {
            out_data[i] = ef[t];
            out_mask[i] = 1;
        }
        else if (kind == 1)
        {
            out_data[i] = (float)mean;
            out_mask[i] = 1;
        }
    }
    return 0;
}

// LVM kriging (lvm_kriging.cpp:16-39): cont_kriging with the box-truncated
// covariance table, SK weights and the per-node mean array as the mean
// provider (combine centres each neighbour on its own mean and adds the
// node's); failures get the node's mean (mean_on_failure).
int ko_lvm_grid(const int *dims, const float *data, const unsigned char *mask, const float *means,
                int cov_type, const double *ranges, const double *angles, double sill, double nugget,
                const int *radiuses, int max_nb, float *out_data, unsigned char *out_mask, double *out_est,
                double *out_var, int *out_status, int n_threads)
{
    long size = (long)dims[0] * dims[1] * dims[2];
    std::vector<int> nodes;
    for (long i = 0; i < size; ++i)
        if (!mask[i]) nodes.push_back((int)i);
    std::vector<float> ef(nodes.size());
    std::vector<double> ed(nodes.size()), vd(nodes.size());
    std::vector<int> st(nodes.size());
    int rc = krige_nodes(1, dims, data, nullptr, -1, mask, cov_type, ranges, angles, sill, nugget, radiuses,
                         max_nb, 0.0, means, nodes.data(), (int)nodes.size(), nullptr, nullptr, nullptr,
                         ed.data(), vd.data(), ef.data(), st.data(), 0, n_threads);
    if (rc) return rc;
    for (long i = 0; i < size; ++i)
        if (mask[i])
        {
            out_data[i] = data[i];
            out_mask[i] = 1;
            if (out_est) out_est[i] = data[i];
            if (out_var) out_var[i] = 0;
            if (out_status) out_status[i] = -1;
        }
    for (size_t t = 0; t < nodes.size(); ++t)
    {
        int i = nodes[t];
        if (out_est) out_est[i] = ed[t];
        if (out_var) out_var[i] = vd[t];
        if (out_status) out_status[i] = st[t];
        out_data[i] = st[t] == KI_SUCCESS ? ef[t] : means[i];
        out_mask[i] = 1;
    }
    return 0;
}

// Full IK (indicator_kriging.h:88-161): every cell (informed ones too), per
// category c an SK with mean = marginal p_c (stored as float,
// ik_params.h:20) on that category's truncated covariance and lookup; failure
// gives p_c; then order relations and the first-max argmax. Per-category
// parameter arrays are indexed [c*3 + axis]. probs (optional) gets the
// corrected probabilities, category-major per cell.
int ko_indicator_grid(const int *dims, const unsigned char *data, const unsigned char *mask,
                      int n_cat, const int *cov_types, const double *ranges, const double *angles,
                      const double *sills, const double *nuggets, const int *radiuses,
                      const int *max_nbs, const double *marginals, unsigned char *out_data,
                      unsigned char *out_mask, float *probs, int n_threads)
{
    long size = (long)dims[0] * dims[1] * dims[2];
    std::vector<int> nodes(size);
    for (long i = 0; i < size; ++i) nodes[i] = (int)i;
    std::vector<std::vector<float>> pc(n_cat, std::vector<float>(size));
    std::vector<std::vector<int>> stc(n_cat, std::vector<int>(size));
    for (int c = 0; c < n_cat; ++c)
    {
        float mc = (float)marginals[c];
        int rc = ko_krige_ind(1, dims, data, mask, c, cov_types[c], ranges + 3 * c, angles + 3 * c,
                              sills[c], nuggets[c], radiuses + 3 * c, max_nbs[c], (double)mc,
                              nodes.data(), (int)size, nullptr, nullptr, nullptr, nullptr, nullptr,
                              pc[c].data(), stc[c].data(), 0, n_threads);
        if (rc) return rc;
        for (long i = 0; i < size; ++i)
            if (stc[c][i] != KI_SUCCESS) pc[c][i] = mc;
    }
    std::vector<float> p(n_cat);
    for (long i = 0; i < size; ++i)
    {
        for (int c = 0; c < n_cat; ++c) p[c] = pc[c][i];
        order_relations(p);
        out_data[i] = (unsigned char)argmax_first(p);
        out_mask[i] = 1;
        if (probs)
            for (int c = 0; c < n_cat; ++c) probs[(size_t)i * n_cat + c] = p[c];
    }
    return 0;
}

// Median IK (median_ik.cpp:24-89): indicator = (data == 1), one truncated
// covariance, mean = marginal_probs[1], double result; prob <= 0.5 -> 0 else 1
// (median_ik.cpp:15-21, through a float). The reference leaves `prob`
// uninitialised when kriging fails; this restatement defines it as the mean.
int ko_median_ik_grid(const int *dims, const unsigned char *data, const unsigned char *mask,
                      int cov_type, const double *ranges, const double *angles, double sill,
                      double nugget, const int *radiuses, int max_nb, const double *marginal_probs,
                      unsigned char *out_data, unsigned char *out_mask, double *out_prob,
                      int *out_status, int n_threads)
{
    long size = (long)dims[0] * dims[1] * dims[2];
    std::vector<int> nodes(size);
    for (long i = 0; i < size; ++i) nodes[i] = (int)i;
    std::vector<double> pd(size);
    std::vector<int> st(size);
    int rc = ko_krige_ind(1, dims, data, mask, 1, cov_type, ranges, angles, sill, nugget, radiuses,
                          max_nb, marginal_probs[1], nodes.data(), (int)size, nullptr, nullptr,
                          nullptr, pd.data(), nullptr, nullptr, st.data(), 0, n_threads);
    if (rc) return rc;
    for (long i = 0; i < size; ++i)
    {
        double p = st[i] == KI_SUCCESS ? pd[i] : (double)(float)marginal_probs[1];
        float pf = (float)p;
        out_data[i] = pf <= 0.5 ? 0 : 1;
        out_mask[i] = 1;
        if (out_prob) out_prob[i] = p;
        if (out_status) out_status[i] = st[i];
    }
    return 0;
}

// SK weights for one system on real coordinates with the analytic model
// (simple_kriging.cpp:67-87, api.cpp:356-410). Returns 1 on success.
int ko_sk_weights(const double *center, const double *xs, const double *ys, const double *zs,
                  int n, int cov_type, const double *ranges, const double *angles, double sill,
                  double nugget, double *out_w, double *out_var)
{
    Model m;
    m.type = cov_type;
    m.r0 = ranges[0];
    m.sill = sill;
    m.nugget = nugget;
    if (!make_transform(ranges, angles, m.T) || n <= 0) return 0;
    std::vector<double> A((size_t)n * n), b(n);
    auto cov = [&](double ax, double ay, double az, double bx, double by, double bz) {
        return m.of_h(m.h_of(ax - bx, ay - by, az - bz));
    };
    for (int i = 0; i < n; ++i)
    {
        for (int j = i; j < n; ++j)
            A[(size_t)i * n + j] = A[(size_t)j * n + i] = cov(xs[i], ys[i], zs[i], xs[j], ys[j], zs[j]);
        b[i] = cov(xs[i], ys[i], zs[i], center[0], center[1], center[2]);
    }
    if (!cholesky(A, n)) return 0;
    std::vector<double> x(b);
    chol_solve(A, n, x);
    double var = cov(center[0], center[1], center[2], center[0], center[1], center[2]);
    for (int i = 0; i < n; ++i)
    {
        out_w[i] = x[i];
        var -= x[i] * b[i];
    }
    if (var < 0) var = 0;
    if (out_var) *out_var = var;
    return 1;
}

// Checks this project's introsort restatement (gnu_introsort.h) against the
// std::sort of the toolchain on keys[0..n): writes both permutations.
void ko_sort_check(const unsigned *keys, int n, int *perm_std, int *perm_gis)
{
    struct E
    {
        unsigned key;
        int pos;
    };
    std::vector<E> a(n);
    for (int i = 0; i < n; ++i) a[i] = {keys[i], i};
    std::vector<E> b = a;
    std::sort(a.begin(), a.end(), [](const E &x, const E &y) { return x.key < y.key; });
    gis::sort(b.data(), (long)n, [](const E &x, const E &y) { return x.key < y.key; });
    for (int i = 0; i < n; ++i)
    {
        perm_std[i] = a[i].pos;
        perm_gis[i] = b[i].pos;
    }
}

// Checks select_first_k (gnu_introsort.h) against std::sort: writes 1 to
// *same_set when the first k elements of both hold the same positions.
void ko_select_check(const unsigned *keys, int n, int k, int *same_set)
{
    struct E
    {
        unsigned key;
        int pos;
    };
    std::vector<E> a(n);
    for (int i = 0; i < n; ++i) a[i] = {keys[i], i};
    std::vector<E> b = a;
    std::sort(a.begin(), a.end(), [](const E &x, const E &y) { return x.key < y.key; });
    gis::select_first_k(b.data(), (long)n, (long)k, [](const E &x, const E &y) { return x.key < y.key; });
    int m = k < n ? k : n;
    std::vector<int> sa(m), sb(m);
    for (int i = 0; i < m; ++i)
    {
        sa[i] = a[i].pos;
        sb[i] = b[i].pos;
    }
    std::sort(sa.begin(), sa.end());
    std::sort(sb.begin(), sb.end());
    *same_set = sa == sb ? 1 : 0;
}

// Sequential Gaussian simulation, do_sequential_gausian_simulation
// (sequential_simulation.h:51-118) as sequential_gaussian_simulation(_lvm)
// instantiates it (sequential_gaussian_simulation.cpp:18-131): the optional
// forward CDF transform of the informed cells (and of the LVM means), then
// every node in the path order that is not informed and whose simulation mask
// is 1 is kriged from the first max_nb informed cells of the template (the
// template-only lookup, sugarbox_neighbour_lookup.h:39-63) with the truncated
// covariances, SK with mean 0 / OK / SK around the LVM means, and set to a
// draw from N(mean, variance) (N(0, 1) on failure) by inverting one
// std::uniform_real_distribution<double> draw of a std::mt19937 seeded with
// `seed`; then the back transform of every informed cell. `data`/`mask` are
// updated in place; out_status (optional) gets the kriging status of each
// simulated node (-1 elsewhere). Returns 0, -1 on bad arguments, -4 when the
// grid exceeds the path generator's 10,000,000-node limit.
int ko_sgs(const int *dims, float *data, unsigned char *mask, const unsigned char *sim_mask,
           const float *cdf_values, const float *cdf_probs, long long cdf_size, const float *means,
           int kind, int cov_type, const double *ranges, const double *angles, double sill, double nugget,
           const int *radiuses, int max_nb, long long seed, int *out_status)
{
    Grid g = {dims[0], dims[1], dims[2]};
    const long size = g.size();
    if (size > 10000000) return -4;
    Flavour f;
    if (!make_flavour(f, true, cov_type, ranges, angles, sill, nugget, radiuses)) return -1;
    PathLcg path;
    if (!path.init(size, seed)) return -1;
    NpCdf cdf;
    const bool use_cdf = cdf_values != nullptr && cdf_probs != nullptr;
    if (use_cdf)
    {
        cdf.v = cdf_values;
        cdf.p = cdf_probs;
        cdf.n = cdf_size;
        for (long i = 0; i < size; ++i)
            if (mask[i]) data[i] = (float)gauss_inverse((double)cdf.prob(data[i]), 0, 1);
    }
    std::vector<float> mv;
    if (means)
    {
        mv.assign(means, means + size);
        if (use_cdf)
            for (long i = 0; i < size; ++i) mv[i] = (float)gauss_inverse((double)cdf.prob(means[i]), 0, 1);
    }
    const std::vector<Off> tmpl = build_template(f);
    const bool ordinary = kind == 0 && !means;
    std::mt19937 gen;
    gen.seed((std::mt19937::result_type)seed);
    if (out_status)
        for (long i = 0; i < size; ++i) out_status[i] = -1;
    std::vector<int> idx, xs, ys, zs;
    std::vector<double> w;
    int node = path.next();
    for (long counter = 0; counter < size; ++counter, node = path.next())
    {
        if (mask[node]) continue;
        if (sim_mask && sim_mask[node] != 1) continue;
        int x, y, z;
        g.coord(node, x, y, z);
        idx.clear();
        for (size_t t = 0; t < tmpl.size() && (int)idx.size() < max_nb; ++t)
        {
            int q = g.index(x + tmpl[t].dx, y + tmpl[t].dy, z + tmpl[t].dz);
            if (q >= 0 && mask[q]) idx.push_back(q);
        }
        int status = KI_NO_NEIGHBOURS;
        float est_f = 0.0f;
        double var = 0.0;
        if (!idx.empty())
        {
            int n = (int)idx.size();
            xs.resize(n);
            ys.resize(n);
            zs.resize(n);
            for (int i = 0; i < n; ++i) g.coord(idx[i], xs[i], ys[i], zs[i]);
            if (weights<double>(f, ordinary, x, y, z, xs, ys, zs, w, var))
            {
                status = KI_SUCCESS;
                // combine (combiner.h:10-25): float accumulation around the means
                float m = means ? mv[node] : 0.0f;
                est_f = m;
                for (int i = 0; i < n; ++i)
                {
                    float d = data[idx[i]] - (means ? mv[idx[i]] : m);
                    est_f += (float)(w[i] * d);
                }
            }
            else
                status = KI_SINGULARITY;
        }
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        double u = dist(gen);
        double value = status == KI_SUCCESS ? gauss_inverse(u, (double)est_f, var) : gauss_inverse(u, 0, 1);
        data[node] = (float)value;
        mask[node] = 1;
        if (out_status) out_status[node] = status;
    }
    if (use_cdf)
        for (long i = 0; i < size; ++i)
            if (mask[i]) data[i] = cdf.inverse((float)gauss_cdf((double)data[i], 0, 1));
    return 0;
}

// n draws of std::uniform_real_distribution<double>(0, 1) on std::mt19937
// seeded as mt_random_generator_t::seed does (bs_random_generator.cpp:9-25).
int ko_mt_draws(long long seed, long long n, double *out)
{
    std::mt19937 gen;
    gen.seed(static_cast<std::mt19937::result_type>((long)seed));
    for (long long i = 0; i < n; ++i)
    {
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        out[i] = dist(gen);
    }
    return 0;
}

// The first `count` nodes of the SGS path for a grid of `size` nodes.
int ko_sgs_path(long long size, long long seed, int *out, long long count)
{
    PathLcg path;
    if (!path.init(size, seed)) return -1;
    for (long long i = 0; i < count; ++i) out[i] = path.next();
    return 0;
}

// Simple collocated cokriging, Markov models I and II
// (simple_cokriging_markI.cpp:19-141, 202-330): for every uninformed cell, the
// first max_nb informed primary cells of the analytic template (the
// template-only lookup), the bordered system of primary covariances, the
// collocated cross covariances coef * C(center, x_i) (Mark I: coef = rho
// sqrt(secondary_variance) / sqrt(C(0)) on the primary model; Mark II: coef =
// rho sqrt(C1(0) / C2(0)) on the secondary model, secondary variance C2(0)),
// solved by gauss_solve; the float result accumulated in double per term
// (combine, :83-106); on failure pm + sv - sm. Informed cells copy the
// primary value; every output cell is informed. out_status: -1 informed,
// 0 kriged, 1 no neighbours, 2 singular.
int ko_cokriging(int mark, const int *dims, const float *pdata, const unsigned char *pmask, const float *sdata,
                 const unsigned char *smask, int cov_type, const double *ranges, const double *angles, double sill,
                 double nugget, int cov_type2, const double *ranges2, const double *angles2, double sill2,
                 double nugget2, const int *radiuses, int max_nb, double primary_mean, double secondary_mean,
                 double secondary_variance, double corr, float *out_data, unsigned char *out_mask, int *out_status,
                 int n_threads)
{
    Grid g = {dims[0], dims[1], dims[2]};
    Flavour fp, fs;
    if (!make_flavour(fp, false, cov_type, ranges, angles, sill, nugget, radiuses)) return -1;
    if (mark == 2 && !make_flavour(fs, false, cov_type2, ranges2, angles2, sill2, nugget2, radiuses)) return -1;
    const double c0p = fp.at(0, 0, 0, 0, 0, 0);
    double coef, sec_var;
    const Flavour *fc;
    if (mark == 1)
    {
        coef = c0p <= 0 ? 0.0 : corr * sqrt(secondary_variance) / sqrt(c0p);
        sec_var = secondary_variance;
        fc = &fp;
    }
    else
    {
        const double c0s = fs.at(0, 0, 0, 0, 0, 0);
        coef = c0s <= 0 ? 0.0 : corr * sqrt(c0p / c0s);
        sec_var = c0s;
        fc = &fs;
    }
    const float pm = (float)primary_mean, sm = (float)secondary_mean; // mean_t is float
    const std::vector<Off> tmpl = build_template(fp);
    const long size = g.size();
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < size; ++i)
    {
        if (pmask[i])
        {
            out_data[i] = pdata[i];
            out_mask[i] = 1;
            if (out_status) out_status[i] = -1;
            continue;
        }
        const float sv = smask[i] ? sdata[i] : sm;
        int x, y, z;
        g.coord((int)i, x, y, z);
        std::vector<int> idx;
        for (size_t t = 0; t < tmpl.size() && (int)idx.size() < max_nb; ++t)
        {
            int q = g.index(x + tmpl[t].dx, y + tmpl[t].dy, z + tmpl[t].dz);
            if (q >= 0 && pmask[q]) idx.push_back(q);
        }
        int status = 1;
        float result = 0.0f;
        if (!idx.empty())
        {
            const int n = (int)idx.size(), m = n + 1;
            std::vector<int> xs(n), ys(n), zs(n);
            for (int k = 0; k < n; ++k) g.coord(idx[k], xs[k], ys[k], zs[k]);
            std::vector<double> A((size_t)m * m), B(m), W;
            for (int a = 0; a < n; ++a)
                for (int b = a; b < n; ++b)
                {
                    A[(size_t)a * m + b] = fp.at(xs[a], ys[a], zs[a], xs[b], ys[b], zs[b]);
                    A[(size_t)b * m + a] = A[(size_t)a * m + b];
                }
            for (int a = 0; a < n; ++a)
            {
                A[(size_t)n * m + a] = coef * fc->at(x, y, z, xs[a], ys[a], zs[a]);
                A[(size_t)a * m + n] = A[(size_t)n * m + a];
                B[a] = fp.at(xs[a], ys[a], zs[a], x, y, z);
            }
            B[n] = coef * fc->at(0, 0, 0, 0, 0, 0);
            A[(size_t)m * m - 1] = sec_var;
            if (gauss_solve_ref(A, B, W, m))
            {
                status = 0;
                result = pm;
                for (int k = 0; k < n; ++k) result += (pdata[idx[k]] - pm) * W[k];
                result += W[n] * (sv - sm);
            }
            else
                status = 2;
        }
        if (status != 0) result = pm + sv - sm;
        out_data[i] = result;
        out_mask[i] = 1;
        if (out_status) out_status[i] = status;
    }
    return 0;
}

// The correlogram scale of an indicator mean (my_kriging_weights.h:407-436):
// sqrt(m (1 - m)) with 0 and 1 moved inside by 1e-5.
static double corr_sigma(double m)
{
    if (m == 0) m += 0.00001;
    if (m == 1) m -= 0.00001;
    return std::sqrt(m * (1 - m));
}

// corellogramed_weights_3 (my_kriging_weights.h:363-505): the SK system with
// A_ij = C_ij (s_i s_j) and b_i = C_ic (s_i s_c), solved by Cholesky; the
// weights are used as they come out (no rescaling).
static bool corr_weights(const Flavour &f, int cx, int cy, int cz, double mean_c, const std::vector<int> &xs,
                         const std::vector<int> &ys, const std::vector<int> &zs, const std::vector<double> &means,
                         std::vector<double> &w)
{
    const int n = (int)xs.size();
    if (n <= 0) return false;
    const double sc = corr_sigma(mean_c);
    std::vector<double> sg(n), A((size_t)n * n);
    for (int i = 0; i < n; ++i) sg[i] = corr_sigma(means[i]);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i)
    {
        for (int j = 0; j < n; ++j)
            A[(size_t)i * n + j] = f.at(xs[i], ys[i], zs[i], xs[j], ys[j], zs[j]) * (sg[i] * sg[j]);
        w[i] = f.at(xs[i], ys[i], zs[i], cx, cy, cz) * (sg[i] * sc);
    }
    if (!cholesky(A, n)) return false;
    chol_solve(A, n, w);
    return true;
}

// Sequential indicator simulation (sequential_indicator_simulation.cpp:24-185):
// the walk of the simulation; per visited node that is not informed and whose
// simulation mask is 1, for every category c (only c = 0 with two categories,
// the other probability being 1 - p) the SK estimate of the indicator
// (category == c) from the first max_nb[c] informed cells of category c's
// truncated template, around float(marginal[c]) or the LVM means of category
// c, accumulated in double (the marginal / mean on failure); then one
// std::uniform_real_distribution draw u picks the first category whose running
// sum of probabilities exceeds u times their sum (sample.cpp:8-21). `params`:
// per category cov_type, ranges[3], angles[3], sill, nugget; radiuses (3 per
// category), max_nb, marginal. means: per category a float per cell, or null;
// with means, `corr` selects the correlogram weights (corellogram_weight_calculator_t).
// Returns 0, -1 on bad arguments, -3 when the walk does not visit every node
// (the reference throws at the end of such a path).
int ko_sis(const int *dims, unsigned char *data, unsigned char *mask, const unsigned char *sim_mask, int ncat,
           const int *cov_types, const double *ranges, const double *angles, const double *sills,
           const double *nuggets, const int *radiuses, const int *max_nb, const double *marginals,
           const float *const *means, long long seed, int *out_status, int corr)
{
    Grid g = {dims[0], dims[1], dims[2]};
    const long size = g.size();
    if (size > 10000000 || ncat < 2) return -1;
    std::vector<Flavour> f(ncat);
    std::vector<std::vector<Off>> tmpl(ncat);
    const int kcat = ncat == 2 ? 1 : ncat;
    for (int c = 0; c < kcat; ++c)
    {
        if (!make_flavour(f[c], true, cov_types[c], ranges + 3 * c, angles + 3 * c, sills[c], nuggets[c],
                          radiuses + 3 * c))
            return -1;
        tmpl[c] = build_template(f[c]);
    }
    PathLcg path;
    if (!path.init(size, (int)seed)) return -1;
    std::mt19937 gen;
    gen.seed((std::mt19937::result_type)(long)(int)seed);
    if (out_status)
        for (long i = 0; i < size; ++i) out_status[i] = -1;
    std::vector<int> idx, xs, ys, zs;
    std::vector<double> w, probs(ncat), nbm;
    const long first = path.R;
    for (long counter = 0; counter < size; ++counter)
    {
        const int node = path.next();
        if (mask[node]) continue;
        if (sim_mask && sim_mask[node] != 1) continue;
        int x, y, z;
        g.coord(node, x, y, z);
        int st_all = 0;
        for (int c = 0; c < kcat; ++c)
        {
            idx.clear();
            for (size_t t = 0; t < tmpl[c].size() && (int)idx.size() < max_nb[c]; ++t)
            {
                int q = g.index(x + tmpl[c][t].dx, y + tmpl[c][t].dy, z + tmpl[c][t].dz);
                if (q >= 0 && mask[q]) idx.push_back(q);
            }
            const float mc = means ? means[c][node] : (float)marginals[c];
            // the failure value: the mean provider at the node (double)
            double prob = means ? (double)means[c][node] : (double)(float)marginals[c];
            int status = KI_NO_NEIGHBOURS;
            if (!idx.empty())
            {
                const int n = (int)idx.size();
                xs.resize(n);
                ys.resize(n);
                zs.resize(n);
                for (int i = 0; i < n; ++i) g.coord(idx[i], xs[i], ys[i], zs[i]);
                double var;
                bool ok;
                if (corr && means)
                {
                    nbm.resize(n);
                    for (int i = 0; i < n; ++i) nbm[i] = (double)means[c][idx[i]];
                    ok = corr_weights(f[c], x, y, z, (double)mc, xs, ys, zs, nbm, w);
                }
                else
                    ok = weights<double>(f[c], false, x, y, z, xs, ys, zs, w, var);
                if (ok)
                {
                    status = KI_SUCCESS;
                    double r = (double)mc;
                    for (int i = 0; i < n; ++i)
                    {
                        const unsigned char v = data[idx[i]] == c ? 1 : 0;
                        const float mi = means ? means[c][idx[i]] : mc;
                        r += w[i] * (v - mi);
                    }
                    prob = r;
                }
                else
                    status = KI_SINGULARITY;
            }
            probs[c] = prob;
            if (status > st_all) st_all = status;
        }
        if (ncat == 2) probs[1] = 1 - probs[0];
        double sum = 0.0;
        for (int c = 0; c < ncat; ++c) sum += probs[c];
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        const double s = dist(gen) * sum;
        double p = 0;
        int pick = ncat - 1;
        for (int c = 0; c < ncat; ++c)
        {
            p += probs[c];
            if (s < p)
            {
                pick = c;
                break;
            }
        }
        data[node] = (unsigned char)pick;
        mask[node] = 1;
        if (out_status) out_status[node] = st_all;
    }
    if (path.R != first) return -3;
    return 0;
}

} // extern "C"
