// Host-side covariance model, search template and selection-key tables.
//
// Compiled by the host C++ compiler with plain IEEE double arithmetic (no
// FMA contraction, no fast-math), the way the reference is compiled, so every
// covariance value that decides a neighbour ordering is bit-identical to the
// value the reference compares.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hb
{
enum CovType
{
    COV_SPHERICAL = 0,
    COV_EXPONENTIAL = 1,
    COV_GAUSSIAN = 2
};

struct CovModel
{
    int type = 0;
    double ranges[3] = {1, 1, 1};
    double angles[3] = {0, 0, 0};
    double sill = 1, nugget = 0;
    double T[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

    // ||T v||_2 with the reference's summation order (cov_model.h:63-77)
    double h_of(double v0, double v1, double v2) const;
    // the three models of cov_model.h:146-183 (C(0) = sill, nugget dropped beyond)
    double of_h(double h) const;
};

// Builds the model; false (with a message) on a zero range or unknown type.
bool make_model(int type, const double *ranges, const double *angles, double sill, double nugget,
                CovModel &m, std::string &err);

// T = S * ((Rx * Ry) * Rz), cov_model.h:16-61 (TNT accumulation order).
bool make_transform(const double *ranges, const double *angles, double *T);

// A covariance flavour as the reference's drivers instantiate it:
//   analytic  — cov_model_t (OK, ordinary_kriging.cpp:29-33);
//   truncated — the +-radius box table (precalculated_covariances_t for SK/IK,
//               covariance_field_t for median IK), 0 outside the box.
struct Flavour
{
    CovModel m;
    bool truncated = false;
    int r[3] = {1, 1, 1};
    // cov(center, center + d), evaluated the way the flavour evaluates it
    double at_offset(int dx, int dy, int dz) const;
    double c0() const { return at_offset(0, 0, 0); }
    // the strict neighbour threshold C(0)/100 (sugarbox_indexed_neighbour_lookup.h:85-90)
    double threshold() const { return c0() / 100; }
};

struct Offset
{
    int dx, dy, dz;
};

// Sorted search template (calc_cov_field, covariance_field.h:62-106).
std::vector<Offset> build_template(const Flavour &f);

// Selection keys over the cluster-search block: offsets d with |d_a| <= 2 r_a - 1
// (the farthest a candidate in the 27 bins around a cell can lie).
// Layout: x fastest, index = ((dz + hz) * ny + (dy + hy)) * nx + (dx + hx),
// h_a = 2 r_a - 1, n_a = 2 h_a + 1.
//   vals[i]  = cov(center, center + d) as the reference computes it
//   rank[i]  = dense rank of vals[i] among kept offsets, descending
//              (0 = largest covariance; equal values share a rank), or
//              KEY_EXCLUDED where the value is not above the threshold.
constexpr uint32_t KEY_EXCLUDED = 0xFFFFFFFFu;
struct KeyTable
{
    int half[3];
    int n[3];
    std::vector<double> vals;
    std::vector<uint32_t> rank;
    uint32_t n_ranks = 0; // distinct kept values
    // per rank the smallest and largest squared anisotropic distance h2 carrying
    // it (||T v||^2 over the offsets of that rank), for the ranks build_key_table
    // assigns; code that assigns other ranks clears them
    std::vector<double> h2_lo, h2_hi;
};
void build_key_table(const Flavour &f, KeyTable &kt, int n_threads);
// The same template as build_template(f), its covariances read from kt.
std::vector<Offset> build_template(const Flavour &f, const KeyTable &kt);
// Its length alone (the clusterizer's limit is length / 250), without the sort.
long template_size(const Flavour &f, const KeyTable &kt);

// Float surrogate of the selection key. Over the kept offsets of the key
// block the dense rank must be a non-decreasing function of the reference's
// squared anisotropic distance h2 = sum_i (sum_j T_ij v_j)^2 (the quantity
// whose square root transfrom_and_norm returns, cov_model.h:63-77).
// build_surrogate checks that on the exact doubles and records, per rank, the
// largest h2 carrying it; when the check holds (ok == true) any candidate whose
// true h2 exceeds that value for the k-th selected rank ranks strictly after
// it, so a float h2 with a bounded error can discard far candidates without
// reading their ranks. With `running_max` the ranks need not follow h2:
// h2_rank[r] is then the largest h2 of any rank <= r, which bounds every rank
// the selection keeps ahead of r all the same (keys that are positions in the
// sorted template, where offsets of one covariance sit in the sort's order).
struct Surrogate
{
    bool ok = false;
    float T[9];                 // the transform rounded to float
    double h2_cut = 0;          // largest h2 of a kept offset
    double e3 = 0;              // bound on || float(T d) - T d ||_2 for the packed offsets
    float step[3] = {0, 0, 0};  // ||T e_a||: a bound on how far the k-th distance moves per unit step
    std::vector<double> h2_rank; // largest h2 of each rank
};
void build_surrogate(const Flavour &f, const KeyTable &kt, Surrogate &sg, bool running_max = false);
// The same for keys that are positions in the sorted template `tmpl` (the
// running maximum of h2 along it).
void build_surrogate_template(const Flavour &f, const std::vector<Offset> &tmpl, Surrogate &sg);

int clamp_threads(int n);
// The simulation's uniform draws: n doubles equal to n calls of
// std::uniform_real_distribution<double>(0, 1) on a std::mt19937 seeded with
// `seed` (as the standard library seeds it: seed mod 2^32).
void sgs_draws(unsigned long long seed, long long n, double *out);

} // namespace hb
