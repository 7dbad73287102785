// Internal interface between the C ABI (api.cpp) and the engine (engine.cu).
#pragma once
#include <cstddef>
#include <string>
#include <vector>

namespace hb
{
struct SkArgs
{
    int cov_type;
    double ranges[3];
    double angles[3];
    double sill, nugget;
    int radiuses[3];
    int max_nb;
    bool auto_mean;
    double mean;
};

struct IkArgs
{
    int cov_type;
    double ranges[3];
    double angles[3];
    double sill, nugget;
    int radiuses[3];
    int max_nb;
    double marginal;
};

struct CovArgs
{
    int cov_type;
    double ranges[3];
    double angles[3];
    double sill, nugget;
};

// Collocated cokriging: mark 1 (one model, the secondary variance given) or
// mark 2 (primary and secondary models).
struct CokArgs
{
    int mark;
    CovArgs primary, secondary;
    int radiuses[3];
    int max_nb;
    double primary_mean, secondary_mean, secondary_variance, corr;
};

struct SgsArgs
{
    int cov_type;
    double ranges[3];
    double angles[3];
    double sill, nugget;
    int radiuses[3];
    int max_nb;
    int kind; // 0 ordinary, 1 simple (ignored with LVM means)
    long long seed;
};

// Non-parametric CDF table (host arrays): ascending values and their probabilities.
struct CdfTable
{
    const float *values = nullptr;
    const float *probs = nullptr;
    long long size = 0;
};

struct Options
{
    int precision = 0;
    int refine_steps = 0;
    unsigned flags = 0;
    void *stream = nullptr;
    double *estimate64 = nullptr;
    double *variance = nullptr;
    signed char *status = nullptr;
    float *ik_probs = nullptr;
    double tolerance = 0.0;
};

enum Stage
{
    STAGE_UPLOAD = 0,   // host->device copies of the inputs
    STAGE_COMPACT,      // informed cells -> points (scan + readback of the count)
    STAGE_TABLES,       // key/value/template uploads and the pair-covariance tables
    STAGE_BINS,         // binning, per-bin path decision (and readback)
    STAGE_SEARCH,       // neighbour search kernel
    STAGE_TIES,         // tie-straddle resolution
    STAGE_PREPARE,      // status + work buckets (and readback)
    STAGE_SOLVE,        // per-bucket solves and FP64 re-solves
    STAGE_FINALIZE,     // outputs of cells not written by a solver
    STAGE_DOWNLOAD,     // device->host copies of the outputs
    kStages
};

struct Stats
{
    double stage_ms[kStages] = {0};
    double total_ms = 0, search_ms = 0, solve_ms = 0, search_kernel_ms = 0;
    long long ties = 0, template_cells = 0, kriged = 0, launches = 0;
    long long h2d = 0, d2h = 0, escalated = 0;
    long long refined = 0; // FP32 systems the four-rows-per-lane check passed on to classic refinement
    long long bucket_items[5] = {0, 0, 0, 0, 0};
    double bucket_ms[5] = {0, 0, 0, 0, 0};
    double bucket_flops[5] = {0, 0, 0, 0, 0};
    long long exact_cells = 0; // cells the float prefilter left to the exact rank path
    bool prefilter = false;
    double plan_ms = 0;        // host time building the covariance tables (overlapped with upload/compaction)
    int sgs_levels = 0;        // SGS: dependency levels (solve launches)
    double draws_ms = 0;       // SGS: host ms generating the uniform draws (overlapped with the search)
    double sgs_flops = 0;      // SGS: algorithmic flops of the kriging solves (same count as the kriging buckets)
};

void set_error(const std::string &msg);
const char *last_error();
void set_threads(int n);
int get_threads();
// the solve-kernel tuning table (tune.cpp): the variant a (bucket, covariance
// type, precision) key runs, and an override returning the previous setting
// (-1 for an invalid key or variant)
int solve_variant(int np, int cov_type, int precision);
int set_solve_variant(int np, int cov_type, int precision, int variant);
// tuning mode on / off; the tuning cache (JSON) read and written, returning
// the number of keys or -1 with `err`; every key back to its built-in pick
int tune_mode();
void set_tune_mode(int on);
int tune_load(const char *path, std::string &err);
int tune_save(const char *path, std::string &err);
void tune_reset();

// kind 0 OK, 1 SK, 2 LVM (SK weights around the per-cell `means`, which kind 2
// requires; lvm_kriging.cpp:16-39)
int cont_kriging(int kind, const int *dims, const float *in_data, const unsigned char *in_mask, const SkArgs &a,
                 float *out_data, unsigned char *out_mask, const Options &opt, const float *means = nullptr);
// Sequential Gaussian simulation in place on data/mask
// (sequential_gaussian_simulation.cpp:18-131). sim_mask, cdf and means
// (LVM) are optional; opt.status receives -1 informed, 0 kriged, 1 no
// neighbours, 2 singular (N(0,1) draw), 3 not simulated.
int sgs_simulation(const int *dims, float *data, unsigned char *mask, const unsigned char *sim_mask,
                   const CdfTable *cdf, const float *means, const SgsArgs &a, const Options &opt);
// Simple collocated cokriging (simple_cokriging_markI.cpp:202-330) of every
// uninformed primary cell; every output cell ends informed. opt.status
// receives -1 informed, 0 kriged, 1 no neighbours, 2 singular.
int cokriging(const int *dims, const float *pdata, const unsigned char *pmask, const float *sdata,
              const unsigned char *smask, const CokArgs &a, float *out_data, unsigned char *out_mask,
              const Options &opt);
// The simulations' dependency levels: level(r) = 1 + the largest level of the
// ranks listed for r (k per rank, -1 for none; each below r in a simulation),
// 0 with none listed.
int sim_levels(long long n_sim, int k, const int *nb_rank, int *levels);
// Sequential indicator simulation in place on data (categories) / mask
// (sequential_indicator_simulation.cpp:24-185): cats per category; means (LVM)
// one float array per category or null, with `correlogram` the correlogram
// weights (my_kriging_weights.h:363-505); opt.status as for the simulation.
int sis_simulation(const int *dims, unsigned char *data, unsigned char *mask, const unsigned char *sim_mask,
                   const std::vector<IkArgs> &cats, const float *const *means, long long seed, const Options &opt,
                   bool correlogram = false);
int indicator_kriging(const int *dims, const unsigned char *in_data, const unsigned char *in_mask,
                      const std::vector<IkArgs> &cats, unsigned char *out_data, unsigned char *out_mask,
                      const Options &opt);
int median_ik(const int *dims, const unsigned char *in_data, const unsigned char *in_mask, const IkArgs &a,
              double marginal1, unsigned char *out_data, unsigned char *out_mask, const Options &opt);
int find_neighbours(int kind, const int *dims, const unsigned char *mask, const SkArgs &a, const int *nodes,
                    int n_nodes, int *out_idx, int *out_count, unsigned char *out_path);
Stats last_stats();
int host_template(int kind, int cov_type, const double *ranges, const double *angles, double sill, double nugget,
                  const int *radiuses, int *out, int cap, int *out_limit);
double host_covariance(int kind, int cov_type, const double *ranges, const double *angles, double sill,
                       double nugget, const int *radiuses, const int *a, const int *b);
int sk_weights(const double *center, const double *xs, const double *ys, const double *zs, int n, int cov_type,
               const double *ranges, const double *angles, double sill, double nugget, double *out_w);
// Property files (inc_io.cpp): INC (read_inc_file.cpp, property_writer.cpp)
// and GSLIB (property_writer.cpp:87-140). Failures throw std::runtime_error
// with the reference's messages.
void read_inc_float(const char *path, float undefined_value, long long size, float *data, unsigned char *mask);
void read_inc_byte(const char *path, int undefined_value, long long size, unsigned char *data, unsigned char *mask);
void write_inc_float(const char *path, const char *name, const float *data, const unsigned char *mask,
                     long long size, float undefined_value, bool gslib);
void write_inc_byte(const char *path, const char *name, const unsigned char *data, const unsigned char *mask,
                    long long size, unsigned char undefined_value, const std::vector<unsigned char> &remap,
                    bool gslib);
void *host_alloc(size_t bytes);
void host_free(void *p);
} // namespace hb
