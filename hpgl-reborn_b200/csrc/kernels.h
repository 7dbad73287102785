// Launchers of the device kernels (search.cu, solve.cu, misc.cu).
#pragma once
#include "engine.cuh"

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace hb
{
constexpr int kBuckets = 5; // neighbour counts 1-8, 9-16, 17-32, 33-64, >64
constexpr int kBucketNP[4] = {8, 16, 32, 64};

struct DevModel
{
    int type;
    double r0, sill, nugget;
    double T[9];
};

struct SolveOut
{
    float *out_data;     // continuous estimate (float) per cell
    uint8_t *out_mask;   // set to 1 where out_data is written
    double *est64;       // optional FP64 estimate per cell
    double *var;         // optional kriging variance per cell
    signed char *status; // per-cell status (0 success, 2 singular)
    float *prob;         // optional: indicator probability of one category (float result)
    int prob_stride;     // distance between cells in `prob` (the category count)
    int write_cont;      // write out_data / out_mask
    const float *cell_mean; // LVM: per-cell mean, added at the centre instead of the SK mean
};

// scan / points / bins (search.cu)
long long scan_tmp_ints(long long n);
void exclusive_scan(int *v, long long n, int *tmp, int *total, cudaStream_t st);
int scan_kernels(long long n); // kernels one exclusive_scan of n ints launches
void launch_flag_informed(const uint8_t *mask, long long n, int *flag, cudaStream_t st);
// `mean_f` (LVM) centres each continuous value on its own cell's mean, in float
void launch_emit_points(const uint8_t *mask, const int *pos, const Geom &g, const float *val_f,
                        const float *mean_f, const uint8_t *val_u8, int *pts_node, unsigned long long *pts_xyz,
                        float *pts_val, uint8_t *pts_cat, int *pid_of_node, cudaStream_t st);
void launch_bin_count(const unsigned long long *pts_xyz, const int *n_pts, const Geom &g, int *bin_cnt,
                      cudaStream_t st);
void launch_bin_fill(const unsigned long long *pts_xyz, const int *n_pts, const Geom &g, const int *bin_start,
                     int *bin_fill, int *bin_pts, cudaStream_t st);
void launch_bin_sort(const Geom &g, const int *bin_start, const int *bin_cnt, int *bin_pts, uint8_t *bin_flag,
                     cudaStream_t st);
// max_cand / max_cand_tmpl: the largest 27-bin candidate count of the cluster-
// path / template-path bins
void launch_bin_region(const Geom &g, uint8_t *bin_flag, const int *bin_cnt, int *max_cand, int *n_tmpl_bins,
                       int *tmpl_bins, int *max_cand_tmpl, cudaStream_t st);
// Template-path search over a bitmap of the grid padded by the radiuses:
// `bits` is scratch of (template_padded_cells + 31) / 32 words; template entries
// carry template_padded_offset(dx, dy, dz) in .w.
long long template_padded_cells(const Geom &g);
int template_padded_offset(const Geom &g, int dx, int dy, int dz);
cudaError_t launch_search_template(const Geom &g, const uint8_t *mask, uint32_t *bits, int all_cells,
                                   const int *tmpl_bins, int n_tmpl_bins, const float *pts_vf, const int4 *tmpl,
                                   int n_tmpl, const int *pid_of_node, int *nb_pid, int2 *nb_rec, int *nb_n,
                                   int *n_template_cells, int n_sm, cudaStream_t st);
size_t search_smem_bytes(int cand_cap, int k, int warps);
cudaError_t launch_search(const Geom &g, const uint8_t *mask, int all_cells, const int *bin_start,
                          const int *bin_cnt, const uint8_t *bin_flag, const int *bin_pts,
                          const unsigned long long *pts_xyz, const float *pts_vf, const uint32_t *keytab,
                          int rank_bits, const int4 *tmpl, int n_tmpl, const int *pid_of_node, int cand_cap,
                          int warps, int *nb_pid, int2 *nb_rec, int *nb_n, int *tie_cells, int *tie_count,
                          int *n_template_cells, cudaStream_t st);
// Float-distance prefilter of the fast selection (host_model.h, Surrogate):
// on == 0 runs the exact rank path for every cell.
struct SurrDev
{
    int on;
    float T[9];
    float step[3];
    double e3;
    double h2_cut;
    const double *h2_rank;
};

size_t search_fast_smem_bytes(int cand_cap, int k, int warps);
// exact_cells (may be null) counts cells the float prefilter left to the exact
// path. template_bins = 0 searches the cluster-path bins; 1 the template-path
// bins, keytab16 then holding template positions (n_template_cells counts them)
cudaError_t launch_search_fast(const Geom &g, const uint8_t *mask, int all_cells, const int *bin_start,
                               const int *bin_cnt, const uint8_t *bin_flag, const int *bin_pts,
                               const unsigned long long *pts_xyz, const float *pts_vf, const uint16_t *keytab16,
                               const SurrDev &sd, int template_bins, const int *pid_of_node, int cand_cap,
                               int warps, int *nb_pid, int2 *nb_rec, int *nb_n, int *tie_cells, int *tie_count,
                               int *n_template_cells, int *exact_cells, cudaStream_t st);
void launch_resolve_ties(const Geom &g, const int *tie_cells, const int *tie_count, int first, int chunk,
                         const int *bin_start, const int *bin_cnt, const int *bin_pts,
                         const unsigned long long *pts_xyz, const float *pts_vf, const uint32_t *keytab,
                         void *scratch, int cap, int *nb_pid, int2 *nb_rec, cudaStream_t st);
size_t tie_entry_bytes();
size_t resolve_ties_fast_smem(int cap, int warps);
cudaError_t launch_resolve_ties_fast(const Geom &g, const int *tie_cells, const int *tie_count, int n_ties,
                                     const int *bin_start, const int *bin_cnt, const int *bin_pts,
                                     const unsigned long long *pts_xyz, const float *pts_vf, const uint16_t *keytab16,
                                     int cap, int *nb_pid, int2 *nb_rec, int n_sm, cudaStream_t st);

// solves (solve.cu, misc.cu)
// Solve-kernel variants (the launch shapes the tuning table chooses between,
// tune.cpp). n <= 32: kVariantFold (two rows per lane: FP32-refined 512-thread
// blocks with in-kernel classic refinement, FP64 384-thread blocks),
// kVariantFoldNarrow (the same with 256-thread blocks and up to 255
// registers); FP32-refined also kVariantQuad (four rows per lane, 384-thread
// blocks, solve_quad.cu) and kVariantQuadNarrow (256-thread blocks), and for
// n 17-32 kVariantTile (four rows per lane reading a union matrix the block
// shares, solve_tile.cu; 384-thread blocks, one per SM) and kVariantTileNarrow
// (192-thread blocks, two per SM). n 33-64: kVariantWide (one warp per system,
// rows shifted in registers, rolled factorisation phases, solve_wide.cu) and
// kVariantFold (one warp per system, fully unrolled, 256-thread blocks).
enum SolveVariant : int
{
    kVariantDefault = 0,
    kVariantFold = 1,
    kVariantQuad = 2,
    kVariantFoldNarrow = 3,
    kVariantQuadNarrow = 4,
    kVariantTile = 5,
    kVariantTileNarrow = 6,
    kVariantWide = 7,
};
constexpr int kVariantCount = 8;
// the four-rows-per-lane FP32 kernels queue failing systems for classic refinement
inline bool is_quad_variant(int v)
{
    return v == kVariantQuad || v == kVariantQuadNarrow || v == kVariantTile || v == kVariantTileNarrow;
}
// the variant that runs for a (bucket, covariance type, precision) key
int solve_variant(int np, int cov_type, int precision);
// whether `variant` can run the key (kVariantDefault always can)
bool solve_variant_valid(int np, int precision, int variant);
// overrides one key; returns its previous setting, or -1 for an invalid key or variant
int set_solve_variant(int np, int cov_type, int precision, int variant);
// tuning mode (tune.cpp): a key without a setting is timed on its first bucket
// of at least kTuneMinItems systems; tune_record takes the ms per 1M systems
// of each variant (<= 0: not run) and sets the fastest
constexpr int kTuneMinItems = 20000;
bool tune_wanted(int np, int cov_type, int precision);
void tune_record(int np, int cov_type, int precision, const double *ms_per_variant);
cudaError_t launch_solve_bucket(int np, int precision, int variant, bool ordinary, const Geom &g, const int2 *cells,
                                const int *n_items, int max_items, const int2 *nb_rec, const int *nb_n, int ind_value,
                                const double *pair64, const float *pair32, double mean, double c0, int steps,
                                double tol, const SolveOut &out, int2 *esc_cells, int *esc_count, int n_sm,
                                cudaStream_t st);
size_t large_scratch_doubles(int k, int blocks);
cudaError_t launch_solve_large(const Geom &g, const int2 *cells, const int *n_items, int blocks, const int2 *nb_rec,
                               const int *nb_n, int ind_value, const double *pair64, bool ordinary, double mean,
                               double c0, double *scratch, const SolveOut &out, cudaStream_t st);

// misc (misc.cu)
void launch_build_pair(const Geom &g, const DevModel &m, int truncated, const double *search_vals, double *pair64,
                       float *pair32, cudaStream_t st);
// tiles of the stable bucket partition; tile_cnt holds kBuckets ints and tile_mom
// 3 kBuckets values per tile
long long prepare_tiles(long long n_cells);
void launch_prepare(const Geom &g, const uint8_t *mask, int all_cells, const int *nb_n, signed char *status,
                    int *bucket_cnt, int *bucket_off, int *tile_cnt, unsigned long long *tile_mom, int2 *cells,
                    unsigned long long *moments, cudaStream_t st);
void launch_finalize_cont(const Geom &g, const float *in_data, signed char *status, int simple, float mean_f,
                          const float *cell_mean, float *out_data, uint8_t *out_mask, double *est64, double *var,
                          cudaStream_t st);
void launch_ik_fail_fill(const Geom &g, const signed char *status, float marginal, int c, int m, float *probs,
                         cudaStream_t st);
void launch_ik_finalize(long long n_cells, int m, float *probs, uint8_t *out_data, uint8_t *out_mask,
                        cudaStream_t st);
void launch_sk_weights(const DevModel &m, const double *pts, int n, double *A, double *w, int *status,
                       cudaStream_t st);
void launch_mik_finalize(long long n_cells, const signed char *status, const double *est64, double marginal1,
                         uint8_t *out_data, uint8_t *out_mask, float *prob_out, cudaStream_t st);

// sequential Gaussian simulation (sgs.cu)
struct SgsWalk
{
    long long A, C, M, R0; // R <- (A R + C) mod M from R0 (a full-period walk)
};
constexpr int kSgsBlockMax = 160; // largest max_neighbours of the SGS solve
void launch_sgs_forward(long long n, float *data, const uint8_t *mask, const float *means_in, float *means_out,
                        const float *cv, const float *cp, long long cn, cudaStream_t st);
void launch_sgs_finalize(long long n, float *data, uint8_t *mask, const int *rank_of, int n_sim,
                         const signed char *st_rank, signed char *status, const float *cv, const float *cp,
                         long long cn, cudaStream_t st);
void launch_sgs_path(const SgsWalk &w, const uint8_t *mask, const uint8_t *sim_mask, int *path_cell, int *flag,
                     cudaStream_t st);
void launch_sgs_index(long long n, const int *path_cell, const int *flag, const int *scan, const uint8_t *mask,
                      int *rank_of, int *sim_cells, cudaStream_t st);
// Template scan with the rank predicate rank_of[q] < rank (or < fixed_rank when
// fixed_rank >= 0); nb_rank may be null.
void launch_sgs_search(const Geom &g, const int4 *tmpl, int n_tmpl, const int *sim_cells, int n_sim,
                       const int *rank_of, int k, int *nb, int *nb_rank, int *nb_cnt, int n_sm, cudaStream_t st,
                       int fixed_rank = -1, int rank_stride = 0);
// SIS (sgs.cu): one launch per level solves every (node, kriged category)
// system and draws each node's category when its last system is done
constexpr int kSisMaxCat = 16;
struct SisCat
{
    const double *pair64; // the category's pair table
    const int *nb;        // its neighbour cells, k per rank
    const int *nb_cnt;
    const float *means;   // LVM: the category's mean per cell, or null
    long long pair_center;
    int pnx, pny;
    int k;
    float marginal;       // the category's mean (float, as the reference stores it)
};
struct SisLevelArgs
{
    const SisCat *cats;  // kcat entries (device)
    int nx, ny;
    const int *order;    // the level's ranks
    int n_nodes;
    int kcat, ncat;
    const int *sim_cells;
    uint8_t *data;       // categories (the draws are written here)
    double *probs;       // per rank, kcat entries
    signed char *st_cat; // per rank, kcat entries
    int *done;           // per rank: systems finished (zeroed per call)
    const double *uniforms;
    signed char *st_rank;
    int correlogram;     // LVM correlogram weights (corellogramed_weights_3)
    int kmax;            // the largest k of the categories
};
cudaError_t launch_sis_level(const SisLevelArgs &a, int n_sm, cudaStream_t st);
void launch_sgs_levels(const int *nb_rank, const int *nb_cnt, int k, int n_sim, int *levp1, int *ticket,
                       int *level_count, int level_cap, int *max_level, int *err, int n_sm, cudaStream_t st);
void launch_sgs_moments(int n_sim, const int *nb_cnt, double *mom, int n_sm, cudaStream_t st); // mom: 3, zeroed
void launch_sgs_level_fill(int n_sim, const int *levp1, const int *level_off, int *level_fill, int *order,
                           cudaStream_t st);
size_t sgs_block_smem(int k);
cudaError_t launch_sgs_solve(const Geom &g, const int *order, int n_items, const int *sim_cells, const int *nb,
                             const int *nb_cnt, int k, const double *pair64, float *data, const float *means,
                             const double *uniforms, signed char *st_rank, bool ordinary, int n_sm, cudaStream_t st);

// collocated cokriging (cokriging.cu)
struct CokParams
{
    double coef;    // cross covariance = coef * cross_tab (Markov models I and II)
    double sec_var; // the secondary variance, A[n][n]
    double b_last;  // coef * C_cross(0), b[n]
    float pm, sm;   // primary and secondary means (float, as the reference stores them)
};
void launch_cok_prepare(long long n, const uint8_t *pmask, int *flag, cudaStream_t st);
void launch_cok_targets(long long n, const int *flag, const int *pos, int *targets, cudaStream_t st);
// cross_tab: the cross model over the +-radius box, x fastest
// nb_rec / nb_n: the kriging search's per-cell neighbour records and counts
cudaError_t launch_cok_solve(const Geom &g, const int *targets, int n_targets, const int2 *nb_rec, const int *nb_n,
                             int k, const double *pair64, const double *cross_tab, const float *pdata,
                             const float *sdata, const uint8_t *smask, const CokParams &p, float *out_data,
                             uint8_t *out_mask, signed char *status, int n_sm, cudaStream_t st);
void launch_cok_finalize(long long n, const float *pdata, const uint8_t *pmask, float *out_data, uint8_t *out_mask,
                         signed char *status, cudaStream_t st);
} // namespace hb
