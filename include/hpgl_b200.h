/*
 * hpgl_b200 — C ABI of the B200 kriging engine.
 *
 * Drop-in for the kriging entry points of HPGL's C API
 * (itohnobue/hpgl-reborn, src/geo_bsd/hpgl/api.h). The structs below are
 * laid out exactly as api.h:18-153 lays them out (same members, same order,
 * natural alignment), so the reference's ctypes bindings
 * (src/geo_bsd/hpgl_wrap.py:44-165) bind to this library unchanged.
 *
 * Ownership: every buffer belongs to the caller. Kriging entry points read
 * and write HOST memory (pinned or pageable) unless the `_ex` flag
 * HPGL_B200_DEVICE_POINTERS says the pointers are CUDA device pointers.
 * Nothing the caller can see is allocated by the library.
 *
 * Errors: the reference-compatible entry points return void (or 0/-1 where
 * the reference does) and keep the message of the last failure for
 * hpgl_get_last_exception_message (api.cpp:30-50). The `_ex` entry points
 * return 0 or a negative HPGL_B200_E* code and never abort.
 */
#ifndef HPGL_B200_H
#define HPGL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ structs */
/* api.h:18-22 */
struct hpgl_shape_t { int m_data[3]; int m_strides[3]; };
/* api.h:24-29 */
struct hpgl_cont_masked_array_t { float *m_data; unsigned char *m_mask; struct hpgl_shape_t m_shape; };
/* api.h:31-37 */
struct hpgl_ind_masked_array_t { unsigned char *m_data; unsigned char *m_mask; struct hpgl_shape_t m_shape; int m_indicator_count; };
/* api.h:51-60 */
struct hpgl_ok_params_t {
    int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget;
    int m_radiuses[3]; int m_max_neighbours;
};
/* api.h:62-73 */
struct hpgl_sk_params_t {
    int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget;
    int m_radiuses[3]; int m_max_neighbours; unsigned char m_automatic_mean; double m_mean;
};
/* api.h:75-82 */
struct hpgl_cov_params_t { int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget; };
/* api.h:98-108 */
struct hpgl_median_ik_params_t {
    int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget;
    int m_radiuses[3]; int m_max_neighbours; double m_marginal_probs[2];
};
/* api.h:110-120 */
struct hpgl_ik_params_t {
    int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget;
    int m_radiuses[3]; int m_max_neighbours; double m_marginal_prob;
};

/* api.h:39-43 */
struct hpgl_float_array_t { float *m_data; struct hpgl_shape_t m_shape; };
/* api.h:45-49 */
struct hpgl_ubyte_array_t { unsigned char *m_data; struct hpgl_shape_t m_shape; };
/* api.h:84-96 (m_kriging_kind 0 ordinary, 1 simple; m_min_neighbours is unused,
 * as in the reference) */
struct hpgl_sgs_params_t {
    int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget;
    int m_radiuses[3]; int m_max_neighbours; int m_kriging_kind; long m_seed; int m_min_neighbours;
};
/* api.h:122-135 */
struct hpgl_cokriging_m1_params_t {
    int m_covariance_type; double m_ranges[3]; double m_angles[3]; double m_sill; double m_nugget;
    int m_radiuses[3]; int m_max_neighbours; double m_primary_mean; double m_secondary_mean;
    double m_secondary_variance; double m_correlation_coef;
};
/* api.h:137-146 */
struct hpgl_cokriging_m2_params_t {
    struct hpgl_cov_params_t m_primary_cov_params; struct hpgl_cov_params_t m_secondary_cov_params;
    int m_radiuses[3]; int m_max_neighbours; double m_primary_mean; double m_secondary_mean;
    double m_correlation_coef;
};
/* api.h:148-153: ascending values with their cumulative probabilities */
struct hpgl_non_parametric_cdf_t { float *m_values; float *m_probs; long long m_size; };

/* -------------------------------------------------- reference-compatible ABI */
/* Replaces api.h:159-160 / api.cpp:38-41. */
char *hpgl_get_last_exception_message(void);
/* Replaces api.h:162-166 / output.cpp:58-68. Handlers run on the calling host
 * thread only, never from a CUDA callback. */
void hpgl_set_output_handler(int (*handler)(char *str, void *param), void *param);
void hpgl_set_progress_handler(int (*handler)(char *stage, int percentage, void *param), void *param);
/* Replaces api.h:168-169 / set_thread_num.cpp:22-33: the host-side worker
 * count used to build covariance tables (the kriging itself runs on the GPU). */
void hpgl_set_thread_num(int n_threads);
int hpgl_get_thread_num(void);

/* Replaces api.h:218-221 / api.cpp:253-293 (ordinary_kriging.cpp:14-48). */
void hpgl_ordinary_kriging(struct hpgl_cont_masked_array_t *input_data, struct hpgl_ok_params_t *params,
                           struct hpgl_cont_masked_array_t *output_data);
/* Replaces api.h:223-230 / api.cpp:323-354 (simple_kriging.cpp:89-124). */
void hpgl_simple_kriging(float *input_data, unsigned char *input_mask, struct hpgl_shape_t *input_data_shape,
                         struct hpgl_sk_params_t *params, float *output_data, unsigned char *output_mask,
                         struct hpgl_shape_t *output_data_shape);
/* Replaces api.h:232-240 / api.cpp:356-410 (simple_kriging.cpp:67-87). */
int hpgl_simple_kriging_weights(float *center_coords, float *neighbours_x, float *neighbours_y,
                                float *neighbours_z, int neighbours_count, struct hpgl_cov_params_t *params,
                                float *weights);
/* Replaces api.h:242-251 / api.cpp:412-455 (lvm_kriging.cpp:16-39): SK weights
 * around a locally varying mean, one float per grid cell; failures take the
 * cell's mean. mean_data_shape, when given, must have the input's volume (the
 * reference does not check it). */
void hpgl_lvm_kriging(float *input_data, unsigned char *input_mask, struct hpgl_shape_t *input_data_shape,
                      float *mean_data, struct hpgl_shape_t *mean_data_shape, struct hpgl_ok_params_t *params,
                      float *output_data, unsigned char *output_mask, struct hpgl_shape_t *output_data_shape);
/* Replaces api.h:267-272 / api.cpp:457-482 (indicator_kriging.h:88-161). */
void hpgl_indicator_kriging(struct hpgl_ind_masked_array_t *in_data, struct hpgl_ind_masked_array_t *out_data,
                            struct hpgl_ik_params_t *params, int indicator_count);
/* Replaces api.h:274-277 / api.cpp:552-601 (median_ik.cpp:24-89). */
void hpgl_median_ik(struct hpgl_ind_masked_array_t *in_data, struct hpgl_median_ik_params_t *params,
                    struct hpgl_ind_masked_array_t *out_data);

/* Replaces api.h:253-258 / api.cpp:484-516 (sequential_gaussian_simulation.cpp:18-77):
 * simulates, in place, every node of data that is not informed and whose
 * simulation_mask byte (when given) is 1. cdf (optional) maps the informed
 * values to the Gaussian space and the result back; `mean` is accepted and, as
 * in the reference, unused (SK runs around 0). Grids above 10,000,000 cells and
 * max_neighbours above 160 are rejected. */
void hpgl_sgs_simulation(struct hpgl_cont_masked_array_t *data, struct hpgl_sgs_params_t *params,
                         struct hpgl_non_parametric_cdf_t *cdf, double *mean,
                         struct hpgl_ubyte_array_t *simulation_mask);
/* Replaces api.h:260-265 / api.cpp:519-550 (sequential_gaussian_simulation.cpp:79-130):
 * SGS with SK weights around a locally varying mean (one float per cell,
 * mapped through cdf when given). */
void hpgl_sgs_lvm_simulation(struct hpgl_cont_masked_array_t *data, struct hpgl_sgs_params_t *params,
                             struct hpgl_non_parametric_cdf_t *cdf, struct hpgl_float_array_t *means,
                             struct hpgl_ubyte_array_t *simulation_mask);

/* Replaces api.h:297-303 / api.cpp:680-749 (simple_cokriging_markI.cpp:202-265):
 * simple collocated cokriging, Markov model I, of every uninformed primary
 * cell; every output cell ends informed (failures take pm + sv - sm). */
void hpgl_simple_cokriging_mark1(struct hpgl_cont_masked_array_t *input_data,
                                 struct hpgl_cont_masked_array_t *secondary_data,
                                 struct hpgl_cokriging_m1_params_t *params,
                                 struct hpgl_cont_masked_array_t *output_data);
/* Replaces api.h:304-310 / api.cpp:751-815 (simple_cokriging_markI.cpp:267-330):
 * Markov model II (the cross covariance from the secondary model). */
void hpgl_simple_cokriging_mark2(struct hpgl_cont_masked_array_t *primary_data,
                                 struct hpgl_cont_masked_array_t *secondary_data,
                                 struct hpgl_cokriging_m2_params_t *params,
                                 struct hpgl_cont_masked_array_t *output_data);

/* Replaces api.h:279-286 / api.cpp:603-635 (sequential_indicator_simulation.cpp:24-145):
 * sequential indicator simulation, in place, of every node of data that is not
 * informed and whose simulation_mask byte (when given) is 1; params: one entry
 * per category (two categories: median SIS, the first kriged). Grids whose
 * walk does not visit every node (2, 4, 6, 8, 12 cells), more than 16
 * categories and max_neighbours above 32 are rejected. */
void hpgl_sis_simulation(struct hpgl_ind_masked_array_t *data, struct hpgl_ik_params_t *params, int indicator_count,
                         int seed, struct hpgl_ubyte_array_t *simulation_mask);
/* Replaces api.h:288-296 / api.cpp:637-677 (sequential_indicator_simulation.cpp:147-183):
 * SIS around a locally varying mean per category (mean_data: indicator_count
 * arrays); use_correlograms != 0 selects the correlogram weights
 * (corellogramed_weights_3, my_kriging_weights.h:363-505: the SK system scaled
 * by sqrt(m (1 - m)) of each cell's mean). */
void hpgl_sis_simulation_lvm(struct hpgl_ind_masked_array_t *data, struct hpgl_ik_params_t *params,
                             struct hpgl_float_array_t *mean_data, int indicator_count, int seed,
                             struct hpgl_ubyte_array_t *simulation_mask, int use_correlograms);

/* Property files. Replace api.h:171-214 / api.cpp:53-252 (read_inc_file.cpp,
 * property_writer.cpp): the INC text format (a property-name line, then
 * whitespace-separated values, "--" comments to the end of a line, a "/"
 * terminator) and the GSLIB format. Readers return 0, or -1 with the message
 * in hpgl_get_last_exception_message (a "/" or a bad token among the first
 * `size` values, or a file with fewer values); the mask marks values other
 * than undefined_value. The byte reader maps values[j] to category j. */
int hpgl_read_inc_file_float(char *filename, float undefined_value, int size, float *data, unsigned char *mask);
int hpgl_read_inc_file_byte(char *filename, int undefined_value, int size, unsigned char *data, unsigned char *mask,
                            unsigned char *values, int values_count);
int hpgl_write_inc_file_float(char *filename, struct hpgl_cont_masked_array_t *arr, float undefined_value,
                              char *name);
int hpgl_write_inc_file_byte(char *filename, struct hpgl_ind_masked_array_t *arr, int undefined_value, char *name,
                             unsigned char *values, int values_count);
int hpgl_write_gslib_cont_property(struct hpgl_cont_masked_array_t *data, const char *filename, const char *name,
                                   double undefined_value);
int hpgl_write_gslib_byte_property(struct hpgl_ind_masked_array_t *data, const char *filename, const char *name,
                                   double undefined_value, unsigned char *values, int values_count);

/* ------------------------------------------------------------ _ex extensions */
/* status codes */
#define HPGL_B200_OK 0
#define HPGL_B200_EINVAL -1     /* bad argument (message says which) */
#define HPGL_B200_ECUDA -2      /* CUDA error, or no usable device */
#define HPGL_B200_ENOMEM -3     /* device memory exhausted */
#define HPGL_B200_ELIMIT -4     /* a size beyond what the engine supports */

/* precision modes */
#define HPGL_B200_FP64_PLAIN 0      /* FP64 assembly, factorisation and solve */
#define HPGL_B200_FP32_REFINED 1    /* FP32 assembly + factorisation, FP64-residual refinement */

/* flags */
#define HPGL_B200_DEVICE_POINTERS 1u   /* data/mask/outputs are device pointers */
#define HPGL_B200_OUT_IS_CLONE 2u      /* output arrays already hold a copy of the input */
#define HPGL_B200_EXACT_SEARCH 4u      /* select neighbours by exact ranks only (no float
                                          distance prefilter); same neighbours, slower */

/* per-cell status codes (written to `status` when non-null) */
#define HPGL_B200_CELL_INFORMED -1     /* conditioning cell, copied */
#define HPGL_B200_CELL_SUCCESS 0       /* kriged (KI_SUCCESS, kriging_interpolation.h:199-204) */
#define HPGL_B200_CELL_NO_NEIGHBOURS 1 /* KI_NO_NEIGHBOURS */
#define HPGL_B200_CELL_SINGULAR 2      /* KI_SINGULARITY: non-SPD factor or OK sum(A^-1 1) ~ 0 */

struct hpgl_b200_options_t {
    int precision;           /* HPGL_B200_FP64_PLAIN or HPGL_B200_FP32_REFINED */
    int refine_steps;        /* FP64-residual refinement steps for FP32_REFINED (1..4; 0 -> 2) */
    unsigned flags;          /* HPGL_B200_* flags */
    void *stream;            /* cudaStream_t to run on; NULL -> the engine's own stream */
    double *estimate64;      /* optional: FP64 estimate per cell (NaN where not kriged) */
    double *variance;        /* optional: kriging variance per cell (-1 where not kriged) */
    signed char *status;     /* optional: per-cell status (HPGL_B200_CELL_*) */
    float *ik_probs;         /* optional (IK): corrected probabilities, cell-major [cell][category] */
    double tolerance;        /* FP32_REFINED: accepted estimate of the remaining relative error of the
                                estimate/variance forms (0 -> 1e-9); systems above it are refined
                                further, then re-solved in FP64 */
};

/* OK / SK over a whole grid with options; dims = (nx, ny, nz), Fortran order.
 * kind 0 = ordinary (params from ok), 1 = simple (sk). The output arrays
 * follow the reference's rules (cont_kriging.h:63-117). */
int hpgl_b200_cont_kriging_ex(int kind, const int *dims, const float *in_data, const unsigned char *in_mask,
                              const struct hpgl_sk_params_t *params, float *out_data, unsigned char *out_mask,
                              const struct hpgl_b200_options_t *opt);
/* LVM kriging with options (hpgl_lvm_kriging's rules); mean_data holds one
 * float per cell, on the device when opt->flags has HPGL_B200_DEVICE_POINTERS. */
int hpgl_b200_lvm_kriging_ex(const int *dims, const float *in_data, const unsigned char *in_mask,
                             const float *mean_data, const struct hpgl_ok_params_t *params, float *out_data,
                             unsigned char *out_mask, const struct hpgl_b200_options_t *opt);
/* SGS with options (hpgl_sgs_simulation's rules): data and mask are updated in
 * place; sim_mask and means (LVM) are optional and, like data and mask, device
 * pointers under HPGL_B200_DEVICE_POINTERS; the cdf tables are host memory.
 * opt->status receives per cell -1 informed, 0 kriged, 1 no neighbours,
 * 2 singular (drawn from N(0,1)), 3 not simulated. */
int hpgl_b200_sgs_ex(const int *dims, float *data, unsigned char *mask, const unsigned char *sim_mask,
                     const struct hpgl_non_parametric_cdf_t *cdf, const float *means,
                     const struct hpgl_sgs_params_t *params, const struct hpgl_b200_options_t *opt);
/* Cokriging with options: mark 1 reads m1 (m2 may be NULL), mark 2 reads m2;
 * arrays of dims' volume (device pointers under HPGL_B200_DEVICE_POINTERS);
 * opt->status receives -1 informed, 0 kriged, 1 no neighbours, 2 singular. */
int hpgl_b200_cokriging_ex(int mark, const int *dims, const float *pdata, const unsigned char *pmask,
                           const float *sdata, const unsigned char *smask,
                           const struct hpgl_cokriging_m1_params_t *m1, const struct hpgl_cokriging_m2_params_t *m2,
                           float *out_data, unsigned char *out_mask, const struct hpgl_b200_options_t *opt);
/* SIS with options (hpgl_sis_simulation's rules): means, when not NULL, holds
 * indicator_count per-cell arrays (LVM, use_correlograms as for
 * hpgl_sis_simulation_lvm); arrays on the device under
 * HPGL_B200_DEVICE_POINTERS; opt->status as for hpgl_b200_sgs_ex (the largest
 * status over the node's categories). */
int hpgl_b200_sis_ex(const int *dims, unsigned char *data, unsigned char *mask, const unsigned char *sim_mask,
                     const struct hpgl_ik_params_t *params, int indicator_count, const float *const *means, int seed,
                     int use_correlograms, const struct hpgl_b200_options_t *opt);
/* The simulation's uniform draws (host): out[i] = the i-th call of
 * std::uniform_real_distribution<double>(0, 1) on a std::mt19937 seeded with
 * `seed` (bs_random_generator.cpp:9-25), as sgs_simulation consumes them, one
 * per simulated node in walk order. */
int hpgl_b200_sgs_draws(long long seed, long long n, double *out);
/* The dependency levels the simulations schedule by (no counterpart in HPGL):
 * for ranks r = 0 .. n_sim-1 with k listed ranks each (nb_rank, host, -1 for
 * none, every other entry in [0, n_sim)), levels[r] = 1 + the largest level of
 * its listed ranks, 0 with none. In a simulation each listed rank is below r;
 * a rank that lists itself or a later rank in a cycle waits, and after 2 s the
 * call returns HPGL_B200_ECUDA ("timed out") with the device still usable. */
int hpgl_b200_sim_levels(long long n_sim, int k, const int *nb_rank, int *levels);
/* Full IK (indicator_count > 2 categories, per-category models) or, with one
 * params entry and indicator_count == 2, median IK (median_ik.cpp:24-89). */
int hpgl_b200_indicator_kriging_ex(const int *dims, const unsigned char *in_data, const unsigned char *in_mask,
                                   const struct hpgl_ik_params_t *params, int indicator_count,
                                   unsigned char *out_data, unsigned char *out_mask,
                                   const struct hpgl_b200_options_t *opt);
int hpgl_b200_median_ik_ex(const int *dims, const unsigned char *in_data, const unsigned char *in_mask,
                           const struct hpgl_median_ik_params_t *params, unsigned char *out_data,
                           unsigned char *out_mask, const struct hpgl_b200_options_t *opt);

/* Neighbour lists exactly as indexed_neighbour_lookup_t::find returns them
 * (sugarbox_indexed_neighbour_lookup.h:67-124) for the listed nodes: node
 * indices, -1 padded to max_neighbours; `path` gets 1 where the template scan
 * ran. kind 0 = analytic covariance (OK), 1 = truncated table (SK / IK /
 * median IK). Host pointers. */
int hpgl_b200_find_neighbours(int kind, const int *dims, const unsigned char *mask,
                              const struct hpgl_sk_params_t *params, const int *nodes, int n_nodes,
                              int *out_idx, int *out_count, unsigned char *out_path);

/* Timing and counters of the last call on the current device's engine.
 * Writes up to `cap` doubles, returns how many:
 *   [0] total_ms (device, whole call)   [1] search_ms (stage)   [2] solve_ms (stage)
 *   [3] tie-resolved cells   [4] template-path cells   [5] kriged cells
 *   [6] kernel launches      [7] h2d bytes   [8] d2h bytes
 *   [9] cells re-solved in FP64 after FP32 refinement did not converge
 *   [10] neighbour-search kernel ms
 *   [11..15] cells per solve bucket (n <= 8, 16, 32, 64, > 64)
 *   [16..20] solve kernel ms per bucket
 *   [21..25] algorithmic flops per bucket, sum of F(n, r) =
 *            n^3/3 + n^2/2 + 2 r n^2 + 30 (n(n+1)/2 + n) + 2 r n (r = 2 OK, 1 SK)
 *   [26..35] ms per stage: upload, compaction, tables, binning, search, tie
 *            resolution, bucketing, solves, finalize, download
 *   [36] cells whose neighbours the float distance prefilter could not
 *        decide (selected by exact ranks over every candidate instead)
 *   [37] 1 when the float distance prefilter was active in the last search
 *   [38] host ms building the covariance tables (overlapped with the upload)
 *   [39] simulation: dependency levels (one solve launch each)
 *   [40] simulation: host ms generating the uniform draws (overlapped)
 *   [41] simulation: algorithmic flops of its kriging solves
 *   [42] FP32_REFINED systems whose first-order check failed in the
 *        four-rows-per-lane kernel and went to classic refinement */
#define HPGL_B200_STATS_LEN 43
int hpgl_b200_last_stats(double *out, int cap);

/* Solve-kernel variants (no counterpart in the reference: HPGL makes one
 * LAPACK call per node). Each (bucket, covariance type, precision) key runs
 * one launch shape: bucket_np 8, 16, 32 or 64 (neighbour counts up to it),
 * cov_type 0 spherical / 1 exponential / 2 Gaussian, precision
 * HPGL_B200_FP64_PLAIN or HPGL_B200_FP32_REFINED. Variants:
 *   HPGL_B200_VARIANT_DEFAULT      the built-in pick of the key
 *   HPGL_B200_VARIANT_FOLD         two rows per lane (FP32: 512-thread blocks,
 *                                  classic refinement in the kernel; FP64:
 *                                  384-thread blocks; bucket 64: one warp per
 *                                  system, 256-thread blocks)
 *   HPGL_B200_VARIANT_FOLD_NARROW  bucket_np <= 32: FOLD in 256-thread blocks
 *                                  (up to 255 registers a thread)
 *   HPGL_B200_VARIANT_QUAD         FP32_REFINED, bucket_np <= 32: four rows
 *                                  per lane, 384-thread blocks; failing systems
 *                                  go on to FOLD's refinement, then to FP64
 *   HPGL_B200_VARIANT_QUAD_NARROW  QUAD in 256-thread blocks
 *   HPGL_B200_VARIANT_TILE         FP32_REFINED, bucket_np == 32: QUAD reading
 *                                  the covariances from a union matrix that the
 *                                  block builds in shared memory for the 48
 *                                  consecutive cells it solves at once
 *   HPGL_B200_VARIANT_TILE_NARROW  TILE in 192-thread blocks, two a
 *                                  multiprocessor, 24 cells at once
 *   HPGL_B200_VARIANT_WIDE         bucket_np == 64 (the built-in pick): one
 *                                  warp per system, the factorisation's steps
 *                                  rolled in phases of eight over rows kept
 *                                  shifted in registers (FOLD is the same
 *                                  layout fully unrolled)
 * hpgl_b200_solve_variant sets a key and returns its previous setting, or
 * HPGL_B200_EINVAL for an invalid key or a variant the key cannot run;
 * hpgl_b200_solve_variant_get returns the variant a key runs now. Results of
 * every variant meet the precision's error bound; they differ in rounding. */
#define HPGL_B200_VARIANT_DEFAULT 0
#define HPGL_B200_VARIANT_FOLD 1
#define HPGL_B200_VARIANT_QUAD 2
#define HPGL_B200_VARIANT_FOLD_NARROW 3
#define HPGL_B200_VARIANT_QUAD_NARROW 4
#define HPGL_B200_VARIANT_TILE 5
#define HPGL_B200_VARIANT_TILE_NARROW 6
#define HPGL_B200_VARIANT_WIDE 7
int hpgl_b200_solve_variant(int bucket_np, int cov_type, int precision, int variant);
int hpgl_b200_solve_variant_get(int bucket_np, int cov_type, int precision);
/* The tuner behind those keys (no counterpart in the reference).
 * hpgl_b200_tune_mode(1): a key without a setting is timed the first time a
 * call meets a bucket of at least 20000 of its systems: that bucket runs with
 * every variant the key can run (twice each, the second run timed), the
 * fastest becomes the key's setting
 * and produces the call's outputs; mode 0 (the default) uses the settings as
 * they are. Returns the previous mode.
 * hpgl_b200_tune_load / hpgl_b200_tune_save read / write the settings as a
 * JSON list of {"np", "cov_type", "precision", "variant", "ms_per_million"}
 * objects (the timings, ms per million systems, are written for keys this
 * process timed); they return the number of keys, or HPGL_B200_EINVAL with
 * the message kept for hpgl_get_last_exception_message.
 * hpgl_b200_tune_reset puts every key back to its built-in pick. */
int hpgl_b200_tune_mode(int on);
int hpgl_b200_tune_load(const char *path);
int hpgl_b200_tune_save(const char *path);
void hpgl_b200_tune_reset(void);

/* No counterpart in the reference. The same SK weights as
 * hpgl_simple_kriging_weights for callers that cannot allocate device memory
 * while they run (device memory owned by another allocator, or a fixed budget
 * reserved up front): the system is solved in a fixed file-scope device array
 * (about 135 KB, held by every GPU that loads the library until exit), so the
 * call never allocates or frees device memory. At most 128 neighbours
 * (HPGL_B200_ELIMIT beyond). Calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller. The first call on a device
 * looks the array's address up (cudaGetSymbolAddress). With lazy module
 * loading (CUDA's default) that first call
 * is also when the device takes the array's memory, so it can fail on a full
 * device: make it before reserving a memory pool; later calls allocate
 * nothing. The call waits on `stream` for its own work before it returns.
 * Host pointers; `stream` may be NULL (the legacy stream).
 * Returns 0, or a negative HPGL_B200_E* code with the message kept for
 * hpgl_get_last_exception_message. */
int hpgl_b200_sk_weights_noalloc(const float *center_coords, const float *neighbours_x, const float *neighbours_y,
                                 const float *neighbours_z, int neighbours_count,
                                 const struct hpgl_cov_params_t *params, float *weights, void *stream);

/* Leave-one-out ordinary kriging of conditioning points, and its adjoint. No
 * counterpart in the reference (HPGL has no cross-validation and computes no
 * gradients); the system of each target is the reference's OK system
 * (ok_kriging_weights_3, my_kriging_weights.h:198-361) in FP64, its covariance
 * evaluated from M = diag(1/r0, 1/r1, 1/r2) Rx Ry Rz, the anisotropy transform of
 * cov_model.h:16-61 divided by ranges[0] (row-major, host pointer to 9 doubles),
 * with C = sill where r0 |M v| < 1e-4 (cov_model.h:146-183).
 *   pts_xyz  [n_pts][3] int grid coordinates, values [n_pts] (device)
 *   targets  [n_targets] point ids; nb_idx [n_targets][k] neighbour point ids
 *            (the target itself excluded), nb_cnt [n_targets] (device); k <= 32
 *   zhat     [n_targets] estimates; status (optional) 0 kriged, 1 no
 *            neighbours, 2 singular (estimate 0)
 * The adjoint takes dL/dzhat and ADDS dL/dvalues to grad_values [n_pts] and
 * dL/dM (9, row-major), dL/dsill, dL/dnugget to grad_params [11]; it recomputes
 * the factors, and targets with status != 0 contribute nothing. Device
 * pointers, work queued on `stream`. */
int hpgl_b200_loo_ok(const int *pts_xyz, const double *values, int n_pts, const int *targets, const int *nb_idx,
                     const int *nb_cnt, int n_targets, int k, int cov_type, const double *M, double r0, double sill,
                     double nugget, double *zhat, signed char *status, void *stream);
int hpgl_b200_loo_ok_adjoint(const int *pts_xyz, const double *values, int n_pts, const int *targets,
                             const int *nb_idx, const int *nb_cnt, int n_targets, int k, int cov_type,
                             const double *M, double r0, double sill, double nugget, const double *grad_zhat,
                             double *grad_values, double *grad_params, void *stream);

/* Page-locked host buffers for fast copies (cudaHostAlloc / cudaFreeHost). */
void *hpgl_b200_host_alloc(size_t bytes);
void hpgl_b200_host_free(void *p);

/* Host-side pieces, callable without a GPU. */
/* The anisotropy transform of cov_model.h:16-61 (row-major, 9 doubles). */
int hpgl_b200_transform(const double *ranges, const double *angles, double *out9);
/* The sorted search template of calc_cov_field (covariance_field.h:62-106):
 * up to `cap` (dx,dy,dz) triples; returns its length, limit = length / 250
 * (sugarbox_indexed_neighbour_lookup.h:59). kind as for find_neighbours. */
int hpgl_b200_template(int kind, const struct hpgl_cov_params_t *cov, const int *radiuses, int *out, int cap,
                       int *out_limit);
/* Covariance between two integer points for a flavour (kind as above). */
double hpgl_b200_covariance(int kind, const struct hpgl_cov_params_t *cov, const int *radiuses, const int *a,
                            const int *b);
/* Library version string. */
const char *hpgl_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif /* HPGL_B200_H */
