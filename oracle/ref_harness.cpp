// Test infrastructure only (never shipped, never on the product path).
//
// White-box harness around the reference's own kriging code, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libref_harness.so. It
// instantiates the reference templates exactly as its drivers do and exposes,
// per grid node:
//   * the neighbour indices chosen by indexed_neighbour_lookup_t::find
//     (src/geo_bsd/hpgl/sugarbox_indexed_neighbour_lookup.h:67-124), plus which
//     of the two search paths was taken (clusterizer.cpp:169-188);
//   * the FP64 estimate and kriging variance of kriging_interpolation
//     (kriging_interpolation.h:277-315) with result_t = double;
//   * the float estimate of the same call with result_t = float, which is what
//     cont_kriging (cont_kriging.h:82-83) stores.
// Covariance flavours follow the drivers: OK uses the analytic cov_model_t
// (ordinary_kriging.cpp:29-33), SK and IK the box-truncated
// precalculated_covariances_t (simple_kriging.cpp:113-115,
// indicator_kriging.h:101-103), median IK covariance_field_t (median_ik.cpp:233).
#include "stdafx.h"
#include "typedefs.h"
#include "sugarbox_grid.h"
#include "property_array.h"
#include "covariance_param.h"
#include "cov_model.h"
#include "precalculated_covariance.h"
#include "covariance_field.h"
#include "neighbourhood_param.h"
#include "sugarbox_indexed_neighbour_lookup.h"
#include "kriging_interpolation.h"
#include "mean_provider.h"
#include "is_informed_predicate.h"

#include <omp.h>
#include <cstring>
#include <memory>

using namespace hpgl;

namespace
{
enum harness_kind { K_OK = 0, K_SK = 1, K_MIK = 2 };

covariance_param_t make_cov(int cov_type, const double *ranges, const double *angles,
                            double sill, double nugget)
{
    covariance_param_t cp;
    cp.m_covariance_type = (covariance_type_t)cov_type;
    cp.set_ranges(ranges[0], ranges[1], ranges[2]);
    cp.set_angles(angles[0], angles[1], angles[2]);
    cp.m_sill = sill;
    cp.m_nugget = nugget;
    return cp;
}

neighbourhood_param_t make_nb(const int *radiuses, int max_nb)
{
    neighbourhood_param_t nb;
    nb.m_radiuses = sugarbox_search_ellipsoid_t(radiuses[0], radiuses[1], radiuses[2]);
    nb.m_max_neighbours = max_nb;
    return nb;
}

template <typename cov_t, typename values_t, typename prop_t, typename means_t, typename wc_t>
void run_nodes(const sugarbox_grid_t &grid, const cov_t &cov, const neighbourhood_param_t &nb,
               const values_t &values, const prop_t &defined_prop, const means_t &means,
               const wc_t &wc, const int *nodes, int n_nodes, int max_nb, int *out_idx,
               int *out_count, unsigned char *out_path, double *out_est, double *out_var,
               float *out_est_f, int *out_status, int n_threads)
{
    typedef indexed_neighbour_lookup_t<sugarbox_grid_t, cov_t> nl_t;
    nl_t nl(&grid, &cov, nb);
    for (node_index_t node = 0; node < defined_prop.size(); ++node)
        if (defined_prop.is_informed(node))
            nl.add_node(node);

    if (n_threads > 0)
        omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int t = 0; t < n_nodes; ++t)
    {
        node_index_t node = nodes[t];
        is_informed_predicate_t<prop_t> pred(defined_prop);
        if (out_idx || out_count)
        {
            std::vector<node_index_t> indices;
            std::vector<sugarbox_location_t> coords;
            sugarbox_location_t nc;
            nl.find(node, pred, nc, indices, coords);
            if (out_count)
                out_count[t] = (int)indices.size();
            if (out_idx)
                for (int i = 0; i < max_nb; ++i)
                    out_idx[(size_t)t * max_nb + i] = i < (int)indices.size() ? indices[i] : -1;
        }
        if (out_est || out_var || out_status)
        {
            double est = 0.0, var = -1.0;
            ki_result_t r = kriging_interpolation(values, pred, node, cov, means, nl, wc, est, var);
            if (out_est) out_est[t] = est;
            if (out_var) out_var[t] = var;
            if (out_status) out_status[t] = (int)r;
        }
        if (out_est_f)
        {
            float est_f = 0.0f;
            kriging_interpolation(values, pred, node, cov, means, nl, wc, est_f);
            out_est_f[t] = est_f;
        }
    }
    (void)out_path; // filled by run_paths
}

// Which search path indexed_neighbour_lookup_t::find takes for each node: the
// clusterizer's limit_exceeded test (clusterizer.cpp:169-188), evaluated with
// the same limit the lookup uses (sugarbox_indexed_neighbour_lookup.h:59).
template <typename cov_t, typename prop_t>
void run_paths(const sugarbox_grid_t &grid, const cov_t &cov, const neighbourhood_param_t &nb,
               const prop_t &defined_prop, const int *nodes, int n_nodes, unsigned char *out_path,
               int *out_template_size, int *out_limit)
{
    neighbour_lookup_t<sugarbox_grid_t, cov_t> tmpl(&grid, &cov, nb);
    std::vector<sugarbox_vector_t> vecs;
    calc_cov_field<cov_t, sugarbox_location_t>(nb.m_radiuses, cov, vecs);
    size_t limit = vecs.size() / detail::MAGIC_NUMBER_2;
    clusterizer_t cl(&grid, nb.m_radiuses, limit);
    for (node_index_t node = 0; node < defined_prop.size(); ++node)
        if (defined_prop.is_informed(node))
            cl.add_node(node);
    if (out_template_size) *out_template_size = (int)vecs.size();
    if (out_limit) *out_limit = (int)limit;
    if (out_path)
        for (int t = 0; t < n_nodes; ++t)
            out_path[t] = cl.limit_exceeded(nodes[t]) ? 1 : 0;
}
} // namespace

extern "C" {

// Continuous kriging (OK when kind == 0, SK when kind == 1) at the listed nodes.
// Any output pointer may be null. Returns 0, or -1 on a C++ exception.
int ref_krige_cont(int kind, const int *dims, const float *data, const unsigned char *mask,
                   int cov_type, const double *ranges, const double *angles, double sill,
                   double nugget, const int *radiuses, int max_nb, double mean,
                   const int *nodes, int n_nodes, int *out_idx, int *out_count,
                   unsigned char *out_path, double *out_est, double *out_var, float *out_est_f,
                   int *out_status, int n_threads)
{
    try
    {
        sugarbox_grid_t grid;
        grid.init(dims[0], dims[1], dims[2]);
        int size = dims[0] * dims[1] * dims[2];
        cont_property_array_t prop(const_cast<float *>(data), const_cast<unsigned char *>(mask), size);
        covariance_param_t cp = make_cov(cov_type, ranges, angles, sill, nugget);
        neighbourhood_param_t nb = make_nb(radiuses, max_nb);
        if (kind == K_OK)
        {
            cov_model_t cov(cp);
            run_nodes(grid, cov, nb, prop, prop, no_mean_t(), ok_weight_calculator_t(), nodes,
                      n_nodes, max_nb, out_idx, out_count, out_path, out_est, out_var, out_est_f,
                      out_status, n_threads);
            if (out_path) run_paths(grid, cov, nb, prop, nodes, n_nodes, out_path, 0, 0);
        }
        else
        {
            precalculated_covariances_t cov(cov_model_t(cp), nb.m_radiuses);
            run_nodes(grid, cov, nb, prop, prop, single_mean_t(mean), sk_weight_calculator_t(),
                      nodes, n_nodes, max_nb, out_idx, out_count, out_path, out_est, out_var,
                      out_est_f, out_status, n_threads);
            if (out_path) run_paths(grid, cov, nb, prop, nodes, n_nodes, out_path, 0, 0);
        }
        return 0;
    }
    catch (const std::exception &)
    {
        return -1;
    }
}

// LVM kriging at the listed nodes, instantiated as lvm_kriging does
// (lvm_kriging.cpp:28-34): truncated covariances, SK weights and the per-cell
// mean array itself as the mean provider.
int ref_krige_lvm(const int *dims, const float *data, const unsigned char *mask, const float *means,
                  int cov_type, const double *ranges, const double *angles, double sill, double nugget,
                  const int *radiuses, int max_nb, const int *nodes, int n_nodes, int *out_idx,
                  int *out_count, unsigned char *out_path, double *out_est, double *out_var,
                  float *out_est_f, int *out_status, int n_threads)
{
    try
    {
        sugarbox_grid_t grid;
        grid.init(dims[0], dims[1], dims[2]);
        int size = dims[0] * dims[1] * dims[2];
        cont_property_array_t prop(const_cast<float *>(data), const_cast<unsigned char *>(mask), size);
        covariance_param_t cp = make_cov(cov_type, ranges, angles, sill, nugget);
        neighbourhood_param_t nb = make_nb(radiuses, max_nb);
        precalculated_covariances_t cov(cov_model_t(cp), nb.m_radiuses);
        const mean_t *mp = means;
        run_nodes(grid, cov, nb, prop, prop, mp, sk_weight_calculator_t(), nodes, n_nodes, max_nb, out_idx,
                  out_count, out_path, out_est, out_var, out_est_f, out_status, n_threads);
        if (out_path) run_paths(grid, cov, nb, prop, nodes, n_nodes, out_path, 0, 0);
        return 0;
    }
    catch (const std::exception &)
    {
        return -1;
    }
}

// Indicator SK at the listed nodes for indicator value `ind_value`: IK per
// category (kind == 1, precalculated covariances, indicator_kriging.h:135) or
// median IK (kind == 2, covariance_field_t, median_ik.cpp:258-264).
int ref_krige_ind(int kind, const int *dims, const unsigned char *data, const unsigned char *mask,
                  int ind_value, int cov_type, const double *ranges, const double *angles,
                  double sill, double nugget, const int *radiuses, int max_nb, double mean,
                  const int *nodes, int n_nodes, int *out_idx, int *out_count,
                  unsigned char *out_path, double *out_est, double *out_var, float *out_est_f,
                  int *out_status, int n_threads)
{
    try
    {
        sugarbox_grid_t grid;
        grid.init(dims[0], dims[1], dims[2]);
        int size = dims[0] * dims[1] * dims[2];
        indicator_property_array_t prop(const_cast<unsigned char *>(data),
                                        const_cast<unsigned char *>(mask), size, 256);
        indicator_array_adapter_t adapter(&prop, (indicator_value_t)ind_value);
        covariance_param_t cp = make_cov(cov_type, ranges, angles, sill, nugget);
        neighbourhood_param_t nb = make_nb(radiuses, max_nb);
        if (kind == K_MIK)
        {
            covariance_field_t cov(nb.m_radiuses, cov_model_t(cp));
            run_nodes(grid, cov, nb, adapter, prop, single_mean_t(mean), sk_weight_calculator_t(),
                      nodes, n_nodes, max_nb, out_idx, out_count, out_path, out_est, out_var,
                      out_est_f, out_status, n_threads);
            if (out_path) run_paths(grid, cov, nb, prop, nodes, n_nodes, out_path, 0, 0);
        }
        else
        {
            precalculated_covariances_t cov(cov_model_t(cp), nb.m_radiuses);
            run_nodes(grid, cov, nb, adapter, prop, single_mean_t(mean), sk_weight_calculator_t(),
                      nodes, n_nodes, max_nb, out_idx, out_count, out_path, out_est, out_var,
                      out_est_f, out_status, n_threads);
            if (out_path) run_paths(grid, cov, nb, prop, nodes, n_nodes, out_path, 0, 0);
        }
        return 0;
    }
    catch (const std::exception &)
    {
        return -1;
    }
}

// The sorted search template of neighbour_lookup_t (calc_cov_field,
// covariance_field.h:62-106) for a covariance flavour (0 OK analytic,
// 1 precalculated, 2 covariance field). Writes up to `cap` offsets as
// (dx,dy,dz) triples; returns the template length and the clusterizer limit.
int ref_template(int kind, int cov_type, const double *ranges, const double *angles, double sill,
                 double nugget, const int *radiuses, int *out_offsets, int cap, int *out_limit)
{
    try
    {
        covariance_param_t cp = make_cov(cov_type, ranges, angles, sill, nugget);
        neighbourhood_param_t nb = make_nb(radiuses, 1);
        std::vector<sugarbox_vector_t> vecs;
        if (kind == K_OK)
        {
            cov_model_t cov(cp);
            calc_cov_field<cov_model_t, sugarbox_location_t>(nb.m_radiuses, cov, vecs);
        }
        else if (kind == K_SK)
        {
            precalculated_covariances_t cov(cov_model_t(cp), nb.m_radiuses);
            calc_cov_field<precalculated_covariances_t, sugarbox_location_t>(nb.m_radiuses, cov, vecs);
        }
        else
        {
            covariance_field_t cov(nb.m_radiuses, cov_model_t(cp));
            calc_cov_field<covariance_field_t, sugarbox_location_t>(nb.m_radiuses, cov, vecs);
        }
        for (int i = 0; i < (int)vecs.size() && i < cap; ++i)
        {
            out_offsets[3 * i + 0] = vecs[i][0];
            out_offsets[3 * i + 1] = vecs[i][1];
            out_offsets[3 * i + 2] = vecs[i][2];
        }
        if (out_limit) *out_limit = (int)(vecs.size() / detail::MAGIC_NUMBER_2);
        return (int)vecs.size();
    }
    catch (const std::exception &)
    {
        return -1;
    }
}

// Covariance between two integer points for a flavour, as the reference evaluates it.
double ref_cov(int kind, int cov_type, const double *ranges, const double *angles, double sill,
               double nugget, const int *radiuses, const int *c1, const int *c2)
{
    covariance_param_t cp = make_cov(cov_type, ranges, angles, sill, nugget);
    sugarbox_location_t a(c1[0], c1[1], c1[2]), b(c2[0], c2[1], c2[2]);
    if (kind == K_OK)
        return cov_model_t(cp)(a, b);
    sugarbox_search_ellipsoid_t r(radiuses[0], radiuses[1], radiuses[2]);
    if (kind == K_SK)
        return precalculated_covariances_t(cov_model_t(cp), r)(a, b);
    return covariance_field_t(r, cov_model_t(cp))(a, b);
}

// The 3x3 anisotropy transform (cov_model.h:16-61), row-major.
int ref_transform(const double *ranges, const double *angles, double *out9)
{
    try
    {
        std::vector<double> t;
        create_transform(ranges, angles, t);
        for (int i = 0; i < 9; ++i) out9[i] = t[i];
        return 0;
    }
    catch (const std::exception &)
    {
        return -1;
    }
}

// Single-system SK weights (simple_kriging.cpp:67-87 via sk_kriging_weights_3
// with real coordinates). Returns 1 on success, 0 on failure.
int ref_sk_weights(const double *center, const double *xs, const double *ys, const double *zs,
                   int n, int cov_type, const double *ranges, const double *angles, double sill,
                   double nugget, double *out_w, double *out_var)
{
    covariance_param_t cp = make_cov(cov_type, ranges, angles, sill, nugget);
    cov_model_t cov(cp);
    real_location_t c(center[0], center[1], center[2]);
    std::vector<real_location_t> pts(n);
    for (int i = 0; i < n; ++i) pts[i] = real_location_t(xs[i], ys[i], zs[i]);
    std::vector<kriging_weight_t> w;
    double var = -1;
    bool ok = sk_kriging_weights_3<cov_model_t, true, real_location_t>(c, pts, cov, w, var);
    for (int i = 0; i < n && ok; ++i) out_w[i] = w[i];
    if (out_var) *out_var = var;
    return ok ? 1 : 0;
}

} // extern "C"
