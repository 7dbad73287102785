// The C ABI declared in include/hpgl_b200.h. Reference-compatible entry
// points keep HPGL's conventions (api.cpp:30-50): void returns, the message of
// the last failure kept for hpgl_get_last_exception_message; nothing aborts.
#include "../../include/hpgl_b200.h"
#include "engine_api.h"
#include "host_model.h"

#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{
std::mutex g_handler_mu;
int (*g_output)(char *, void *) = nullptr;
void *g_output_param = nullptr;
int (*g_progress)(char *, int, void *) = nullptr;
void *g_progress_param = nullptr;

void emit(const std::string &s)
{
    std::lock_guard<std::mutex> lk(g_handler_mu);
    if (g_output)
    {
        std::vector<char> buf(s.begin(), s.end());
        buf.push_back(0);
        g_output(buf.data(), g_output_param);
    }
    else
    {
        fputs(s.c_str(), stdout);
        fflush(stdout);
    }
}

void progress(const char *stage, int pct)
{
    std::lock_guard<std::mutex> lk(g_handler_mu);
    if (g_progress)
    {
        std::string s(stage);
        std::vector<char> buf(s.begin(), s.end());
        buf.push_back(0);
        g_progress(buf.data(), pct, g_progress_param);
    }
}

// get_shape_volume (api_helpers.cpp:29-42)
bool shape_dims(const hpgl_shape_t *sh, int *dims)
{
    if (!sh) return false;
    long long v = 1;
    for (int i = 0; i < 3; ++i)
    {
        dims[i] = sh->m_data[i];
        v *= sh->m_data[i];
    }
    if (v > INT_MAX || v <= 0)
    {
        hb::set_error("get_shape_volume: grid volume exceeds INT_MAX");
        return false;
    }
    return true;
}

hb::SkArgs sk_args_from(const hpgl_sk_params_t *p)
{
    hb::SkArgs a{};
    a.cov_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        a.ranges[i] = p->m_ranges[i];
        a.angles[i] = p->m_angles[i];
        a.radiuses[i] = p->m_radiuses[i];
    }
    a.sill = p->m_sill;
    a.nugget = p->m_nugget;
    a.max_nb = p->m_max_neighbours;
    a.auto_mean = p->m_automatic_mean != 0;
    a.mean = p->m_mean;
    return a;
}

hb::SkArgs ok_args_from(const hpgl_ok_params_t *p)
{
    hb::SkArgs a{};
    a.cov_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        a.ranges[i] = p->m_ranges[i];
        a.angles[i] = p->m_angles[i];
        a.radiuses[i] = p->m_radiuses[i];
    }
    a.sill = p->m_sill;
    a.nugget = p->m_nugget;
    a.max_nb = p->m_max_neighbours;
    a.auto_mean = false;
    a.mean = 0;
    return a;
}

hb::IkArgs ik_args_from(const hpgl_ik_params_t *p)
{
    hb::IkArgs a{};
    a.cov_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        a.ranges[i] = p->m_ranges[i];
        a.angles[i] = p->m_angles[i];
        a.radiuses[i] = p->m_radiuses[i];
    }
    a.sill = p->m_sill;
    a.nugget = p->m_nugget;
    a.max_nb = p->m_max_neighbours;
    a.marginal = p->m_marginal_prob;
    return a;
}

hb::SgsArgs sgs_args_from(const hpgl_sgs_params_t *p)
{
    hb::SgsArgs a{};
    a.cov_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        a.ranges[i] = p->m_ranges[i];
        a.angles[i] = p->m_angles[i];
        a.radiuses[i] = p->m_radiuses[i];
    }
    a.sill = p->m_sill;
    a.nugget = p->m_nugget;
    a.max_nb = p->m_max_neighbours;
    a.kind = p->m_kriging_kind;
    a.seed = p->m_seed;
    return a;
}

hb::CovArgs cov_args_from(const hpgl_cov_params_t *p)
{
    hb::CovArgs c{};
    c.cov_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        c.ranges[i] = p->m_ranges[i];
        c.angles[i] = p->m_angles[i];
    }
    c.sill = p->m_sill;
    c.nugget = p->m_nugget;
    return c;
}

bool cok_args_from(int mark, const hpgl_cokriging_m1_params_t *m1, const hpgl_cokriging_m2_params_t *m2,
                   hb::CokArgs &a)
{
    a = hb::CokArgs{};
    a.mark = mark;
    if (mark == 1 && m1)
    {
        a.primary.cov_type = m1->m_covariance_type;
        for (int i = 0; i < 3; ++i)
        {
            a.primary.ranges[i] = m1->m_ranges[i];
            a.primary.angles[i] = m1->m_angles[i];
            a.radiuses[i] = m1->m_radiuses[i];
        }
        a.primary.sill = m1->m_sill;
        a.primary.nugget = m1->m_nugget;
        a.secondary = a.primary;
        a.max_nb = m1->m_max_neighbours;
        a.primary_mean = m1->m_primary_mean;
        a.secondary_mean = m1->m_secondary_mean;
        a.secondary_variance = m1->m_secondary_variance;
        a.corr = m1->m_correlation_coef;
        return true;
    }
    if (mark == 2 && m2)
    {
        a.primary = cov_args_from(&m2->m_primary_cov_params);
        a.secondary = cov_args_from(&m2->m_secondary_cov_params);
        for (int i = 0; i < 3; ++i) a.radiuses[i] = m2->m_radiuses[i];
        a.max_nb = m2->m_max_neighbours;
        a.primary_mean = m2->m_primary_mean;
        a.secondary_mean = m2->m_secondary_mean;
        a.corr = m2->m_correlation_coef;
        return true;
    }
    return false;
}

// the size checks of api.cpp:690-706
bool cok_shapes(const char *fn, const hpgl_shape_t *a, const hpgl_shape_t *b, const hpgl_shape_t *c, int *dims)
{
    int d2[3], d3[3];
    if (!shape_dims(a, dims) || !shape_dims(b, d2) || !shape_dims(c, d3)) return false;
    const long long s1 = (long long)dims[0] * dims[1] * dims[2], s2 = (long long)d2[0] * d2[1] * d2[2],
                    s3 = (long long)d3[0] * d3[1] * d3[2];
    if (s1 != s2)
    {
        hb::set_error(std::string(fn) + ": Size of secondary data (" + std::to_string(s2) +
                      ") is different from size of primary data (" + std::to_string(s1) + ")");
        return false;
    }
    if (s1 != s3)
    {
        hb::set_error(std::string(fn) + ": Size of output data (" + std::to_string(s3) +
                      ") is different from size of primary data (" + std::to_string(s1) + ")");
        return false;
    }
    return true;
}

// init_remap_table (api.cpp:143-167): the given values when there is one per
// indicator (the first indicator_count of more, with a warning), else 0, 1, 2 ...
std::vector<unsigned char> remap_table(const unsigned char *values, int values_count, int indicator_count)
{
    std::vector<unsigned char> t;
    if (values_count == indicator_count)
        t.assign(values, values + values_count);
    else if (values_count > indicator_count)
    {
        emit("Given " + std::to_string(values_count) + " values for " + std::to_string(indicator_count) +
             " indicators. Ignoring extra values.\n");
        t.assign(values, values + indicator_count);
    }
    else
    {
        if (values_count > 0)
            emit("Warning: Given " + std::to_string(values_count) + " values for " + std::to_string(indicator_count) +
                 " indicators. Ignoring values. Using [0, 1, 2 ..]\n");
        for (int i = 0; i < indicator_count; ++i) t.push_back((unsigned char)i);
    }
    return t;
}

hb::Options options_from(const hpgl_b200_options_t *o)
{
    hb::Options r;
    if (!o) return r;
    r.precision = o->precision;
    r.refine_steps = o->refine_steps;
    r.flags = o->flags;
    r.stream = o->stream;
    r.estimate64 = o->estimate64;
    r.variance = o->variance;
    r.status = o->status;
    r.ik_probs = o->ik_probs;
    r.tolerance = o->tolerance;
    return r;
}

void report_done(const char *algo)
{
    hb::Stats s = hb::last_stats();
    char buf[256];
    double secs = s.total_ms / 1000.0;
    snprintf(buf, sizeof(buf), "%s done on the GPU. Average speed: %.0f point/sec.\n", algo,
             secs > 0 ? (double)s.kriged / secs : 0.0);
    emit(buf);
    progress(algo, 100);
}
} // namespace

extern "C" {

char *hpgl_get_last_exception_message(void) { return const_cast<char *>(hb::last_error()); }

void hpgl_set_output_handler(int (*handler)(char *, void *), void *param)
{
    std::lock_guard<std::mutex> lk(g_handler_mu);
    g_output = handler;
    g_output_param = param;
}

void hpgl_set_progress_handler(int (*handler)(char *, int, void *), void *param)
{
    std::lock_guard<std::mutex> lk(g_handler_mu);
    g_progress = handler;
    g_progress_param = param;
}

void hpgl_set_thread_num(int n_threads) { hb::set_threads(n_threads); }
int hpgl_get_thread_num(void) { return hb::get_threads(); }

void hpgl_ordinary_kriging(hpgl_cont_masked_array_t *input_data, hpgl_ok_params_t *params,
                           hpgl_cont_masked_array_t *output_data)
{
    if (!input_data || !params || !output_data)
    {
        hb::set_error("hpgl_ordinary_kriging: null argument");
        return;
    }
    int dims[3];
    if (!shape_dims(&input_data->m_shape, dims)) return;
    hb::Options opt;
    progress("Ordinary Kriging", 0);
    if (hb::cont_kriging(0, dims, input_data->m_data, input_data->m_mask, ok_args_from(params), output_data->m_data,
                         output_data->m_mask, opt) == 0)
        report_done("Ordinary Kriging");
}

void hpgl_simple_kriging(float *input_data, unsigned char *input_mask, hpgl_shape_t *input_data_shape,
                         hpgl_sk_params_t *params, float *output_data, unsigned char *output_mask,
                         hpgl_shape_t *output_data_shape)
{
    (void)output_data_shape;
    if (!params)
    {
        hb::set_error("hpgl_simple_kriging: null argument");
        return;
    }
    int dims[3];
    if (!shape_dims(input_data_shape, dims)) return;
    hb::Options opt;
    progress("Simple Kriging", 0);
    if (hb::cont_kriging(1, dims, input_data, input_mask, sk_args_from(params), output_data, output_mask, opt) == 0)
        report_done("Simple Kriging");
}

void hpgl_lvm_kriging(float *input_data, unsigned char *input_mask, hpgl_shape_t *input_data_shape,
                      float *mean_data, hpgl_shape_t *mean_data_shape, hpgl_ok_params_t *params, float *output_data,
                      unsigned char *output_mask, hpgl_shape_t *output_data_shape)
{
    (void)output_data_shape;
    if (!params || !mean_data)
    {
        hb::set_error("hpgl_lvm_kriging: null argument");
        return;
    }
    int dims[3], mdims[3];
    if (!shape_dims(input_data_shape, dims)) return;
    if (mean_data_shape)
    {
        if (!shape_dims(mean_data_shape, mdims)) return;
        if ((long long)mdims[0] * mdims[1] * mdims[2] != (long long)dims[0] * dims[1] * dims[2])
        {
            hb::set_error("hpgl_lvm_kriging: mean and input size mismatch");
            return;
        }
    }
    hb::Options opt;
    progress("LVM Kriging", 0);
    if (hb::cont_kriging(2, dims, input_data, input_mask, ok_args_from(params), output_data, output_mask, opt,
                         mean_data) == 0)
        report_done("LVM Kriging");
}

void hpgl_sgs_simulation(hpgl_cont_masked_array_t *data, hpgl_sgs_params_t *params, hpgl_non_parametric_cdf_t *cdf,
                         double *mean, hpgl_ubyte_array_t *simulation_mask)
{
    (void)mean; // sequential_gaussian_simulation.cpp:39-41: SK runs around 0 whatever the mean
    if (!data || !params)
    {
        hb::set_error("hpgl_sgs_simulation: null argument");
        return;
    }
    int dims[3];
    if (!shape_dims(&data->m_shape, dims)) return;
    hb::CdfTable t;
    if (cdf) t = {cdf->m_values, cdf->m_probs, cdf->m_size};
    hb::Options opt;
    progress("Sequential Gaussian Simulation", 0);
    if (hb::sgs_simulation(dims, data->m_data, data->m_mask, simulation_mask ? simulation_mask->m_data : nullptr,
                           cdf ? &t : nullptr, nullptr, sgs_args_from(params), opt) == 0)
        report_done("Sequential Gaussian Simulation");
}

void hpgl_sgs_lvm_simulation(hpgl_cont_masked_array_t *data, hpgl_sgs_params_t *params,
                             hpgl_non_parametric_cdf_t *cdf, hpgl_float_array_t *means,
                             hpgl_ubyte_array_t *simulation_mask)
{
    if (!data || !params || !means || !means->m_data)
    {
        hb::set_error("hpgl_sgs_lvm_simulation: null argument");
        return;
    }
    int dims[3];
    if (!shape_dims(&data->m_shape, dims)) return;
    hb::CdfTable t;
    if (cdf) t = {cdf->m_values, cdf->m_probs, cdf->m_size};
    hb::Options opt;
    progress("Sequential Gaussian Simulation with Local Varying Mean", 0);
    if (hb::sgs_simulation(dims, data->m_data, data->m_mask, simulation_mask ? simulation_mask->m_data : nullptr,
                           cdf ? &t : nullptr, means->m_data, sgs_args_from(params), opt) == 0)
        report_done("Sequential Gaussian Simulation with Local Varying Mean");
}

void hpgl_simple_cokriging_mark1(hpgl_cont_masked_array_t *input_data, hpgl_cont_masked_array_t *secondary_data,
                                 hpgl_cokriging_m1_params_t *params, hpgl_cont_masked_array_t *output_data)
{
    if (!input_data || !secondary_data || !params || !output_data)
    {
        hb::set_error("hpgl_simple_cokriging_mark1: null argument");
        return;
    }
    int dims[3];
    if (!cok_shapes("hpgl_simple_cokriging_mark1", &input_data->m_shape, &secondary_data->m_shape,
                    &output_data->m_shape, dims))
        return;
    hb::CokArgs a;
    cok_args_from(1, params, nullptr, a);
    hb::Options opt;
    progress("Simple Colocated Cokriging Markov Model I", 0);
    if (hb::cokriging(dims, input_data->m_data, input_data->m_mask, secondary_data->m_data, secondary_data->m_mask,
                      a, output_data->m_data, output_data->m_mask, opt) == 0)
        report_done("Simple Colocated Cokriging Markov Model I");
}

void hpgl_simple_cokriging_mark2(hpgl_cont_masked_array_t *primary_data, hpgl_cont_masked_array_t *secondary_data,
                                 hpgl_cokriging_m2_params_t *params, hpgl_cont_masked_array_t *output_data)
{
    if (!primary_data || !secondary_data || !params || !output_data)
    {
        hb::set_error("hpgl_simple_cokriging_mark2: null argument");
        return;
    }
    int dims[3];
    if (!cok_shapes("hpgl_simple_cokriging_mark2", &primary_data->m_shape, &secondary_data->m_shape,
                    &output_data->m_shape, dims))
        return;
    hb::CokArgs a;
    cok_args_from(2, nullptr, params, a);
    hb::Options opt;
    progress("Simple Colocated Cokriging Markov Model II", 0);
    if (hb::cokriging(dims, primary_data->m_data, primary_data->m_mask, secondary_data->m_data,
                      secondary_data->m_mask, a, output_data->m_data, output_data->m_mask, opt) == 0)
        report_done("Simple Colocated Cokriging Markov Model II");
}

int hpgl_read_inc_file_float(char *filename, float undefined_value, int size, float *data, unsigned char *mask)
{
    try
    {
        if (!filename || !data || size < 0) throw std::runtime_error("hpgl_read_inc_file_float: bad argument");
        hb::read_inc_float(filename, undefined_value, size, data, mask);
        return 0;
    }
    catch (const std::exception &ex)
    {
        hb::set_error(ex.what());
        return -1;
    }
}

int hpgl_read_inc_file_byte(char *filename, int undefined_value, int size, unsigned char *data, unsigned char *mask,
                            unsigned char *values, int values_count)
{
    try
    {
        if (!filename || !data || !mask || size < 0 || (values_count > 0 && !values))
            throw std::runtime_error("hpgl_read_inc_file_byte: bad argument");
        hb::read_inc_byte(filename, undefined_value, size, data, mask);
        // values -> category indices (api.cpp:95-108): the first matching entry
        for (int i = 0; i < size; ++i)
            if (mask[i] != 0)
                for (int j = 0; j < values_count; ++j)
                    if (data[i] == values[j])
                    {
                        data[i] = (unsigned char)j;
                        break;
                    }
        return 0;
    }
    catch (const std::exception &ex)
    {
        hb::set_error(ex.what());
        return -1;
    }
}

int hpgl_write_inc_file_float(char *filename, hpgl_cont_masked_array_t *arr, float undefined_value, char *name)
{
    try
    {
        if (!filename || !arr || !name) throw std::runtime_error("hpgl_write_inc_file_float: bad argument");
        int dims[3];
        if (!shape_dims(&arr->m_shape, dims)) return -1;
        hb::write_inc_float(filename, name, arr->m_data, arr->m_mask, (long long)dims[0] * dims[1] * dims[2],
                            undefined_value, false);
        return 0;
    }
    catch (const std::exception &ex)
    {
        hb::set_error(ex.what());
        return -1;
    }
}

int hpgl_write_inc_file_byte(char *filename, hpgl_ind_masked_array_t *arr, int undefined_value, char *name,
                             unsigned char *values, int values_count)
{
    try
    {
        if (!filename || !arr || !name) throw std::runtime_error("hpgl_write_inc_file_byte: bad argument");
        int dims[3];
        if (!shape_dims(&arr->m_shape, dims)) return -1;
        hb::write_inc_byte(filename, name, arr->m_data, arr->m_mask, (long long)dims[0] * dims[1] * dims[2],
                           (unsigned char)undefined_value, remap_table(values, values_count, arr->m_indicator_count),
                           false);
        return 0;
    }
    catch (const std::exception &ex)
    {
        hb::set_error(ex.what());
        return -1;
    }
}

int hpgl_write_gslib_cont_property(hpgl_cont_masked_array_t *data, const char *filename, const char *name,
                                   double undefined_value)
{
    try
    {
        if (!filename || !data || !name) throw std::runtime_error("hpgl_write_gslib_cont_property: bad argument");
        int dims[3];
        if (!shape_dims(&data->m_shape, dims)) return -1;
        // the undefined value passes through cont_value_t (float), property_writer.cpp:95-99
        hb::write_inc_float(filename, name, data->m_data, data->m_mask, (long long)dims[0] * dims[1] * dims[2],
                            (float)undefined_value, true);
        return 0;
    }
    catch (const std::exception &ex)
    {
        hb::set_error(ex.what());
        return -1;
    }
}

int hpgl_write_gslib_byte_property(hpgl_ind_masked_array_t *data, const char *filename, const char *name,
                                   double undefined_value, unsigned char *values, int values_count)
{
    try
    {
        if (!filename || !data || !name) throw std::runtime_error("hpgl_write_gslib_byte_property: bad argument");
        int dims[3];
        if (!shape_dims(&data->m_shape, dims)) return -1;
        hb::write_inc_byte(filename, name, data->m_data, data->m_mask, (long long)dims[0] * dims[1] * dims[2],
                           (unsigned char)undefined_value, remap_table(values, values_count, data->m_indicator_count),
                           true);
        return 0;
    }
    catch (const std::exception &ex)
    {
        hb::set_error(ex.what());
        return -1;
    }
}

void hpgl_sis_simulation(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, int indicator_count, int seed,
                         hpgl_ubyte_array_t *simulation_mask)
{
    if (!data || !params || indicator_count <= 0)
    {
        hb::set_error("hpgl_sis_simulation: bad argument");
        return;
    }
    int dims[3];
    if (!shape_dims(&data->m_shape, dims)) return;
    std::vector<hb::IkArgs> cats;
    for (int i = 0; i < indicator_count; ++i) cats.push_back(ik_args_from(params + i));
    hb::Options opt;
    progress("Sequential Indicator Simulation", 0);
    if (hb::sis_simulation(dims, data->m_data, data->m_mask, simulation_mask ? simulation_mask->m_data : nullptr,
                           cats, nullptr, seed, opt) == 0)
        report_done("Sequential Indicator Simulation");
}

void hpgl_sis_simulation_lvm(hpgl_ind_masked_array_t *data, hpgl_ik_params_t *params, hpgl_float_array_t *mean_data,
                             int indicator_count, int seed, hpgl_ubyte_array_t *simulation_mask,
                             int use_correlograms)
{
    if (!data || !params || !mean_data || indicator_count <= 0)
    {
        hb::set_error("hpgl_sis_simulation_lvm: bad argument");
        return;
    }
    int dims[3];
    if (!shape_dims(&data->m_shape, dims)) return;
    std::vector<hb::IkArgs> cats;
    std::vector<const float *> means;
    for (int i = 0; i < indicator_count; ++i)
    {
        cats.push_back(ik_args_from(params + i));
        means.push_back(mean_data[i].m_data);
    }
    hb::Options opt;
    progress("Sequential Indicator Simulation", 0);
    if (hb::sis_simulation(dims, data->m_data, data->m_mask, simulation_mask ? simulation_mask->m_data : nullptr,
                           cats, means.data(), seed, opt, use_correlograms != 0) == 0)
        report_done("Sequential Indicator Simulation");
}

int hpgl_simple_kriging_weights(float *center_coords, float *neighbours_x, float *neighbours_y,
                                float *neighbours_z, int neighbours_count, hpgl_cov_params_t *params,
                                float *weights)
{
    if (!center_coords || !params || !weights || neighbours_count < 0)
    {
        hb::set_error("hpgl_simple_kriging_weights: bad argument");
        return -1;
    }
    const int n = neighbours_count;
    double c[3] = {center_coords[0], center_coords[1], center_coords[2]};
    std::vector<double> xs(n), ys(n), zs(n), w(n);
    for (int i = 0; i < n; ++i)
    {
        xs[i] = neighbours_x[i];
        ys[i] = neighbours_y[i];
        zs[i] = neighbours_z[i];
    }
    int rc = hb::sk_weights(c, xs.data(), ys.data(), zs.data(), n, params->m_covariance_type, params->m_ranges,
                            params->m_angles, params->m_sill, params->m_nugget, w.data());
    if (rc != 0) return -1;
    for (int i = 0; i < n; ++i) weights[i] = (float)w[i];
    return 0;
}

void hpgl_indicator_kriging(hpgl_ind_masked_array_t *in_data, hpgl_ind_masked_array_t *out_data,
                            hpgl_ik_params_t *params, int indicator_count)
{
    if (!in_data || !out_data || !params || indicator_count <= 0)
    {
        hb::set_error("hpgl_indicator_kriging: bad argument");
        return;
    }
    int dims[3], dims2[3];
    if (!shape_dims(&in_data->m_shape, dims) || !shape_dims(&out_data->m_shape, dims2)) return;
    if ((long long)dims[0] * dims[1] * dims[2] != (long long)dims2[0] * dims2[1] * dims2[2])
    {
        hb::set_error("hpgl_indicator_kriging: input and output size mismatch");
        return;
    }
    std::vector<hb::IkArgs> cats;
    for (int i = 0; i < indicator_count; ++i) cats.push_back(ik_args_from(params + i));
    hb::Options opt;
    progress("Indicator Kriging", 0);
    if (hb::indicator_kriging(dims, in_data->m_data, in_data->m_mask, cats, out_data->m_data, out_data->m_mask,
                              opt) == 0)
        report_done("Indicator Kriging");
}

void hpgl_median_ik(hpgl_ind_masked_array_t *in_data, hpgl_median_ik_params_t *params,
                    hpgl_ind_masked_array_t *out_data)
{
    if (!in_data || !out_data || !params)
    {
        hb::set_error("hpgl_median_ik: bad argument");
        return;
    }
    int dims[3];
    if (!shape_dims(&in_data->m_shape, dims)) return;
    hb::IkArgs a{};
    a.cov_type = params->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        a.ranges[i] = params->m_ranges[i];
        a.angles[i] = params->m_angles[i];
        a.radiuses[i] = params->m_radiuses[i];
    }
    a.sill = params->m_sill;
    a.nugget = params->m_nugget;
    a.max_nb = params->m_max_neighbours;
    a.marginal = params->m_marginal_probs[1];
    hb::Options opt;
    progress("Median IK", 0);
    if (hb::median_ik(dims, in_data->m_data, in_data->m_mask, a, params->m_marginal_probs[1], out_data->m_data,
                      out_data->m_mask, opt) == 0)
        report_done("Median IK");
}

int hpgl_b200_cont_kriging_ex(int kind, const int *dims, const float *in_data, const unsigned char *in_mask,
                              const hpgl_sk_params_t *params, float *out_data, unsigned char *out_mask,
                              const hpgl_b200_options_t *opt)
{
    if (!params || (kind != 0 && kind != 1))
    {
        hb::set_error("hpgl_b200_cont_kriging_ex: bad argument");
        return HPGL_B200_EINVAL;
    }
    return hb::cont_kriging(kind, dims, in_data, in_mask, sk_args_from(params), out_data, out_mask, options_from(opt));
}

int hpgl_b200_lvm_kriging_ex(const int *dims, const float *in_data, const unsigned char *in_mask,
                             const float *mean_data, const hpgl_ok_params_t *params, float *out_data,
                             unsigned char *out_mask, const hpgl_b200_options_t *opt)
{
    if (!params || !mean_data)
    {
        hb::set_error("hpgl_b200_lvm_kriging_ex: bad argument");
        return HPGL_B200_EINVAL;
    }
    return hb::cont_kriging(2, dims, in_data, in_mask, ok_args_from(params), out_data, out_mask, options_from(opt),
                            mean_data);
}

int hpgl_b200_cokriging_ex(int mark, const int *dims, const float *pdata, const unsigned char *pmask,
                           const float *sdata, const unsigned char *smask, const hpgl_cokriging_m1_params_t *m1,
                           const hpgl_cokriging_m2_params_t *m2, float *out_data, unsigned char *out_mask,
                           const hpgl_b200_options_t *opt)
{
    hb::CokArgs a;
    if (!cok_args_from(mark, m1, m2, a))
    {
        hb::set_error("hpgl_b200_cokriging_ex: mark must be 1 (with m1) or 2 (with m2)");
        return HPGL_B200_EINVAL;
    }
    return hb::cokriging(dims, pdata, pmask, sdata, smask, a, out_data, out_mask, options_from(opt));
}

int hpgl_b200_sis_ex(const int *dims, unsigned char *data, unsigned char *mask, const unsigned char *sim_mask,
                     const hpgl_ik_params_t *params, int indicator_count, const float *const *means, int seed,
                     int use_correlograms, const hpgl_b200_options_t *opt)
{
    if (!params || indicator_count <= 0)
    {
        hb::set_error("hpgl_b200_sis_ex: bad argument");
        return HPGL_B200_EINVAL;
    }
    std::vector<hb::IkArgs> cats;
    for (int i = 0; i < indicator_count; ++i) cats.push_back(ik_args_from(params + i));
    return hb::sis_simulation(dims, data, mask, sim_mask, cats, means, seed, options_from(opt), use_correlograms != 0);
}

int hpgl_b200_sgs_draws(long long seed, long long n, double *out)
{
    if (n < 0 || (n > 0 && !out))
    {
        hb::set_error("hpgl_b200_sgs_draws: bad argument");
        return HPGL_B200_EINVAL;
    }
    hb::sgs_draws((unsigned long long)seed, n, out);
    return HPGL_B200_OK;
}

int hpgl_b200_sim_levels(long long n_sim, int k, const int *nb_rank, int *levels)
{
    return hb::sim_levels(n_sim, k, nb_rank, levels);
}

int hpgl_b200_sgs_ex(const int *dims, float *data, unsigned char *mask, const unsigned char *sim_mask,
                     const hpgl_non_parametric_cdf_t *cdf, const float *means, const hpgl_sgs_params_t *params,
                     const hpgl_b200_options_t *opt)
{
    if (!params)
    {
        hb::set_error("hpgl_b200_sgs_ex: bad argument");
        return HPGL_B200_EINVAL;
    }
    hb::CdfTable t;
    if (cdf) t = {cdf->m_values, cdf->m_probs, cdf->m_size};
    return hb::sgs_simulation(dims, data, mask, sim_mask, cdf ? &t : nullptr, means, sgs_args_from(params),
                              options_from(opt));
}

int hpgl_b200_indicator_kriging_ex(const int *dims, const unsigned char *in_data, const unsigned char *in_mask,
                                   const hpgl_ik_params_t *params, int indicator_count, unsigned char *out_data,
                                   unsigned char *out_mask, const hpgl_b200_options_t *opt)
{
    if (!params || indicator_count <= 0)
    {
        hb::set_error("hpgl_b200_indicator_kriging_ex: bad argument");
        return HPGL_B200_EINVAL;
    }
    std::vector<hb::IkArgs> cats;
    for (int i = 0; i < indicator_count; ++i) cats.push_back(ik_args_from(params + i));
    return hb::indicator_kriging(dims, in_data, in_mask, cats, out_data, out_mask, options_from(opt));
}

int hpgl_b200_median_ik_ex(const int *dims, const unsigned char *in_data, const unsigned char *in_mask,
                           const hpgl_median_ik_params_t *params, unsigned char *out_data, unsigned char *out_mask,
                           const hpgl_b200_options_t *opt)
{
    if (!params)
    {
        hb::set_error("hpgl_b200_median_ik_ex: bad argument");
        return HPGL_B200_EINVAL;
    }
    hb::IkArgs a{};
    a.cov_type = params->m_covariance_type;
    for (int i = 0; i < 3; ++i)
    {
        a.ranges[i] = params->m_ranges[i];
        a.angles[i] = params->m_angles[i];
        a.radiuses[i] = params->m_radiuses[i];
    }
    a.sill = params->m_sill;
    a.nugget = params->m_nugget;
    a.max_nb = params->m_max_neighbours;
    a.marginal = params->m_marginal_probs[1];
    return hb::median_ik(dims, in_data, in_mask, a, params->m_marginal_probs[1], out_data, out_mask,
                         options_from(opt));
}

int hpgl_b200_find_neighbours(int kind, const int *dims, const unsigned char *mask, const hpgl_sk_params_t *params,
                              const int *nodes, int n_nodes, int *out_idx, int *out_count, unsigned char *out_path)
{
    if (!params || !dims || !mask || !nodes || !out_idx)
    {
        hb::set_error("hpgl_b200_find_neighbours: bad argument");
        return HPGL_B200_EINVAL;
    }
    return hb::find_neighbours(kind, dims, mask, sk_args_from(params), nodes, n_nodes, out_idx, out_count, out_path);
}

int hpgl_b200_last_stats(double *out, int cap)
{
    hb::Stats s = hb::last_stats();
    double v[HPGL_B200_STATS_LEN] = {s.total_ms, s.search_ms, s.solve_ms, (double)s.ties, (double)s.template_cells,
                                     (double)s.kriged, (double)s.launches, (double)s.h2d, (double)s.d2h,
                                     (double)s.escalated, s.search_kernel_ms};
    for (int b = 0; b < 5; ++b)
    {
        v[11 + b] = (double)s.bucket_items[b];
        v[16 + b] = s.bucket_ms[b];
        v[21 + b] = s.bucket_flops[b];
    }
    for (int i = 0; i < hb::kStages; ++i) v[26 + i] = s.stage_ms[i];
    v[36] = (double)s.exact_cells;
    v[37] = s.prefilter ? 1.0 : 0.0;
    v[38] = s.plan_ms;
    v[39] = (double)s.sgs_levels;
    v[40] = s.draws_ms;
    v[41] = s.sgs_flops;
    v[42] = (double)s.refined;
    int n = cap < HPGL_B200_STATS_LEN ? cap : HPGL_B200_STATS_LEN;
    for (int i = 0; i < n; ++i) out[i] = v[i];
    return n;
}

int hpgl_b200_solve_variant(int bucket_np, int cov_type, int precision, int variant)
{
    const int prev = hb::set_solve_variant(bucket_np, cov_type, precision, variant);
    if (prev < 0)
    {
        hb::set_error("hpgl_b200_solve_variant: invalid key or variant");
        return HPGL_B200_EINVAL;
    }
    return prev;
}

int hpgl_b200_solve_variant_get(int bucket_np, int cov_type, int precision)
{
    return hb::solve_variant(bucket_np, cov_type, precision);
}

int hpgl_b200_tune_mode(int on)
{
    const int prev = hb::tune_mode();
    hb::set_tune_mode(on);
    return prev;
}

int hpgl_b200_tune_load(const char *path)
{
    std::string err;
    const int n = path ? hb::tune_load(path, err) : -1;
    if (n < 0)
    {
        hb::set_error("hpgl_b200_tune_load: " + (path ? err : std::string("null path")));
        return HPGL_B200_EINVAL;
    }
    return n;
}

int hpgl_b200_tune_save(const char *path)
{
    std::string err;
    const int n = path ? hb::tune_save(path, err) : -1;
    if (n < 0)
    {
        hb::set_error("hpgl_b200_tune_save: " + (path ? err : std::string("null path")));
        return HPGL_B200_EINVAL;
    }
    return n;
}

void hpgl_b200_tune_reset(void) { hb::tune_reset(); }

void *hpgl_b200_host_alloc(size_t bytes) { return hb::host_alloc(bytes); }
void hpgl_b200_host_free(void *p) { hb::host_free(p); }

int hpgl_b200_transform(const double *ranges, const double *angles, double *out9)
{
    hb::CovModel m;
    std::string err;
    if (!hb::make_model(0, ranges, angles, 1.0, 0.0, m, err))
    {
        hb::set_error(err);
        return HPGL_B200_EINVAL;
    }
    for (int i = 0; i < 9; ++i) out9[i] = m.T[i];
    return 0;
}

int hpgl_b200_template(int kind, const hpgl_cov_params_t *cov, const int *radiuses, int *out, int cap,
                       int *out_limit)
{
    if (!cov || !radiuses || (cap > 0 && !out))
    {
        hb::set_error("hpgl_b200_template: bad argument");
        return HPGL_B200_EINVAL;
    }
    return hb::host_template(kind, cov->m_covariance_type, cov->m_ranges, cov->m_angles, cov->m_sill,
                             cov->m_nugget, radiuses, out, cap, out_limit);
}

double hpgl_b200_covariance(int kind, const hpgl_cov_params_t *cov, const int *radiuses, const int *a, const int *b)
{
    return hb::host_covariance(kind, cov->m_covariance_type, cov->m_ranges, cov->m_angles, cov->m_sill,
                               cov->m_nugget, radiuses, a, b);
}

const char *hpgl_b200_version(void) { return "hpgl_b200 0.1 (sm_100a)"; }

} // extern "C"
