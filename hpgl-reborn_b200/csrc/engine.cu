// Engine: host orchestration of one kriging call on the GPU.
//
//   host  : validate, build the flavour's search template (std::sort, as the
//           reference does), the selection-key table (exact double covariances
//           and their dense descending ranks), geometry;
//   device: upload, compact points, bin, search, resolve ties, bucket by
//           neighbour count, solve per bucket, finalize; download.
//
// Device buffers are cached per engine (grow-only) so repeated calls do not
// allocate. One engine per CUDA device, used under a mutex.
#include "engine_api.h"
#include "host_model.h"
#include "kernels.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <exception>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace hb
{
// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;
static std::string g_last_error_global;
static std::mutex g_err_mu;

void set_error(const std::string &msg)
{
    g_last_error = msg;
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_error_global = msg;
}
const char *last_error()
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    static std::string copy;
    copy = g_last_error_global;
    return copy.c_str();
}

struct CudaFail
{
    int code;
    std::string msg;
};

#define HB_CK(expr)                                                                                            \
    do                                                                                                         \
    {                                                                                                          \
        cudaError_t _e = (expr);                                                                               \
        if (_e != cudaSuccess)                                                                                 \
            throw CudaFail{_e == cudaErrorMemoryAllocation ? -3 : -2,                                          \
                           std::string(#expr) + ": " + cudaGetErrorString(_e)};                                \
    } while (0)

// ------------------------------------------------------------------ buffers
struct DevBuf
{
    void *p = nullptr;
    size_t cap = 0;
};

class Engine
{
  public:
    explicit Engine(int dev) : device_(dev)
    {
        HB_CK(cudaSetDevice(dev));
        HB_CK(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
        cudaDeviceProp prop;
        HB_CK(cudaGetDeviceProperties(&prop, dev));
        n_sm_ = prop.multiProcessorCount;
        max_smem_ = (int)prop.sharedMemPerBlockOptin;
        for (int i = 0; i < kNumEvents; ++i) HB_CK(cudaEventCreate(&ev_[i]));
        for (int i = 0; i < 64; ++i) HB_CK(cudaEventCreate(&stage_ev_[i]));
        HB_CK(cudaEventCreate(&stage_start_));
    }

    template <typename T>
    T *buf(const char *name, size_t count)
    {
        DevBuf &b = bufs_[name];
        size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        if (b.cap < bytes)
        {
            if (b.p) cudaFree(b.p);
            b.p = nullptr;
            b.cap = 0;
            size_t want = bytes + bytes / 8;
            HB_CK(cudaMalloc(&b.p, want));
            b.cap = want;
        }
        return reinterpret_cast<T *>(b.p);
    }

    // Stage timing: mark(id) records the end of stage `id` on the stream; the
    // stage lasts from the previous mark (or the call start).
    void mark(int id, cudaStream_t st)
    {
        if (id < 0 || id >= kStages) return;
        HB_CK(cudaEventRecord(stage_ev_[n_marks_ % 64], st));
        mark_id_[n_marks_ % 64] = id;
        ++n_marks_;
    }
    void reset_marks(cudaStream_t st)
    {
        n_marks_ = 0;
        HB_CK(cudaEventRecord(stage_start_, st));
    }
    void collect_marks()
    {
        cudaEvent_t prev = stage_start_;
        for (int i = 0; i < n_marks_ && i < 64; ++i)
        {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, prev, stage_ev_[i]) == cudaSuccess) stats.stage_ms[mark_id_[i]] += ms;
            prev = stage_ev_[i];
        }
    }
    // Page-locked host staging for table uploads. The contents must not be
    // rewritten before the copies issued from them have completed (the engine
    // synchronises its stream between the uses).
    unsigned char *staging(size_t bytes)
    {
        if (stage_cap_ < bytes)
        {
            if (stage_) cudaFreeHost(stage_);
            stage_ = nullptr;
            stage_cap_ = 0;
            const size_t want = bytes + bytes / 4;
            HB_CK(cudaHostAlloc(reinterpret_cast<void **>(&stage_), want, cudaHostAllocDefault));
            stage_cap_ = want;
        }
        return stage_;
    }
    // A second page-locked area (the SGS draws), same rules as staging().
    unsigned char *staging2(size_t bytes)
    {
        if (stage2_cap_ < bytes)
        {
            if (stage2_) cudaFreeHost(stage2_);
            stage2_ = nullptr;
            stage2_cap_ = 0;
            const size_t want = bytes + bytes / 4;
            HB_CK(cudaHostAlloc(reinterpret_cast<void **>(&stage2_), want, cudaHostAllocDefault));
            stage2_cap_ = want;
        }
        return stage2_;
    }
    // Page-locked host areas for the copies of user arrays that are not
    // page-locked, one per name (so the areas of one call never alias); the
    // engine synchronises its stream before a name is used again.
    unsigned char *pinned(const std::string &name, size_t bytes)
    {
        DevBuf &b = pinned_[name];
        if (b.cap < bytes)
        {
            if (b.p) cudaFreeHost(b.p);
            b.p = nullptr;
            b.cap = 0;
            const size_t want = bytes + bytes / 8;
            HB_CK(cudaHostAlloc(&b.p, want, cudaHostAllocDefault));
            b.cap = want;
        }
        return reinterpret_cast<unsigned char *>(b.p);
    }
    // Downloads through a page-locked area, finished on the host after the
    // call's stream synchronisation (end_call).
    struct PendingCopy
    {
        void *dst;
        const void *src;
        size_t bytes;
    };
    std::vector<PendingCopy> pending;
    int n_downloads = 0;
    int n_sm() const { return n_sm_; }
    int max_smem() const { return max_smem_; }
    cudaStream_t stream(const void *user) const { return user ? (cudaStream_t)user : own_stream_; }
    static constexpr int kNumEvents = 32;
    cudaEvent_t ev_[kNumEvents];
    Stats stats;

  private:
    cudaEvent_t stage_ev_[64];
    cudaEvent_t stage_start_;
    int mark_id_[64];
    int n_marks_ = 0;
    unsigned char *stage2_ = nullptr;
    size_t stage2_cap_ = 0;
    int device_;
    cudaStream_t own_stream_ = nullptr;
    int n_sm_ = 148;
    int max_smem_ = 227 * 1024;
    std::map<std::string, DevBuf> bufs_;
    std::map<std::string, DevBuf> pinned_;
    unsigned char *stage_ = nullptr;
    size_t stage_cap_ = 0;
};

static std::mutex g_engine_mu;
static std::map<int, std::unique_ptr<Engine>> g_engines;
static int g_threads = 0;

void set_threads(int n) { g_threads = n; }
int get_threads() { return clamp_threads(g_threads); }

static Engine &engine_for_current_device()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) throw CudaFail{-2, std::string("no usable CUDA device: ") + cudaGetErrorString(e)};
    int n = 0;
    e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) throw CudaFail{-2, "no usable CUDA device"};
    auto it = g_engines.find(dev);
    if (it == g_engines.end()) it = g_engines.emplace(dev, std::make_unique<Engine>(dev)).first;
    return *it->second;
}

// ------------------------------------------------------------------ plan
struct Plan
{
    Flavour f;
    long tmpl_count = 0; // length of the search template (built only when a bin needs it)
    KeyTable kt;
    Surrogate sg;
    Geom g;
    int rank_bits = 0;
};

static int bits_for(uint32_t max_value)
{
    int b = 0;
    while (b < 32 && (max_value >> b) != 0) ++b;
    return b;
}

static void check_model_args(int cov_type, const double *ranges, const double *angles, double sill, double nugget,
                             const int *radiuses, int k)
{
    for (int i = 0; i < 3; ++i)
    {
        if (!std::isfinite(ranges[i]) || !std::isfinite(angles[i]))
            throw CudaFail{-1, "ranges and angles must be finite"};
        if (radiuses[i] <= 0)
            throw CudaFail{-1, "search radiuses must be positive integers (a zero radius makes the reference's "
                               "clusterizer index out of range)"};
        if (radiuses[i] > 4096) throw CudaFail{-4, "search radius above 4096 is not supported"};
    }
    if (!std::isfinite(sill) || !std::isfinite(nugget)) throw CudaFail{-1, "sill and nugget must be finite"};
    // a negative sill makes the strict C(0)/100 threshold negative, so zero
    // (out-of-box) covariances would pass it; the reference's validation
    // rejects it too (validation.py:397-430)
    if (sill < 0) throw CudaFail{-1, "sill must be >= 0"};
    if (k < 1) throw CudaFail{-1, "max_neighbours must be >= 1"};
    if (k > 1024) throw CudaFail{-4, "max_neighbours above 1024 is not supported"};
    if (cov_type < 0 || cov_type > 2) throw CudaFail{-1, "unknown covariance type"};
}

static long long check_dims(const int *dims)
{
    if (!dims) throw CudaFail{-1, "null dims"};
    long long n = (long long)dims[0] * dims[1] * dims[2];
    if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || n > 2147483647LL)
        throw CudaFail{-1, "get_shape_volume: grid volume exceeds INT_MAX"};
    if (dims[0] >= (1 << 21) || dims[1] >= (1 << 21) || dims[2] >= (1 << 21))
        throw CudaFail{-4, "grid axis longer than 2^21 cells is not supported"};
    return n;
}

static Plan make_plan(bool truncated, int cov_type, const double *ranges, const double *angles, double sill,
                      double nugget, const int *radiuses, int k, const int *dims, bool surrogate = true)
{
    check_model_args(cov_type, ranges, angles, sill, nugget, radiuses, k);
    Plan pl;
    std::string err;
    if (!make_model(cov_type, ranges, angles, sill, nugget, pl.f.m, err)) throw CudaFail{-1, err};
    pl.f.truncated = truncated;
    for (int a = 0; a < 3; ++a) pl.f.r[a] = radiuses[a];
    build_key_table(pl.f, pl.kt, g_threads);
    pl.tmpl_count = template_size(pl.f, pl.kt);
    if (surrogate && k <= 64 && pl.kt.n_ranks <= 0xFFFE) build_surrogate(pl.f, pl.kt, pl.sg);
    pl.rank_bits = pl.kt.n_ranks > 1 ? bits_for(pl.kt.n_ranks - 1) : 0;

    Geom &g = pl.g;
    g.nx = dims[0];
    g.ny = dims[1];
    g.nz = dims[2];
    g.n_cells = (long long)dims[0] * dims[1] * dims[2];
    g.rx = radiuses[0];
    g.ry = radiuses[1];
    g.rz = radiuses[2];
    // clusterizer.cpp:87-89: bins per axis = (int)(g / (double)r + 2)
    g.bx = (int)(g.nx / (double)g.rx + 2);
    g.by = (int)(g.ny / (double)g.ry + 2);
    g.bz = (int)(g.nz / (double)g.rz + 2);
    long long nb = (long long)g.bx * g.by * g.bz;
    if (nb > (1LL << 30)) throw CudaFail{-4, "too many search bins"};
    g.n_bins = (int)nb;
    g.limit = (int)(pl.tmpl_count / 250);
    g.k = k;
    g.khx = pl.kt.half[0];
    g.khy = pl.kt.half[1];
    g.khz = pl.kt.half[2];
    g.knx = pl.kt.n[0];
    g.kny = pl.kt.n[1];
    int ph[3];
    for (int a = 0; a < 3; ++a) ph[a] = truncated ? 2 * radiuses[a] : 4 * radiuses[a] - 2;
    for (int a = 0; a < 3; ++a) ph[a] = std::max(ph[a], pl.kt.half[a]);
    g.phx = ph[0];
    g.phy = ph[1];
    g.phz = ph[2];
    g.pnx = 2 * ph[0] + 1;
    g.pny = 2 * ph[1] + 1;
    long long pn = (long long)g.pnx * g.pny * (2 * ph[2] + 1);
    if (pn > (1LL << 31) - 1) throw CudaFail{-4, "covariance table too large for these radiuses"};
    g.pair_center = ((long long)ph[2] * g.pny + ph[1]) * g.pnx + ph[0];
    return pl;
}

// Geometry of the grid alone: what the upload and point compaction read.
static Geom grid_geom(const int *dims)
{
    Geom g = {};
    g.nx = dims[0];
    g.ny = dims[1];
    g.nz = dims[2];
    g.n_cells = (long long)dims[0] * dims[1] * dims[2];
    return g;
}

static DevModel dev_model(const CovModel &m)
{
    DevModel d;
    d.type = m.type;
    d.r0 = m.ranges[0];
    d.sill = m.sill;
    d.nugget = m.nugget;
    for (int i = 0; i < 9; ++i) d.T[i] = m.T[i];
    return d;
}

// ------------------------------------------------------------------ stages
struct DevPoints
{
    int *n_pts = nullptr; // device scalar
    int m = 0;            // host copy
    int *pts_node = nullptr;
    unsigned long long *pts_xyz = nullptr;
    float *pts_val = nullptr;
    uint8_t *pts_cat = nullptr;
    int *pid_of_node = nullptr;
};

static DevPoints compact_points(Engine &E, const Geom &g, const uint8_t *d_mask, const float *d_val_f,
                                const uint8_t *d_val_u8, cudaStream_t st, const float *d_mean = nullptr)
{
    DevPoints P;
    long long n = g.n_cells;
    int *pos = E.buf<int>("pos", (size_t)n);
    int *tmp = E.buf<int>("scan_tmp", (size_t)scan_tmp_ints(n) + 4);
    P.n_pts = E.buf<int>("n_pts", 1);
    E.mark(STAGE_UPLOAD, st);
    launch_flag_informed(d_mask, n, pos, st);
    exclusive_scan(pos, n, tmp, P.n_pts, st);
    HB_CK(cudaGetLastError());
    HB_CK(cudaMemcpyAsync(&P.m, P.n_pts, sizeof(int), cudaMemcpyDeviceToHost, st));
    HB_CK(cudaStreamSynchronize(st));
    size_t m = std::max(P.m, 1);
    P.pts_node = E.buf<int>("pts_node", m);
    P.pts_xyz = E.buf<unsigned long long>("pts_xyz", m);
    P.pts_val = E.buf<float>("pts_val", m);
    if (d_val_u8) P.pts_cat = E.buf<uint8_t>("pts_cat", m);
    P.pid_of_node = E.buf<int>("pid_of_node", (size_t)n);
    launch_emit_points(d_mask, pos, g, d_val_f, d_mean, d_val_u8, P.pts_node, P.pts_xyz, P.pts_val, P.pts_cat,
                       P.pid_of_node, st);
    HB_CK(cudaGetLastError());
    E.mark(STAGE_COMPACT, st);
    return P;
}

struct DevSearch
{
    int2 *nb_rec = nullptr;
    int *nb_pid = nullptr;
    int *nb_n = nullptr;
    uint8_t *bin_flag = nullptr;
    double *search_vals = nullptr;
    double *pair64 = nullptr;
    float *pair32 = nullptr;
    int ties = 0;
    int template_cells = 0;
};

// Search for one flavour; `all_cells` selects every cell (IK) or only the
// uninformed ones. Table slots are suffixed with `tag` so several flavours can
// coexist (IK categories run one after another and reuse them).
static DevSearch run_search(Engine &E, const Plan &pl, const DevPoints &P, const uint8_t *d_mask, int all_cells,
                            cudaStream_t st, bool want_pids = false, bool exact_search = false)
{
    const Geom &g = pl.g;
    DevSearch S;
    // tables: the exact covariances of the key block (for the pair tables), the
    // 16-bit ranks of the fast selection and the prefilter's per-rank h2, staged
    // through page-locked memory; the 32-bit ranks only when a slow path needs them
    const size_t nk = pl.kt.rank.size();
    const bool fast_keys = g.k <= 64 && pl.kt.n_ranks <= 0xFFFE;
    const bool use_sd = fast_keys && pl.sg.ok && !exact_search;
    const size_t nh = use_sd ? pl.sg.h2_rank.size() : 0;
    const size_t off_k16 = nk * 8, off_h2 = (off_k16 + (fast_keys ? nk * 2 : 0) + 15) / 16 * 16;
    unsigned char *stg = E.staging(off_h2 + nh * 8);
    std::memcpy(stg, pl.kt.vals.data(), nk * 8);
    S.search_vals = E.buf<double>("search_vals", nk);
    HB_CK(cudaMemcpyAsync(S.search_vals, stg, nk * 8, cudaMemcpyHostToDevice, st));
    uint16_t *keytab16 = nullptr;
    if (fast_keys)
    {
        uint16_t *k16 = reinterpret_cast<uint16_t *>(stg + off_k16);
        for (size_t i = 0; i < nk; ++i)
            k16[i] = pl.kt.rank[i] == KEY_EXCLUDED ? (uint16_t)0xFFFF : (uint16_t)pl.kt.rank[i];
        keytab16 = E.buf<uint16_t>("keytab16", nk);
        HB_CK(cudaMemcpyAsync(keytab16, k16, nk * 2, cudaMemcpyHostToDevice, st));
    }
    uint32_t *keytab32 = nullptr;
    auto keytab = [&]() {
        if (!keytab32)
        {
            keytab32 = E.buf<uint32_t>("keytab", nk);
            HB_CK(cudaMemcpyAsync(keytab32, pl.kt.rank.data(), nk * 4, cudaMemcpyHostToDevice, st));
        }
        return keytab32;
    };
    SurrDev sd = {};
    if (use_sd)
    {
        std::memcpy(stg + off_h2, pl.sg.h2_rank.data(), nh * 8);
        double *h2r = E.buf<double>("h2_rank", nh);
        HB_CK(cudaMemcpyAsync(h2r, stg + off_h2, nh * 8, cudaMemcpyHostToDevice, st));
        sd.on = 1;
        for (int i = 0; i < 9; ++i) sd.T[i] = pl.sg.T[i];
        for (int a = 0; a < 3; ++a) sd.step[a] = pl.sg.step[a];
        sd.e3 = pl.sg.e3;
        sd.h2_cut = pl.sg.h2_cut;
        sd.h2_rank = h2r;
    }
    long long pn = (long long)g.pnx * g.pny * (2 * g.phz + 1);
    S.pair64 = E.buf<double>("pair64", (size_t)pn);
    S.pair32 = E.buf<float>("pair32", (size_t)pn);
    launch_build_pair(g, dev_model(pl.f.m), pl.f.truncated ? 1 : 0, S.search_vals, S.pair64, S.pair32, st);
    E.mark(STAGE_TABLES, st);

    // bins
    int *bin_cnt = E.buf<int>("bin_cnt", g.n_bins);
    int *bin_start = E.buf<int>("bin_start", g.n_bins);
    int *bin_fill = E.buf<int>("bin_fill", g.n_bins);
    S.bin_flag = E.buf<uint8_t>("bin_flag", g.n_bins);
    int *bin_pts = E.buf<int>("bin_pts", std::max(P.m, 1));
    int *tmpl_bins = E.buf<int>("tmpl_bins", g.n_bins);
    // 0 total, 1 max_cand, 2 tmpl bins, 3 ties, 4 tmpl cells, 5 exact cells, 6 max_cand of the template bins
    int *scal = E.buf<int>("scalars", 8);
    int *tmp = E.buf<int>("scan_tmp2", (size_t)scan_tmp_ints(g.n_bins) + 4);
    HB_CK(cudaMemsetAsync(bin_cnt, 0, sizeof(int) * g.n_bins, st));
    HB_CK(cudaMemsetAsync(bin_fill, 0, sizeof(int) * g.n_bins, st));
    HB_CK(cudaMemsetAsync(scal, 0, sizeof(int) * 8, st));
    launch_bin_count(P.pts_xyz, P.n_pts, g, bin_cnt, st);
    HB_CK(cudaMemcpyAsync(bin_start, bin_cnt, sizeof(int) * g.n_bins, cudaMemcpyDeviceToDevice, st));
    exclusive_scan(bin_start, g.n_bins, tmp, scal + 0, st);
    launch_bin_fill(P.pts_xyz, P.n_pts, g, bin_start, bin_fill, bin_pts, st);
    launch_bin_sort(g, bin_start, bin_cnt, bin_pts, S.bin_flag, st);
    launch_bin_region(g, S.bin_flag, bin_cnt, scal + 1, scal + 2, tmpl_bins, scal + 6, st);
    HB_CK(cudaGetLastError());
    int host_scal[8];
    HB_CK(cudaMemcpyAsync(host_scal, scal, sizeof(host_scal), cudaMemcpyDeviceToHost, st));
    HB_CK(cudaStreamSynchronize(st));
    E.mark(STAGE_BINS, st);
    int max_cand = host_scal[1];
    const int n_tmpl_bins = host_scal[2];
    const int max_cand_tmpl = host_scal[6];
    // Template-path bins (sugarbox_neighbour_lookup.h:171-197: the first k informed
    // cells of the sorted template, in its order) as a selection: the informed
    // cells of the 27 bins around a cell keyed by their offset's position in the
    // template, unique keys whose k smallest are those cells, through the fast
    // search; the template scan over the informed-cell bitmap beyond its limits.
    int n_tmpl = 0;
    int4 *tmpl = E.buf<int4>("tmpl", std::max<long>(pl.tmpl_count, 1));
    bool tmpl_select = false;
    uint16_t *keypos16 = nullptr;
    SurrDev sdp = {};
    int cand_cap_t = 0, warps_t = 8;
    if (n_tmpl_bins > 0 && pl.tmpl_count > 0)
    {
        const std::vector<Offset> tv = build_template(pl.f, pl.kt);
        if (g.k <= 64 && tv.size() <= 0xFFFE)
        {
            cand_cap_t = std::max(4, (max_cand_tmpl + 3) / 4 * 4);
            while (warps_t > 1 && search_fast_smem_bytes(cand_cap_t, g.k, warps_t) > (size_t)E.max_smem()) --warps_t;
            tmpl_select = cand_cap_t <= 65536 && search_fast_smem_bytes(cand_cap_t, g.k, warps_t) <= (size_t)E.max_smem();
        }
        if (tmpl_select)
        {
            std::vector<uint16_t> kp(nk, (uint16_t)0xFFFF);
            for (size_t i = 0; i < tv.size(); ++i) kp[key_index(g, tv[i].dx, tv[i].dy, tv[i].dz)] = (uint16_t)i;
            keypos16 = E.buf<uint16_t>("keypos16", nk);
            HB_CK(cudaMemcpyAsync(keypos16, kp.data(), nk * 2, cudaMemcpyHostToDevice, st));
            Surrogate sgp;
            build_surrogate_template(pl.f, tv, sgp);
            double *h2p = E.buf<double>("h2_pos", sgp.h2_rank.size());
            HB_CK(cudaMemcpyAsync(h2p, sgp.h2_rank.data(), sgp.h2_rank.size() * 8, cudaMemcpyHostToDevice, st));
            sdp.on = sgp.ok && !exact_search ? 1 : 0;
            for (int i = 0; i < 9; ++i) sdp.T[i] = sgp.T[i];
            for (int a = 0; a < 3; ++a) sdp.step[a] = sgp.step[a];
            sdp.e3 = sgp.e3;
            sdp.h2_cut = sgp.h2_cut;
            sdp.h2_rank = h2p;
            HB_CK(cudaStreamSynchronize(st)); // kp and sgp are temporaries
        }
        else
        {
            // the template probes a bitmap of the grid padded by the radiuses; its
            // linear offsets are 32-bit
            const long long PX = g.nx + 2LL * g.rx, PY = g.ny + 2LL * g.ry;
            if ((long long)g.rz * PY * PX + (long long)g.ry * PX + g.rx > 2147483647LL)
                throw CudaFail{-4, "grid too large for the template search path at these radiuses"};
            std::vector<int4> t4(tv.size());
            for (size_t i = 0; i < tv.size(); ++i)
                t4[i] = make_int4(tv[i].dx, tv[i].dy, tv[i].dz, template_padded_offset(g, tv[i].dx, tv[i].dy, tv[i].dz));
            HB_CK(cudaMemcpyAsync(tmpl, t4.data(), t4.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
            HB_CK(cudaStreamSynchronize(st)); // t4 is a temporary
            n_tmpl = (int)tv.size();
        }
    }

    // search
    int cand_cap = std::max(4, (max_cand + 3) / 4 * 4);
    const bool fast = fast_keys && cand_cap <= 65536;
    auto smem_need = [&](int w) {
        return fast ? search_fast_smem_bytes(cand_cap, g.k, w) : search_smem_bytes(cand_cap, g.k, w);
    };
    int warps = 8;
    while (warps > 1 && smem_need(warps) > (size_t)E.max_smem()) --warps;
    if (smem_need(warps) > (size_t)E.max_smem())
        throw CudaFail{-4, "neighbour candidate list too long for shared memory (" + std::to_string(max_cand) +
                               " candidates)"};
    S.nb_rec = E.buf<int2>("nb_rec", (size_t)g.n_cells * g.k);
    S.nb_pid = want_pids ? E.buf<int>("nb_pid", (size_t)g.n_cells * g.k) : nullptr;
    S.nb_n = E.buf<int>("nb_n", (size_t)g.n_cells);
    int *tie_cells = E.buf<int>("tie_cells", (size_t)g.n_cells);
    HB_CK(cudaMemsetAsync(S.nb_n, 0, sizeof(int) * g.n_cells, st));
    HB_CK(cudaEventRecord(E.ev_[8], st));
    if (fast)
        HB_CK(launch_search_fast(g, d_mask, all_cells, bin_start, bin_cnt, S.bin_flag, bin_pts, P.pts_xyz, P.pts_val,
                                 keytab16, sd, 0, P.pid_of_node, cand_cap, warps, S.nb_pid,
                                 S.nb_rec, S.nb_n, tie_cells, scal + 3, scal + 4, scal + 5, st));
    else
        HB_CK(launch_search(g, d_mask, all_cells, bin_start, bin_cnt, S.bin_flag, bin_pts, P.pts_xyz, P.pts_val,
                            keytab(), pl.rank_bits, tmpl, n_tmpl, P.pid_of_node, cand_cap, warps,
                            S.nb_pid, S.nb_rec, S.nb_n, tie_cells, scal + 3, scal + 4, st));
    if (n_tmpl_bins > 0 && tmpl_select)
        HB_CK(launch_search_fast(g, d_mask, all_cells, bin_start, bin_cnt, S.bin_flag, bin_pts, P.pts_xyz, P.pts_val,
                                 keypos16, sdp, 1, P.pid_of_node, cand_cap_t, warps_t, S.nb_pid, S.nb_rec, S.nb_n,
                                 tie_cells, scal + 3, scal + 4, scal + 5, st));
    else if (n_tmpl_bins > 0)
        HB_CK(launch_search_template(g, d_mask, E.buf<uint32_t>("mask_bits", (size_t)(template_padded_cells(g) + 31) / 32), all_cells,
                                     tmpl_bins, n_tmpl_bins, P.pts_val, tmpl, n_tmpl, P.pid_of_node, S.nb_pid,
                                     S.nb_rec, S.nb_n, scal + 4, E.n_sm(), st));
    HB_CK(cudaEventRecord(E.ev_[9], st));
    HB_CK(cudaMemcpyAsync(host_scal, scal, sizeof(host_scal), cudaMemcpyDeviceToHost, st));
    HB_CK(cudaStreamSynchronize(st));
    S.ties = host_scal[3];
    S.template_cells = host_scal[4];
    E.stats.exact_cells += host_scal[5];
    E.stats.prefilter = E.stats.prefilter || (fast && sd.on);
    E.mark(STAGE_SEARCH, st);
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, E.ev_[8], E.ev_[9]);
        E.stats.search_kernel_ms += ms;
    }
    // flag, scan tiles (+add), emit, pair table, bin count, bin scan, fill, sort, region, search
    E.stats.launches += 10 + (g.n_cells > 1024 ? 2 : 0) + (n_tmpl_bins > 0 ? (tmpl_select ? 1 : 2) : 0);

    // tie groups straddling the k-th slot: std::sort's choice, replayed
    if (S.ties > 0)
    {
        int cap = std::max(max_cand, 1);
        if (fast && cap <= 65535 && resolve_ties_fast_smem(cap, 1) <= (size_t)E.max_smem())
        {
            HB_CK(launch_resolve_ties_fast(g, tie_cells, scal + 3, S.ties, bin_start, bin_cnt, bin_pts, P.pts_xyz,
                                           P.pts_val, keytab16, cap, S.nb_pid, S.nb_rec, E.n_sm(), st));
            E.stats.launches += 1;
        }
        else
        {
            size_t per = (size_t)cap * tie_entry_bytes();
            size_t budget = (size_t)512 << 20;
            int chunk = (int)std::max<size_t>(1, std::min<size_t>(budget / per, (size_t)S.ties));
            void *scratch = E.buf<unsigned char>("tie_scratch", per * chunk);
            for (int first = 0; first < S.ties; first += chunk)
            {
                launch_resolve_ties(g, tie_cells, scal + 3, first, chunk, bin_start, bin_cnt, bin_pts, P.pts_xyz,
                                    P.pts_val, keytab(), scratch, cap, S.nb_pid, S.nb_rec, st);
                E.stats.launches += 1;
            }
        }
        HB_CK(cudaGetLastError());
    }
    E.mark(STAGE_TIES, st);
    return S;
}

// Solve every bucket for one search result. FP32-refined systems that do not
// converge (or whose float factor breaks down) are re-solved in FP64.
static void run_solves(Engine &E, const Plan &pl, const DevPoints &P, const DevSearch &S, const uint8_t *d_mask,
                       int all_cells, bool ordinary, int precision, int steps, double tol, double mean,
                       int ind_value, signed char *d_status, const SolveOut &out, cudaStream_t st)
{
    if (!(tol > 0.0)) tol = 1e-9;
    (void)P;
    const Geom &g = pl.g;
    int *bucket_cnt = E.buf<int>("bucket_cnt", kBuckets);
    int *bucket_off = E.buf<int>("bucket_off", kBuckets + 1);
    const size_t n_tiles = (size_t)prepare_tiles(g.n_cells);
    int *tile_cnt = E.buf<int>("tile_cnt", n_tiles * kBuckets);
    unsigned long long *tile_mom = E.buf<unsigned long long>("tile_mom", n_tiles * kBuckets * 3);
    int2 *cells = E.buf<int2>("cells", (size_t)g.n_cells);
    unsigned long long *moments = E.buf<unsigned long long>("moments", kBuckets * 3);
    // FP32-refined systems that fail the four-rows-per-lane kernel's check go
    // first to the two-rows-per-lane kernel (classic refinement), and what
    // that does not converge to the FP64 kernel
    int *esc_cnt = E.buf<int>("esc_cnt", 2 * kBuckets);
    int *ref_cnt = esc_cnt + kBuckets;
    int2 *esc_cells = precision ? E.buf<int2>("esc_cells", (size_t)g.n_cells) : nullptr;
    int2 *ref_cells = nullptr;
    int variant[kBuckets];
    bool any_quad = false;
    for (int b = 0; b < kBuckets; ++b)
    {
        variant[b] = b < 4 ? solve_variant(kBucketNP[b], pl.f.m.type, precision) : kVariantFold;
        any_quad = any_quad || (precision && b < 4 && kBucketNP[b] <= 32 &&
                                (is_quad_variant(variant[b]) || tune_wanted(kBucketNP[b], pl.f.m.type, precision)));
    }
    if (any_quad) ref_cells = E.buf<int2>("ref_cells", (size_t)g.n_cells);
    launch_prepare(g, d_mask, all_cells, S.nb_n, d_status, bucket_cnt, bucket_off, tile_cnt, tile_mom, cells, moments,
                   st);
    HB_CK(cudaMemsetAsync(esc_cnt, 0, sizeof(int) * 2 * kBuckets, st));
    HB_CK(cudaGetLastError());
    E.stats.launches += 3;
    int cnt[kBuckets];
    unsigned long long mom[kBuckets * 3];
    HB_CK(cudaMemcpyAsync(cnt, bucket_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    HB_CK(cudaMemcpyAsync(mom, moments, sizeof(mom), cudaMemcpyDeviceToHost, st));
    HB_CK(cudaStreamSynchronize(st));
    E.mark(STAGE_PREPARE, st);
    int off = 0;
    const double c0 = pl.f.c0();
    const double rhs = ordinary ? 2.0 : 1.0;
    int esc_off[kBuckets];
    // Tuning mode: the first large bucket of a key without a setting runs
    // every variant the key can run twice, the second run timed (the first
    // loads the kernel), and the fastest becomes the key's setting (and runs
    // below, leaving this call's outputs).
    auto tune_bucket = [&](int b, const int2 *bcells, int first) {
        const int np = kBucketNP[b];
        double ms[kVariantCount] = {0};
        for (int v = 1; v < kVariantCount; ++v)
        {
            if (!solve_variant_valid(np, precision, v)) continue;
            const bool quad = precision && is_quad_variant(v);
            for (int rep = 0; rep < 2; ++rep)
            {
                HB_CK(cudaMemsetAsync(esc_cnt + b, 0, sizeof(int), st));
                HB_CK(cudaMemsetAsync(ref_cnt + b, 0, sizeof(int), st));
                HB_CK(cudaEventRecord(E.ev_[10 + 2 * b], st));
                HB_CK(launch_solve_bucket(np, precision, v, ordinary, g, bcells, bucket_cnt + b, cnt[b], S.nb_rec,
                                          S.nb_n, ind_value, S.pair64, S.pair32, mean, c0, steps, tol, out,
                                          quad ? ref_cells + first : (esc_cells ? esc_cells + first : nullptr),
                                          quad ? ref_cnt + b : esc_cnt + b, E.n_sm(), st));
                HB_CK(cudaEventRecord(E.ev_[11 + 2 * b], st));
                E.stats.launches += 1;
            }
            HB_CK(cudaEventSynchronize(E.ev_[11 + 2 * b]));
            float t = 0.0f;
            HB_CK(cudaEventElapsedTime(&t, E.ev_[10 + 2 * b], E.ev_[11 + 2 * b]));
            ms[v] = t * 1e6 / (double)cnt[b];
        }
        tune_record(np, pl.f.m.type, precision, ms);
        HB_CK(cudaMemsetAsync(esc_cnt + b, 0, sizeof(int), st));
        HB_CK(cudaMemsetAsync(ref_cnt + b, 0, sizeof(int), st));
        variant[b] = solve_variant(np, pl.f.m.type, precision);
    };
    for (int b = 0; b < kBuckets; ++b)
    {
        esc_off[b] = off;
        if (cnt[b] > 0)
        {
            const int2 *bcells = cells + off;
            if (b < 4 && cnt[b] >= kTuneMinItems && tune_wanted(kBucketNP[b], pl.f.m.type, precision))
                tune_bucket(b, bcells, off);
            const bool quad = precision && b < 4 && kBucketNP[b] <= 32 && is_quad_variant(variant[b]);
            HB_CK(cudaEventRecord(E.ev_[10 + 2 * b], st));
            if (b < 4)
            {
                int2 *first_esc = quad ? ref_cells + off : (esc_cells ? esc_cells + off : nullptr);
                HB_CK(launch_solve_bucket(kBucketNP[b], precision, variant[b], ordinary, g, bcells, bucket_cnt + b,
                                          cnt[b], S.nb_rec, S.nb_n, ind_value, S.pair64, S.pair32, mean, c0, steps,
                                          tol, out, first_esc, quad ? ref_cnt + b : esc_cnt + b, E.n_sm(), st));
            }
            else
            {
                int blocks = std::min(cnt[b], E.n_sm() * 2);
                double *scratch = E.buf<double>("large_scratch", large_scratch_doubles(g.k, blocks));
                HB_CK(launch_solve_large(g, bcells, bucket_cnt + b, blocks, S.nb_rec, S.nb_n, ind_value, S.pair64,
                                         ordinary, mean, c0, scratch, out, st));
            }
            HB_CK(cudaEventRecord(E.ev_[11 + 2 * b], st));
            E.stats.launches += 1;
            E.stats.kriged += cnt[b];
            E.stats.bucket_items[b] += cnt[b];
            const double s1 = (double)mom[3 * b], s2 = (double)mom[3 * b + 1], s3 = (double)mom[3 * b + 2];
            // F(n, r) = n^3/3 + n^2/2 + 2 r n^2 + 30 (n(n+1)/2 + n) + 2 r n, summed over the bucket
            E.stats.bucket_flops[b] += s3 / 3.0 + s2 * (0.5 + 2.0 * rhs + 15.0) + s1 * (45.0 + 2.0 * rhs);
        }
        off += cnt[b];
    }
    if (precision)
    {
        // classic refinement of what the four-rows-per-lane kernel queued
        for (int b = 0; b < 4; ++b)
        {
            if (cnt[b] == 0 || !(kBucketNP[b] <= 32 && is_quad_variant(variant[b]))) continue;
            HB_CK(launch_solve_bucket(kBucketNP[b], 1, kVariantFold, ordinary, g, ref_cells + esc_off[b], ref_cnt + b,
                                      std::min(cnt[b], E.n_sm() * 8), S.nb_rec, S.nb_n, ind_value, S.pair64,
                                      S.pair32, mean, c0, steps, tol, out, esc_cells + esc_off[b], esc_cnt + b,
                                      E.n_sm(), st));
            E.stats.launches += 1;
        }
        // FP64 re-solve of escalated systems, one persistent launch per bucket
        for (int b = 0; b < 4; ++b)
        {
            if (cnt[b] == 0) continue;
            HB_CK(launch_solve_bucket(kBucketNP[b], 0, kVariantDefault, ordinary, g, esc_cells + esc_off[b],
                                      esc_cnt + b, std::min(cnt[b], E.n_sm() * 8), S.nb_rec, S.nb_n, ind_value,
                                      S.pair64, S.pair32, mean, c0, 0, tol, out, nullptr, nullptr, E.n_sm(), st));
            E.stats.launches += 1;
        }
        int esc[2 * kBuckets];
        HB_CK(cudaMemcpyAsync(esc, esc_cnt, sizeof(esc), cudaMemcpyDeviceToHost, st));
        HB_CK(cudaStreamSynchronize(st));
        for (int b = 0; b < kBuckets; ++b)
        {
            E.stats.escalated += esc[b];
            E.stats.refined += esc[kBuckets + b];
        }
    }
    else
        HB_CK(cudaStreamSynchronize(st));
    E.mark(STAGE_SOLVE, st);
    for (int b = 0; b < kBuckets; ++b)
        if (cnt[b] > 0)
        {
            float ms = 0;
            cudaEventElapsedTime(&ms, E.ev_[10 + 2 * b], E.ev_[11 + 2 * b]);
            E.stats.bucket_ms[b] += ms;
        }
}

// ------------------------------------------------------------------ io helpers
struct IoPlan
{
    bool device;
    cudaStream_t st;
};

// Host arrays that are not page-locked (numpy arrays, std::vector) and hold at
// least kStageMin bytes are copied through a page-locked area by several host
// threads: a pageable cudaMemcpy moved the benchmark's 42 MB of inputs at about
// 11 GB/s and its outputs at about 5 GB/s into freshly allocated arrays (the
// first touch of each page in the copy's path), a third of the Python API's
// call time.
constexpr size_t kStageMin = 4u << 20;

// true for ordinary pageable host memory (not page-locked, registered, device
// or managed memory: those go to cudaMemcpyAsync as they are)
static bool host_pageable(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// memcpy split over up to eight host threads (4 MB at least each)
static void par_memcpy(void *dst, const void *src, size_t bytes)
{
    int nt = (int)std::min<size_t>(8, bytes / kStageMin);
    nt = std::min(nt, get_threads());
    if (nt <= 1)
    {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t chunk = (bytes / nt + 4095) & ~(size_t)4095;
    std::vector<std::thread> pool;
    for (int i = 0; i < nt; ++i)
    {
        const size_t off = (size_t)i * chunk;
        if (off >= bytes) break;
        const size_t len = std::min(chunk, bytes - off);
        pool.emplace_back([=]() { std::memcpy((char *)dst + off, (const char *)src + off, len); });
    }
    for (auto &th : pool) th.join();
}

template <typename T>
static T *to_device(Engine &E, const char *slot, const T *src, size_t n, const IoPlan &io)
{
    if (io.device) return const_cast<T *>(src);
    T *d = E.buf<T>(slot, n);
    const size_t bytes = n * sizeof(T);
    if (bytes < kStageMin || !host_pageable(src))
        HB_CK(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, io.st));
    else
    {
        unsigned char *h = E.pinned(slot, bytes);
        par_memcpy(h, src, bytes);
        HB_CK(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, io.st));
    }
    E.stats.h2d += bytes;
    return d;
}

template <typename T>
static void to_host(Engine &E, T *dst, const T *dsrc, size_t n, const IoPlan &io)
{
    if (io.device || dst == dsrc) return;
    const size_t bytes = n * sizeof(T);
    if (bytes < kStageMin || !host_pageable(dst))
        HB_CK(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToHost, io.st));
    else
    {
        unsigned char *h = E.pinned("download_" + std::to_string(E.n_downloads++), bytes);
        HB_CK(cudaMemcpyAsync(h, dsrc, bytes, cudaMemcpyDeviceToHost, io.st));
        E.pending.push_back({dst, h, bytes});
    }
    E.stats.d2h += bytes;
}

static void begin_call(Engine &E, cudaStream_t st)
{
    if (!E.pending.empty()) HB_CK(cudaStreamSynchronize(st)); // a call that failed after queuing downloads
    E.pending.clear();
    E.n_downloads = 0;
    E.stats = Stats();
    HB_CK(cudaEventRecord(E.ev_[0], st));
    E.reset_marks(st);
}
static void end_call(Engine &E, cudaStream_t st)
{
    HB_CK(cudaEventRecord(E.ev_[1], st));
    HB_CK(cudaEventSynchronize(E.ev_[1]));
    float ms = 0;
    HB_CK(cudaEventElapsedTime(&ms, E.ev_[0], E.ev_[1]));
    E.stats.total_ms = ms;
    E.collect_marks();
    for (const Engine::PendingCopy &c : E.pending) par_memcpy(c.dst, c.src, c.bytes);
    E.pending.clear();
}

// ------------------------------------------------------------------ entry points
int cont_kriging(int kind, const int *dims, const float *in_data, const unsigned char *in_mask,
                 const SkArgs &a, float *out_data, unsigned char *out_mask, const Options &opt, const float *means)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (!dims || !in_data || !in_mask || !out_data || !out_mask) throw CudaFail{-1, "null array argument"};
        if (kind < 0 || kind > 2) throw CudaFail{-1, "unknown kriging kind"};
        const bool lvm = kind == 2;
        if (lvm && !means) throw CudaFail{-1, "LVM kriging needs the mean array"};
        long long n = check_dims(dims);
        const bool simple = kind != 0; // SK and LVM share the truncated covariance and SK weights
        check_model_args(a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb);
        // the host tables are built while the grid is uploaded and compacted
        double plan_ms = 0.0;
        auto plan_f = std::async(std::launch::async, [&]() {
            const auto t0 = std::chrono::steady_clock::now();
            Plan p = make_plan(simple, a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb, dims);
            plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return p;
        });
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(opt.stream);
        IoPlan io{(opt.flags & 1u) != 0, st};
        begin_call(E, st);

        const float *d_in = to_device(E, "in_data", in_data, (size_t)n, io);
        const uint8_t *d_mask = to_device(E, "in_mask", in_mask, (size_t)n, io);
        const float *d_means = lvm ? to_device(E, "in_means", means, (size_t)n, io) : nullptr;
        float *d_out = io.device ? out_data : E.buf<float>("out_data", (size_t)n);
        uint8_t *d_omask = io.device ? out_mask : E.buf<uint8_t>("out_mask", (size_t)n);
        if (!io.device)
        {
            if (opt.flags & 2u)
            {
                HB_CK(cudaMemcpyAsync(d_out, d_in, n * 4, cudaMemcpyDeviceToDevice, st));
                HB_CK(cudaMemcpyAsync(d_omask, d_mask, n, cudaMemcpyDeviceToDevice, st));
            }
            else
            {
                HB_CK(cudaMemcpyAsync(d_out, out_data, n * 4, cudaMemcpyHostToDevice, st));
                HB_CK(cudaMemcpyAsync(d_omask, out_mask, n, cudaMemcpyHostToDevice, st));
                E.stats.h2d += n * 5;
            }
        }
        double *d_est = nullptr, *d_var = nullptr;
        signed char *d_status = nullptr;
        if (opt.estimate64) d_est = io.device ? opt.estimate64 : E.buf<double>("est64", (size_t)n);
        if (opt.variance) d_var = io.device ? opt.variance : E.buf<double>("var", (size_t)n);
        d_status = (io.device && opt.status) ? opt.status : E.buf<signed char>("status", (size_t)n);

        // SK mean: calc_mean over informed cells (calc_mean.cpp:6-30), on the host
        // data. LVM centres the values on their own means as they are compacted,
        // so the uniform mean stays 0 there.
        double mean = 0.0;
        if (kind == 1)
        {
            if (a.auto_mean)
            {
                std::vector<float> hv;
                std::vector<uint8_t> hm;
                const float *pv = in_data;
                const uint8_t *pm = in_mask;
                if (io.device)
                {
                    hv.resize(n);
                    hm.resize(n);
                    HB_CK(cudaMemcpyAsync(hv.data(), in_data, n * 4, cudaMemcpyDeviceToHost, st));
                    HB_CK(cudaMemcpyAsync(hm.data(), in_mask, n, cudaMemcpyDeviceToHost, st));
                    HB_CK(cudaStreamSynchronize(st));
                    pv = hv.data();
                    pm = hm.data();
                }
                double sum = 0;
                long long cnt = 0;
                for (long long i = 0; i < n; ++i)
                    if (pm[i])
                    {
                        sum += pv[i];
                        cnt += 1;
                    }
                mean = cnt ? sum / cnt : 0.0;
            }
            else
                mean = a.mean;
        }

        HB_CK(cudaEventRecord(E.ev_[2], st));
        DevPoints P = compact_points(E, grid_geom(dims), d_mask, d_in, nullptr, st, d_means);
        const Plan pl = plan_f.get();
        E.stats.plan_ms = plan_ms;
        DevSearch S = run_search(E, pl, P, d_mask, 0, st, false, (opt.flags & 4u) != 0);
        HB_CK(cudaEventRecord(E.ev_[3], st));
        SolveOut so{};
        so.out_data = d_out;
        so.out_mask = d_omask;
        so.est64 = d_est;
        so.var = d_var;
        so.status = d_status;
        so.write_cont = 1;
        so.cell_mean = d_means;
        int steps = opt.refine_steps > 0 ? opt.refine_steps : 2;
        run_solves(E, pl, P, S, d_mask, 0, !simple, opt.precision, steps, opt.tolerance, mean, -1, d_status, so, st);
        launch_finalize_cont(pl.g, d_in, d_status, simple ? 1 : 0, (float)mean, d_means, d_out, d_omask, d_est, d_var,
                             st);
        HB_CK(cudaGetLastError());
        E.stats.launches += 1;
        HB_CK(cudaEventRecord(E.ev_[4], st));
        E.mark(STAGE_FINALIZE, st);

        to_host(E, out_data, d_out, (size_t)n, io);
        to_host(E, out_mask, d_omask, (size_t)n, io);
        if (opt.estimate64) to_host(E, opt.estimate64, d_est, (size_t)n, io);
        if (opt.variance) to_host(E, opt.variance, d_var, (size_t)n, io);
        if (opt.status) to_host(E, opt.status, d_status, (size_t)n, io);
        E.mark(STAGE_DOWNLOAD, st);
        end_call(E, st);
        float ms_search = 0, ms_solve = 0;
        cudaEventElapsedTime(&ms_search, E.ev_[2], E.ev_[3]);
        cudaEventElapsedTime(&ms_solve, E.ev_[3], E.ev_[4]);
        E.stats.search_ms = ms_search;
        E.stats.solve_ms = ms_solve;
        E.stats.ties = S.ties;
        E.stats.template_cells = S.template_cells;
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

int indicator_kriging(const int *dims, const unsigned char *in_data, const unsigned char *in_mask,
                      const std::vector<IkArgs> &cats, unsigned char *out_data, unsigned char *out_mask,
                      const Options &opt)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (!dims || !in_data || !in_mask || !out_data || !out_mask) throw CudaFail{-1, "null array argument"};
        long long n = check_dims(dims);
        const int m = (int)cats.size();
        if (m < 1) throw CudaFail{-1, "indicator_count must be positive"};
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(opt.stream);
        IoPlan io{(opt.flags & 1u) != 0, st};
        begin_call(E, st);
        const uint8_t *d_in = to_device(E, "in_u8", in_data, (size_t)n, io);
        const uint8_t *d_mask = to_device(E, "in_mask", in_mask, (size_t)n, io);
        uint8_t *d_out = io.device ? out_data : E.buf<uint8_t>("out_u8", (size_t)n);
        uint8_t *d_omask = io.device ? out_mask : E.buf<uint8_t>("out_mask", (size_t)n);
        float *d_probs = (io.device && opt.ik_probs) ? opt.ik_probs : E.buf<float>("ik_probs", (size_t)n * m);
        signed char *d_status = E.buf<signed char>("status", (size_t)n);
        HB_CK(cudaEventRecord(E.ev_[2], st));
        Plan pl0 = make_plan(true, cats[0].cov_type, cats[0].ranges, cats[0].angles, cats[0].sill, cats[0].nugget,
                             cats[0].radiuses, cats[0].max_nb, dims);
        DevPoints P = compact_points(E, pl0.g, d_mask, nullptr, d_in, st);
        float search_ms = 0, solve_ms = 0;
        for (int c = 0; c < m; ++c)
        {
            const IkArgs &a = cats[c];
            Plan pl = c == 0 ? pl0
                             : make_plan(true, a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb,
                                         dims);
            HB_CK(cudaEventRecord(E.ev_[5], st));
            DevSearch S = run_search(E, pl, P, d_mask, 1, st, false, (opt.flags & 4u) != 0);
            HB_CK(cudaEventRecord(E.ev_[6], st));
            SolveOut so{};
            so.status = d_status;
            so.prob = d_probs + c;
            so.prob_stride = m;
            // marginal stored as float (ik_params.h:20); the mean provider widens it back
            const float mc = (float)a.marginal;
            run_solves(E, pl, P, S, d_mask, 1, false, opt.precision, opt.refine_steps > 0 ? opt.refine_steps : 2,
                       opt.tolerance, (double)mc, c, d_status, so, st);
            launch_ik_fail_fill(pl.g, d_status, mc, c, m, d_probs, st);
            HB_CK(cudaEventRecord(E.ev_[7], st));
            HB_CK(cudaEventSynchronize(E.ev_[7]));
            float a1 = 0, a2 = 0;
            cudaEventElapsedTime(&a1, E.ev_[5], E.ev_[6]);
            cudaEventElapsedTime(&a2, E.ev_[6], E.ev_[7]);
            search_ms += a1;
            solve_ms += a2;
            E.stats.ties += S.ties;
            E.stats.template_cells += S.template_cells;
        }
        launch_ik_finalize(n, m, d_probs, d_out, d_omask, st);
        HB_CK(cudaGetLastError());
        to_host(E, out_data, d_out, (size_t)n, io);
        to_host(E, out_mask, d_omask, (size_t)n, io);
        if (opt.ik_probs) to_host(E, opt.ik_probs, d_probs, (size_t)n * m, io);
        end_call(E, st);
        E.stats.search_ms = search_ms;
        E.stats.solve_ms = solve_ms;
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

int median_ik(const int *dims, const unsigned char *in_data, const unsigned char *in_mask, const IkArgs &a,
              double marginal1, unsigned char *out_data, unsigned char *out_mask, const Options &opt)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (!dims || !in_data || !in_mask || !out_data || !out_mask) throw CudaFail{-1, "null array argument"};
        long long n = check_dims(dims);
        check_model_args(a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb);
        auto plan_f = std::async(std::launch::async, [&]() {
            return make_plan(true, a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb, dims);
        });
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(opt.stream);
        IoPlan io{(opt.flags & 1u) != 0, st};
        begin_call(E, st);
        const uint8_t *d_in = to_device(E, "in_u8", in_data, (size_t)n, io);
        const uint8_t *d_mask = to_device(E, "in_mask", in_mask, (size_t)n, io);
        uint8_t *d_out = io.device ? out_data : E.buf<uint8_t>("out_u8", (size_t)n);
        uint8_t *d_omask = io.device ? out_mask : E.buf<uint8_t>("out_mask", (size_t)n);
        signed char *d_status = E.buf<signed char>("status", (size_t)n);
        double *d_est = E.buf<double>("est64", (size_t)n);
        float *d_prob = opt.ik_probs ? ((io.device) ? opt.ik_probs : E.buf<float>("ik_probs", (size_t)n)) : nullptr;
        HB_CK(cudaEventRecord(E.ev_[2], st));
        DevPoints P = compact_points(E, grid_geom(dims), d_mask, nullptr, d_in, st);
        const Plan pl = plan_f.get();
        DevSearch S = run_search(E, pl, P, d_mask, 1, st, false, (opt.flags & 4u) != 0);
        HB_CK(cudaEventRecord(E.ev_[3], st));
        SolveOut so{};
        so.status = d_status;
        so.est64 = d_est;
        run_solves(E, pl, P, S, d_mask, 1, false, opt.precision, opt.refine_steps > 0 ? opt.refine_steps : 2,
                   opt.tolerance, marginal1, 1, d_status, so, st);
        launch_mik_finalize(n, d_status, d_est, marginal1, d_out, d_omask, d_prob, st);
        HB_CK(cudaGetLastError());
        HB_CK(cudaEventRecord(E.ev_[4], st));
        to_host(E, out_data, d_out, (size_t)n, io);
        to_host(E, out_mask, d_omask, (size_t)n, io);
        if (opt.ik_probs) to_host(E, opt.ik_probs, d_prob, (size_t)n, io);
        end_call(E, st);
        float a1 = 0, a2 = 0;
        cudaEventElapsedTime(&a1, E.ev_[2], E.ev_[3]);
        cudaEventElapsedTime(&a2, E.ev_[3], E.ev_[4]);
        E.stats.search_ms = a1;
        E.stats.solve_ms = a2;
        E.stats.ties = S.ties;
        E.stats.template_cells = S.template_cells;
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

// ------------------------------------------------------------------ SGS
// The walk of path_random_generator.cpp:24-67: R <- (A R + C) mod size from
// seed % size, A = 1 + the product of the primes dividing size (doubled when 4
// divides size), C = the largest prime not above size / 3 that does not divide
// size, 2 when there is none. Returns false when the walk is not a permutation
// (C = 2 dividing size: grids of a few cells).
static bool is_prime_ll(long long p)
{
    if (p < 2) return false;
    for (long long d = 2; d * d <= p; ++d)
        if (p % d == 0) return false;
    return true;
}

static bool sgs_walk(long long size, long long seed, SgsWalk &w)
{
    long long A = 1, m = size;
    for (long long p = 2; p * p <= m; ++p)
        if (m % p == 0)
        {
            A *= p;
            while (m % p == 0) m /= p;
        }
    if (m > 1) A *= m;
    if (size % 4 == 0) A *= 2;
    A += 1;
    long long C = 2;
    for (long long p = size / 3; p >= 3; --p)
        if (size % p != 0 && is_prime_ll(p))
        {
            C = p;
            break;
        }
    w.A = A;
    w.C = C;
    w.M = size;
    w.R0 = seed % size;
    return size % C != 0;
}

int sgs_simulation(const int *dims, float *data, unsigned char *mask, const unsigned char *sim_mask,
                   const CdfTable *cdf, const float *means, const SgsArgs &a, const Options &opt)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (!dims || !data || !mask) throw CudaFail{-1, "null array argument"};
        const long long n = check_dims(dims);
        if (n > 10000000) throw CudaFail{-4, "the simulation path supports at most 10,000,000 cells"};
        check_model_args(a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb);
        if (a.max_nb > kSgsBlockMax)
            throw CudaFail{-4, "simulation supports max_neighbours up to " + std::to_string(kSgsBlockMax)};
        SgsWalk walk;
        const bool full_period = sgs_walk(n, a.seed, walk);
        if (walk.R0 < 0) throw CudaFail{-1, "seed % grid size must not be negative"};
        const bool use_cdf = cdf && cdf->values && cdf->probs && cdf->size > 0;
        const bool lvm = means != nullptr;
        const bool ordinary = !lvm && a.kind == 0;
        double plan_ms = 0.0;
        auto plan_f = std::async(std::launch::async, [&]() {
            const auto t0 = std::chrono::steady_clock::now();
            // the simulation's search is the template scan alone: no float prefilter tables
            Plan p = make_plan(true, a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb, dims,
                               false);
            std::vector<Offset> tv = build_template(p.f, p.kt);
            plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return std::make_pair(std::move(p), std::move(tv));
        });
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(opt.stream);
        IoPlan io{(opt.flags & 1u) != 0, st};
        begin_call(E, st);

        // in/out property: data and mask are simulated in place
        float *d_data = io.device ? data : E.buf<float>("sgs_data", (size_t)n);
        uint8_t *d_mask = io.device ? mask : E.buf<uint8_t>("sgs_mask", (size_t)n);
        if (!io.device)
        {
            HB_CK(cudaMemcpyAsync(d_data, data, n * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaMemcpyAsync(d_mask, mask, n, cudaMemcpyHostToDevice, st));
            E.stats.h2d += n * 5;
        }
        const uint8_t *d_sim = sim_mask ? to_device(E, "sgs_sim_mask", sim_mask, (size_t)n, io) : nullptr;
        const float *d_means_in = lvm ? to_device(E, "sgs_means_in", means, (size_t)n, io) : nullptr;
        float *d_means = lvm ? E.buf<float>("sgs_means", (size_t)n) : nullptr;
        float *d_cv = nullptr, *d_cp = nullptr;
        if (use_cdf)
        {
            d_cv = E.buf<float>("sgs_cdf_v", (size_t)cdf->size);
            d_cp = E.buf<float>("sgs_cdf_p", (size_t)cdf->size);
            HB_CK(cudaMemcpyAsync(d_cv, cdf->values, cdf->size * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaMemcpyAsync(d_cp, cdf->probs, cdf->size * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaStreamSynchronize(st)); // the tables are caller memory, possibly pageable
        }
        E.mark(STAGE_UPLOAD, st);

        // the walk -> ranks of the simulated nodes
        int *rank_of = E.buf<int>("sgs_rank_of", (size_t)n);
        int *sim_cells = E.buf<int>("sgs_sim_cells", (size_t)n);
        int n_sim = 0;
        if (full_period)
        {
            int *path_cell = E.buf<int>("sgs_path", (size_t)n);
            int *flag = E.buf<int>("sgs_flag", (size_t)n);
            int *tmp = E.buf<int>("scan_tmp", (size_t)scan_tmp_ints(n) + 4);
            int *total = E.buf<int>("sgs_total", 1);
            launch_sgs_path(walk, d_mask, d_sim, path_cell, flag, st);
            int *scan = E.buf<int>("sgs_scan", (size_t)n);
            HB_CK(cudaMemcpyAsync(scan, flag, n * 4, cudaMemcpyDeviceToDevice, st));
            exclusive_scan(scan, n, tmp, total, st);
            launch_sgs_index(n, path_cell, flag, scan, d_mask, rank_of, sim_cells, st);
            HB_CK(cudaGetLastError());
            E.stats.launches += 2 + scan_kernels(n);
            HB_CK(cudaMemcpyAsync(&n_sim, total, sizeof(int), cudaMemcpyDeviceToHost, st));
            HB_CK(cudaStreamSynchronize(st));
        }
        else
        {
            // a walk that revisits nodes (grids of a few cells): the first visit of
            // an uninformed node with simulation mask 1 simulates it
            std::vector<uint8_t> hm(n), hs(sim_mask ? n : 0), seen(n, 0);
            std::vector<int> hr(n), hc;
            HB_CK(cudaMemcpyAsync(hm.data(), d_mask, n, cudaMemcpyDeviceToHost, st));
            if (d_sim) HB_CK(cudaMemcpyAsync(hs.data(), d_sim, n, cudaMemcpyDeviceToHost, st));
            HB_CK(cudaStreamSynchronize(st));
            for (long long i = 0; i < n; ++i) hr[i] = hm[i] ? -1 : INT_MAX;
            long long R = walk.R0;
            for (long long p = 0; p < n; ++p)
            {
                const int c = (int)R;
                if (!hm[c] && !seen[c] && (!d_sim || hs[c] == 1))
                {
                    seen[c] = 1;
                    hr[c] = (int)hc.size();
                    hc.push_back(c);
                }
                R = (walk.A * R + walk.C) % walk.M;
            }
            n_sim = (int)hc.size();
            HB_CK(cudaMemcpyAsync(rank_of, hr.data(), n * 4, cudaMemcpyHostToDevice, st));
            if (n_sim) HB_CK(cudaMemcpyAsync(sim_cells, hc.data(), (size_t)n_sim * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaStreamSynchronize(st));
        }
        E.mark(STAGE_COMPACT, st);

        // the draws: one uniform per simulated node in walk order, generated on
        // the host while the device searches and levels
        double *h_u = reinterpret_cast<double *>(E.staging2((size_t)std::max(n_sim, 1) * 8));
        double draws_ms = 0.0;
        auto draws_f = std::async(std::launch::async, [&, n_sim]() {
            const auto t0 = std::chrono::steady_clock::now();
            sgs_draws((unsigned long long)a.seed, n_sim, h_u);
            draws_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        });

        auto plan_pair = plan_f.get();
        const Plan &pl = plan_pair.first;
        const std::vector<Offset> &tv = plan_pair.second;
        E.stats.plan_ms = plan_ms;
        const Geom &g = pl.g;
        const size_t nk = pl.kt.vals.size();
        double *search_vals = E.buf<double>("search_vals", nk);
        HB_CK(cudaMemcpyAsync(search_vals, pl.kt.vals.data(), nk * 8, cudaMemcpyHostToDevice, st));
        const long long pn = (long long)g.pnx * g.pny * (2 * g.phz + 1);
        double *pair64 = E.buf<double>("pair64", (size_t)pn);
        float *pair32 = E.buf<float>("pair32", (size_t)pn);
        launch_build_pair(g, dev_model(pl.f.m), 1, search_vals, pair64, pair32, st);
        E.stats.launches += 1 + ((use_cdf || lvm) ? 1 : 0) + (n_sim > 0 ? 4 : 0); // + search, moments, levels x2
        std::vector<int4> t4(tv.size());
        for (size_t i = 0; i < tv.size(); ++i) t4[i] = make_int4(tv[i].dx, tv[i].dy, tv[i].dz, 0);
        int4 *tmpl = E.buf<int4>("sgs_tmpl", std::max<size_t>(t4.size(), 1));
        if (!t4.empty())
            HB_CK(cudaMemcpyAsync(tmpl, t4.data(), t4.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
        if (use_cdf || lvm)
            launch_sgs_forward(n, d_data, d_mask, d_means_in, d_means, use_cdf ? d_cv : nullptr, d_cp,
                               use_cdf ? cdf->size : 0, st);
        HB_CK(cudaGetLastError());
        HB_CK(cudaStreamSynchronize(st)); // t4 and the key values are host temporaries
        E.mark(STAGE_TABLES, st);

        // neighbours of every simulated node
        const int k = a.max_nb;
        int *nb = E.buf<int>("sgs_nb", (size_t)std::max(n_sim, 1) * k);
        int *nb_rank = E.buf<int>("sgs_nb_rank", (size_t)std::max(n_sim, 1) * k);
        int *nb_cnt = E.buf<int>("sgs_nb_cnt", (size_t)std::max(n_sim, 1));
        if (n_sim > 0)
            launch_sgs_search(g, tmpl, (int)t4.size(), sim_cells, n_sim, rank_of, k, nb, nb_rank, nb_cnt, E.n_sm(),
                              st);
        HB_CK(cudaGetLastError());
        E.mark(STAGE_SEARCH, st);

        // dependency levels
        const int level_cap = 1 << 20;
        int *levp1 = E.buf<int>("sgs_levp1", (size_t)std::max(n_sim, 1));
        int *lvl_count = E.buf<int>("sgs_lvl_count", (size_t)level_cap + 1);
        int *scal = E.buf<int>("sgs_scal", 4); // ticket, max level, error
        double *mom = E.buf<double>("sgs_mom", 3);
        HB_CK(cudaMemsetAsync(mom, 0, 24, st));
        if (n_sim > 0) launch_sgs_moments(n_sim, nb_cnt, mom, E.n_sm(), st);
        HB_CK(cudaMemsetAsync(levp1, 0, (size_t)std::max(n_sim, 1) * 4, st));
        HB_CK(cudaMemsetAsync(lvl_count, 0, ((size_t)level_cap + 1) * 4, st));
        HB_CK(cudaMemsetAsync(scal, 0, 16, st));
        if (n_sim > 0)
            launch_sgs_levels(nb_rank, nb_cnt, k, n_sim, levp1, scal + 0, lvl_count, level_cap, scal + 1, scal + 2,
                              E.n_sm(), st);
        HB_CK(cudaGetLastError());
        int hs[4] = {0, 0, 0, 0};
        double hmom[3] = {0, 0, 0};
        HB_CK(cudaMemcpyAsync(hs, scal, 16, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaMemcpyAsync(hmom, mom, 24, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaStreamSynchronize(st));
        {
            // F(n, r) = n^3/3 + n^2/2 + 2 r n^2 + 30 (n(n+1)/2 + n) + 2 r n, r = 1 (SK) or 2 (OK):
            // the kriging buckets' count, its triangular solves being here a forward and a back pass
            const double rhs = ordinary ? 2.0 : 1.0;
            E.stats.sgs_flops = hmom[2] / 3.0 + hmom[1] * (0.5 + 2.0 * rhs + 15.0) + hmom[0] * (45.0 + 2.0 * rhs);
        }
        if (hs[2] == 1) throw CudaFail{-2, "simulation level pass: a dependency wait timed out"};
        if (hs[2] == 2) throw CudaFail{-4, "simulation needs more than 2^20 dependency levels"};
        const int n_levels = n_sim > 0 ? hs[1] + 1 : 0;
        std::vector<int> counts(std::max(n_levels, 1)), offs(std::max(n_levels, 1) + 1, 0);
        if (n_levels > 0)
        {
            HB_CK(cudaMemcpyAsync(counts.data(), lvl_count, (size_t)n_levels * 4, cudaMemcpyDeviceToHost, st));
            HB_CK(cudaStreamSynchronize(st));
        }
        for (int l = 0; l < n_levels; ++l) offs[l + 1] = offs[l] + counts[l];
        int *order = E.buf<int>("sgs_order", (size_t)std::max(n_sim, 1));
        int *level_off = E.buf<int>("sgs_level_off", (size_t)n_levels + 1);
        int *level_fill = E.buf<int>("sgs_level_fill", (size_t)n_levels + 1);
        if (n_levels > 0)
        {
            HB_CK(cudaMemcpyAsync(level_off, offs.data(), ((size_t)n_levels + 1) * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaMemsetAsync(level_fill, 0, ((size_t)n_levels + 1) * 4, st));
            launch_sgs_level_fill(n_sim, levp1, level_off, level_fill, order, st);
            HB_CK(cudaGetLastError());
            E.stats.launches += 1;
        }
        E.stats.sgs_levels = n_levels;
        E.mark(STAGE_TIES, st);

        // draws in, then one solve launch per level
        draws_f.get();
        E.stats.draws_ms = draws_ms;
        double *d_u = E.buf<double>("sgs_uniforms", (size_t)std::max(n_sim, 1));
        if (n_sim > 0)
        {
            HB_CK(cudaMemcpyAsync(d_u, h_u, (size_t)n_sim * 8, cudaMemcpyHostToDevice, st));
            E.stats.h2d += (long long)n_sim * 8;
        }
        E.mark(STAGE_PREPARE, st);
        signed char *st_rank = E.buf<signed char>("sgs_st_rank", (size_t)std::max(n_sim, 1));
        for (int l = 0; l < n_levels; ++l)
        {
            HB_CK(launch_sgs_solve(g, order + offs[l], counts[l], sim_cells, nb, nb_cnt, k, pair64, d_data, d_means,
                                   d_u, st_rank, ordinary, E.n_sm(), st));
            E.stats.launches += 1;
        }
        E.mark(STAGE_SOLVE, st);
        signed char *d_status =
            opt.status ? (io.device ? opt.status : E.buf<signed char>("status", (size_t)n)) : nullptr;
        launch_sgs_finalize(n, d_data, d_mask, rank_of, n_sim, st_rank, d_status, use_cdf ? d_cv : nullptr, d_cp,
                            use_cdf ? cdf->size : 0, st);
        HB_CK(cudaGetLastError());
        E.stats.launches += 1;
        E.mark(STAGE_FINALIZE, st);
        if (!io.device)
        {
            to_host(E, data, d_data, (size_t)n, io);
            to_host(E, mask, d_mask, (size_t)n, io);
            if (opt.status) to_host(E, opt.status, d_status, (size_t)n, io);
        }
        E.mark(STAGE_DOWNLOAD, st);
        E.stats.kriged = n_sim;
        end_call(E, st);
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

// ------------------------------------------------------------------ levels
int sim_levels(long long n_sim, int k, const int *nb_rank, int *levels)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (n_sim < 0 || n_sim > 10000000 || k <= 0 || k > 4096 || (n_sim > 0 && (!nb_rank || !levels)))
            throw CudaFail{-1, "bad argument"};
        // every listed rank is read by the pass: it must name a rank or be -1
        for (long long i = 0; i < n_sim * k; ++i)
            if (nb_rank[i] < -1 || nb_rank[i] >= n_sim) throw CudaFail{-1, "neighbour rank out of range"};
        if (n_sim == 0) return 0;
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(nullptr);
        begin_call(E, st);
        const size_t ns = (size_t)n_sim;
        int *d_rank = E.buf<int>("lv_nb_rank", ns * k);
        HB_CK(cudaMemcpyAsync(d_rank, nb_rank, ns * k * 4, cudaMemcpyHostToDevice, st));
        const int level_cap = 1 << 20;
        int *levp1 = E.buf<int>("sgs_levp1", ns);
        int *lvl_count = E.buf<int>("sgs_lvl_count", (size_t)level_cap + 1);
        int *scal = E.buf<int>("sgs_scal", 4);
        HB_CK(cudaMemsetAsync(levp1, 0, ns * 4, st));
        HB_CK(cudaMemsetAsync(lvl_count, 0, ((size_t)level_cap + 1) * 4, st));
        HB_CK(cudaMemsetAsync(scal, 0, 16, st));
        launch_sgs_levels(d_rank, nullptr, k, (int)n_sim, levp1, scal + 0, lvl_count, level_cap, scal + 1, scal + 2,
                          E.n_sm(), st);
        HB_CK(cudaGetLastError());
        E.stats.launches += 2;
        int hs[4] = {0, 0, 0, 0};
        HB_CK(cudaMemcpyAsync(hs, scal, 16, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaMemcpyAsync(levels, levp1, ns * 4, cudaMemcpyDeviceToHost, st));
        end_call(E, st);
        if (hs[2] == 1) throw CudaFail{-2, "simulation level pass: a dependency wait timed out"};
        if (hs[2] == 2) throw CudaFail{-4, "simulation needs more than 2^20 dependency levels"};
        for (size_t i = 0; i < ns; ++i) levels[i] -= 1;
        E.stats.sgs_levels = hs[1] + 1;
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

// ------------------------------------------------------------------ SIS
int sis_simulation(const int *dims, unsigned char *data, unsigned char *mask, const unsigned char *sim_mask,
                   const std::vector<IkArgs> &cats, const float *const *means, long long seed, const Options &opt,
                   bool correlogram)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (!dims || !data || !mask) throw CudaFail{-1, "null array argument"};
        const long long n = check_dims(dims);
        if (n > 10000000) throw CudaFail{-4, "the simulation path supports at most 10,000,000 cells"};
        const int ncat = (int)cats.size();
        if (ncat < 2) throw CudaFail{-1, "indicator simulation needs at least two categories"};
        if (ncat > kSisMaxCat)
            throw CudaFail{-4, "indicator simulation supports up to " + std::to_string(kSisMaxCat) + " categories"};
        // median SIS (two categories) krige the first only
        const int kcat = ncat == 2 ? 1 : ncat;
        for (int c = 0; c < kcat; ++c)
        {
            const IkArgs &a = cats[c];
            check_model_args(a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb);
            if (a.max_nb > 32) throw CudaFail{-4, "indicator simulation supports max_neighbours up to 32"};
        }
        SgsWalk walk;
        if (!sgs_walk(n, seed, walk))
            throw CudaFail{-1, "the simulation path does not visit every node of a grid of this size"};
        if (walk.R0 < 0) throw CudaFail{-1, "seed % grid size must not be negative"};
        double plan_ms = 0.0;
        auto plan_f = std::async(std::launch::async, [&]() {
            const auto t0 = std::chrono::steady_clock::now();
            std::vector<std::pair<Plan, std::vector<Offset>>> v;
            for (int c = 0; c < kcat; ++c)
            {
                const IkArgs &a = cats[c];
                Plan p = make_plan(true, a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb, dims,
                                   false);
                std::vector<Offset> tv = build_template(p.f, p.kt);
                v.emplace_back(std::move(p), std::move(tv));
            }
            plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return v;
        });
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(opt.stream);
        IoPlan io{(opt.flags & 1u) != 0, st};
        begin_call(E, st);
        uint8_t *d_data = io.device ? data : E.buf<uint8_t>("sis_data", (size_t)n);
        uint8_t *d_mask = io.device ? mask : E.buf<uint8_t>("sis_mask", (size_t)n);
        if (!io.device)
        {
            HB_CK(cudaMemcpyAsync(d_data, data, n, cudaMemcpyHostToDevice, st));
            HB_CK(cudaMemcpyAsync(d_mask, mask, n, cudaMemcpyHostToDevice, st));
            E.stats.h2d += n * 2;
        }
        const uint8_t *d_sim = sim_mask ? to_device(E, "sgs_sim_mask", sim_mask, (size_t)n, io) : nullptr;
        std::vector<const float *> d_means(kcat, nullptr);
        if (means)
            for (int c = 0; c < kcat; ++c)
            {
                if (!means[c]) throw CudaFail{-1, "LVM indicator simulation needs a mean array per category"};
                const std::string slot = "sis_means_" + std::to_string(c);
                d_means[c] = to_device(E, slot.c_str(), means[c], (size_t)n, io);
            }
        E.mark(STAGE_UPLOAD, st);

        // the walk -> ranks (the same walk as the Gaussian simulation's)
        int *rank_of = E.buf<int>("sgs_rank_of", (size_t)n);
        int *sim_cells = E.buf<int>("sgs_sim_cells", (size_t)n);
        int n_sim = 0;
        {
            int *path_cell = E.buf<int>("sgs_path", (size_t)n);
            int *flag = E.buf<int>("sgs_flag", (size_t)n);
            int *tmp = E.buf<int>("scan_tmp", (size_t)scan_tmp_ints(n) + 4);
            int *total = E.buf<int>("sgs_total", 1);
            int *scan = E.buf<int>("sgs_scan", (size_t)n);
            launch_sgs_path(walk, d_mask, d_sim, path_cell, flag, st);
            HB_CK(cudaMemcpyAsync(scan, flag, n * 4, cudaMemcpyDeviceToDevice, st));
            exclusive_scan(scan, n, tmp, total, st);
            launch_sgs_index(n, path_cell, flag, scan, d_mask, rank_of, sim_cells, st);
            HB_CK(cudaGetLastError());
            HB_CK(cudaMemcpyAsync(&n_sim, total, sizeof(int), cudaMemcpyDeviceToHost, st));
            HB_CK(cudaStreamSynchronize(st));
            E.stats.launches += 2 + scan_kernels(n);
        }
        E.mark(STAGE_COMPACT, st);
        double *h_u = reinterpret_cast<double *>(E.staging2((size_t)std::max(n_sim, 1) * 8));
        double draws_ms = 0.0;
        auto draws_f = std::async(std::launch::async, [&, n_sim]() {
            const auto t0 = std::chrono::steady_clock::now();
            sgs_draws((unsigned long long)seed, n_sim, h_u);
            draws_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        });

        // per category: pair table, template, search (ranks into one merged row per node)
        auto plans = plan_f.get();
        E.stats.plan_ms = plan_ms;
        int ktot = 0;
        std::vector<int> koff(kcat);
        for (int c = 0; c < kcat; ++c)
        {
            koff[c] = ktot;
            ktot += cats[c].max_nb;
        }
        const size_t ns = (size_t)std::max(n_sim, 1);
        int *nb_rank = E.buf<int>("sis_nb_rank", ns * ktot);
        HB_CK(cudaMemsetAsync(nb_rank, 0xFF, ns * ktot * 4, st)); // -1: no neighbour
        std::vector<double *> pair64(kcat);
        std::vector<int *> nb(kcat), nb_cnt(kcat);
        for (int c = 0; c < kcat; ++c)
        {
            const Plan &pl = plans[c].first;
            const std::vector<Offset> &tv = plans[c].second;
            const Geom &g = pl.g;
            const std::string sfx = std::to_string(c);
            const size_t nk = pl.kt.vals.size();
            double *sv = E.buf<double>(("sis_vals_" + sfx).c_str(), nk);
            HB_CK(cudaMemcpyAsync(sv, pl.kt.vals.data(), nk * 8, cudaMemcpyHostToDevice, st));
            const long long pn = (long long)g.pnx * g.pny * (2 * g.phz + 1);
            pair64[c] = E.buf<double>(("sis_pair64_" + sfx).c_str(), (size_t)pn);
            float *p32 = E.buf<float>(("sis_pair32_" + sfx).c_str(), (size_t)pn);
            launch_build_pair(g, dev_model(pl.f.m), 1, sv, pair64[c], p32, st);
            std::vector<int4> t4(tv.size());
            for (size_t i = 0; i < tv.size(); ++i) t4[i] = make_int4(tv[i].dx, tv[i].dy, tv[i].dz, 0);
            int4 *tmpl = E.buf<int4>(("sis_tmpl_" + sfx).c_str(), std::max<size_t>(t4.size(), 1));
            if (!t4.empty())
                HB_CK(cudaMemcpyAsync(tmpl, t4.data(), t4.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
            nb[c] = E.buf<int>(("sis_nb_" + sfx).c_str(), ns * cats[c].max_nb);
            nb_cnt[c] = E.buf<int>(("sis_nb_cnt_" + sfx).c_str(), ns);
            if (n_sim > 0)
                launch_sgs_search(g, tmpl, (int)t4.size(), sim_cells, n_sim, rank_of, cats[c].max_nb, nb[c],
                                  nb_rank + koff[c], nb_cnt[c], E.n_sm(), st, -1, ktot);
            HB_CK(cudaGetLastError());
            HB_CK(cudaStreamSynchronize(st)); // the host tables of this category
            E.stats.launches += 1 + (n_sim > 0 ? 1 : 0);
        }
        E.mark(STAGE_SEARCH, st);

        // the solves' size moments over every category's systems
        double *mom = E.buf<double>("sgs_mom", 3);
        HB_CK(cudaMemsetAsync(mom, 0, 24, st));
        if (n_sim > 0)
        {
            for (int c = 0; c < kcat; ++c) launch_sgs_moments(n_sim, nb_cnt[c], mom, E.n_sm(), st);
            E.stats.launches += kcat;
        }
        // dependency levels over the union of the categories' neighbours
        const int level_cap = 1 << 20;
        int *levp1 = E.buf<int>("sgs_levp1", ns);
        int *lvl_count = E.buf<int>("sgs_lvl_count", (size_t)level_cap + 1);
        int *scal = E.buf<int>("sgs_scal", 4);
        HB_CK(cudaMemsetAsync(levp1, 0, ns * 4, st));
        HB_CK(cudaMemsetAsync(lvl_count, 0, ((size_t)level_cap + 1) * 4, st));
        HB_CK(cudaMemsetAsync(scal, 0, 16, st));
        if (n_sim > 0)
        {
            launch_sgs_levels(nb_rank, nullptr, ktot, n_sim, levp1, scal + 0, lvl_count, level_cap, scal + 1,
                              scal + 2, E.n_sm(), st);
            E.stats.launches += 2;
        }
        HB_CK(cudaGetLastError());
        int hs[4] = {0, 0, 0, 0};
        double hmom[3] = {0, 0, 0};
        HB_CK(cudaMemcpyAsync(hs, scal, 16, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaMemcpyAsync(hmom, mom, 24, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaStreamSynchronize(st));
        // the simple-kriging count F(n, 1) of the Gaussian simulation, per category system
        E.stats.sgs_flops = hmom[2] / 3.0 + hmom[1] * (0.5 + 2.0 + 15.0) + hmom[0] * (45.0 + 2.0);
        if (hs[2] == 1) throw CudaFail{-2, "simulation level pass: a dependency wait timed out"};
        if (hs[2] == 2) throw CudaFail{-4, "simulation needs more than 2^20 dependency levels"};
        const int n_levels = n_sim > 0 ? hs[1] + 1 : 0;
        std::vector<int> counts(std::max(n_levels, 1)), offs(std::max(n_levels, 1) + 1, 0);
        if (n_levels > 0)
        {
            HB_CK(cudaMemcpyAsync(counts.data(), lvl_count, (size_t)n_levels * 4, cudaMemcpyDeviceToHost, st));
            HB_CK(cudaStreamSynchronize(st));
        }
        for (int l = 0; l < n_levels; ++l) offs[l + 1] = offs[l] + counts[l];
        int *order = E.buf<int>("sgs_order", ns);
        int *level_off = E.buf<int>("sgs_level_off", (size_t)n_levels + 1);
        int *level_fill = E.buf<int>("sgs_level_fill", (size_t)n_levels + 1);
        if (n_levels > 0)
        {
            HB_CK(cudaMemcpyAsync(level_off, offs.data(), ((size_t)n_levels + 1) * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaMemsetAsync(level_fill, 0, ((size_t)n_levels + 1) * 4, st));
            launch_sgs_level_fill(n_sim, levp1, level_off, level_fill, order, st);
            HB_CK(cudaGetLastError());
            E.stats.launches += 1;
        }
        E.stats.sgs_levels = n_levels;
        E.mark(STAGE_TIES, st);

        draws_f.get();
        E.stats.draws_ms = draws_ms;
        double *d_u = E.buf<double>("sgs_uniforms", ns);
        if (n_sim > 0)
        {
            HB_CK(cudaMemcpyAsync(d_u, h_u, (size_t)n_sim * 8, cudaMemcpyHostToDevice, st));
            E.stats.h2d += (long long)n_sim * 8;
        }
        E.mark(STAGE_PREPARE, st);
        double *probs = E.buf<double>("sis_probs", ns * kcat);
        signed char *st_cat = E.buf<signed char>("sis_st_cat", ns * kcat);
        int *done = E.buf<int>("sis_done", ns);
        signed char *st_rank = E.buf<signed char>("sgs_st_rank", ns);
        std::vector<SisCat> hc(kcat);
        for (int c = 0; c < kcat; ++c)
        {
            const Geom &g = plans[c].first.g;
            hc[c] = SisCat{pair64[c], nb[c], nb_cnt[c], d_means[c], g.pair_center, g.pnx, g.pny, cats[c].max_nb,
                           (float)cats[c].marginal};
        }
        int kmax = 0;
        for (int c = 0; c < kcat; ++c) kmax = std::max(kmax, cats[c].max_nb);
        SisCat *d_cats = E.buf<SisCat>("sis_cats", kSisMaxCat);
        HB_CK(cudaMemcpyAsync(d_cats, hc.data(), kcat * sizeof(SisCat), cudaMemcpyHostToDevice, st));
        HB_CK(cudaMemsetAsync(done, 0, ns * 4, st));
        for (int l = 0; l < n_levels; ++l)
        {
            SisLevelArgs la{d_cats, dims[0], dims[1], order + offs[l], counts[l], kcat, ncat, sim_cells, d_data,
                            probs, st_cat, done, d_u, st_rank, correlogram && means ? 1 : 0, kmax};
            HB_CK(launch_sis_level(la, E.n_sm(), st));
            E.stats.launches += 1;
        }
        HB_CK(cudaGetLastError());
        E.mark(STAGE_SOLVE, st);
        signed char *d_status =
            opt.status ? (io.device ? opt.status : E.buf<signed char>("status", (size_t)n)) : nullptr;
        // masks and status (no transform): the simulation's finalize on an empty CDF
        launch_sgs_finalize(n, nullptr, d_mask, rank_of, n_sim, st_rank, d_status, nullptr, nullptr, 0, st);
        HB_CK(cudaGetLastError());
        E.stats.launches += 1;
        E.mark(STAGE_FINALIZE, st);
        if (!io.device)
        {
            to_host(E, data, d_data, (size_t)n, io);
            to_host(E, mask, d_mask, (size_t)n, io);
            if (opt.status) to_host(E, opt.status, d_status, (size_t)n, io);
        }
        E.mark(STAGE_DOWNLOAD, st);
        E.stats.kriged = n_sim;
        end_call(E, st);
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

// ------------------------------------------------------------------ cokriging
int cokriging(const int *dims, const float *pdata, const unsigned char *pmask, const float *sdata,
              const unsigned char *smask, const CokArgs &a, float *out_data, unsigned char *out_mask,
              const Options &opt)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (!dims || !pdata || !pmask || !sdata || !smask || !out_data || !out_mask)
            throw CudaFail{-1, "null array argument"};
        if (a.mark != 1 && a.mark != 2) throw CudaFail{-1, "cokriging: mark must be 1 or 2"};
        const long long n = check_dims(dims);
        const CovArgs &pc = a.primary;
        check_model_args(pc.cov_type, pc.ranges, pc.angles, pc.sill, pc.nugget, a.radiuses, a.max_nb);
        if (a.mark == 2)
            check_model_args(a.secondary.cov_type, a.secondary.ranges, a.secondary.angles, a.secondary.sill,
                             a.secondary.nugget, a.radiuses, a.max_nb);
        if (a.max_nb > kSgsBlockMax)
            throw CudaFail{-4, "cokriging supports max_neighbours up to " + std::to_string(kSgsBlockMax)};
        if (!std::isfinite(a.primary_mean) || !std::isfinite(a.secondary_mean) ||
            !std::isfinite(a.secondary_variance) || !std::isfinite(a.corr))
            throw CudaFail{-1, "cokriging means, variance and correlation must be finite"};
        // the analytic primary model (the template and A, b), and the cross model
        double plan_ms = 0.0;
        auto plan_f = std::async(std::launch::async, [&]() {
            const auto t0 = std::chrono::steady_clock::now();
            Plan p = make_plan(false, pc.cov_type, pc.ranges, pc.angles, pc.sill, pc.nugget, a.radiuses, a.max_nb,
                               dims, false);
            std::vector<Offset> tv = build_template(p.f, p.kt);
            plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return std::make_pair(std::move(p), std::move(tv));
        });
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(opt.stream);
        IoPlan io{(opt.flags & 1u) != 0, st};
        begin_call(E, st);
        const float *d_pd = to_device(E, "cok_pdata", pdata, (size_t)n, io);
        const uint8_t *d_pm = to_device(E, "cok_pmask", pmask, (size_t)n, io);
        const float *d_sd = to_device(E, "cok_sdata", sdata, (size_t)n, io);
        const uint8_t *d_sm = to_device(E, "cok_smask", smask, (size_t)n, io);
        float *d_out = io.device ? out_data : E.buf<float>("out_data", (size_t)n);
        uint8_t *d_omask = io.device ? out_mask : E.buf<uint8_t>("out_mask", (size_t)n);
        signed char *d_status =
            opt.status ? (io.device ? opt.status : E.buf<signed char>("status", (size_t)n)) : nullptr;
        E.mark(STAGE_UPLOAD, st);

        // targets: the uninformed primary cells in ascending order
        int *flag = E.buf<int>("cok_flag", (size_t)n);
        int *pos = E.buf<int>("cok_pos", (size_t)n);
        int *tmp = E.buf<int>("scan_tmp", (size_t)scan_tmp_ints(n) + 4);
        int *total = E.buf<int>("cok_total", 1);
        int *targets = E.buf<int>("cok_targets", (size_t)n);
        launch_cok_prepare(n, d_pm, flag, st);
        HB_CK(cudaMemcpyAsync(pos, flag, n * 4, cudaMemcpyDeviceToDevice, st));
        exclusive_scan(pos, n, tmp, total, st);
        launch_cok_targets(n, flag, pos, targets, st);
        HB_CK(cudaGetLastError());
        int n_t = 0;
        HB_CK(cudaMemcpyAsync(&n_t, total, sizeof(int), cudaMemcpyDeviceToHost, st));
        HB_CK(cudaStreamSynchronize(st));
        E.stats.launches += 2 + scan_kernels(n);
        E.mark(STAGE_COMPACT, st);

        auto plan_pair = plan_f.get();
        Plan &pl = plan_pair.first;
        const std::vector<Offset> &tv = plan_pair.second;
        E.stats.plan_ms = plan_ms;
        const Geom &g = pl.g;
        const int k = a.max_nb;
        // the cross model over the +-radius box and the border's constants
        // (cross_cov_model_mark_i_t / _mark_ii_t, simple_cokriging_markI.cpp:145-193)
        Flavour fs = pl.f;
        if (a.mark == 2)
        {
            std::string err;
            if (!make_model(a.secondary.cov_type, a.secondary.ranges, a.secondary.angles, a.secondary.sill,
                            a.secondary.nugget, fs.m, err))
                throw CudaFail{-1, err};
        }
        const double c0p = pl.f.c0(), c0s = fs.c0();
        CokParams cp;
        if (a.mark == 1)
        {
            cp.coef = c0p <= 0 ? 0.0 : a.corr * sqrt(a.secondary_variance) / sqrt(c0p);
            cp.sec_var = a.secondary_variance;
        }
        else
        {
            cp.coef = c0s <= 0 ? 0.0 : a.corr * sqrt(c0p / c0s);
            cp.sec_var = c0s;
        }
        cp.b_last = cp.coef * fs.c0();
        cp.pm = (float)a.primary_mean;
        cp.sm = (float)a.secondary_mean;
        const int bx = 2 * g.rx + 1, by = 2 * g.ry + 1, bz = 2 * g.rz + 1;
        std::vector<double> cross((size_t)bx * by * bz);
        for (int dz = -g.rz; dz <= g.rz; ++dz)
            for (int dy = -g.ry; dy <= g.ry; ++dy)
                for (int dx = -g.rx; dx <= g.rx; ++dx)
                    cross[((size_t)(dz + g.rz) * by + (dy + g.ry)) * bx + (dx + g.rx)] = fs.at_offset(dx, dy, dz);
        double *d_cross = E.buf<double>("cok_cross", cross.size());
        HB_CK(cudaMemcpyAsync(d_cross, cross.data(), cross.size() * 8, cudaMemcpyHostToDevice, st));
        HB_CK(cudaStreamSynchronize(st)); // host temporaries
        E.mark(STAGE_TABLES, st);

        DevPoints P = compact_points(E, grid_geom(dims), d_pm, d_pd, nullptr, st);
        E.stats.launches += 2 + scan_kernels(n);
        // The reference's lookup here is the template scan alone
        // (sugarbox_neighbour_lookup.h:39-63): the first k informed cells in
        // template order. As a selection: every informed cell of the 27 bins
        // around a cell keyed by its offset's position in the sorted template
        // (unique keys, so the k smallest are those cells, in that order), through
        // the kriging path's binned search with every bin selecting. The scan of
        // the template over the informed-cell bitmap remains for configurations
        // the selection does not take (k > 64, templates past 65534 offsets,
        // candidate lists past shared memory).
        int2 *nb_rec = nullptr;
        int *nb_n = nullptr;
        double *pair64 = nullptr;
        bool selected = false;
        if (k <= 64 && tv.size() <= 0xFFFE)
        {
            std::fill(pl.kt.rank.begin(), pl.kt.rank.end(), KEY_EXCLUDED);
            for (size_t i = 0; i < tv.size(); ++i) pl.kt.rank[key_index(g, tv[i].dx, tv[i].dy, tv[i].dz)] = (uint32_t)i;
            pl.kt.n_ranks = (uint32_t)tv.size();
            pl.kt.h2_lo.clear(); // the key table's h2 ranges belong to its own ranks
            pl.kt.h2_hi.clear();
            pl.rank_bits = pl.kt.n_ranks > 1 ? bits_for(pl.kt.n_ranks - 1) : 0;
            pl.sg = Surrogate();
            build_surrogate(pl.f, pl.kt, pl.sg, true);
            pl.g.limit = INT_MAX; // no bin takes the template path
            try
            {
                DevSearch S = run_search(E, pl, P, d_pm, 0, st);
                if (S.ties != 0) throw CudaFail{-2, "cokriging search: equal template keys"};
                nb_rec = S.nb_rec;
                nb_n = S.nb_n;
                pair64 = S.pair64;
                selected = true;
            }
            catch (const CudaFail &f)
            {
                if (f.code != -4) throw;
            }
        }
        if (!selected)
        {
            const size_t nk = pl.kt.vals.size();
            double *search_vals = E.buf<double>("search_vals", nk);
            HB_CK(cudaMemcpyAsync(search_vals, pl.kt.vals.data(), nk * 8, cudaMemcpyHostToDevice, st));
            const long long pn = (long long)g.pnx * g.pny * (2 * g.phz + 1);
            pair64 = E.buf<double>("pair64", (size_t)pn);
            float *pair32 = E.buf<float>("pair32", (size_t)pn);
            launch_build_pair(g, dev_model(pl.f.m), 0, search_vals, pair64, pair32, st);
            // the template over the informed-cell bitmap of the grid padded by
            // the radiuses, for every bin; its linear offsets are 32-bit
            const long long PX = g.nx + 2LL * g.rx, PY = g.ny + 2LL * g.ry;
            if ((long long)g.rz * PY * PX + (long long)g.ry * PX + g.rx > 2147483647LL)
                throw CudaFail{-4, "grid too large for the template search at these radiuses"};
            std::vector<int4> t4(tv.size());
            for (size_t i = 0; i < tv.size(); ++i)
                t4[i] = make_int4(tv[i].dx, tv[i].dy, tv[i].dz, template_padded_offset(g, tv[i].dx, tv[i].dy, tv[i].dz));
            int4 *tmpl = E.buf<int4>("tmpl", std::max<size_t>(t4.size(), 1));
            if (!t4.empty())
                HB_CK(cudaMemcpyAsync(tmpl, t4.data(), t4.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
            std::vector<int> all_bins(g.n_bins);
            for (int b = 0; b < g.n_bins; ++b) all_bins[b] = b;
            int *tmpl_bins = E.buf<int>("tmpl_bins", (size_t)g.n_bins);
            HB_CK(cudaMemcpyAsync(tmpl_bins, all_bins.data(), (size_t)g.n_bins * 4, cudaMemcpyHostToDevice, st));
            HB_CK(cudaStreamSynchronize(st)); // host temporaries
            E.stats.launches += 1;
            nb_rec = E.buf<int2>("nb_rec", (size_t)n * k);
            nb_n = E.buf<int>("nb_n", (size_t)n);
            int *tcount = E.buf<int>("cok_tcount", 1);
            HB_CK(cudaMemsetAsync(tcount, 0, 4, st));
            if (n_t > 0)
            {
                HB_CK(launch_search_template(g, d_pm, E.buf<uint32_t>("mask_bits", (size_t)(template_padded_cells(g) + 31) / 32),
                                             0, tmpl_bins, g.n_bins, P.pts_val, tmpl, (int)t4.size(), P.pid_of_node,
                                             nullptr, nb_rec, nb_n, tcount, E.n_sm(), st));
                E.stats.launches += 2;
            }
        }
        E.mark(STAGE_SEARCH, st);
        HB_CK(launch_cok_solve(g, targets, n_t, nb_rec, nb_n, k, pair64, d_cross, d_pd, d_sd, d_sm, cp, d_out, d_omask,
                               d_status, E.n_sm(), st));
        if (n_t > 0) E.stats.launches += 1;
        E.mark(STAGE_SOLVE, st);
        launch_cok_finalize(n, d_pd, d_pm, d_out, d_omask, d_status, st);
        HB_CK(cudaGetLastError());
        E.stats.launches += 1;
        E.mark(STAGE_FINALIZE, st);
        to_host(E, out_data, d_out, (size_t)n, io);
        to_host(E, out_mask, d_omask, (size_t)n, io);
        if (opt.status) to_host(E, opt.status, d_status, (size_t)n, io);
        E.mark(STAGE_DOWNLOAD, st);
        E.stats.kriged = n_t;
        end_call(E, st);
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

int find_neighbours(int kind, const int *dims, const unsigned char *mask, const SkArgs &a, const int *nodes,
                    int n_nodes, int *out_idx, int *out_count, unsigned char *out_path)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        long long n = check_dims(dims);
        Plan pl = make_plan(kind != 0, a.cov_type, a.ranges, a.angles, a.sill, a.nugget, a.radiuses, a.max_nb, dims);
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(nullptr);
        IoPlan io{false, st};
        begin_call(E, st);
        const uint8_t *d_mask = to_device(E, "in_mask", mask, (size_t)n, io);
        DevPoints P = compact_points(E, pl.g, d_mask, nullptr, nullptr, st);
        DevSearch S = run_search(E, pl, P, d_mask, 1, st, true);
        std::vector<int> nb_n(n), pts(std::max(P.m, 1));
        std::vector<uint8_t> flags(pl.g.n_bins);
        HB_CK(cudaMemcpyAsync(nb_n.data(), S.nb_n, n * 4, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaMemcpyAsync(pts.data(), P.pts_node, pts.size() * 4, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaMemcpyAsync(flags.data(), S.bin_flag, flags.size(), cudaMemcpyDeviceToHost, st));
        std::vector<int> lst((size_t)pl.g.k);
        for (int t = 0; t < n_nodes; ++t)
        {
            int node = nodes[t];
            if (node < 0 || node >= n) throw CudaFail{-1, "node index out of range"};
            HB_CK(cudaMemcpyAsync(lst.data(), S.nb_pid + (size_t)node * pl.g.k, pl.g.k * 4, cudaMemcpyDeviceToHost,
                                  st));
            HB_CK(cudaStreamSynchronize(st));
            int cnt = nb_n[node];
            if (out_count) out_count[t] = cnt;
            for (int i = 0; i < pl.g.k; ++i) out_idx[(size_t)t * pl.g.k + i] = i < cnt ? pts[lst[i]] : -1;
            if (out_path)
            {
                int x = node % dims[0], y = node % (dims[0] * dims[1]) / dims[0], z = node / (dims[0] * dims[1]);
                int b = ((z / pl.g.rz) * pl.g.by + (y / pl.g.ry)) * pl.g.bx + (x / pl.g.rx);
                out_path[t] = (flags[b] & 2) ? 1 : 0;
            }
        }
        end_call(E, st);
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
    catch (const std::exception &ex)
    {
        set_error(ex.what());
        return -1;
    }
}

Stats last_stats()
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return Stats();
    auto it = g_engines.find(dev);
    return it == g_engines.end() ? Stats() : it->second->stats;
}

int host_template(int kind, int cov_type, const double *ranges, const double *angles, double sill, double nugget,
                  const int *radiuses, int *out, int cap, int *out_limit)
{
    try
    {
        check_model_args(cov_type, ranges, angles, sill, nugget, radiuses, 1);
        Flavour f;
        std::string err;
        if (!make_model(cov_type, ranges, angles, sill, nugget, f.m, err)) throw CudaFail{-1, err};
        f.truncated = kind != 0;
        for (int a = 0; a < 3; ++a) f.r[a] = radiuses[a];
        KeyTable kt;
        build_key_table(f, kt, g_threads);
        std::vector<Offset> t = build_template(f, kt);
        for (int i = 0; i < (int)t.size() && i < cap; ++i)
        {
            out[3 * i] = t[i].dx;
            out[3 * i + 1] = t[i].dy;
            out[3 * i + 2] = t[i].dz;
        }
        if (out_limit) *out_limit = (int)(t.size() / 250);
        return (int)t.size();
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
}

double host_covariance(int kind, int cov_type, const double *ranges, const double *angles, double sill,
                       double nugget, const int *radiuses, const int *a, const int *b)
{
    Flavour f;
    std::string err;
    if (!make_model(cov_type, ranges, angles, sill, nugget, f.m, err))
    {
        set_error(err);
        return NAN;
    }
    f.truncated = kind != 0;
    for (int i = 0; i < 3; ++i) f.r[i] = radiuses ? radiuses[i] : 1;
    return f.at_offset(b[0] - a[0], b[1] - a[1], b[2] - a[2]);
}
} // namespace hb

namespace hb
{
int sk_weights(const double *center, const double *xs, const double *ys, const double *zs, int n, int cov_type,
               const double *ranges, const double *angles, double sill, double nugget, double *out_w)
{
    std::lock_guard<std::mutex> lk(g_engine_mu);
    try
    {
        if (n <= 0) throw CudaFail{-1, "sk_kriging_weights: no neighbours"};
        CovModel m;
        std::string err;
        if (!make_model(cov_type, ranges, angles, sill, nugget, m, err)) throw CudaFail{-1, err};
        Engine &E = engine_for_current_device();
        cudaStream_t st = E.stream(nullptr);
        std::vector<double> h(3 + 3 * (size_t)n);
        h[0] = center[0];
        h[1] = center[1];
        h[2] = center[2];
        for (int i = 0; i < n; ++i)
        {
            h[3 + i] = xs[i];
            h[3 + n + i] = ys[i];
            h[3 + 2 * n + i] = zs[i];
        }
        double *d_pts = E.buf<double>("skw_pts", h.size());
        double *d_A = E.buf<double>("skw_A", (size_t)n * n);
        double *d_w = E.buf<double>("skw_w", (size_t)n);
        int *d_st = E.buf<int>("skw_status", 1);
        HB_CK(cudaMemcpyAsync(d_pts, h.data(), h.size() * 8, cudaMemcpyHostToDevice, st));
        launch_sk_weights(dev_model(m), d_pts, n, d_A, d_w, d_st, st);
        HB_CK(cudaGetLastError());
        int ok = 0;
        HB_CK(cudaMemcpyAsync(out_w, d_w, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaMemcpyAsync(&ok, d_st, 4, cudaMemcpyDeviceToHost, st));
        HB_CK(cudaStreamSynchronize(st));
        if (!ok) throw CudaFail{-1, "sk_kriging_weights: covariance matrix is not positive definite"};
        return 0;
    }
    catch (const CudaFail &f)
    {
        set_error(f.msg);
        return f.code;
    }
}

void *host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) return nullptr;
    return p;
}
void host_free(void *p)
{
    if (p) cudaFreeHost(p);
}
} // namespace hb
