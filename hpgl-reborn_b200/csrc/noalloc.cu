// SK weights of one kriging system without any device allocation.
//
// Some callers cannot allocate device memory while they run: a process whose
// GPU memory is owned by another allocator (a framework's caching pool sized
// to fill the device), or a service that reserves a fixed memory budget up
// front and must not grow it or fail with out-of-memory mid-request. The
// regular hpgl_simple_kriging_weights entry point allocates (and caches)
// device buffers for its matrix and vectors on first use, so those callers
// cannot use it. This entry point computes the same weights using a fixed,
// file-scope device array instead: the array is part of the library's device
// image, so every GPU that loads the library holds it (about 135 KB) until the
// process exits, and no call ever allocates or frees device memory.
//
// Limits and sharing:
//   * at most kNoAllocMaxN neighbours per call (larger systems are rejected);
//   * every call uses the same array; calls that overlap on the GPU (two
//     streams, or two host threads) race on it and must be serialised by the
//     caller. The array keeps the previous call's contents; every element this
//     kernel reads is written earlier in the same call, so nothing carries over
//     between calls;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress) with that device current and caches it;
//   * with lazy module loading (CUDA's default since 12.2) the device holds
//     the array only from the moment this file's device code is loaded onto
//     it, which the first call's set-up forces (cudaFuncGetAttributes on the
//     kernel). That first call can therefore allocate the array's memory and
//     fail when the device is already full: make it before the caller reserves
//     its memory pool. Later calls allocate nothing;
//   * the call waits on `stream` for its own copies and kernel before it
//     returns the weights.
#include "../../include/hpgl_b200.h"
#include "engine_api.h"
#include "host_model.h"
#include "sk_single.cuh"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace
{
constexpr int kNoAllocMaxN = 128;
constexpr int kMaxDevices = 64;
// layout in doubles: centre (3) | x, y, z (3 n) | A (n n) | w (n) | status (1)
constexpr size_t kScratchDoubles = 3 + 3 * kNoAllocMaxN + (size_t)kNoAllocMaxN * kNoAllocMaxN + kNoAllocMaxN + 1;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// One CTA solves the system held in `s` (the static array's address): builds A
// and b, factors A = L L^T and solves for the weights, all in FP64, with the
// same device code as the regular entry point (sk_single.cuh).
__global__ void k_sk_weights_noalloc(hb::DevModel m, double *__restrict__ s, int n)
{
    double *A = s + 3 + 3 * kNoAllocMaxN;
    double *w = A + (size_t)kNoAllocMaxN * kNoAllocMaxN;
    const bool fail = hb::sk_single_solve(m, s, n, A, w);
    if (threadIdx.x == 0) w[kNoAllocMaxN] = fail ? 0.0 : 1.0;
}

std::mutex g_setup_mu;
double *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the static array on the current device, looked up once;
// the kernel's module (and with it the array) is loaded onto the device here.
cudaError_t scratch_address(int dev, double **out)
{
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev])
    {
        cudaFuncAttributes fa{};
        cudaError_t e = cudaFuncGetAttributes(&fa, k_sk_weights_noalloc);
        if (e != cudaSuccess) return e;
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}
} // namespace

extern "C" int hpgl_b200_sk_weights_noalloc(const float *center_coords, const float *neighbours_x,
                                            const float *neighbours_y, const float *neighbours_z, int neighbours_count,
                                            const struct hpgl_cov_params_t *params, float *weights, void *stream)
{
    const int n = neighbours_count;
    if (!center_coords || !neighbours_x || !neighbours_y || !neighbours_z || !params || !weights)
    {
        hb::set_error("hpgl_b200_sk_weights_noalloc: null argument");
        return HPGL_B200_EINVAL;
    }
    if (n < 1 || n > kNoAllocMaxN)
    {
        hb::set_error("hpgl_b200_sk_weights_noalloc: neighbours_count " + std::to_string(n) +
                      " outside 1.." + std::to_string(kNoAllocMaxN) +
                      " (the fixed device array holds at most " + std::to_string(kNoAllocMaxN) + " neighbours)");
        return HPGL_B200_ELIMIT;
    }
    hb::CovModel cm;
    std::string err;
    if (!hb::make_model(params->m_covariance_type, params->m_ranges, params->m_angles, params->m_sill,
                        params->m_nugget, cm, err))
    {
        hb::set_error("hpgl_b200_sk_weights_noalloc: " + err);
        return HPGL_B200_EINVAL;
    }
    hb::DevModel m;
    m.type = cm.type;
    m.r0 = cm.ranges[0];
    m.sill = cm.sill;
    m.nugget = cm.nugget;
    for (int i = 0; i < 9; ++i) m.T[i] = cm.T[i];

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    {
        hb::set_error(std::string("hpgl_b200_sk_weights_noalloc: no usable CUDA device: ") + cudaGetErrorString(e));
        return HPGL_B200_ECUDA;
    }
    double *s = nullptr;
    e = scratch_address(dev, &s);
    if (e != cudaSuccess)
    {
        hb::set_error(std::string("hpgl_b200_sk_weights_noalloc: cudaGetSymbolAddress failed: ") +
                      cudaGetErrorString(e));
        return HPGL_B200_ECUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // inputs staged through a stack buffer into the device array (no heap either)
    double in[3 + 3 * kNoAllocMaxN];
    in[0] = center_coords[0];
    in[1] = center_coords[1];
    in[2] = center_coords[2];
    for (int i = 0; i < n; ++i)
    {
        in[3 + i] = neighbours_x[i];
        in[3 + n + i] = neighbours_y[i];
        in[3 + 2 * n + i] = neighbours_z[i];
    }
    double out[kNoAllocMaxN + 1];
    const size_t w_off = 3 + 3 * kNoAllocMaxN + (size_t)kNoAllocMaxN * kNoAllocMaxN;
    e = cudaMemcpyAsync(s, in, (3 + 3 * (size_t)n) * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
    {
        k_sk_weights_noalloc<<<1, 256, 0, st>>>(m, s, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, s + w_off, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out + kNoAllocMaxN, s + w_off + kNoAllocMaxN, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
    {
        hb::set_error(std::string("hpgl_b200_sk_weights_noalloc: ") + cudaGetErrorString(e));
        return HPGL_B200_ECUDA;
    }
    if (out[kNoAllocMaxN] != 1.0)
    {
        hb::set_error("hpgl_b200_sk_weights_noalloc: covariance matrix is not positive definite");
        return HPGL_B200_EINVAL;
    }
    for (int i = 0; i < n; ++i) weights[i] = (float)out[i];
    return 0;
}
