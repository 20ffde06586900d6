// Allocation-free variant of the time-step reduction (main.rs:375-408
// calc_global_dt, dt.rs:5-34 get_local_dt) for callers that cannot allocate
// device memory themselves: code running where the memory is owned by a host
// framework or a pool that forbids cudaMalloc, or inside a region where an
// allocation would synchronise the device. The caller passes its own device
// buffers for the inputs and the output; the only scratch, one partial
// minimum per block, lives in the file-scope array below, which every GPU
// that loads the library holds until the process exits.
//
// Rules of use (also in include/rh3t.h):
//   - at most RH3T_DT_NOALLOC_MAX_CELLS fluid-grid nodes (nx*ny) per call;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, that device current); make that
//     first call before any stream capture;
//   - all calls share the array: two calls that overlap on the GPU (other
//     streams, other host threads) race on it; calls on one stream are safe.
//     Each call writes every entry it later reads, so nothing needs clearing.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/rh3t.h"
#include "physics.cuh"

namespace rh3t {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = RH3T_DT_NOALLOC_MAX_CELLS / kNoAllocThreads;

static __device__ __align__(256) double g_dt_partial[kNoAllocMaxBlocks];

__global__ void __launch_bounds__(kNoAllocThreads)
    k_dt_noalloc_partial(const double* __restrict__ value, const uint8_t* __restrict__ fluid, long long n, double dx,
                         double dy, DevParams P, double* __restrict__ partial) {
    __shared__ double red[kNoAllocThreads / 32];
    const long long l = (long long)blockIdx.x * kNoAllocThreads + threadIdx.x;
    double m = INFINITY;
    if (l < n && fluid[l]) {
        double s[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) s[c] = value[l * 6 + c];
        m = fmin(m, local_dt(s, dx, dy, P));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = red[0];
        for (int k = 1; k < kNoAllocThreads / 32; ++k) b = fmin(b, red[k]);
        partial[blockIdx.x] = b;
    }
}

__global__ void __launch_bounds__(kNoAllocThreads)
    k_dt_noalloc_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    __shared__ double red[kNoAllocThreads / 32];
    double m = INFINITY;
    for (int k = threadIdx.x; k < nb; k += kNoAllocThreads) m = fmin(m, partial[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = red[0];
        for (int k = 1; k < kNoAllocThreads / 32; ++k) b = fmin(b, red[k]);
        out[0] = b;
    }
}

// device address of g_dt_partial, looked up once per device
constexpr int kMaxDevices = 64;
static double* g_partial_ptr[kMaxDevices] = {nullptr};
static std::mutex g_partial_mu;

static int partial_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return RH3T_ERR_NO_DEVICE;
    if (dev < 0 || dev >= kMaxDevices) return RH3T_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_partial_mu);
    if (!g_partial_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_dt_partial);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "rh3t_calc_global_dt_noalloc: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e));
            return RH3T_ERR_CUDA;
        }
        g_partial_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_partial_ptr[dev];
    return RH3T_OK;
}

} // namespace rh3t

extern "C" int rh3t_calc_global_dt_noalloc(const rh3t_grid* grid, const rh3t_params* params, const double* d_value,
                                           const uint8_t* d_fluid, double* d_dt_cfl, void* stream) {
    using namespace rh3t;
    if (!grid || !params || !d_value || !d_fluid || !d_dt_cfl || grid->nx <= 0 || grid->ny <= 0 ||
        !(grid->dx > 0.0) || !(grid->dy > 0.0))
        return RH3T_ERR_INVALID_ARGUMENT;
    const long long n = (long long)grid->nx * grid->ny;
    if (n > RH3T_DT_NOALLOC_MAX_CELLS) {
        std::fprintf(stderr,
                     "rh3t_calc_global_dt_noalloc: grid of %lld nodes exceeds the allocation-free limit of %d "
                     "nodes; use rh3t_calc_global_dt\n",
                     n, RH3T_DT_NOALLOC_MAX_CELLS);
        return RH3T_ERR_INVALID_ARGUMENT;
    }
    double* partial = nullptr;
    int rc = partial_for_current_device(&partial);
    if (rc) return rc;
    DevParams P;
    static_assert(sizeof(DevParams) == sizeof(rh3t_params), "DevParams mirrors rh3t_params");
    memcpy(&P, params, sizeof(P));
    const int nb = (int)((n + kNoAllocThreads - 1) / kNoAllocThreads);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_dt_noalloc_partial<<<nb, kNoAllocThreads, 0, s>>>(d_value, d_fluid, n, grid->dx, grid->dy, P, partial);
    k_dt_noalloc_final<<<1, kNoAllocThreads, 0, s>>>(partial, nb, d_dt_cfl);
    return cudaGetLastError() == cudaSuccess ? RH3T_OK : RH3T_ERR_CUDA;
}
