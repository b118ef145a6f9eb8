// rdst_noalloc.cu -- allocation-free residual-norm reduction.
//
// rdst_residual_norms_noalloc() computes, for a per-unit-volume residual
// R[n][5] and cell volumes V[n] already in device memory, the same norms the
// step reports: out[0] = sqrt(sum_i |R_i|^2) and out[1+k] = ||R_k V||_2.
// It is the norm part of the step's residual kernel, made usable by callers
// that may not allocate device memory: code that runs while a CUDA stream is
// being captured into a graph (cudaMalloc is not a capturable operation),
// applications whose device memory is owned by a pool allocator (a PyTorch
// or RMM pool that must see every allocation), and latency-bound paths that
// cannot afford cudaMalloc's implicit device synchronisation.
//
// The per-block partial sums live in a file-scope __device__ array of fixed
// size, so the entry point allocates nothing.  That array exists once per
// GPU that loads the library and stays resident until process exit.  Every
// call shares it: two calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race on it and must be serialised by
// the caller.  Each call overwrites exactly the partials it later reads, so
// no clearing is needed between calls.
//
// The GPU a call runs on is the one that holds R (V and out must be on the
// same one; host memory is rejected): the library carries its own CUDA
// runtime, whose current device is not the caller's, so the call selects
// that device for its set-up and launches and restores the thread's
// previous device afterwards.  `stream` must belong to that device.
#include "../../include/rdst.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#define RDST_API extern "C" __attribute__((visibility("default")))

namespace {

constexpr int NA_TPB = 256;                         // threads per block, one cell each
constexpr int NA_MAX_BLOCKS = 4096;                 // scratch capacity in blocks
constexpr long NA_MAX_CELLS = (long)NA_MAX_BLOCKS * NA_TPB;   // 1,048,576 cells
constexpr int NA_NV = 6;                            // |R|^2 and (R_k V)^2, k < 5
constexpr int NA_MAX_DEVICES = 128;

// 4096 x 6 doubles = 192 KiB per GPU
static __device__ __align__(256) double g_noalloc_partial[NA_MAX_BLOCKS * NA_NV];

// device address of g_noalloc_partial per device (host code cannot use the
// symbol itself: on the host it only names a stand-in)
std::mutex g_mu;
double* g_scratch[NA_MAX_DEVICES] = {nullptr};
thread_local std::string g_err;

__device__ __forceinline__ double na_warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// fixed-order block sum, result in thread 0
__device__ __forceinline__ double na_block_sum(double v) {
    __shared__ double sh[NA_TPB / 32];
    v = na_warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < NA_TPB / 32) ? sh[threadIdx.x] : 0.0;
    if (wid == 0) v = na_warp_sum(v);
    return v;
}

__global__ void __launch_bounds__(NA_TPB) k_na_norm_partials(int n, const double* __restrict__ R,
                                                             const double* __restrict__ V,
                                                             double* __restrict__ partial) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double sq_mag = 0.0, sq_c[5] = {0, 0, 0, 0, 0};
    if (i < n) {
        const double Vi = V[i];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const double Rc = R[5 * i + c];
            sq_mag += Rc * Rc;
            const double rv = Rc * Vi;
            sq_c[c] = rv * rv;
        }
    }
    double v = na_block_sum(sq_mag);
    if (threadIdx.x == 0) partial[blockIdx.x * NA_NV] = v;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        v = na_block_sum(sq_c[c]);
        if (threadIdx.x == 0) partial[blockIdx.x * NA_NV + 1 + c] = v;
    }
}

__global__ void k_na_norm_final(const double* __restrict__ partial, int nb, double* __restrict__ out) {
    const int c = threadIdx.x;
    if (c >= NA_NV) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += partial[b * NA_NV + c];
    out[c] = sqrt(s);
}

// Device of a caller buffer: device memory (or managed memory) only, taken
// from the pointer itself, since the library's own CUDA runtime does not
// follow the caller's current device.
bool device_of(const void* p, int& dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return false;
    dev = a.device;
    return true;
}

// Set-up on the first call per device (with that device current): the
// device address of the scratch array.
double* scratch_for_device(int dev, cudaError_t& err) {
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[dev]) {
        void* p = nullptr;
        err = cudaGetSymbolAddress(&p, g_noalloc_partial);
        if (err != cudaSuccess) return nullptr;
        g_scratch[dev] = static_cast<double*>(p);
    }
    return g_scratch[dev];
}

// Makes `dev` current on this thread for the lifetime of the guard and
// restores the previous device afterwards.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

// Message of the last failing context-free call on this thread.
const char* rdst_noalloc_error_message() { return g_err.c_str(); }

RDST_API rdst_status rdst_residual_norms_noalloc(int32_t n_cells, const double* R, const double* V, double* out,
                                                 void* stream) {
    g_err.clear();
    if (n_cells <= 0 || !R || !V || !out) {
        g_err = "rdst_residual_norms_noalloc: null pointer or n_cells <= 0";
        return RDST_ERR_ARG;
    }
    if ((long)n_cells > NA_MAX_CELLS) {
        g_err = "rdst_residual_norms_noalloc: n_cells = " + std::to_string(n_cells) +
                " exceeds the fixed scratch capacity of " + std::to_string(NA_MAX_CELLS) + " cells";
        return RDST_ERR_ARG;
    }
    // the GPU is the one holding the buffers, checked before any launch
    int dev = -1, dev_v = -1, dev_o = -1;
    if (!device_of(R, dev) || !device_of(V, dev_v) || !device_of(out, dev_o)) {
        g_err = "rdst_residual_norms_noalloc: R, V and out must be device memory";
        return RDST_ERR_ARG;
    }
    if (dev_v != dev || dev_o != dev) {
        g_err = "rdst_residual_norms_noalloc: R, V and out are on different devices (" + std::to_string(dev) +
                ", " + std::to_string(dev_v) + ", " + std::to_string(dev_o) + ")";
        return RDST_ERR_ARG;
    }
    DeviceGuard guard(dev);
    if (guard.err != cudaSuccess) {
        g_err = std::string("rdst_residual_norms_noalloc: cannot select device ") + std::to_string(dev) + ": " +
                cudaGetErrorString(guard.err);
        return RDST_ERR_CUDA;
    }
    cudaError_t e = cudaSuccess;
    double* partial = scratch_for_device(dev, e);
    if (!partial) {
        g_err = std::string("rdst_residual_norms_noalloc: scratch set-up failed: ") + cudaGetErrorString(e);
        return RDST_ERR_CUDA;
    }
    const int nb = (int)((n_cells + NA_TPB - 1) / NA_TPB);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_na_norm_partials<<<nb, NA_TPB, 0, s>>>(n_cells, R, V, partial);
    k_na_norm_final<<<1, 32, 0, s>>>(partial, nb, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_err = std::string("rdst_residual_norms_noalloc: launch failed: ") + cudaGetErrorString(e);
        return RDST_ERR_CUDA;
    }
    return RDST_OK;
}
