// Batched dot products for callers that must not allocate device memory.
//
// The regular reductions of the engine keep their per-block partial sums in scratch
// that the library allocates itself (a buffer per stream, created on first use).  Some
// callers cannot allow that: an application that owns every byte of device memory
// through its own arena (a memory pool sized at start-up, or a framework's caching
// allocator) and forbids libraries to allocate behind its back, because an allocation
// it does not know of can push its own pool out of memory or make its accounting
// wrong.  ccsd_dot_batch_noalloc gives them the same computation as the DIIS
// error-matrix row (out[j] = <x, y_j>) with the scratch placed in a fixed file-scope
// device array instead: the caller passes inputs and outputs, the library allocates
// nothing.
//
// Limits and rules:
//  * at most kMaxVectors (16) vectors per call; larger requests are rejected;
//  * the scratch array (kBlocks x kMaxVectors doubles = 32 KiB) lives in every device
//    that loads the library until the process exits;
//  * every call shares that array, so calls whose kernels overlap on the GPU (two
//    streams, or two threads) race; serialise them on one stream;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (no allocation); make that first call before any stream
//    capture begins;
//  * that address is kept per device number for the life of the process: it does not
//    survive cudaDeviceReset (or a reset of the primary context by other code), after
//    which the entry point must not be called again in this process;
//  * a CUDA error left pending by earlier work on the calling thread is reported and
//    left in place for its owner: the call then launches nothing.
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "ccsd_b200.h"

namespace ccsd {
void set_global_error(const std::string& msg);
}

namespace {

constexpr int kBlocks = 256;
constexpr int kThreads = 256;
constexpr int kMaxVectors = 16;
constexpr int kMaxDevices = 64;

// scratch: the partial sum of block b for vector j sits at [b * ny + j]
static __device__ __align__(256) double g_dot_batch_scratch[kBlocks * kMaxVectors];

struct Vectors {
    const double* y[kMaxVectors];
};

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kThreads) dot_partials(const double* __restrict__ x, Vectors ys, int ny, int64_t n,
                                                         double* scratch) {
    __shared__ double red[32];
    double s[kMaxVectors];
#pragma unroll
    for (int j = 0; j < kMaxVectors; j++) s[j] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double xv = x[i];
#pragma unroll
        for (int j = 0; j < kMaxVectors; j++)
            if (j < ny) s[j] += xv * ys.y[j][i];
    }
    for (int j = 0; j < ny; j++) {
        double t = block_sum(s[j], red);
        if (threadIdx.x == 0) scratch[blockIdx.x * ny + j] = t;
    }
}

__global__ void __launch_bounds__(kThreads) dot_fold(const double* scratch, int nblocks, int ny, double* out) {
    __shared__ double red[32];
    for (int j = 0; j < ny; j++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += scratch[b * ny + j];
        s = block_sum(s, red);
        if (threadIdx.x == 0) out[j] = s;
    }
}

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

}  // namespace

extern "C" int ccsd_dot_batch_noalloc(void* stream, const double* x, const double* const* ys, int ny, int64_t n,
                                      double* out) {
    if (ny < 1 || ny > kMaxVectors) {
        ccsd::set_global_error("ccsd_dot_batch_noalloc: ny=" + std::to_string(ny) + " outside 1.." +
                               std::to_string(kMaxVectors) + " (the fixed scratch holds at most " +
                               std::to_string(kMaxVectors) + " vectors per call)");
        return CCSD_ERR_ARG;
    }
    if (n < 0 || !x || !ys || !out) {
        ccsd::set_global_error("ccsd_dot_batch_noalloc: null pointer or negative length");
        return CCSD_ERR_ARG;
    }
    Vectors v{};
    for (int j = 0; j < ny; j++) {
        if (!ys[j]) {
            ccsd::set_global_error("ccsd_dot_batch_noalloc: null vector pointer");
            return CCSD_ERR_ARG;
        }
        v.y[j] = ys[j];
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        ccsd::set_global_error(std::string("ccsd_dot_batch_noalloc: no current device: ") + cudaGetErrorString(e));
        return CCSD_ERR_CUDA;
    }
    double* scratch = nullptr;
    {
        // once per device, with that device current: the device address of the array
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_dot_batch_scratch);
            if (e != cudaSuccess || !p) {
                ccsd::set_global_error(std::string("ccsd_dot_batch_noalloc: cudaGetSymbolAddress failed: ") +
                                       cudaGetErrorString(e));
                return CCSD_ERR_CUDA;
            }
            g_scratch_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    int64_t want = (n + kThreads - 1) / kThreads;
    const int nblocks = (int)(want < 1 ? 1 : (want > kBlocks ? kBlocks : want));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an error pending from earlier, unrelated work belongs to that work: report it without
    // consuming it, and launch nothing
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        ccsd::set_global_error(std::string("ccsd_dot_batch_noalloc: a CUDA error from earlier work is pending: ") +
                               cudaGetErrorString(e));
        return CCSD_ERR_CUDA;
    }
    dot_partials<<<nblocks, kThreads, 0, s>>>(x, v, ny, n, scratch);
    e = cudaGetLastError();   // nothing was pending, so an error here is this launch's
    if (e != cudaSuccess) {
        ccsd::set_global_error(std::string("ccsd_dot_batch_noalloc: launch of the partial sums failed: ") +
                               cudaGetErrorString(e));
        return CCSD_ERR_CUDA;
    }
    dot_fold<<<1, kThreads, 0, s>>>(scratch, nblocks, ny, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ccsd::set_global_error(std::string("ccsd_dot_batch_noalloc: launch of the fold failed: ") +
                               cudaGetErrorString(e));
        return CCSD_ERR_CUDA;
    }
    return CCSD_OK;
}
