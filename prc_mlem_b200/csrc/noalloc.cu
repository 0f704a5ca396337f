// noalloc.cu -- an FP64 volume sum that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc at the point where they need a count
// sum: reconstruction services that reserve all of their device memory once at start-up and
// forbid any later allocation (a fixed budget, so a long-running scanner process can neither
// fragment nor exhaust the GPU), hot loops that must not pay the device-wide synchronisation
// that cudaMalloc / cudaFree can cause, and operators embedded in another framework whose
// device memory must come from that framework's own allocator.  prc_sum needs a handle, and
// creating one allocates.  prc_sum_static gives those callers the same FP64 sum with its
// scratch (block partials and a completion counter) in a file-scope __device__ array that is
// part of the library image: every GPU that loads the library holds it (kStaticBlocks * 8 + 256
// bytes, about 512 KiB) until the process exits.
//
// When the array is committed: under CUDA's lazy module loading (the default since CUDA 12.2)
// the module holding it is loaded on a device by the first address lookup, i.e. by the first
// prc_sum_static call made with that device current; with CUDA_MODULE_LOADING=EAGER it is
// loaded with the library.  A caller that must not allocate after start-up therefore makes one
// warm-up call per device at start-up (before reserving its memory and before any stream
// capture); every later call allocates nothing.
#include "../../include/prc_b200.h"
#include "engine.h"

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>

namespace {

constexpr int kStaticThreads = 256;
constexpr int kStaticItems = 16;                             // elements per thread
constexpr long long kPerBlock = (long long)kStaticThreads * kStaticItems;
constexpr int kStaticBlocks = 65536;                         // partials the array holds
constexpr long long kStaticMaxElements = kPerBlock * kStaticBlocks;  // 2^28 floats
constexpr int kMaxDevices = 64;

// [0, 256): the completion counter (first 4 bytes); [256, 256 + 8 * kStaticBlocks): partials.
static __device__ __align__(256) unsigned char g_sum_scratch[256 + sizeof(double) * kStaticBlocks];

// Per-device address of g_sum_scratch (the name is only a host stand-in for the device symbol;
// a kernel must be given the device address).  Only a successful lookup is kept, so a lookup
// that failed for a passing reason (for example inside a stream capture) is retried by the
// next call.
std::atomic<void*> g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

cudaError_t scratch_address(int dev, unsigned char** out) {
    void* p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
        if (!p) {
            const cudaError_t e = cudaGetSymbolAddress(&p, g_sum_scratch);  // with `dev` current
            if (e != cudaSuccess) {
                cudaGetLastError();  // a failed lookup leaves no error behind for the caller
                return e;
            }
            g_scratch_ptr[dev].store(p, std::memory_order_release);
        }
    }
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

__global__ void __launch_bounds__(kStaticThreads) static_sum_kernel(const float* __restrict__ x, long long n,
                                                                    unsigned char* scratch, double* out) {
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    double* partials = reinterpret_cast<double*>(scratch + 256);
    __shared__ double sh[kStaticThreads / 32];
    __shared__ bool last;
    const long long start = (long long)blockIdx.x * kPerBlock;
    double v = 0.0;
#pragma unroll 4
    for (int k = 0; k < kStaticItems; ++k) {
        const long long i = start + (long long)k * kStaticThreads + threadIdx.x;
        if (i < n) v += x[i];
    }
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kStaticThreads / 32; ++w) t += sh[w];
        partials[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block adds the partials in block order: the result does not depend on timing
    double acc = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kStaticThreads) acc += __ldcg(partials + b);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kStaticThreads / 32; ++w) t += sh[w];
        *out = t;
    }
}

}  // namespace

extern "C" int prc_sum_static(const float* d_x, int64_t n, double* d_sum, void* stream) {
    if (!d_x || !d_sum || n < 0) {
        prc::set_last_error("Invalid argument");
        return PRC_ERR_ARGUMENT;
    }
    if (n > kStaticMaxElements) {
        prc::set_last_error("prc_sum_static: " + std::to_string(n) + " elements exceed its static scratch limit of " +
                            std::to_string(kStaticMaxElements) + " (2^28) elements");
        return PRC_ERR_LIMIT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess && (dev < 0 || dev >= kMaxDevices)) e = cudaErrorInvalidDevice;
    // The device address of the scratch array, looked up once per device with it current.
    unsigned char* scratch = nullptr;
    if (e == cudaSuccess) e = scratch_address(dev, &scratch);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The array keeps the previous call's contents: the counter must start at zero.
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        if (n == 0) {
            e = cudaMemsetAsync(d_sum, 0, sizeof(double), s);
        } else {
            const int blocks = (int)((n + kPerBlock - 1) / kPerBlock);
            static_sum_kernel<<<blocks, kStaticThreads, 0, s>>>(d_x, (long long)n, scratch, d_sum);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess) {
        prc::set_last_error(std::string("CUDA error '") + cudaGetErrorString(e) + "' in prc_sum_static");
        return PRC_ERR_CUDA;
    }
    return PRC_OK;
}
