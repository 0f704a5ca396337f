// sampling.cu -- Poisson counts on the device, for synthetic measurement data.
//
// The reference's tests make their measured data by blurring a phantom and Poisson-sampling it
// on the host.  prc_poisson draws out[i] ~ Poisson(scale * mean[i]) for every voxel in one
// grid-stride pass.  Random numbers come from Philox4x32-10 (Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), keyed by the seed with the voxel
// index as counter, so a voxel's count depends only on (mean, scale, seed, index), not on the
// launch shape.  Means below 10 are sampled by inversion of the cumulative distribution; larger
// means by the transformed rejection method with squeeze, PTRS (W. Hormann, "The transformed
// rejection method for generating Poisson random variables", Insurance: Mathematics and
// Economics 12, 1993), in double precision.
#include "../../include/prc_data.h"
#include "engine.h"

#include <cuda_runtime.h>

#include <cmath>
#include <string>

namespace {

// Ten rounds of the Philox-4x32 bijection (multipliers and Weyl key increments of the paper).
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
    constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u, kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(kM0, ctr.x), lo0 = kM0 * ctr.x;
        const uint32_t hi1 = __umulhi(kM1, ctr.z), lo1 = kM1 * ctr.z;
        ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
        key.x += kW0;
        key.y += kW1;
    }
    return ctr;
}

// Uniform in (0, 1) from 32 random bits.
__device__ __forceinline__ double uniform01(uint32_t u) { return ((double)u + 0.5) * (1.0 / 4294967296.0); }

// Stream of uniforms for one voxel: counter (index lo, index hi, draw block, 0).
struct Uniforms {
    uint2 key;
    uint32_t lo, hi, block = 0;
    uint4 bits{};
    int used = 4;
    __device__ double next() {
        if (used == 4) {
            bits = philox4x32_10(make_uint4(lo, hi, block++, 0u), key);
            used = 0;
        }
        const uint32_t v = used == 0 ? bits.x : used == 1 ? bits.y : used == 2 ? bits.z : bits.w;
        ++used;
        return uniform01(v);
    }
};

__device__ double poisson_sample(double lambda, Uniforms& u) {
    if (!(lambda > 0.0)) return 0.0;
    if (lambda < 10.0) {  // inversion: the first k whose cumulative probability exceeds u
        const double x = u.next();
        double p = exp(-lambda), F = p;
        int k = 0;
        while (x > F && k < 1000) {
            ++k;
            p *= lambda / k;
            F += p;
        }
        return (double)k;
    }
    // PTRS (Hormann 1993, algorithm PTRS with the paper's constants)
    const double slam = sqrt(lambda), loglam = log(lambda);
    const double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4), v_r = 0.9277 - 3.6224 / (b - 2.0);
    for (int attempt = 0; attempt < 1000; ++attempt) {
        const double U = u.next() - 0.5, V = u.next();
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + lambda + 0.43);
        if (us >= 0.07 && V <= v_r) return k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(inv_alpha) - log(a / (us * us) + b) <= -lambda + k * loglam - lgamma(k + 1.0)) return k;
    }
    return floor(lambda + 0.5);  // not reached in practice (acceptance is above 0.9 per attempt)
}

__global__ void poisson_kernel(const float* __restrict__ mean, long long n, double scale, uint2 key,
                               float* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float m = mean[i];
        Uniforms u;
        u.key = key;
        u.lo = (uint32_t)i;
        u.hi = (uint32_t)((unsigned long long)i >> 32);
        const double lambda = isfinite(m) && m > 0.0f ? scale * (double)m : 0.0;
        out[i] = (float)poisson_sample(lambda, u);
    }
}

}  // namespace

extern "C" int prc_poisson(const float* d_mean, int64_t n, double scale, uint64_t seed, float* d_out, void* stream) {
    if (n < 0 || (n > 0 && (!d_mean || !d_out)) || !(scale >= 0.0) || !std::isfinite(scale)) {
        prc::set_last_error("Invalid argument");
        return PRC_ERR_ARGUMENT;
    }
    if (n == 0) return PRC_OK;
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    poisson_kernel<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_mean, (long long)n, scale, key, d_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        prc::set_last_error(std::string("CUDA error '") + cudaGetErrorString(e) + "' in prc_poisson");
        return PRC_ERR_CUDA;
    }
    return PRC_OK;
}
