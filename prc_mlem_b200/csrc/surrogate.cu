// surrogate.cu -- the learned range-kernel surrogate: tensor-core (tcgen05) GEMMs, the 3D CNN
// that maps a voxel's 9^3 density patch and isotope to per-direction radial far-field kernel
// coefficients, its training (forward, backward, Adam) and its inference into a coefficient
// field.  The GEMM engine is umma.cuh.
#include "../../include/prc_surrogate.h"
#include "../../include/prc_b200.h"
#include "engine.h"
#include "umma.cuh"

#include <string>
#include <vector>

namespace {

using bf16 = __nv_bfloat16;

// ---- plain GEMM: C[M][N] = A[M][K] . B[N][K]^T (both row-major, K contiguous) ----------------
struct PlainGemm {
    const bf16* a;
    const bf16* b;
    float* c;
    int M, N, K;
};

template <int BN>
__global__ void __launch_bounds__(prc::umma::kThreads) plain_gemm_kernel(PlainGemm g, unsigned int* error) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const bool ok = prc::umma::gemm_tile<BN>(
        g.M, g.N, g.K, blockIdx.x * prc::umma::kM, blockIdx.y * BN, 0, g.K,
        [&](int m, int k) { return g.a[(size_t)m * g.K + k]; }, [&](int n, int k) { return g.b[(size_t)n * g.K + k]; },
        [&](int m, int n, float v) { g.c[(size_t)m * g.N + n] = v; }, smem, &bar, &tmem_slot);
    if (!ok && threadIdx.x == 0) atomicOr(error, 1u);
}

}  // namespace

extern "C" int prc_nn_gemm_bf16(const void* d_a, const void* d_b, float* d_c, int M, int N, int K,
                                unsigned int* d_error, void* stream) {
    if (!d_a || !d_b || !d_c || !d_error || M <= 0 || N <= 0 || K <= 0) {
        prc::set_last_error("Invalid argument");
        return PRC_ERR_ARGUMENT;
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    PlainGemm g{static_cast<const bf16*>(d_a), static_cast<const bf16*>(d_b), d_c, M, N, K};
    constexpr int BN = 64;
    dim3 grid((M + prc::umma::kM - 1) / prc::umma::kM, (N + BN - 1) / BN);
    cudaError_t e = cudaFuncSetAttribute(plain_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)prc::umma::smem_bytes<BN>());
    if (e == cudaSuccess) {
        plain_gemm_kernel<BN><<<grid, prc::umma::kThreads, prc::umma::smem_bytes<BN>(), s>>>(g, d_error);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        prc::set_last_error(std::string("CUDA error '") + cudaGetErrorString(e) + "' in prc_nn_gemm_bf16");
        return PRC_ERR_CUDA;
    }
    return PRC_OK;
}

// ================================================================================================
// The network: 4 valid 3x3x3 convolutions (32 channels, ReLU) on a 9^3 patch, then a linear head
// to 128 directions x 16 radial bins.  Tensors are channels-last; conv weights [cout][27][cin].
// Every GEMM below is an implicit GEMM on the tensor cores: the loaders compute the im2col (or
// its transpose) addresses, the store functors apply bias, ReLU and the bf16 rounding.
// ================================================================================================
namespace {

constexpr int kC = 32;           // channels of the hidden layers
constexpr int kIn = 4;           // density + one-hot isotope (18F, 68Ga, 82Rb)
constexpr int kOut = 2048;       // 128 directions x 16 radial bins
constexpr int kLayers = 5;       // 4 convolutions + head
constexpr int kSide[5] = {9, 7, 5, 3, 1};  // spatial side of the input of layer l (l = 0..3), and a4

__device__ __forceinline__ void decode3(int p, int S, int& z, int& y, int& x) {
    z = p / (S * S);
    y = (p / S) % S;
    x = p % S;
}

// Forward convolution: out[(b,p)][cout] = relu(sum_{kpos,cin} x[b][p+kpos][cin] w[cout][kpos][cin] + bias)
struct ConvFwd {
    const bf16* x;
    const bf16* w;
    const float* bias;
    bf16* out;
    int S, cin;  // input side and channels
    __device__ bf16 a(int m, int k) const {
        const int So = S - 2, n3 = So * So * So, b = m / n3;
        int oz, oy, ox, kz, ky, kx;
        decode3(m % n3, So, oz, oy, ox);
        decode3(k / cin, 3, kz, ky, kx);
        return x[((((size_t)b * S + oz + kz) * S + oy + ky) * S + ox + kx) * cin + k % cin];
    }
    __device__ bf16 b(int n, int k) const { return w[(size_t)n * 27 * cin + k]; }
    __device__ void store(int m, int n, float v) const {
        out[(size_t)m * kC + n] = __float2bfloat16_rn(fmaxf(v + bias[n], 0.0f));
    }
};

// Data gradient of a convolution, masked by the previous layer's ReLU:
// dz_prev[(b,pin)][cin] = (x[b][pin][cin] > 0) * sum_{kpos,cout} dz[b][pin-kpos][cout] w[cout][kpos][cin]
struct ConvDx {
    const bf16* dz;
    const bf16* w;
    const bf16* x;
    bf16* dz_prev;
    int S;  // input side (output side S - 2); cin = cout = 32
    __device__ bf16 a(int m, int k) const {
        const int So = S - 2, n3 = S * S * S, b = m / n3;
        int iz, iy, ix, kz, ky, kx;
        decode3(m % n3, S, iz, iy, ix);
        decode3(k / kC, 3, kz, ky, kx);
        const int oz = iz - kz, oy = iy - ky, ox = ix - kx;
        if (oz < 0 || oy < 0 || ox < 0 || oz >= So || oy >= So || ox >= So) return __float2bfloat16(0.0f);
        return dz[((((size_t)b * So + oz) * So + oy) * So + ox) * kC + k % kC];
    }
    __device__ bf16 b(int n, int k) const { return w[((size_t)(k % kC) * 27 + k / kC) * kC + n]; }
    __device__ void store(int m, int n, float v) const {
        const size_t i = (size_t)m * kC + n;
        dz_prev[i] = __float2bfloat16_rn(__bfloat162float(x[i]) > 0.0f ? v : 0.0f);
    }
};

// Weight gradient: gw[cout][(kpos,cin)] = sum_{b,p} dz[b][p][cout] x[b][p+kpos][cin]; split-K
// slices add into gw.
struct ConvDw {
    const bf16* x;
    const bf16* dz;
    float* gw;
    int S, cin;
    __device__ bf16 a(int m, int k) const {
        const int So = S - 2, n3 = So * So * So, b = k / n3;
        int oz, oy, ox, kz, ky, kx;
        decode3(k % n3, So, oz, oy, ox);
        decode3(m / cin, 3, kz, ky, kx);
        return x[((((size_t)b * S + oz + kz) * S + oy + ky) * S + ox + kx) * cin + m % cin];
    }
    __device__ bf16 b(int n, int k) const { return dz[(size_t)k * kC + n]; }
    __device__ void store(int m, int n, float v) const { atomicAdd(gw + (size_t)n * 27 * cin + m, v); }
};

struct HeadFwd {
    const bf16* a4;
    const bf16* wh;
    const float* bh;
    float* y;
    __device__ bf16 a(int m, int k) const { return a4[(size_t)m * kC + k]; }
    __device__ bf16 b(int n, int k) const { return wh[(size_t)n * kC + k]; }
    __device__ void store(int m, int n, float v) const { y[(size_t)m * kOut + n] = v + bh[n]; }
};

struct HeadDx {
    const bf16* dy;
    const bf16* wh;
    const bf16* a4;
    bf16* dz4;
    __device__ bf16 a(int m, int k) const { return dy[(size_t)m * kOut + k]; }
    __device__ bf16 b(int n, int k) const { return wh[(size_t)k * kC + n]; }
    __device__ void store(int m, int n, float v) const {
        const size_t i = (size_t)m * kC + n;
        dz4[i] = __float2bfloat16_rn(__bfloat162float(a4[i]) > 0.0f ? v : 0.0f);
    }
};

struct HeadDw {
    const bf16* dy;
    const bf16* a4;
    float* gwh;
    __device__ bf16 a(int m, int k) const { return dy[(size_t)k * kOut + m]; }
    __device__ bf16 b(int n, int k) const { return a4[(size_t)k * kC + n]; }
    __device__ void store(int m, int n, float v) const { atomicAdd(gwh + (size_t)m * kC + n, v); }
};

template <int BN, class P>
__global__ void __launch_bounds__(prc::umma::kThreads) problem_kernel(P prob, int M, int N, int K, int k_split,
                                                                      unsigned int* error) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int k_lo = blockIdx.z * k_split;
    const bool ok = prc::umma::gemm_tile<BN>(
        M, N, K, blockIdx.x * prc::umma::kM, blockIdx.y * BN, k_lo, k_lo + k_split,
        [&](int m, int k) { return prob.a(m, k); }, [&](int n, int k) { return prob.b(n, k); },
        [&](int m, int n, float v) { prob.store(m, n, v); }, smem, &bar, &tmem_slot);
    if (!ok && threadIdx.x == 0) atomicOr(error, 1u);
}

// splits > 1 only for problems whose store adds (weight gradients).
template <int BN, class P>
cudaError_t run_problem(const P& prob, int M, int N, int K, int splits, unsigned int* error, cudaStream_t s) {
    const int tiles = (K + prc::umma::kKT - 1) / prc::umma::kKT;
    if (splits > tiles) splits = tiles;
    if (splits < 1) splits = 1;
    const int k_split = (tiles + splits - 1) / splits * prc::umma::kKT;
    splits = (K + k_split - 1) / k_split;
    static bool attr = false;
    if (!attr) {
        const cudaError_t e = cudaFuncSetAttribute(problem_kernel<BN, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)prc::umma::smem_bytes<BN>());
        if (e != cudaSuccess) return e;
        attr = true;
    }
    dim3 grid((M + prc::umma::kM - 1) / prc::umma::kM, (N + BN - 1) / BN, splits);
    problem_kernel<BN, P><<<grid, prc::umma::kThreads, prc::umma::smem_bytes<BN>(), s>>>(prob, M, N, K, k_split, error);
    return cudaGetLastError();
}

// loss and dy = bf16(2 (y - t) / (B * 2048)); FP64 sum of squared errors into *sse
__global__ void loss_kernel(const float* y, const float* t, bf16* dy, size_t n, double* sse) {
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        dy[i] = __float2bfloat16_rn(2.0f * d / (float)n);
        acc += (double)d * d;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sse, acc);
}

// gb[n] = sum over rows of dz[row][n] (n < cols); one block per column.
__global__ void colsum_kernel(const bf16* dz, int rows, int cols, float* gb) {
    const int n = blockIdx.x;
    float acc = 0.0f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) acc += __bfloat162float(dz[(size_t)r * cols + n]);
    __shared__ float sh[32];
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        gb[n] = t;
    }
}

// Adam on fp32 master weights (bias-corrected), then the bf16 copy the GEMMs read.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, bf16* wb, size_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi, v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(const float* w, bf16* wb, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

}  // namespace

// Parameter tensors: index 0..3 conv layers (weights [32][27][cin], bias [32]), 4 head
// (weights [2048][32], bias [2048]).
struct prc_net {
    int max_batch = 0;
    float* w[kLayers] = {};
    float* b[kLayers] = {};
    bf16* wb[kLayers] = {};
    float* gw[kLayers] = {};
    float* gb[kLayers] = {};
    float* mw[kLayers] = {};
    float* vw[kLayers] = {};
    float* mb[kLayers] = {};
    float* vb[kLayers] = {};
    size_t nw[kLayers] = {}, nb[kLayers] = {};
    bf16* act[5] = {};  // a0 (input patches) .. a4
    bf16* dz[5] = {};   // dz[l]: gradient wrt the pre-activation of conv layer l (1..4)
    float* y = nullptr;
    bf16* dy = nullptr;
    double* sse = nullptr;
    unsigned int* error = nullptr;
    int step = 0;
    std::vector<void*> allocs;
    cudaStream_t stream = nullptr;
};

namespace {

template <class T>
cudaError_t net_alloc(prc_net* n, T** p, size_t count) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, count * sizeof(T) + 16);
    if (e != cudaSuccess) return e;
    n->allocs.push_back(v);
    *p = static_cast<T*>(v);
    return cudaMemset(v, 0, count * sizeof(T) + 16);
}

int nn_fail(cudaError_t e, const char* what) {
    prc::set_last_error(std::string("CUDA error '") + cudaGetErrorString(e) + "' in " + what);
    return e == cudaErrorMemoryAllocation ? PRC_ERR_MEMORY : PRC_ERR_CUDA;
}

#define NN_CUDA(call, what)                                 \
    do {                                                    \
        const cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return nn_fail(e_, what);    \
    } while (0)

}  // namespace

extern "C" {

int prc_nn_create(int max_batch, prc_net** out) {
    if (!out || max_batch <= 0) {
        prc::set_last_error("Invalid argument");
        return PRC_ERR_ARGUMENT;
    }
    *out = nullptr;
    prc_net* n = new prc_net();
    n->max_batch = max_batch;
    const int cin[kLayers] = {kIn, kC, kC, kC, kC};
    auto fail_cleanup = [&](int code) {
        for (void* p : n->allocs) cudaFree(p);
        delete n;
        return code;
    };
    for (int l = 0; l < kLayers; ++l) {
        n->nw[l] = l < 4 ? (size_t)kC * 27 * cin[l] : (size_t)kOut * kC;
        n->nb[l] = l < 4 ? kC : kOut;
        cudaError_t e = cudaSuccess;
        for (float** p : {&n->w[l], &n->gw[l], &n->mw[l], &n->vw[l]})
            if (e == cudaSuccess) e = net_alloc(n, p, n->nw[l]);
        for (float** p : {&n->b[l], &n->gb[l], &n->mb[l], &n->vb[l]})
            if (e == cudaSuccess) e = net_alloc(n, p, n->nb[l]);
        if (e == cudaSuccess) e = net_alloc(n, &n->wb[l], n->nw[l]);
        if (e != cudaSuccess) return fail_cleanup(nn_fail(e, "prc_nn_create"));
    }
    const size_t B = (size_t)max_batch;
    const size_t act_sizes[5] = {B * 729 * kIn, B * 343 * kC, B * 125 * kC, B * 27 * kC, B * kC};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = net_alloc(n, &n->act[i], act_sizes[i]);
    for (int i = 1; i < 5 && e == cudaSuccess; ++i) e = net_alloc(n, &n->dz[i], act_sizes[i]);
    if (e == cudaSuccess) e = net_alloc(n, &n->y, B * kOut);
    if (e == cudaSuccess) e = net_alloc(n, &n->dy, B * kOut);
    if (e == cudaSuccess) e = net_alloc(n, &n->sse, 1);
    if (e == cudaSuccess) e = net_alloc(n, &n->error, 1);
    if (e != cudaSuccess) return fail_cleanup(nn_fail(e, "prc_nn_create"));
    *out = n;
    return PRC_OK;
}

void prc_nn_destroy(prc_net* n) {
    if (!n) return;
    cudaDeviceSynchronize();
    for (void* p : n->allocs) cudaFree(p);
    delete n;
}

// Parameters from / to host memory: tensor order w1, b1, w2, b2, w3, b3, w4, b4, wh, bh.
int prc_nn_set_params(prc_net* n, const float* host) {
    if (!n || !host) return prc::set_last_error("Invalid argument"), PRC_ERR_ARGUMENT;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        NN_CUDA(cudaMemcpy(n->w[l], host + off, n->nw[l] * 4, cudaMemcpyHostToDevice), "prc_nn_set_params");
        off += n->nw[l];
        NN_CUDA(cudaMemcpy(n->b[l], host + off, n->nb[l] * 4, cudaMemcpyHostToDevice), "prc_nn_set_params");
        off += n->nb[l];
        to_bf16_kernel<<<64, 256>>>(n->w[l], n->wb[l], n->nw[l]);
        NN_CUDA(cudaMemset(n->mw[l], 0, n->nw[l] * 4), "prc_nn_set_params");
        NN_CUDA(cudaMemset(n->vw[l], 0, n->nw[l] * 4), "prc_nn_set_params");
        NN_CUDA(cudaMemset(n->mb[l], 0, n->nb[l] * 4), "prc_nn_set_params");
        NN_CUDA(cudaMemset(n->vb[l], 0, n->nb[l] * 4), "prc_nn_set_params");
    }
    n->step = 0;
    NN_CUDA(cudaDeviceSynchronize(), "prc_nn_set_params");
    return PRC_OK;
}

int64_t prc_nn_param_count(void) {
    return (int64_t)kC * 27 * kIn + kC + 3 * ((int64_t)kC * 27 * kC + kC) + (int64_t)kOut * kC + kOut;
}

int prc_nn_get(prc_net* n, int what, float* host) {
    if (!n || !host) return prc::set_last_error("Invalid argument"), PRC_ERR_ARGUMENT;
    NN_CUDA(cudaDeviceSynchronize(), "prc_nn_get");
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        const float* w = what == 0 ? n->w[l] : n->gw[l];
        const float* b = what == 0 ? n->b[l] : n->gb[l];
        NN_CUDA(cudaMemcpy(host + off, w, n->nw[l] * 4, cudaMemcpyDeviceToHost), "prc_nn_get");
        off += n->nw[l];
        NN_CUDA(cudaMemcpy(host + off, b, n->nb[l] * 4, cudaMemcpyDeviceToHost), "prc_nn_get");
        off += n->nb[l];
    }
    return PRC_OK;
}

// Forward pass of a batch of patches d_x0 ([batch][9][9][9][4] bf16) into d_y ([batch][2048] fp32;
// NULL = the network's own buffer), keeping the activations for a backward pass.
int prc_nn_forward(prc_net* n, const void* d_x0, int batch, float* d_y, void* stream) {
    if (!n || !d_x0 || batch <= 0 || batch > n->max_batch)
        return prc::set_last_error("Invalid argument"), PRC_ERR_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    NN_CUDA(cudaMemcpyAsync(n->act[0], d_x0, (size_t)batch * 729 * kIn * sizeof(bf16), cudaMemcpyDeviceToDevice, s),
            "prc_nn_forward");
    for (int l = 0; l < 4; ++l) {
        const int S = kSide[l], So = S - 2, cin = l == 0 ? kIn : kC;
        ConvFwd p{n->act[l], n->wb[l], n->b[l], n->act[l + 1], S, cin};
        NN_CUDA((run_problem<32>(p, batch * So * So * So, kC, 27 * cin, 1, n->error, s)), "prc_nn_forward");
    }
    HeadFwd h{n->act[4], n->wb[4], n->b[4], d_y ? d_y : n->y};
    NN_CUDA((run_problem<256>(h, batch, kOut, kC, 1, n->error, s)), "prc_nn_forward");
    return PRC_OK;
}

// Loss against d_target ([batch][2048] fp32) after prc_nn_forward on the same batch (output in
// the network's own buffer), all gradients, and -- with lr > 0 -- one Adam step.  The mean
// squared error is written to *loss (host; synchronises) when loss is not NULL.
int prc_nn_backward(prc_net* n, const float* d_target, int batch, float lr, double* loss, void* stream) {
    if (!n || !d_target || batch <= 0 || batch > n->max_batch)
        return prc::set_last_error("Invalid argument"), PRC_ERR_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t ny = (size_t)batch * kOut;
    NN_CUDA(cudaMemsetAsync(n->sse, 0, sizeof(double), s), "prc_nn_backward");
    loss_kernel<<<256, 256, 0, s>>>(n->y, d_target, n->dy, ny, n->sse);
    for (int l = 0; l < kLayers; ++l) NN_CUDA(cudaMemsetAsync(n->gw[l], 0, n->nw[l] * 4, s), "prc_nn_backward");
    // head
    HeadDw hw{n->dy, n->act[4], n->gw[4]};
    NN_CUDA((run_problem<32>(hw, kOut, kC, batch, 8, n->error, s)), "prc_nn_backward");
    colsum_kernel<<<kOut, 256, 0, s>>>(n->dy, batch, kOut, n->gb[4]);
    HeadDx hx{n->dy, n->wb[4], n->act[4], n->dz[4]};
    NN_CUDA((run_problem<32>(hx, batch, kC, kOut, 1, n->error, s)), "prc_nn_backward");
    // convolutions, last to first
    for (int l = 3; l >= 0; --l) {
        const int S = kSide[l], So = S - 2, cin = l == 0 ? kIn : kC;
        const int rows_out = batch * So * So * So;
        ConvDw dw{n->act[l], n->dz[l + 1], n->gw[l], S, cin};
        const int k_tiles = (rows_out + prc::umma::kKT - 1) / prc::umma::kKT;
        NN_CUDA((run_problem<32>(dw, 27 * cin, kC, rows_out, (k_tiles + 7) / 8, n->error, s)), "prc_nn_backward");
        colsum_kernel<<<kC, 256, 0, s>>>(n->dz[l + 1], rows_out, kC, n->gb[l]);
        if (l > 0) {
            ConvDx dx{n->dz[l + 1], n->wb[l], n->act[l], n->dz[l], S};
            NN_CUDA((run_problem<32>(dx, batch * S * S * S, kC, 27 * kC, 1, n->error, s)), "prc_nn_backward");
        }
    }
    if (lr > 0.0f) {
        n->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - powf(b1, (float)n->step), c2 = 1.0f - powf(b2, (float)n->step);
        for (int l = 0; l < kLayers; ++l) {
            adam_kernel<<<128, 256, 0, s>>>(n->w[l], n->gw[l], n->mw[l], n->vw[l], n->wb[l], n->nw[l], lr, b1, b2, 1e-8f,
                                            c1, c2);
            adam_kernel<<<8, 256, 0, s>>>(n->b[l], n->gb[l], n->mb[l], n->vb[l], nullptr, n->nb[l], lr, b1, b2, 1e-8f,
                                          c1, c2);
        }
    }
    NN_CUDA(cudaGetLastError(), "prc_nn_backward");
    if (loss) {
        double sse = 0.0;
        unsigned int err = 0;
        NN_CUDA(cudaMemcpyAsync(&sse, n->sse, sizeof(double), cudaMemcpyDeviceToHost, s), "prc_nn_backward");
        NN_CUDA(cudaMemcpyAsync(&err, n->error, sizeof(err), cudaMemcpyDeviceToHost, s), "prc_nn_backward");
        NN_CUDA(cudaStreamSynchronize(s), "prc_nn_backward");
        if (err) return prc::set_last_error("a tensor-core MMA wait gave up"), PRC_ERR_CUDA;
        *loss = sse / (double)ny;
    }
    return PRC_OK;
}

}  // extern "C"
