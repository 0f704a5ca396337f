// surrogate.cu -- the learned range-kernel surrogate: tensor-core (tcgen05) GEMMs, the 3D CNN
// that maps a voxel's 9^3 density patch and isotope to per-direction radial far-field kernel
// coefficients, its training (forward, backward, Adam) and its inference into a coefficient
// field.  The GEMM engine is umma.cuh.
#include "../../include/prc_surrogate.h"
#include "../../include/prc_b200.h"
#include "engine.h"
#include "umma.cuh"

#include <string>
#include <type_traits>
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
// The network: 4 valid 3x3x3 convolutions (32 channels, ReLU) with dilations 1, 2, 3 and 4 on a
// 21^3 patch (a voxel sees 10 voxels in every direction), then a linear head to 128 directions x
// 16 radial bins.  Tensors are channels-last; conv weights [cout][27][cin].
// Every GEMM below is an implicit GEMM on the tensor cores: the loaders compute the im2col (or
// its transpose) addresses, the store functors apply bias, ReLU and the bf16 rounding.
// ================================================================================================
namespace {

constexpr int kC = 32;           // channels of the hidden layers
constexpr int kIn = 8;           // density, inside-the-volume flag, one-hot isotope (18F, 68Ga, 82Rb), 3 zeros
constexpr int kOut = 2048;       // 128 directions x 16 radial bins
constexpr int kLayers = 5;       // 4 convolutions + head
constexpr int kDil[4] = {1, 2, 3, 4};       // tap spacing of convolution l
constexpr int kSide[5] = {21, 19, 15, 9, 1};  // spatial side of the input of layer l (l = 0..3), and a4
static_assert(kSide[0] == 1 + 2 * (kDil[0] + kDil[1] + kDil[2] + kDil[3]) && kSide[1] == kSide[0] - 2 * kDil[0] &&
                  kSide[2] == kSide[1] - 2 * kDil[1] && kSide[3] == kSide[2] - 2 * kDil[2] &&
                  kSide[4] == kSide[3] - 2 * kDil[3],
              "each convolution trims its dilation from both sides");

__device__ __forceinline__ void decode3(int p, int S, int& z, int& y, int& x) {
    z = p / (S * S);
    y = (p / S) % S;
    x = p % S;
}

// Forward convolution with taps d apart:
// out[(b,p)][cout] = relu(sum_{kpos,cin} x[b][p + d kpos][cin] w[cout][kpos][cin] + bias)
struct ConvFwd {
    const bf16* x;
    const bf16* w;
    const float* bias;
    bf16* out;
    int S, cin, d;  // input side, channels and dilation
    __device__ bf16 a(int m, int k) const {
        const int So = S - 2 * d, n3 = So * So * So, b = m / n3;
        int oz, oy, ox, kz, ky, kx;
        decode3(m % n3, So, oz, oy, ox);
        decode3(k / cin, 3, kz, ky, kx);
        return x[((((size_t)b * S + oz + kz * d) * S + oy + ky * d) * S + ox + kx * d) * cin + k % cin];
    }
    // 8 channels of one tap are contiguous when cin is a multiple of 8 (the 32-channel layers)
    __device__ bool vec_a() const { return cin % 8 == 0; }
    __device__ uint4 a8(int m, int k) const {
        const int So = S - 2 * d, n3 = So * So * So, b = m / n3;
        int oz, oy, ox, kz, ky, kx;
        decode3(m % n3, So, oz, oy, ox);
        decode3(k / cin, 3, kz, ky, kx);
        return *reinterpret_cast<const uint4*>(
            x + ((((size_t)b * S + oz + kz * d) * S + oy + ky * d) * S + ox + kx * d) * cin + k % cin);
    }
    __device__ bf16 b(int n, int k) const { return w[(size_t)n * 27 * cin + k]; }
    __device__ void store(int m, int n, float v) const {
        out[(size_t)m * kC + n] = __float2bfloat16_rn(fmaxf(v + bias[n], 0.0f));
    }
};

// Data gradient of a convolution, masked by the previous layer's ReLU:
// dz_prev[(b,pin)][cin] = (x[b][pin][cin] > 0) * sum_{kpos,cout} dz[b][pin - d kpos][cout] w[cout][kpos][cin]
struct ConvDx {
    const bf16* dz;
    const bf16* w;
    const bf16* x;
    bf16* dz_prev;
    int S, d;  // input side (output side S - 2d) and dilation; cin = cout = 32
    __device__ bf16 a(int m, int k) const {
        const int So = S - 2 * d, n3 = S * S * S, b = m / n3;
        int iz, iy, ix, kz, ky, kx;
        decode3(m % n3, S, iz, iy, ix);
        decode3(k / kC, 3, kz, ky, kx);
        const int oz = iz - kz * d, oy = iy - ky * d, ox = ix - kx * d;
        if (oz < 0 || oy < 0 || ox < 0 || oz >= So || oy >= So || ox >= So) return __float2bfloat16(0.0f);
        return dz[((((size_t)b * So + oz) * So + oy) * So + ox) * kC + k % kC];
    }
    __device__ bool vec_a() const { return true; }
    __device__ uint4 a8(int m, int k) const {
        const int So = S - 2 * d, n3 = S * S * S, b = m / n3;
        int iz, iy, ix, kz, ky, kx;
        decode3(m % n3, S, iz, iy, ix);
        decode3(k / kC, 3, kz, ky, kx);
        const int oz = iz - kz * d, oy = iy - ky * d, ox = ix - kx * d;
        if (oz < 0 || oy < 0 || ox < 0 || oz >= So || oy >= So || ox >= So) return make_uint4(0u, 0u, 0u, 0u);
        return *reinterpret_cast<const uint4*>(dz + ((((size_t)b * So + oz) * So + oy) * So + ox) * kC + k % kC);
    }
    __device__ bf16 b(int n, int k) const { return w[((size_t)(k % kC) * 27 + k / kC) * kC + n]; }
    static constexpr bool kRowsA = false, kRowsB = true;
    __device__ void store(int m, int n, float v) const {
        const size_t i = (size_t)m * kC + n;
        dz_prev[i] = __float2bfloat16_rn(__bfloat162float(x[i]) > 0.0f ? v : 0.0f);
    }
};

// Weight gradient: gw[cout][(kpos,cin)] = sum_{b,p} dz[b][p][cout] x[b][p + d kpos][cin]; split-K
// slices add into gw.
struct ConvDw {
    const bf16* x;
    const bf16* dz;
    float* gw;
    int S, cin, d;
    __device__ bf16 a(int m, int k) const {
        const int So = S - 2 * d, n3 = So * So * So, b = k / n3;
        int oz, oy, ox, kz, ky, kx;
        decode3(k % n3, So, oz, oy, ox);
        decode3(m / cin, 3, kz, ky, kx);
        return x[((((size_t)b * S + oz + kz * d) * S + oy + ky * d) * S + ox + kx * d) * cin + m % cin];
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
    __device__ bool vec_a() const { return true; }
    __device__ uint4 a8(int m, int k) const { return *reinterpret_cast<const uint4*>(a4 + (size_t)m * kC + k); }
    __device__ bf16 b(int n, int k) const { return wh[(size_t)n * kC + k]; }
    __device__ void store(int m, int n, float v) const { y[(size_t)m * kOut + n] = v + bh[n]; }
};

struct HeadDx {
    const bf16* dy;
    const bf16* wh;
    const bf16* a4;
    bf16* dz4;
    __device__ bf16 a(int m, int k) const { return dy[(size_t)m * kOut + k]; }
    __device__ bool vec_a() const { return true; }
    __device__ uint4 a8(int m, int k) const { return *reinterpret_cast<const uint4*>(dy + (size_t)m * kOut + k); }
    __device__ bf16 b(int n, int k) const { return wh[(size_t)k * kC + n]; }
    static constexpr bool kRowsA = false, kRowsB = true;
    // run split over K (SplitK); relu_grad_epilogue_kernel then writes
    // dz4 = bf16(a4 > 0 ? sum : 0)
};

struct HeadDw {
    const bf16* dy;
    const bf16* a4;
    float* gwh;
    __device__ bf16 a(int m, int k) const { return dy[(size_t)k * kOut + m]; }
    __device__ bf16 b(int n, int k) const { return a4[(size_t)k * kC + n]; }
    __device__ void store(int m, int n, float v) const { atomicAdd(gwh + (size_t)m * kC + n, v); }
};

// Problems whose A operand has 16-byte rows in memory offer a8(m, k) (8 values at once) and
// vec_a() (whether this instance may use it).
template <class P, class = void>
struct HasVecA : std::false_type {};
template <class P>
struct HasVecA<P, decltype((void)&P::a8)> : std::true_type {};
// kRowsA / kRowsB (default false): the operand is contiguous along M / N, so its element loader
// walks rows fastest.
template <class P, class = void>
struct RowsA : std::false_type {};
template <class P>
struct RowsA<P, std::enable_if_t<P::kRowsA>> : std::true_type {};
template <class P, class = void>
struct RowsB : std::false_type {};
template <class P>
struct RowsB<P, std::enable_if_t<P::kRowsB>> : std::true_type {};

// (Measured: walking rows fastest helps the weight operand of the data gradients, whose rows are
// contiguous channels, but slows the weight-gradient GEMMs down, whose operands are read from
// several positions per row anyway; those keep the K-fastest order.)
static_assert(!RowsA<ConvDx>::value && RowsB<ConvDx>::value && RowsB<HeadDx>::value && !RowsA<ConvDw>::value &&
                  !RowsB<ConvDw>::value && !RowsA<ConvFwd>::value && !RowsB<ConvFwd>::value,
              "loader order per operand");
static_assert(HasVecA<ConvFwd>::value && HasVecA<ConvDx>::value && HasVecA<HeadFwd>::value && HasVecA<HeadDx>::value &&
                  !HasVecA<ConvDw>::value && !HasVecA<HeadDw>::value,
              "channels-last problems offer 16-byte A rows");

// Few output rows (the 3^3 -> 1 convolution and the head's data gradient have one row per
// sample) leave most SMs idle, so those GEMMs also split K: every slice adds into an fp32
// buffer and a second pass applies the epilogue.  Same operands as the wrapped problem.
template <class P>
struct SplitK {
    P p;
    float* acc;  // [M][kC]
    __device__ bf16 a(int m, int k) const { return p.a(m, k); }
    __device__ bool vec_a() const { return p.vec_a(); }
    __device__ uint4 a8(int m, int k) const { return p.a8(m, k); }
    __device__ bf16 b(int n, int k) const { return p.b(n, k); }
    __device__ void store(int m, int n, float v) const { atomicAdd(acc + (size_t)m * kC + n, v); }
    static constexpr bool kRowsA = RowsA<P>::value, kRowsB = RowsB<P>::value;
};

static_assert(HasVecA<SplitK<ConvFwd>>::value && HasVecA<SplitK<HeadDx>>::value, "the split keeps the vector loader");

// out = bf16(relu(acc + bias))
__global__ void conv_epilogue_kernel(const float* acc, const float* bias, bf16* out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(fmaxf(acc[i] + bias[i % kC], 0.0f));
}
// dz = bf16(a > 0 ? acc : 0)
__global__ void relu_grad_epilogue_kernel(const float* acc, const bf16* a, bf16* dz, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dz[i] = __float2bfloat16_rn(__bfloat162float(a[i]) > 0.0f ? acc[i] : 0.0f);
}

template <int BN, class P>
__global__ void __launch_bounds__(prc::umma::kThreads) problem_kernel(P prob, int M, int N, int K, int k_split,
                                                                      unsigned int* error) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int k_lo = blockIdx.z * k_split;
    bool ok;
    if constexpr (HasVecA<P>::value) {
        ok = prc::umma::gemm_tile<BN, RowsA<P>::value, RowsB<P>::value>(
            M, N, K, blockIdx.x * prc::umma::kM, blockIdx.y * BN, k_lo, k_lo + k_split,
            [&](int m, int k) { return prob.a(m, k); }, prob.vec_a(), [&](int m, int k) { return prob.a8(m, k); },
            [&](int n, int k) { return prob.b(n, k); }, [&](int m, int n, float v) { prob.store(m, n, v); }, smem, &bar,
            &tmem_slot);
    } else {
        ok = prc::umma::gemm_tile<BN, RowsA<P>::value, RowsB<P>::value>(
            M, N, K, blockIdx.x * prc::umma::kM, blockIdx.y * BN, k_lo, k_lo + k_split,
            [&](int m, int k) { return prob.a(m, k); }, false, prc::umma::NoVecA{},
            [&](int n, int k) { return prob.b(n, k); }, [&](int m, int n, float v) { prob.store(m, n, v); }, smem,
            &bar, &tmem_slot);
    }
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

// loss and dy = bf16(2 (y - t) / (B * 2048)); FP64 sum of squared errors into *sse.  A negative
// target marks an output the surrogate field never uses (no loss, no gradient).
__global__ void loss_kernel(const float* y, const float* t, bf16* dy, size_t n, double* sse) {
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float d = t[i] < 0.0f ? 0.0f : y[i] - t[i];
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
    float* split_acc = nullptr;  // [max_batch][kC] fp32 partial sums of the split-K GEMMs
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
    auto cube = [](int side) { return (size_t)side * side * side; };
    const size_t act_sizes[5] = {B * cube(kSide[0]) * kIn, B * cube(kSide[1]) * kC, B * cube(kSide[2]) * kC,
                                 B * cube(kSide[3]) * kC, B * cube(kSide[4]) * kC};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = net_alloc(n, &n->act[i], act_sizes[i]);
    for (int i = 1; i < 5 && e == cudaSuccess; ++i) e = net_alloc(n, &n->dz[i], act_sizes[i]);
    if (e == cudaSuccess) e = net_alloc(n, &n->y, B * kOut);
    if (e == cudaSuccess) e = net_alloc(n, &n->dy, B * kOut);
    if (e == cudaSuccess) e = net_alloc(n, &n->sse, 1);
    if (e == cudaSuccess) e = net_alloc(n, &n->split_acc, B * kC);
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

int prc_nn_patch_side(void) { return kSide[0]; }

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

// Forward pass of a batch of patches d_x0 ([batch][21][21][21][8] bf16) into d_y ([batch][2048]
// fp32; NULL = the network's own buffer), keeping the activations for a backward pass.
int prc_nn_forward(prc_net* n, const void* d_x0, int batch, float* d_y, void* stream) {
    if (!n || !d_x0 || batch <= 0 || batch > n->max_batch)
        return prc::set_last_error("Invalid argument"), PRC_ERR_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t patch = (size_t)kSide[0] * kSide[0] * kSide[0];
    NN_CUDA(cudaMemcpyAsync(n->act[0], d_x0, (size_t)batch * patch * kIn * sizeof(bf16), cudaMemcpyDeviceToDevice, s),
            "prc_nn_forward");
    for (int l = 0; l < 4; ++l) {
        const int S = kSide[l], So = kSide[l + 1], cin = l == 0 ? kIn : kC;
        ConvFwd p{n->act[l], n->wb[l], n->b[l], n->act[l + 1], S, cin, kDil[l]};
        const int rows = batch * So * So * So;
        if (So == 1) {  // one row per sample: split K, then bias + ReLU
            NN_CUDA(cudaMemsetAsync(n->split_acc, 0, (size_t)rows * kC * sizeof(float), s), "prc_nn_forward");
            NN_CUDA((run_problem<32>(SplitK<ConvFwd>{p, n->split_acc}, rows, kC, 27 * cin, 14, n->error, s)),
                    "prc_nn_forward");
            conv_epilogue_kernel<<<64, 256, 0, s>>>(n->split_acc, n->b[l], n->act[l + 1], (size_t)rows * kC);
        } else {
            NN_CUDA((run_problem<32>(p, rows, kC, 27 * cin, 1, n->error, s)), "prc_nn_forward");
        }
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
    NN_CUDA(cudaMemsetAsync(n->split_acc, 0, (size_t)batch * kC * sizeof(float), s), "prc_nn_backward");
    NN_CUDA((run_problem<32>(SplitK<HeadDx>{hx, n->split_acc}, batch, kC, kOut, 32, n->error, s)), "prc_nn_backward");
    relu_grad_epilogue_kernel<<<64, 256, 0, s>>>(n->split_acc, n->act[4], n->dz[4], (size_t)batch * kC);
    // convolutions, last to first
    for (int l = 3; l >= 0; --l) {
        const int S = kSide[l], So = kSide[l + 1], cin = l == 0 ? kIn : kC;
        const int rows_out = batch * So * So * So;
        ConvDw dw{n->act[l], n->dz[l + 1], n->gw[l], S, cin, kDil[l]};
        const int k_tiles = (rows_out + prc::umma::kKT - 1) / prc::umma::kKT;
        NN_CUDA((run_problem<32>(dw, 27 * cin, kC, rows_out, (k_tiles + 7) / 8, n->error, s)), "prc_nn_backward");
        colsum_kernel<<<kC, 256, 0, s>>>(n->dz[l + 1], rows_out, kC, n->gb[l]);
        if (l > 0) {
            ConvDx dx{n->dz[l + 1], n->wb[l], n->act[l], n->dz[l], S, kDil[l]};
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

// ================================================================================================
// Training data and whole-volume inference.
// ================================================================================================
namespace {

constexpr int kPatch = kSide[0], kPatch3 = kPatch * kPatch * kPatch, kHalo = kPatch / 2;
constexpr int kEllipsoids = 10;  // parameter slots per volume
constexpr float kAir = 0.0012f;

__device__ __forceinline__ uint32_t hash32(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return (uint32_t)x;
}
__device__ __forceinline__ float unit(uint64_t key) { return (hash32(key) >> 8) * (1.0f / 16777216.0f); }

// Volume v: air, then up to 10 ellipsoids (cx, cy, cz, rx, ry, rz [voxels], density, used) painted
// in order, then Gaussian multiplicative jitter of relative spread `jitter` (Box-Muller on a hash
// of the voxel).
__global__ void paint_kernel(float* rho, int n, const float* ell, int n_vol, uint64_t seed, float jitter) {
    const size_t per = (size_t)n * n * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < per * n_vol; i += (size_t)gridDim.x * blockDim.x) {
        const int v = (int)(i / per);
        const int j = (int)(i % per);
        const float x = j % n, y = (j / n) % n, z = j / (n * n);
        float r = kAir;
        const float* e = ell + (size_t)v * kEllipsoids * 8;
        for (int k = 0; k < kEllipsoids; ++k, e += 8) {
            if (e[7] == 0.0f) continue;
            const float dx = (x - e[0]) / e[3], dy = (y - e[1]) / e[4], dz = (z - e[2]) / e[5];
            if (dx * dx + dy * dy + dz * dz <= 1.0f) r = e[6];
        }
        const float u1 = fmaxf(unit(seed * 0x9E3779B97F4A7C15ULL + 2 * i), 1e-7f), u2 = unit(seed * 0x9E3779B97F4A7C15ULL + 2 * i + 1);
        const float g = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
        rho[i] = fmaxf(r * (1.0f + jitter * g), prc::kMinDensity);
    }
}

// Sample i of volume v: a hashed random voxel, re-drawn (at most 64 times) until it is tissue.
__global__ void pick_kernel(const float* rho, int n, int n_vol, int per_vol, float support_rho, uint64_t seed,
                            int* src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_vol * per_vol) return;
    const int v = i / per_vol;
    const int n3 = n * n * n;
    int pick = 0;
    for (int t = 0; t < 64; ++t) {
        pick = (int)(hash32(seed * 1315423911ULL + (uint64_t)i * 64 + t) % (uint32_t)n3);
        if (rho[(size_t)v * n3 + pick] >= support_rho) break;
    }
    src[i] = pick;
}

// The input channels of one voxel: density / 2 (air beyond the volume), 1 inside the volume and 0
// beyond it (a ray stops at the volume's edge but runs on through air inside it), the one-hot
// isotope, and three zeros (8 channels: one 16-byte row per tap for the tensor-core loader).
__device__ __forceinline__ void write_input(bf16* o, float r, bool inside, int iso) {
    o[0] = __float2bfloat16_rn(0.5f * r);
    o[1] = __float2bfloat16_rn(inside ? 1.0f : 0.0f);
    for (int c = 0; c < 3; ++c) o[2 + c] = __float2bfloat16_rn(c == iso ? 1.0f : 0.0f);
    for (int c = 5; c < kIn; ++c) o[c] = __float2bfloat16_rn(0.0f);
}

// Patch of sample i (channels of write_input).
__global__ void patch_kernel(const float* rho, int n, int per_vol, const int* src, int n_src, int iso, bf16* out) {
    const size_t total = (size_t)n_src * kPatch3;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int smp = (int)(i / kPatch3), q = (int)(i % kPatch3);
        const int v = smp / per_vol, s = src[smp];
        const int x = s % n + q % kPatch - kHalo, y = (s / n) % n + (q / kPatch) % kPatch - kHalo,
                  z = s / (n * n) + q / (kPatch * kPatch) - kHalo;
        const bool in = (unsigned)x < (unsigned)n && (unsigned)y < (unsigned)n && (unsigned)z < (unsigned)n;
        const float r = in ? rho[(size_t)v * n * n * n + ((size_t)z * n + y) * n + x] : kAir;
        write_input(out + i * kIn, r, in, iso);
    }
}

__global__ void scale_kernel(float* x, size_t n, float s) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] *= s;
}

// Marks (-1) the targets a surrogate field never takes from the network: the bins past the
// water range, and every bin of a ray with more than `beyond` of its mass past it (the tracer's
// judge keeps such rays exact).  One thread per (sample, ray) of 16 bins.
__global__ void mask_targets_kernel(float* t, size_t n_rays_total, int water_bins, float beyond) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_rays_total; i += (size_t)gridDim.x * blockDim.x) {
        float* r = t + i * 16;
        float mass = 0.0f, far = 0.0f;
        for (int b = 0; b < 16; ++b) {
            mass += r[b];
            far += b >= water_bins ? r[b] : 0.0f;
        }
        const bool drop = far > beyond * mass;
        for (int b = 0; b < 16; ++b)
            if (drop || b >= water_bins) r[b] = -1.0f;
    }
}

// Whole-volume inference.  The input lives on the volume padded by kHalo voxels of air on every
// side; every layer is a 'same' dilated 3x3x3 convolution on that padded grid (zero beyond it),
// which equals the valid convolutions of training on the 21^3 patch of every voxel of the volume
// (the halo is the sum of the dilations, so no tap of a volume voxel's cone reaches the zeros).
struct ConvSame {
    const bf16* x;
    const bf16* w;
    const float* bias;
    bf16* out;
    int pz, py, px, cin, d;
    __device__ bf16 a(int m, int k) const {
        int z, y, x0, kz, ky, kx;
        z = m / (py * px);
        y = (m / px) % py;
        x0 = m % px;
        decode3(k / cin, 3, kz, ky, kx);
        const int zz = z + (kz - 1) * d, yy = y + (ky - 1) * d, xx = x0 + (kx - 1) * d;
        if ((unsigned)zz >= (unsigned)pz || (unsigned)yy >= (unsigned)py || (unsigned)xx >= (unsigned)px)
            return __float2bfloat16(0.0f);
        return x[(((size_t)zz * py + yy) * px + xx) * cin + k % cin];
    }
    __device__ bool vec_a() const { return cin % 8 == 0; }
    __device__ uint4 a8(int m, int k) const {
        const int z = m / (py * px), y = (m / px) % py, x0 = m % px;
        int kz, ky, kx;
        decode3(k / cin, 3, kz, ky, kx);
        const int zz = z + (kz - 1) * d, yy = y + (ky - 1) * d, xx = x0 + (kx - 1) * d;
        if ((unsigned)zz >= (unsigned)pz || (unsigned)yy >= (unsigned)py || (unsigned)xx >= (unsigned)px)
            return make_uint4(0u, 0u, 0u, 0u);
        return *reinterpret_cast<const uint4*>(x + (((size_t)zz * py + yy) * px + xx) * cin + k % cin);
    }
    __device__ bf16 b(int n, int k) const { return w[(size_t)n * 27 * cin + k]; }
    __device__ void store(int m, int n, float v) const {
        out[(size_t)m * kC + n] = __float2bfloat16_rn(fmaxf(v + bias[n], 0.0f));
    }
};

// Head on the tissue voxels: coef[src][n] = bf16(max(scale * (a4 . wh[n] + bh[n]), 0)).
struct HeadActive {
    const bf16* a4;
    const int* active;
    const bf16* wh;
    const float* bh;
    bf16* coef;
    int nx, ny, py, px;
    float scale;
    __device__ bf16 a(int m, int k) const {
        const int s = active[m];
        const int x = s % nx + kHalo, y = (s / nx) % ny + kHalo, z = s / (nx * ny) + kHalo;
        return a4[(((size_t)z * py + y) * px + x) * kC + k];
    }
    __device__ bool vec_a() const { return true; }
    __device__ uint4 a8(int m, int k) const {
        const int s = active[m];
        const int x = s % nx + kHalo, y = (s / nx) % ny + kHalo, z = s / (nx * ny) + kHalo;
        return *reinterpret_cast<const uint4*>(a4 + (((size_t)z * py + y) * px + x) * kC + k);
    }
    __device__ bf16 b(int n, int k) const { return wh[(size_t)n * kC + k]; }
    __device__ void store(int m, int n, float v) const {
        coef[(size_t)m * kOut + n] = __float2bfloat16_rn(fmaxf(scale * (v + bh[n]), 0.0f));
    }
};

__global__ void padded_input_kernel(const float* rho, int nx, int ny, int nz, int iso, bf16* out) {
    const int px = nx + 2 * kHalo, py = ny + 2 * kHalo, pz = nz + 2 * kHalo;
    const size_t total = (size_t)px * py * pz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % px) - kHalo, y = (int)((i / px) % py) - kHalo, z = (int)(i / ((size_t)px * py)) - kHalo;
        const bool in = (unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz;
        const float r = in ? rho[((size_t)z * ny + y) * nx + x] : kAir;
        write_input(out + i * kIn, r, in, iso);
    }
}

// Judge (see surrogate_judge in engine.h); one warp per source, a half-warp per far ray (the 16
// radial bins of a ray are one lane each).
__global__ void judge_kernel(bf16* coef, const float* traced, int n_src, int n_rays, int first, float threshold,
                             float beyond, int water_bins, const int* active, const int* bin_xyz, int nx, int ny,
                             int nz, unsigned char* flags) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n_src) return;
    const int s = active[first + warp];
    const int vx = s % nx, vy = (s / nx) % ny, vz = s / (nx * ny);
    const size_t per_src = (size_t)n_rays * 16;
    bf16* c = coef + (size_t)(first + warp) * per_src;
    const float* t = traced + (size_t)warp * per_src;
    unsigned char* f = flags + (size_t)(first + warp) * n_rays;
    const int bin = lane & 15;
    float ray_energy = 0.0f;  // mean over the source's rays of the traced squared norm
    for (int k = lane; k < n_rays * 16; k += 32) ray_energy += t[k] * t[k];
    for (int off = 16; off > 0; off >>= 1) ray_energy += __shfl_xor_sync(0xffffffffu, ray_energy, off);
    ray_energy /= n_rays;
    for (int r0 = 0; r0 < n_rays; r0 += 2) {
        const int r = r0 + (lane >> 4), k = r * 16 + bin;
        const bool ray = r < n_rays;  // the second half-warp idles on an odd last ray
        const float tv = ray ? t[k] : 0.0f;
        float err = 0.0f;
        if (ray && threshold >= 0.0f) {
            const float d = bin < water_bins ? __bfloat162float(c[k]) - tv : -tv;  // what the field stores
            err = d * d;
        } else if (ray) {
            c[k] = __float2bfloat16_rn(tv);
        }
        float mass = tv, far = bin >= water_bins ? tv : 0.0f;
        for (int off = 8; off > 0; off >>= 1) {  // within the half-warp of this ray
            err += __shfl_xor_sync(0xffffffffu, err, off);
            mass += __shfl_xor_sync(0xffffffffu, mass, off);
            far += __shfl_xor_sync(0xffffffffu, far, off);
        }
        // a ray cut by the volume's edge inside the water range (the voxel of its last water bin
        // lies outside; the volume is convex, so the earlier bins lie inside): a truncated kernel
        bool cut = false;
        if (ray) {
            const int xyz = bin_xyz[r * 16 + water_bins - 1];
            const int x = vx + (xyz & 1023) - 512, y = vy + ((xyz >> 10) & 1023) - 512, z = vz + ((xyz >> 20) & 1023) - 512;
            cut = (unsigned)x >= (unsigned)nx || (unsigned)y >= (unsigned)ny || (unsigned)z >= (unsigned)nz;
        }
        const bool bad = (threshold >= 0.0f && (cut || err > threshold * threshold * ray_energy)) || far > beyond * mass;
        if (ray && bin == 0) f[r] = bad ? 1 : 0;
    }
}

}  // namespace

namespace prc {

// Whole-volume inference of `net` on the clamped density rho (device, nx*ny*nz) for isotope
// index iso; coef[src][2048] for the sources of `active` (device), scaled back by 1 / target
// scale.  Scratch: two padded activation volumes (allocated and freed here).
int surrogate_infer(prc_net* net, const float* rho, int nx, int ny, int nz, int iso, const int* active, int n_active,
                    float inv_target_scale, bf16* coef, cudaStream_t s) {
    const int px = nx + 2 * kHalo, py = ny + 2 * kHalo, pz = nz + 2 * kHalo;
    const size_t pv = (size_t)px * py * pz;
    bf16 *buf0 = nullptr, *buf1 = nullptr;
    NN_CUDA(cudaMalloc(&buf0, pv * kC * sizeof(bf16)), "surrogate inference");
    cudaError_t e = cudaMalloc(&buf1, pv * kC * sizeof(bf16));
    if (e != cudaSuccess) {
        cudaFree(buf0);
        return nn_fail(e, "surrogate inference");
    }
    struct Free {
        bf16* a;
        bf16* b;
        ~Free() {
            cudaFree(a);
            cudaFree(b);
        }
    } free_bufs{buf0, buf1};
    padded_input_kernel<<<1024, 256, 0, s>>>(rho, nx, ny, nz, iso, buf0);
    bf16* in = buf0;
    bf16* out = buf1;
    for (int l = 0; l < 4; ++l) {
        const int cin = l == 0 ? kIn : kC;
        ConvSame c{in, net->wb[l], net->b[l], out, pz, py, px, cin, kDil[l]};
        NN_CUDA((run_problem<32>(c, (int)pv, kC, 27 * cin, 1, net->error, s)), "surrogate inference");
        bf16* t = in;
        in = out;
        out = t;
    }
    HeadActive h{in, active, net->wb[4], net->b[4], coef, nx, ny, py, px, inv_target_scale};
    NN_CUDA((run_problem<256>(h, n_active, kOut, kC, 1, net->error, s)), "surrogate inference");
    NN_CUDA(cudaStreamSynchronize(s), "surrogate inference");
    unsigned int err = 0;
    NN_CUDA(cudaMemcpy(&err, net->error, sizeof(err), cudaMemcpyDeviceToHost), "surrogate inference");
    if (err) return prc::set_last_error("a tensor-core MMA wait gave up"), PRC_ERR_CUDA;
    return PRC_OK;
}

cudaError_t surrogate_judge(bf16* coef, const float* traced, int n_src, int n_rays, int first, float threshold,
                            float beyond, int water_bins, const int* active, const int* bin_xyz, int nx, int ny,
                            int nz, unsigned char* flags, cudaStream_t s) {
    judge_kernel<<<(n_src * 32 + 255) / 256, 256, 0, s>>>(coef, traced, n_src, n_rays, first, threshold, beyond,
                                                          water_bins, active, bin_xyz, nx, ny, nz, flags);
    return cudaGetLastError();
}

}  // namespace prc

extern "C" int prc_nn_make_samples(const char* isotope, int n_vol, int side, float spacing_mm, const float* ellipsoids,
                                   uint64_t seed, int per_vol, void* d_patches, float* d_targets, float target_scale,
                                   float jitter, void* stream) {
    using namespace prc;
    static const char* kIsos[3] = {"18F", "68Ga", "82Rb"};
    int iso = -1;
    for (int i = 0; i < 3; ++i)
        if (isotope && std::string(isotope) == kIsos[i]) iso = i;
    if (iso < 0 || n_vol <= 0 || side < 8 || per_vol <= 0 || per_vol % kLanes || !ellipsoids || !d_patches ||
        !d_targets || !(spacing_mm > 0) || !(jitter >= 0.0f && jitter <= 0.5f))
        return set_last_error("Invalid argument: isotope must be 18F, 68Ga or 82Rb; per_vol a multiple of 32; "
                              "jitter in [0, 0.5]"),
               PRC_ERR_ARGUMENT;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    RangeModel model;
    model.resolve(kIsos[iso]);
    Grid g{side, side, side, spacing_mm, spacing_mm, spacing_mm, model.cutoff, 0.05f, 50.0f};
    const int n_rays = 128;
    const int tmpl_len = ((3 * side + 6) / 4) * 4;
    const size_t n3 = (size_t)side * side * side;
    std::vector<void*> allocs;
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return (void*)nullptr;
        allocs.push_back(p);
        return p;
    };
    struct FreeAll {
        std::vector<void*>& v;
        ~FreeAll() {
            for (void* p : v) cudaFree(p);
        }
    } free_all{allocs};
    float* rho = (float*)alloc(n3 * n_vol * sizeof(float));
    float* ell = (float*)alloc((size_t)n_vol * kEllipsoids * 8 * sizeof(float));
    int* src = (int*)alloc((size_t)n_vol * per_vol * sizeof(int));
    RayStep* far = (RayStep*)alloc(n_rays * sizeof(RayStep));
    RayStep* near = (RayStep*)alloc(kNearRays * sizeof(RayStep));
    float* table = (float*)alloc((kRangeBins + 1) * sizeof(float));
    RadialTables tab;
    tab.bin_of = (unsigned char*)alloc((size_t)n_rays * tmpl_len);
    tab.offset = (int*)alloc(n_rays * kRadialBins * sizeof(int));
    tab.xyz = (int*)alloc(n_rays * kRadialBins * sizeof(int));
    for (void* p : allocs)
        if (!p) return set_last_error("Device allocation failed in prc_nn_make_samples"), PRC_ERR_MEMORY;
    if (allocs.size() != 9) return set_last_error("Device allocation failed in prc_nn_make_samples"), PRC_ERR_MEMORY;
    const std::vector<float> t = model.table();
    NN_CUDA(cudaMemcpyAsync(table, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, s), "make_samples");
    NN_CUDA(cudaMemcpyAsync(ell, ellipsoids, (size_t)n_vol * kEllipsoids * 8 * sizeof(float), cudaMemcpyHostToDevice, s),
            "make_samples");
    NN_CUDA(setup_rays(g, n_rays, far, near, s), "make_samples");
    ProjParams p{};
    p.g = g;
    p.nxy = side * side;
    p.n_rays = n_rays;
    p.rho = rho;
    p.far = far;
    p.near = near;
    p.table = table;
    p.table_scale = model.table_scale();
    p.n_branch = model.n;
    for (int b = 0; b < 3; ++b) p.br[b] = model.br[b];
    p.tmpl_len = tmpl_len;
    NN_CUDA(build_radial_tables(p, tab, s), "make_samples");
    paint_kernel<<<2048, 256, 0, s>>>(rho, side, ell, n_vol, seed, jitter);
    pick_kernel<<<(n_vol * per_vol + 255) / 256, 256, 0, s>>>(rho, side, n_vol, per_vol, g.support_rho, seed, src);
    NN_CUDA(radial_kernels(p, tab, src, n_vol * per_vol, per_vol / kLanes, d_targets, s), "make_samples");
    scale_kernel<<<1024, 256, 0, s>>>(d_targets, (size_t)n_vol * per_vol * kOut, target_scale);
    mask_targets_kernel<<<1024, 256, 0, s>>>(d_targets, (size_t)n_vol * per_vol * (kOut / 16), radial_water_bins(),
                                             kBeyondShare);
    patch_kernel<<<2048, 256, 0, s>>>(rho, side, per_vol, src, n_vol * per_vol, iso, static_cast<bf16*>(d_patches));
    NN_CUDA(cudaGetLastError(), "make_samples");
    NN_CUDA(cudaStreamSynchronize(s), "make_samples");
    return PRC_OK;
}

