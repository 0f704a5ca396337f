// metrics.cu -- reference-based image-quality metrics of a reconstruction, on the device.
//
// The reference scores corrected images against a known truth with tools/evaluate.py
// (Evaluator.__call__, tools/evaluate.py:105-154): global and tissue NRMSE, MSE, MAE, count
// bias, PSNR over the dilated-body box, 3D SSIM (Gaussian window, sigma 1.5, 11 voxels),
// recovery coefficients of hot regions, background bias and CoV, local-range (ringing)
// violations on the edge band, and the halo around hot regions.  The masks those metrics use
// are fixed by the truth alone, so they are built once (prc_eval_create); every scored image
// then costs one pass for the FP64 sums below plus three separable filter passes for SSIM.
// The host turns the sums into the reference's metric values.
#include "../../include/prc_metrics.h"
#include "engine.h"

#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <string>
#include <vector>

struct prc_eval {
    int nz = 0, ny = 0, nx = 0;
    size_t n = 0;
    int n_labels = 0;
    int roi[6] = {};  // z0, z1, y0, y1, x0, x1
    double data_range = 0.0;
    double* t = nullptr;
    unsigned char* cls = nullptr;
    int* label = nullptr;
    double* lo = nullptr;
    double* hi = nullptr;
    double* sums = nullptr;
    double* fields = nullptr;  // 2 x 5 filtered volumes over the ROI box (SSIM)
    std::vector<void*> allocations;
    ~prc_eval() {
        for (void* p : allocations) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T** p, size_t count) {
        void* v = nullptr;
        const cudaError_t e = cudaMalloc(&v, count * sizeof(T) > 0 ? count * sizeof(T) : 1);
        if (e != cudaSuccess) return e;
        allocations.push_back(v);
        *p = static_cast<T*>(v);
        return cudaSuccess;
    }
};

namespace {

constexpr int kThreads = 256;
constexpr int kRadius = 5;  // int(3.5 * 1.5 + 0.5): the 11-voxel Gaussian window
constexpr double kSigma = 1.5;

__constant__ double c_gauss[2 * kRadius + 1];

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-reduces NV per-thread partials and adds them to out[0..NV).
template <int NV>
__device__ void block_add(double (&v)[NV], double* out) {
    __shared__ double part[kThreads / 32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double s = warp_sum(v[i]);
        if (lane == 0) part[warp][i] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += part[w][threadIdx.x];
        atomicAdd(out + threadIdx.x, s);
    }
}

// One pass over the volume: every sum that is not SSIM (PRC_EVAL_* indices).
template <typename TF>
__global__ void __launch_bounds__(kThreads) sums_kernel(const TF* __restrict__ f, const double* __restrict__ t,
                                                         const unsigned char* __restrict__ cls,
                                                         const int* __restrict__ label, const double* __restrict__ lo,
                                                         const double* __restrict__ hi, size_t n, double* out) {
    double v[PRC_EVAL_SSIM_SUM] = {};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double fi = f[i], ti = t[i];
        if (!isfinite(fi)) {
            v[PRC_EVAL_NONFINITE] += 1.0;
            continue;
        }
        const unsigned c = cls[i];
        const double d = fi - ti, d2 = d * d, t2 = ti * ti;
        v[PRC_EVAL_D2] += d2;
        v[PRC_EVAL_T2] += t2;
        v[PRC_EVAL_F] += fi;
        v[PRC_EVAL_T] += ti;
        if (c & PRC_CLASS_BODY) {
            v[PRC_EVAL_D2_BODY] += d2;
            v[PRC_EVAL_T2_BODY] += t2;
            v[PRC_EVAL_ABS_BODY] += fabs(d);
            v[PRC_EVAL_N_BODY] += 1.0;
        }
        if (c & PRC_CLASS_ROI) {
            v[PRC_EVAL_D2_ROI] += d2;
            v[PRC_EVAL_N_ROI] += 1.0;
        }
        if (c & PRC_CLASS_HOT) {
            v[PRC_EVAL_F_HOT] += fi;
            v[PRC_EVAL_T_HOT] += ti;
            const int l = label[i];
            if (l > 0) {
                atomicAdd(out + PRC_EVAL_NUM_SUMS + 2 * (l - 1), fi);
                atomicAdd(out + PRC_EVAL_NUM_SUMS + 2 * (l - 1) + 1, ti);
            }
        }
        if (c & PRC_CLASS_BACKGROUND) {
            v[PRC_EVAL_F_BG] += fi;
            v[PRC_EVAL_F2_BG] += fi * fi;
            v[PRC_EVAL_N_BG] += 1.0;
        }
        if (c & PRC_CLASS_EDGE) {
            const double over = fmax(fi - hi[i], 0.0), under = fmax(lo[i] - fi, 0.0);
            v[PRC_EVAL_RING2] += (over + under) * (over + under);
            v[PRC_EVAL_OVER2] += over * over;
            v[PRC_EVAL_UNDER2] += under * under;
            v[PRC_EVAL_N_EDGE] += 1.0;
            v[PRC_EVAL_D2_EDGE] += d2;
            v[PRC_EVAL_T2_EDGE] += t2;
        }
        if (c & PRC_CLASS_HALO) {
            v[PRC_EVAL_F_HALO] += fi;
            v[PRC_EVAL_N_HALO] += 1.0;
        }
    }
    block_add<PRC_EVAL_SSIM_SUM>(v, out);
}

// Half-sample symmetric extension ("reflect": d c b a | a b c d | d c b a), n > kRadius.
__device__ __forceinline__ int reflect(int i, int n) {
    if (i < 0) return -i - 1;
    if (i >= n) return 2 * n - i - 1;
    return i;
}

struct Box {
    int z0, y0, x0, cz, cy, cx, nx, nxy;
    __device__ size_t vol(int z, int y, int x) const { return ((size_t)(z0 + z) * (size_t)nxy) + (size_t)(y0 + y) * nx + (x0 + x); }
    __device__ size_t box(int z, int y, int x) const { return ((size_t)z * cy + y) * cx + x; }
    __device__ size_t size() const { return (size_t)cz * cy * cx; }
};

// SSIM pass 1 (x axis): the five fields t, f, t*t, f*f, t*f of the box, filtered along x.
template <typename TF>
__global__ void ssim_x_kernel(const TF* __restrict__ f, const double* __restrict__ t, Box b, double* out) {
    const size_t m = b.size();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % b.cx), y = (int)(i / b.cx % b.cy), z = (int)(i / ((size_t)b.cx * b.cy));
        double a[5] = {};
        for (int k = -kRadius; k <= kRadius; ++k) {
            const size_t j = b.vol(z, y, reflect(x + k, b.cx));
            const double tv = t[j], fv = (double)f[j], w = c_gauss[k + kRadius];
            a[0] += w * tv, a[1] += w * fv, a[2] += w * (tv * tv), a[3] += w * (fv * fv), a[4] += w * (tv * fv);
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) out[q * m + i] = a[q];
    }
}

// SSIM pass 2 (y axis) on the five fields.
__global__ void ssim_y_kernel(const double* __restrict__ in, Box b, double* __restrict__ out) {
    const size_t m = b.size();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 5 * m; i += (size_t)gridDim.x * blockDim.x) {
        const size_t q = i / m, r = i % m;
        const int x = (int)(r % b.cx), y = (int)(r / b.cx % b.cy), z = (int)(r / ((size_t)b.cx * b.cy));
        double a = 0.0;
        for (int k = -kRadius; k <= kRadius; ++k) a += c_gauss[k + kRadius] * in[q * m + b.box(z, reflect(y + k, b.cy), x)];
        out[i] = a;
    }
}

// SSIM pass 3 (z axis), the SSIM map (Wang et al. 2004, Gaussian window, population
// covariances) and its sums over the valid interior (kRadius from every face of the box):
// all voxels, tissue voxels and edge-band voxels.
__global__ void __launch_bounds__(kThreads) ssim_z_kernel(const double* __restrict__ in, Box b,
                                                           const unsigned char* __restrict__ cls, double c1, double c2,
                                                           double* sums) {
    const size_t m = b.size();
    double v[6] = {};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % b.cx), y = (int)(i / b.cx % b.cy), z = (int)(i / ((size_t)b.cx * b.cy));
        if (x < kRadius || y < kRadius || z < kRadius || x >= b.cx - kRadius || y >= b.cy - kRadius ||
            z >= b.cz - kRadius)
            continue;
        double a[5] = {};
        for (int k = -kRadius; k <= kRadius; ++k) {
            const size_t j = b.box(z + k, y, x);  // interior: no extension needed along z
            const double w = c_gauss[k + kRadius];
#pragma unroll
            for (int q = 0; q < 5; ++q) a[q] += w * in[q * m + j];
        }
        const double ux = a[0], uy = a[1];
        const double vx = a[2] - ux * ux, vy = a[3] - uy * uy, vxy = a[4] - ux * uy;
        const double s = ((2.0 * ux * uy + c1) * (2.0 * vxy + c2)) / ((ux * ux + uy * uy + c1) * (vx + vy + c2));
        const unsigned c = cls[b.vol(z, y, x)];
        v[0] += s, v[1] += 1.0;
        if (c & PRC_CLASS_BODY) v[2] += s, v[3] += 1.0;
        if (c & PRC_CLASS_EDGE) v[4] += s, v[5] += 1.0;
    }
    block_add<6>(v, sums + PRC_EVAL_SSIM_SUM);
}

int fail(int code, const std::string& msg) {
    prc::set_last_error(msg);
    return code;
}

#define EVAL_CUDA(call)                                                                                  \
    do {                                                                                                 \
        const cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(PRC_ERR_CUDA, std::string("CUDA error '") + cudaGetErrorString(e_) + "' in " #call); \
    } while (0)

}  // namespace

extern "C" {

int prc_eval_create(int nz, int ny, int nx, const double* truth, const unsigned char* classes, const int* labels,
                    int n_labels, const double* lo, const double* hi, const int* roi, double data_range,
                    prc_eval** out) {
    if (!out) return fail(PRC_ERR_ARGUMENT, "Invalid argument: null evaluator pointer");
    *out = nullptr;
    if (nz <= 0 || ny <= 0 || nx <= 0 || !truth || !classes || !lo || !hi || !roi || n_labels < 0 ||
        (n_labels > 0 && !labels) || !(data_range > 0) || !std::isfinite(data_range))
        return fail(PRC_ERR_ARGUMENT, "Invalid evaluator arguments");
    if ((size_t)nx * ny > (size_t)INT_MAX || (size_t)nx * ny * nz > ((size_t)1 << 40))
        return fail(PRC_ERR_LIMIT, "Volume too large for the evaluator");
    if (roi[0] < 0 || roi[1] > nz || roi[0] >= roi[1] || roi[2] < 0 || roi[3] > ny || roi[2] >= roi[3] || roi[4] < 0 ||
        roi[5] > nx || roi[4] >= roi[5])
        return fail(PRC_ERR_ARGUMENT, "Invalid evaluator ROI box");
    prc_eval* e = new prc_eval();
    e->nz = nz, e->ny = ny, e->nx = nx;
    e->n = (size_t)nz * ny * nx;
    e->n_labels = n_labels;
    for (int i = 0; i < 6; ++i) e->roi[i] = roi[i];
    e->data_range = data_range;
    auto bail = [&](cudaError_t err, const char* what) {
        delete e;
        return fail(PRC_ERR_CUDA, std::string("CUDA error '") + cudaGetErrorString(err) + "' in " + what);
    };
    cudaError_t err;
    if ((err = e->alloc(&e->t, e->n)) != cudaSuccess) return bail(err, "prc_eval_create");
    if ((err = e->alloc(&e->cls, e->n)) != cudaSuccess) return bail(err, "prc_eval_create");
    if ((err = e->alloc(&e->label, n_labels ? e->n : 1)) != cudaSuccess) return bail(err, "prc_eval_create");
    if ((err = e->alloc(&e->lo, e->n)) != cudaSuccess) return bail(err, "prc_eval_create");
    if ((err = e->alloc(&e->hi, e->n)) != cudaSuccess) return bail(err, "prc_eval_create");
    if ((err = e->alloc(&e->sums, (size_t)PRC_EVAL_NUM_SUMS + 2 * (size_t)n_labels)) != cudaSuccess)
        return bail(err, "prc_eval_create");
    const size_t box = (size_t)(roi[1] - roi[0]) * (roi[3] - roi[2]) * (roi[5] - roi[4]);
    if ((err = e->alloc(&e->fields, 10 * box)) != cudaSuccess) return bail(err, "prc_eval_create");
    if ((err = cudaMemcpy(e->t, truth, e->n * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemcpy(e->cls, classes, e->n, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (n_labels && (err = cudaMemcpy(e->label, labels, e->n * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) ||
        (err = cudaMemcpy(e->lo, lo, e->n * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (err = cudaMemcpy(e->hi, hi, e->n * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(err, "prc_eval_create");
    // Gaussian window of scipy.ndimage.gaussian_filter1d (sigma 1.5, truncate 3.5), normalised.
    double g[2 * kRadius + 1], total = 0.0;
    for (int k = -kRadius; k <= kRadius; ++k) total += g[k + kRadius] = std::exp(-0.5 / (kSigma * kSigma) * k * k);
    for (double& w : g) w /= total;
    if ((err = cudaMemcpyToSymbol(c_gauss, g, sizeof(g))) != cudaSuccess) return bail(err, "prc_eval_create");
    *out = e;
    return PRC_OK;
}

}  // extern "C"

template <typename TF>
static int eval_sums(prc_eval* e, const TF* d_f, double* sums, void* stream) {
    if (!e || !d_f || !sums) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n_sums = (size_t)PRC_EVAL_NUM_SUMS + 2 * (size_t)e->n_labels;
    EVAL_CUDA(cudaMemsetAsync(e->sums, 0, n_sums * sizeof(double), s));
    sums_kernel<TF><<<592, kThreads, 0, s>>>(d_f, e->t, e->cls, e->label, e->lo, e->hi, e->n, e->sums);
    EVAL_CUDA(cudaGetLastError());
    const Box b{e->roi[0], e->roi[2], e->roi[4], e->roi[1] - e->roi[0], e->roi[3] - e->roi[2], e->roi[5] - e->roi[4],
                e->nx, e->nx * e->ny};
    if (b.cz >= 2 * kRadius + 1 && b.cy >= 2 * kRadius + 1 && b.cx >= 2 * kRadius + 1) {  // tools/evaluate.py:124
        const size_t m = (size_t)b.cz * b.cy * b.cx;
        const double c1 = (0.01 * e->data_range) * (0.01 * e->data_range);
        const double c2 = (0.03 * e->data_range) * (0.03 * e->data_range);
        ssim_x_kernel<TF><<<592, kThreads, 0, s>>>(d_f, e->t, b, e->fields);
        ssim_y_kernel<<<592, kThreads, 0, s>>>(e->fields, b, e->fields + 5 * m);
        ssim_z_kernel<<<592, kThreads, 0, s>>>(e->fields + 5 * m, b, e->cls, c1, c2, e->sums);
        EVAL_CUDA(cudaGetLastError());
    }
    EVAL_CUDA(cudaMemcpyAsync(sums, e->sums, n_sums * sizeof(double), cudaMemcpyDeviceToHost, s));
    EVAL_CUDA(cudaStreamSynchronize(s));
    return PRC_OK;
}

extern "C" {

int prc_eval_sums(prc_eval* e, const float* d_f, double* sums, void* stream) { return eval_sums(e, d_f, sums, stream); }

int prc_eval_sums_f64(prc_eval* e, const double* d_f, double* sums, void* stream) {
    return eval_sums(e, d_f, sums, stream);
}

void prc_eval_destroy(prc_eval* e) { delete e; }

}  // extern "C"
