// em.cu -- the MAP-EM image-update chain around the projector (prc.cu:269-332, 659-700).
//
// Every kernel is a grid-stride pass over the volume with a fixed grid of kReduceBlocks blocks.
// The three scalars that the reference reads back to the host every iteration (the count sum
// for the rescale and the two Biggs-Andrews inner products, prc.cu:689, 695-696) are reduced
// on the device in FP64 instead: each block writes its partial, and the last block to finish
// combines the partials in block order (deterministic) and writes the derived scalar (scale,
// lambda) into EmScalars, where the next kernel reads it.  So an iteration enqueues without a
// single host synchronisation.
#include "engine.h"

#include <algorithm>

namespace prc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = kEmThreads / 32;

// Grid-wide FP64 reduction of NV values.  Must be reached by every thread of every block.
// The last block calls fin(totals) from thread 0 and re-arms the counter for the next launch.
template <int NV, class Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[NV], const Reduction& r, Fin&& fin) {
    __shared__ double sh[NV][kWarpsPerBlock];
    __shared__ bool am_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(kFull, v[k], off);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
            for (int w = 0; w < kWarpsPerBlock; ++w) t += sh[k][w];
            r.partials[blockIdx.x * NV + k] = t;
        }
        __threadfence();
        am_last = atomicAdd(r.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(r.partials + b * NV + k);
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) acc[k] += __shfl_xor_sync(kFull, acc[k], off);
    __syncthreads();  // sh is reused below
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = acc[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            tot[k] = 0.0;
            for (int w = 0; w < kWarpsPerBlock; ++w) tot[k] += sh[k][w];
        }
        fin(tot);
        *r.counter = 0u;
    }
}

#define GRID_STRIDE(i, n) \
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

// The streaming passes move 16 bytes per access: element 4q + c of a volume is component c of
// float4 q.  They take that path when every pointer they touch is 16-byte aligned (allocations
// are; a caller's offset pointer may not be) and finish the last n % 4 elements one at a time.
// Each element is computed by the same expression on both paths.
#define TAIL_STRIDE(i, start, n)                                                                 \
    for (size_t i = (start) + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n);          \
         i += (size_t)gridDim.x * blockDim.x)

__device__ __forceinline__ bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// g = support ? max(g_in, 0) : 0 (prc.cu:604-612); f = g; support_sum, eps and the floor.
__device__ __forceinline__ void begin_body(const float* __restrict__ g_in, const unsigned char* __restrict__ support,
                                           float* __restrict__ g, float* __restrict__ f, size_t n, int n_active,
                                           EmScalars* sc, Reduction r) {
    double v[1] = {0.0};
    GRID_STRIDE(i, n) {
        const float x = support[i] ? fmaxf(g_in[i], 0.0f) : 0.0f;
        g[i] = x;
        f[i] = x;
        v[0] += x;
    }
    grid_reduce<1>(v, r, [&](const double* t) {
        sc->support_sum = t[0];
        const float eps = (float)(1.0e-6 * t[0] / n_active);  // prc.cu:668
        sc->eps = eps;
        sc->floor = 1000.0f * eps;  // prc.cu:670
        sc->lambda = 0.0f;
        sc->scale = 1.0f;
    });
}

// initialize_kernel (prc.cu:311-314) fused with the FP64 sum that sets the initial rescale.
__device__ __forceinline__ void floor_body(float* __restrict__ f, const unsigned char* __restrict__ support, size_t n,
                                           EmScalars* sc, Reduction r) {
    const float fl = sc->floor;
    double v[1] = {0.0};
    GRID_STRIDE(i, n) {
        float x = f[i];
        if (support[i]) x = fmaxf(x, fl);
        f[i] = x;
        v[0] += x;
    }
    grid_reduce<1>(v, r, [&](const double* t) { sc->init_scale = (float)(sc->support_sum / t[0]); });
}

// finish_kernel without a residual (prc.cu:325-332, called at prc.cu:671).
__device__ __forceinline__ void init_scale_body(float* __restrict__ f, size_t n, const EmScalars* sc) {
    const float scale = sc->init_scale;
    GRID_STRIDE(i, n) f[i] = __fmul_rn(f[i], scale);
}

// Biggs-Andrews prediction, kept above f/2 (prc.cu:318-321).
__device__ __forceinline__ void extrapolate_body(const float* __restrict__ f, const float* __restrict__ prev,
                                                 float* __restrict__ y, size_t n, const EmScalars* sc) {
    const float lambda = sc->lambda;
    auto predict = [lambda](float fi, float pi) { return fmaxf(fi + lambda * (fi - pi), 0.5f * fi); };
    const size_t n4 = aligned16(f) && aligned16(prev) && aligned16(y) ? n / 4 : 0;
    const float4* f4 = reinterpret_cast<const float4*>(f);
    const float4* p4 = reinterpret_cast<const float4*>(prev);
    float4* y4 = reinterpret_cast<float4*>(y);
    GRID_STRIDE(q, n4) {
        const float4 a = f4[q], b = p4[q];
        y4[q] = make_float4(predict(a.x, b.x), predict(a.y, b.y), predict(a.z, b.z), predict(a.w, b.w));
    }
    TAIL_STRIDE(i, 4 * n4, n) y[i] = predict(f[i], prev[i]);
}

// EM ratio g / max(A y, eps) on the support (prc.cu:270-274).
__device__ __forceinline__ void ratio_body(const float* __restrict__ g, float* __restrict__ est,
                                           const unsigned char* __restrict__ support, size_t n, const EmScalars* sc) {
    const float eps = sc->eps;
    auto ratio = [eps](unsigned char s, float gi, float ei) { return s ? gi / fmaxf(ei, eps) : 0.0f; };
    const size_t n4 = aligned16(g) && aligned16(est) && ((uintptr_t)support & 3u) == 0 ? n / 4 : 0;
    const float4* g4 = reinterpret_cast<const float4*>(g);
    const uchar4* s4 = reinterpret_cast<const uchar4*>(support);
    float4* e4 = reinterpret_cast<float4*>(est);
    GRID_STRIDE(q, n4) {
        const uchar4 m = s4[q];
        const float4 a = g4[q], e = e4[q];
        e4[q] = make_float4(ratio(m.x, a.x, e.x), ratio(m.y, a.y, e.y), ratio(m.z, a.z, e.z), ratio(m.w, a.w, e.w));
    }
    TAIL_STRIDE(i, 4 * n4, n) est[i] = ratio(support[i], g[i], est[i]);
}

__device__ __forceinline__ bool in_grid(const Grid& g, int i, int j, int k) {
    return i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz;
}

// RDP MAP-EM update over the 26 tissue neighbours (prc.cu:279-309), with the FP64 sum of the
// new estimate that drives the count rescale (prc.cu:688-691) when SUM is set.
template <bool SUM>
__device__ __forceinline__ void update_body(const float* __restrict__ f, const float* __restrict__ back,
                                            const unsigned char* __restrict__ support, float* __restrict__ next,
                                            const Grid& g, float beta, float gamma, EmScalars* sc, Reduction r) {
    const float eps = sc->eps;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    double v[1] = {0.0};
    GRID_STRIDE(idx, n) {
        float out;
        if (!support[idx]) {
            out = 0.0f;
        } else {
            const float fj = f[idx], f_em = fj * back[idx];
            if (beta == 0.0f) {
                out = fmaxf(f_em, 0.0f);
            } else {
                int i, j, k;
                if (n <= 0xffffffffull) {  // 32-bit division (the usual case)
                    const unsigned u = (unsigned)idx, row = u / (unsigned)g.nx;
                    i = (int)(u - row * (unsigned)g.nx);
                    j = (int)(row % (unsigned)g.ny);
                    k = (int)(row / (unsigned)g.ny);
                } else {
                    i = (int)(idx % g.nx);
                    j = (int)((idx / g.nx) % g.ny);
                    k = (int)(idx / ((size_t)g.nx * g.ny));
                }
                float grad = 0.0f, curv = 0.0f;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            if (!(dx | dy | dz) || !in_grid(g, i + dx, j + dy, k + dz)) continue;
                            const size_t nb = idx + ((long)dz * g.ny + dy) * g.nx + dx;
                            if (!support[nb]) continue;
                            const float mx = dx * g.sx, my = dy * g.sy, mz = dz * g.sz;
                            const float w = fminf(g.sx, fminf(g.sy, g.sz)) * rsqrtf(mx * mx + my * my + mz * mz);
                            const float fk = f[nb], d = fj - fk, ad = fabsf(d);
                            const float D = fj + fk + gamma * ad + eps, invD = 1.0f / D;
                            grad += w * d * (fj + 3.0f * fk + gamma * ad + 2.0f * eps) * invD * invD;
                            const float half_quad = (2.0f * (fj + fk + eps) + gamma * ad) * invD * invD;
                            const float hess = 2.0f * (2.0f * fk + eps) * (2.0f * fk + eps) * invD * invD * invD;
                            curv += 2.0f * w * fmaxf(half_quad, hess);
                        }
                // positive root of a x^2 + B x - f_em = 0, stable form for each sign of B
                const float a = beta * curv, B = 1.0f + beta * (grad - curv * fj);
                const float root = sqrtf(B * B + 4.0f * a * f_em);
                out = B >= 0.0f ? (f_em > 0.0f ? 2.0f * f_em / (B + root) : 0.0f) : (root - B) / (2.0f * a);
            }
        }
        next[idx] = out;
        if (SUM) v[0] += out;
    }
    if (SUM)
        grid_reduce<1>(v, r, [&](const double* t) {
            sc->sum = t[0];
            sc->scale = t[0] > 0.0 ? (float)(sc->support_sum / t[0]) : 1.0f;
        });
}

// Distance weight of neighbour offset (dx, dy, dz): min(dx, dy, dz) / |offset| with the
// reciprocal square root of prc.cu:293-296; computed once per run for the 26 offsets.
__global__ void geometry_weights_kernel(Grid g, float* geo_w) {
    const int q = threadIdx.x;
    if (q >= 27) return;
    const int dx = q % 3 - 1, dy = q / 3 % 3 - 1, dz = q / 9 - 1;
    const float mx = dx * g.sx, my = dy * g.sy, mz = dz * g.sz;
    geo_w[q] = (dx | dy | dz) ? fminf(g.sx, fminf(g.sy, g.sz)) * rsqrtf(mx * mx + my * my + mz * mz) : 0.0f;
}

// The RDP update of update_body, one thread per tissue voxel: threads walk the tissue list, so
// no lane idles on air, and the distance weights are read from geo_w (uniform across the warp)
// instead of being recomputed per neighbour.  An interior voxel (one voxel away from every
// face) reads its 26 neighbours at fixed linear offsets with no bounds tests; only voxels on
// the volume's faces test each neighbour.  Per neighbour the arithmetic is update_body's, in the
// same order, so the result is the same for every voxel.
template <bool SUM>
__device__ __forceinline__ void update_active_body(
    const float* __restrict__ f, const float* __restrict__ back, const unsigned char* __restrict__ support,
    float* __restrict__ next, const int* __restrict__ active, int n_active, const Grid& g, const float* __restrict__ geo_w,
    float beta, float gamma, EmScalars* sc, const Reduction& r) {
    __shared__ float w_sh[27];
    if (threadIdx.x < 27) w_sh[threadIdx.x] = geo_w[threadIdx.x];
    __syncthreads();
    const float eps = sc->eps;
    const int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
    double v[1] = {0.0};
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n_active; a += gridDim.x * blockDim.x) {
        const int idx = __ldg(active + a);
        const float fj = __ldg(f + idx), f_em = fj * __ldg(back + idx);
        float out;
        if (beta == 0.0f) {
            out = fmaxf(f_em, 0.0f);
        } else {
            const unsigned row = (unsigned)idx / (unsigned)nx;
            const int i = idx - (int)row * nx, j = (int)(row % (unsigned)ny), k = (int)(row / (unsigned)ny);
            const bool interior = i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k > 0 && k < nz - 1;
            float grad = 0.0f, curv = 0.0f;
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int dx = q % 3 - 1, dy = q / 3 % 3 - 1, dz = q / 9 - 1;
                if (q == 13) continue;  // the voxel itself
                if (!interior && !(i + dx >= 0 && i + dx < nx && j + dy >= 0 && j + dy < ny && k + dz >= 0 &&
                                   k + dz < nz))
                    continue;
                const int nb = idx + dz * nxy + dy * nx + dx;
                if (!__ldg(support + nb)) continue;
                const float w = w_sh[q];
                const float fk = __ldg(f + nb), d = fj - fk, ad = fabsf(d);
                // the correctly rounded reciprocal: the same value as 1.0f / D, without the
                // general division's numerator handling
                const float D = fj + fk + gamma * ad + eps, invD = __frcp_rn(D);
                grad += w * d * (fj + 3.0f * fk + gamma * ad + 2.0f * eps) * invD * invD;
                const float half_quad = (2.0f * (fj + fk + eps) + gamma * ad) * invD * invD;
                const float hess = 2.0f * (2.0f * fk + eps) * (2.0f * fk + eps) * invD * invD * invD;
                curv += 2.0f * w * fmaxf(half_quad, hess);
            }
            const float a2 = beta * curv, B = 1.0f + beta * (grad - curv * fj);
            const float root = sqrtf(B * B + 4.0f * a2 * f_em);
            out = B >= 0.0f ? (f_em > 0.0f ? 2.0f * f_em / (B + root) : 0.0f) : (root - B) / (2.0f * a2);
        }
        next[idx] = out;
        if (SUM) v[0] += out;
    }
    if (SUM)
        grid_reduce<1>(v, r, [&](const double* t) {
            sc->sum = t[0];
            sc->scale = t[0] > 0.0 ? (float)(sc->support_sum / t[0]) : 1.0f;
        });
}

template <bool SUM>
__global__ void __launch_bounds__(kEmThreads) update_active_kernel(
    const float* __restrict__ f, const float* __restrict__ back, const unsigned char* __restrict__ support,
    float* __restrict__ next, const int* __restrict__ active, int n_active, Grid g, const float* __restrict__ geo_w,
    float beta, float gamma, EmScalars* sc, Reduction r) {
    update_active_body<SUM>(f, back, support, next, active, n_active, g, geo_w, beta, gamma, sc, r);
}

// Count rescale and, when accelerating, the step h = next - y and the two FP64 inner products
// that give lambda = clamp(<h, h_prev> / <h_prev, h_prev>, 0, 1) (prc.cu:325-332, 693-696).
template <bool RESIDUAL>
__device__ __forceinline__ void finish_body(float* __restrict__ next, float* __restrict__ residual,
                                            const float* __restrict__ h_prev, size_t n, bool use_scale, EmScalars* sc,
                                            Reduction r) {
    const float scale = use_scale ? sc->scale : 1.0f;
    double v[2] = {0.0, 0.0};
    // one element: rescale, step h = next - y into residual, and the two products
    auto step = [&](float& nx, float& res, float hp_f) {
        nx = __fmul_rn(nx, scale);
        if (RESIDUAL) {
            res = nx - res;
            const double hp = hp_f;
            v[0] += (double)res * hp;
            v[1] += hp * hp;
        }
    };
    const size_t n4 = aligned16(next) && (!RESIDUAL || (aligned16(residual) && aligned16(h_prev))) ? n / 4 : 0;
    float4* x4 = reinterpret_cast<float4*>(next);
    float4* r4 = reinterpret_cast<float4*>(residual);
    const float4* h4 = reinterpret_cast<const float4*>(h_prev);
    GRID_STRIDE(q, n4) {
        float4 x = x4[q];
        float4 res = RESIDUAL ? r4[q] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float4 hp = RESIDUAL ? h4[q] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        step(x.x, res.x, hp.x);
        step(x.y, res.y, hp.y);
        step(x.z, res.z, hp.z);
        step(x.w, res.w, hp.w);
        x4[q] = x;
        if (RESIDUAL) r4[q] = res;
    }
    TAIL_STRIDE(i, 4 * n4, n) {
        float x = next[i];
        float res = RESIDUAL ? residual[i] : 0.0f;
        step(x, res, RESIDUAL ? h_prev[i] : 0.0f);
        next[i] = x;
        if (RESIDUAL) residual[i] = res;
    }
    if (RESIDUAL)
        grid_reduce<2>(v, r, [&](const double* t) {
            const double hh = t[1];
            sc->lambda = hh > 0.0 ? (float)fmin(1.0, fmax(0.0, t[0] / hh)) : 0.0f;
        });
}

__global__ void begin_kernel(const float* g_in, const unsigned char* support, float* g, float* f, size_t n,
                             int n_active, EmScalars* sc, Reduction r) {
    begin_body(g_in, support, g, f, n, n_active, sc, r);
}
__global__ void floor_kernel(float* f, const unsigned char* support, size_t n, EmScalars* sc, Reduction r) {
    floor_body(f, support, n, sc, r);
}
__global__ void init_scale_kernel(float* f, size_t n, const EmScalars* sc) { init_scale_body(f, n, sc); }
__global__ void extrapolate_kernel(const float* f, const float* prev, float* y, size_t n, const EmScalars* sc) {
    extrapolate_body(f, prev, y, n, sc);
}
__global__ void ratio_kernel(const float* g, float* est, const unsigned char* support, size_t n, const EmScalars* sc) {
    ratio_body(g, est, support, n, sc);
}
template <bool SUM>
__global__ void update_kernel(const float* f, const float* back, const unsigned char* support, float* next, Grid g,
                              float beta, float gamma, EmScalars* sc, Reduction r) {
    update_body<SUM>(f, back, support, next, g, beta, gamma, sc, r);
}
template <bool RESIDUAL>
__global__ void finish_kernel(float* next, float* residual, const float* h_prev, size_t n, bool use_scale,
                              EmScalars* sc, Reduction r) {
    finish_body<RESIDUAL>(next, residual, h_prev, n, use_scale, sc, r);
}

// Batched forms: blockIdx.y selects the volume; its grid reductions use its own scratch.
__global__ void begin_batch_kernel(const EmItem* items, bool initialize_phase, int phase) {
    const EmItem& it = items[blockIdx.y];
    if (phase == 0) begin_body(it.g_in, it.v.support, it.g, it.f, it.v.n, it.n_active, it.v.scalars, it.v.red);
    else if (phase == 1) floor_body(it.f, it.v.support, it.v.n, it.v.scalars, it.v.red);
    else init_scale_body(it.f, it.v.n, it.v.scalars);
    (void)initialize_phase;
}
__global__ void extrapolate_batch_kernel(const EmItem* items) {
    const EmItem& it = items[blockIdx.y];
    extrapolate_body(it.f, it.prev, it.y, it.v.n, it.v.scalars);
}
__global__ void ratio_batch_kernel(const EmItem* items) {
    const EmItem& it = items[blockIdx.y];
    ratio_body(it.g, it.est, it.v.support, it.v.n, it.v.scalars);
}
// The batched RDP update over each item's tissue list (the single-volume em_update_active); `est`
// is 0 off the support already (the forward preparation, the ratio or the chunk's epilogue put it there).
template <bool SUM>
__global__ void __launch_bounds__(kEmThreads) update_batch_kernel(const EmItem* items, float beta, float gamma,
                                                                  bool accelerate) {
    const EmItem& it = items[blockIdx.y];
    update_active_body<SUM>(accelerate ? it.y : it.f, it.prev, it.v.support, it.est, it.active, it.n_active, it.grid,
                            it.geo_w, beta, gamma, it.v.scalars, it.v.red);
}
template <bool RESIDUAL>
__global__ void finish_batch_kernel(const EmItem* items, bool use_scale) {
    const EmItem& it = items[blockIdx.y];
    finish_body<RESIDUAL>(it.est, RESIDUAL ? it.y : nullptr, it.h_prev, it.v.n, use_scale, it.v.scalars, it.v.red);
}

__global__ void sum_kernel(const float* __restrict__ x, size_t n, EmScalars* sc, Reduction r) {
    double v[1] = {0.0};
    GRID_STRIDE(i, n) v[0] += x[i];
    grid_reduce<1>(v, r, [&](const double* t) { sc->sum = t[0]; });
}

__global__ void mask_copy_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                 const unsigned char* __restrict__ support, size_t n, float fill) {
    GRID_STRIDE(i, n) dst[i] = support[i] ? src[i] : fill;
}

}  // namespace

cudaError_t em_begin(const EmVolumes& v, const float* g_in, float* g, float* f, int n_active, bool initialize,
                     cudaStream_t s) {
    begin_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(g_in, v.support, g, f, v.n, n_active, v.scalars, v.red);
    if (initialize) {
        floor_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(f, v.support, v.n, v.scalars, v.red);
        init_scale_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(f, v.n, v.scalars);
    }
    return cudaGetLastError();
}

cudaError_t em_extrapolate(const EmVolumes& v, const float* f, const float* prev, float* y, cudaStream_t s) {
    extrapolate_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(f, prev, y, v.n, v.scalars);
    return cudaGetLastError();
}

cudaError_t em_ratio(const EmVolumes& v, const float* g, float* est, cudaStream_t s) {
    ratio_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(g, est, v.support, v.n, v.scalars);
    return cudaGetLastError();
}

cudaError_t em_update(const EmVolumes& v, const Grid& grid, const float* start, const float* back, float* next,
                      float beta, float gamma, cudaStream_t s) {
    if (beta > 0.0f)
        update_kernel<true><<<kReduceBlocks, kEmThreads, 0, s>>>(start, back, v.support, next, grid, beta, gamma,
                                                                 v.scalars, v.red);
    else
        update_kernel<false><<<kReduceBlocks, kEmThreads, 0, s>>>(start, back, v.support, next, grid, beta, gamma,
                                                                  v.scalars, v.red);
    return cudaGetLastError();
}

cudaError_t em_geometry_weights(const Grid& grid, float* geo_w, cudaStream_t s) {
    geometry_weights_kernel<<<1, 32, 0, s>>>(grid, geo_w);
    return cudaGetLastError();
}

cudaError_t em_update_active(const EmVolumes& v, const Grid& grid, const int* active, int n_active,
                             const float* geo_w, const float* start, const float* back, float* next, float beta,
                             float gamma, cudaStream_t s) {
    // one tissue voxel per thread where the reduction scratch allows (kReduceBlocks * 4 block
    // partials): many warps in flight hide the latency of the neighbour loads and divisions
    const int blocks = std::max(1, std::min(kReduceBlocks * 4, (n_active + kEmThreads - 1) / kEmThreads));
    if (beta > 0.0f)
        update_active_kernel<true><<<blocks, kEmThreads, 0, s>>>(start, back, v.support, next, active, n_active, grid,
                                                                 geo_w, beta, gamma, v.scalars, v.red);
    else
        update_active_kernel<false><<<blocks, kEmThreads, 0, s>>>(start, back, v.support, next, active, n_active,
                                                                  grid, geo_w, beta, gamma, v.scalars, v.red);
    return cudaGetLastError();
}

cudaError_t em_finish(const EmVolumes& v, float* next, float* residual, const float* h_prev, bool use_scale,
                      cudaStream_t s) {
    if (residual)
        finish_kernel<true><<<kReduceBlocks, kEmThreads, 0, s>>>(next, residual, h_prev, v.n, use_scale, v.scalars,
                                                                 v.red);
    else
        finish_kernel<false><<<kReduceBlocks, kEmThreads, 0, s>>>(next, nullptr, nullptr, v.n, use_scale, v.scalars,
                                                                  v.red);
    return cudaGetLastError();
}

cudaError_t em_batch_phase(EmPhase phase, const EmItem* d_items, int n_items, int blocks, float beta, float gamma,
                           bool accelerate, cudaStream_t s) {
    if (n_items == 0) return cudaSuccess;
    if (blocks > kReduceBlocks) blocks = kReduceBlocks;
    const dim3 grid(blocks, n_items);
    switch (phase) {
        case EmPhase::Begin:
            begin_batch_kernel<<<grid, kEmThreads, 0, s>>>(d_items, true, 0);
            begin_batch_kernel<<<grid, kEmThreads, 0, s>>>(d_items, true, 1);
            begin_batch_kernel<<<grid, kEmThreads, 0, s>>>(d_items, true, 2);
            break;
        case EmPhase::Extrapolate: extrapolate_batch_kernel<<<grid, kEmThreads, 0, s>>>(d_items); break;
        case EmPhase::Ratio: ratio_batch_kernel<<<grid, kEmThreads, 0, s>>>(d_items); break;
        case EmPhase::Update:
            if (beta > 0.0f) update_batch_kernel<true><<<grid, kEmThreads, 0, s>>>(d_items, beta, gamma, accelerate);
            else update_batch_kernel<false><<<grid, kEmThreads, 0, s>>>(d_items, beta, gamma, accelerate);
            break;
        case EmPhase::Finish:
            if (accelerate) finish_batch_kernel<true><<<grid, kEmThreads, 0, s>>>(d_items, beta > 0.0f);
            else finish_batch_kernel<false><<<grid, kEmThreads, 0, s>>>(d_items, beta > 0.0f);
            break;
    }
    return cudaGetLastError();
}

cudaError_t em_sum(const EmVolumes& v, const float* x, cudaStream_t s) {
    sum_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(x, v.n, v.scalars, v.red);
    return cudaGetLastError();
}

cudaError_t em_mask_copy(const EmVolumes& v, const float* src, float* dst, float fill, cudaStream_t s) {
    mask_copy_kernel<<<kReduceBlocks, kEmThreads, 0, s>>>(src, dst, v.support, v.n, fill);
    return cudaGetLastError();
}

}  // namespace prc
