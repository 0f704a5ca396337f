// projector.cu -- the heterogeneous range-blur projector A (normalisation, forward, adjoint).
//
// Model (jlherraiz/PRC_MLEM prc.cu:131-267): every tissue voxel s emits mirrored ray pairs; a
// ray marches voxel faces (3D DDA), accumulating water-equivalent path w += rho * dt, and
// deposits S(w_in) - S(w_out) into each tissue voxel it crosses.  2048 "near" rays fill the
// 5x5x5 block around s; n_rays "far" rays deposit outside it.  W_s = sum_t w_st, and
//   forward:  (A f)_t  = sum_s f_s / W_s * w_st      (scatter)
//   adjoint:  (A^T y)_s = sum_t w_st * y_t / W_s     (gather)
//
// B200 mapping (the reference gives one warp to one source and strides its lanes over rays):
// here a warp owns 32 consecutive tissue voxels (lanes) and all lanes trace the SAME ray k at
// the same time.  Because ray k starts at the same sub-voxel offset with the same direction
// in every source voxel and the grid is uniform, the face-crossing sequence (which axis, and
// the path length dt of each segment) is identical in every lane: it is warp-uniform control
// flow, computed once per ray with prc.cu's own float arithmetic, so the weights are the
// reference's bit for bit.  Only the density along the path differs per lane, which decides
// where each lane stops.  The 32 lanes are x-neighbours in one image row, so every density
// read, gather and scatter of a step touches 32 consecutive voxels: coalesced 128-byte lines
// from L2, where the 10 MB volumes stay resident.  The near block is either traced into a
// per-warp shared-memory tile laid out [offset][lane] (conflict-free, no atomics: each lane
// owns its column) or read from the group-interleaved cache.
#include "engine.h"

#include <cstdio>

namespace prc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;  // groups per block
constexpr int kBlock = kWarps * kLanes;
constexpr size_t kNearSmemBytes = size_t(kWarps) * kNear * kLanes * sizeof(float);

// Direction and sub-voxel start (voxel units) of ray k of n.  Rays 2m and 2m+1 are mirror
// images (start and direction negated), which centres the emission on the voxel.  The
// direction of pair m is the m-th point of a Fibonacci lattice on the hemisphere (even steps in
// z, golden-ratio steps in azimuth); the start is the m-th point of the R3 sequence.  The
// integer hashing wraps modulo 2^32 and the float operations are those of prc.cu:118-129, in
// the same order, so both projectors trace identical rays.
__device__ __forceinline__ void ray_geometry(int k, int n, float3& start, float3& dir) {
    const unsigned pair = static_cast<unsigned>(k) >> 1;
    const float mirror = (k & 1) ? -1.0f : 1.0f;
    const float cz = 1.0f - (pair + 0.5f) / ((n + 1) >> 1);
    const float rxy = sqrtf(fmaxf(0.0f, 1.0f - cz * cz));
    const float inv2p32 = 2.3283064e-10f;
    float sn, cs;
    sincospif(2.0f * inv2p32 * (pair * 2654435769u), &sn, &cs);
    dir = make_float3(mirror * rxy * cs, mirror * rxy * sn, mirror * cz);
    start = make_float3(mirror * (inv2p32 * (0x80000000u + pair * 3518319155u) - 0.5f),
                        mirror * (inv2p32 * (0x80000000u + pair * 2882110345u) - 0.5f),
                        mirror * (inv2p32 * (0x80000000u + pair * 2360945575u) - 0.5f));
}

__device__ RayStep derive_step(const Grid& g, int k, int n) {
    float3 x, d;
    ray_geometry(k, n, x, d);
    const float big = 1.0e30f;
    RayStep r;
    r.di = d.x > 0.0f ? 1 : -1;
    r.dj = d.y > 0.0f ? 1 : -1;
    r.dk = d.z > 0.0f ? 1 : -1;
    r.tx = d.x != 0.0f ? (0.5f * r.di - x.x) * g.sx / d.x : big;
    r.ty = d.y != 0.0f ? (0.5f * r.dj - x.y) * g.sy / d.y : big;
    r.tz = d.z != 0.0f ? (0.5f * r.dk - x.z) * g.sz / d.z : big;
    r.dtx = d.x != 0.0f ? g.sx / fabsf(d.x) : big;
    r.dty = d.y != 0.0f ? g.sy / fabsf(d.y) : big;
    r.dtz = d.z != 0.0f ? g.sz / fabsf(d.z) : big;
    r.pad = 0;
    return r;
}

__global__ void ray_setup_kernel(Grid g, int n_far, RayStep* far, RayStep* near) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n_far) far[k] = derive_step(g, k, n_far);
    if (k < kNearRays) near[k] = derive_step(g, k, kNearRays);
}

// S(w) for 0 <= w <= cutoff: the float table with an fmaf lerp (prc.cu:74-80) or analytic.
template <bool EXACT>
__device__ __forceinline__ float survival_lookup(const ProjParams& p, float w) {
    if constexpr (EXACT) {
        return survival(p.br, p.n_branch, w);
    } else {
        const float u = w * p.table_scale;
        const int i = min((int)u, kRangeBins - 1);
        const float lo = __ldg(p.table + i), hi = __ldg(p.table + i + 1);
        return fmaf(fminf(u - i, 1.0f), hi - lo, lo);
    }
}

// One ray for the 32 sources of a warp.  `run` is this lane's participation, (idx, ci, cj, ck)
// its source voxel.  The loop runs while any lane is still marching; the per-lane stopping
// rules are those of prc.cu:145-164: range cutoff, air cap, leaving the image, and (near rays)
// leaving the block.  visit(t, weight, q) gets the target voxel, the deposit and the block
// offset code q = ((dz+2)*5 + dy+2)*5 + dx+2 and, for far rays, the post-block step index m
// (the position of the step in the ray template).
template <bool NEAR, bool EXACT, class Visit>
__device__ __forceinline__ void march(const ProjParams& p, const RayStep& R, bool run, int idx, int ci, int cj,
                                      int ck, Visit&& visit) {
    float tx = R.tx, ty = R.ty, tz = R.tz, t = 0.0f;
    float w = 0.0f, surv = 1.0f, air = 0.0f;
    int oi = 0, oj = 0, ok = 0;  // offset from the source: identical in every lane
    int m = 0;                   // post-block steps taken (far rays)
    const int step_y = R.dj * p.g.nx, step_z = R.dk * p.nxy;
    const float cutoff = p.g.cutoff, srho = p.g.support_rho, cap = p.g.air_cap;
    while (__any_sync(kFull, run)) {
        const bool in_block = abs(oi) <= kNearR && abs(oj) <= kNearR && abs(ok) <= kNearR;
        if (NEAR && !in_block) break;
        const float t_next = fminf(tx, fminf(ty, tz));
        const float dt = t_next - t;
        if (run) {
            const float rho = __ldg(p.rho + idx);
            const float w_next = fminf(w + rho * dt, cutoff);
            const float surv_next = survival_lookup<EXACT>(p, w_next);
            if (rho >= srho) {
                air = 0.0f;
                if (in_block == NEAR && surv > surv_next)
                    visit(idx, surv - surv_next, ((ok + kNearR) * kNearSide + oj + kNearR) * kNearSide + oi + kNearR, m);
            } else if ((air += dt) > cap) {
                run = false;
            }
            if (w_next >= cutoff) run = false;
            w = w_next;
            surv = surv_next;
        }
        t = t_next;
        m += !in_block;
        if (t_next == tx) {
            oi += R.di, ci += R.di, idx += R.di, tx += R.dtx;
            if ((unsigned)ci >= (unsigned)p.g.nx) run = false;
        } else if (t_next == ty) {
            oj += R.dj, cj += R.dj, idx += step_y, ty += R.dty;
            if ((unsigned)cj >= (unsigned)p.g.ny) run = false;
        } else {
            ok += R.dk, ck += R.dk, idx += step_z, tz += R.dtz;
            if ((unsigned)ck >= (unsigned)p.g.nz) run = false;
        }
    }
}

enum NearMode : int { kTraceNear = 0, kCacheF32 = 1, kCacheBF16 = 2 };
enum FarMode : int { kMarch = 0, kFieldF32 = 1, kFieldBF16 = 2 };

// kPack consecutive steps of one lane are stored together (one vector load per lane).
constexpr int kPack = 4;

// Streaming (evict-first) vector load of kPack stored weights of this lane.
template <int FAR_MODE>
__device__ __forceinline__ void load_pack(const FarField& f, long long e, float* w) {
    if constexpr (FAR_MODE == kFieldF32) {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(f.f32 + e));
        w[0] = v.x, w[1] = v.y, w[2] = v.z, w[3] = v.w;
    } else {
        const uint2 v = __ldcs(reinterpret_cast<const uint2*>(f.b16 + e));
        w[0] = __uint_as_float(v.x << 16), w[1] = __uint_as_float(v.x & 0xffff0000u);
        w[2] = __uint_as_float(v.y << 16), w[3] = __uint_as_float(v.y & 0xffff0000u);
    }
}

// One warp per group of 32 consecutive sources.  NEAR_MODE says where the 5x5x5 weights come
// from, FAR_MODE whether far rays are marched or read from the stored field.  Norm always
// marches and, when the caches are allocated, writes them; Layout marches to size the field.
template <Op OP, bool EXACT, int NEAR_MODE, int FAR_MODE>
__global__ void __launch_bounds__(kBlock) project_kernel(const ProjParams p, const OpArgs a) {
    extern __shared__ float near_sum[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int group = blockIdx.x * kWarps + warp;
    if (group * kLanes >= p.n_active) return;  // the whole warp leaves together
    const int src = group * kLanes + lane;
    const bool valid = src < p.n_active;
    const int s = valid ? __ldg(p.active + src) : 0;
    bool live = valid;
    float scale = 0.0f, acc = 0.0f;
    unsigned long long cnt = 0;
    if constexpr (OP == Op::Forward) {  // prc.cu:244-248
        const float fs = valid ? __ldg(a.in + s) : 0.0f, ws = valid ? __ldg(a.W + src) : 0.0f;
        scale = ws > 0.0f ? fs / ws : 0.0f;
        live = valid && scale > 0.0f;
    } else if constexpr (OP == Op::Adjoint) {  // prc.cu:260-264
        const float ws = valid ? __ldg(a.W + src) : 0.0f;
        live = valid && ws > 0.0f;
        if (valid && !live) a.out[s] = 0.0f;
    }
    if (!__any_sync(kFull, live)) return;
    const int nx = p.g.nx, ny = p.g.ny;
    const int vx = s % nx, vy = (s / nx) % ny, vz = s / p.nxy;
    // Norm: W must sum exactly the weights later projections use, so stored bf16 weights are
    // rounded before they are accumulated.
    const bool near_bf16 = OP == Op::Norm && a.near.b16, far_bf16 = OP == Op::Norm && a.far.b16;

    auto deposit = [&](int t, float w) {
        if constexpr (OP == Op::Norm) acc += w;
        else if constexpr (OP == Op::Forward) atomicAdd(a.out + t, scale * w);
        else if constexpr (OP == Op::Adjoint) acc += w * __ldg(a.in + t);
        else cnt += 1;
    };

    // Near block (prc.cu:193-218).
    if constexpr (OP != Op::Layout) {
        float* sum = near_sum + warp * (kNear * kLanes);
        if constexpr (NEAR_MODE == kTraceNear) {
            for (int q = 0; q < kNear; ++q) sum[q * kLanes + lane] = 0.0f;
            for (int r = 0; r < kNearRays; ++r) {
                const RayStep R = p.near[r];
                march<true, EXACT>(p, R, live, s, vx, vy, vz,
                                   [&](int, float w, int q, int) { sum[q * kLanes + lane] += w; });
            }
        }
        const size_t cache_base = (size_t)group * kNear * kLanes + lane;
        const float near_scale = (float)p.n_rays / kNearRays;
        for (int q = 0; q < kNear; ++q) {
            const int dx = q % kNearSide - kNearR, dy = q / kNearSide % kNearSide - kNearR,
                      dz = q / (kNearSide * kNearSide) - kNearR;
            float w;
            if constexpr (NEAR_MODE == kTraceNear) {
                const bool in = (unsigned)(vx + dx) < (unsigned)nx && (unsigned)(vy + dy) < (unsigned)ny &&
                                (unsigned)(vz + dz) < (unsigned)p.g.nz;
                w = in ? sum[q * kLanes + lane] * near_scale : 0.0f;
                if constexpr (OP == Op::Norm) {
                    if (near_bf16) w = __bfloat162float(__float2bfloat16_rn(w));
                    if (valid && a.near.b16) a.near.b16[cache_base + (size_t)q * kLanes] = __float2bfloat16_rn(w);
                    if (valid && a.near.f32) a.near.f32[cache_base + (size_t)q * kLanes] = w;
                }
            } else if constexpr (NEAR_MODE == kCacheF32) {
                w = live ? __ldg(a.near.f32 + cache_base + (size_t)q * kLanes) : 0.0f;
            } else {
                w = live ? __bfloat162float(a.near.b16[cache_base + (size_t)q * kLanes]) : 0.0f;
            }
            if (live && w > 0.0f) deposit(s + (dz * ny + dy) * nx + dx, w);
        }
    }

    // Far field (prc.cu:220-226).
    if constexpr (FAR_MODE == kMarch) {
        long long fbase = 0;  // Norm: element offset of this ray's field block, plus this lane's slot
        if constexpr (OP == Op::Norm) {
            if (a.far.on()) fbase = p.group_base[group] + lane * kPack;
        }
        for (int r = 0; r < p.n_rays; ++r) {
            const RayStep R = p.far[r];
            if constexpr (OP == Op::Layout) {
                int last = -1;
                march<false, EXACT>(p, R, live, s, vx, vy, vz, [&](int, float, int, int m) { last = m; });
                const int L = (__reduce_max_sync(kFull, last + 1) + kPack - 1) / kPack * kPack;
                if (lane == 0) a.len[(size_t)group * p.n_rays + r] = (unsigned short)L;
                acc += (float)L;  // exact: totals stay far below 2^24 per group
            } else if constexpr (OP == Op::Norm) {
                const int L = a.far.on() ? (int)p.len[(size_t)group * p.n_rays + r] : 0;
                march<false, EXACT>(p, R, live, s, vx, vy, vz, [&](int, float w, int, int m) {
                    if (far_bf16) w = __bfloat162float(__float2bfloat16_rn(w));
                    acc += w;
                    const long long e = fbase + (long long)(m / kPack) * (kPack * kLanes) + m % kPack;
                    if (a.far.f32) a.far.f32[e] = w;
                    else if (a.far.b16) a.far.b16[e] = __float2bfloat16_rn(w);
                });
                fbase += (long long)L * kLanes;
            } else {
                march<false, EXACT>(p, R, live, s, vx, vy, vz, [&](int t, float w, int, int) { deposit(t, w); });
            }
        }
    } else {
        // Stored field: the weights of one ray for the 32 lanes are one contiguous block of
        // len * 32 entries, packed so that each lane reads kPack consecutive steps with one
        // vector load (16 B fp32, 8 B bf16); target voxels are the source plus the template
        // offsets, read as int4 broadcasts.  Eight steps are loaded before any is used.  The
        // adjoint's gathers do not wait for the weights: their index is clamped into the volume
        // and a zero weight discards the value.
        const int4* tmpl4 = reinterpret_cast<const int4*>(p.tmpl);
        const unsigned short* len = p.len + (size_t)group * p.n_rays;
        long long fbase = p.group_base[group] + lane * kPack;
        const int n_vox = p.nxy * p.g.nz;
        for (int r = 0; r < p.n_rays; ++r, tmpl4 += p.tmpl_len / kPack) {
            const int L = len[r];
            for (int m = 0; m < L; m += 2 * kPack) {
                const bool two = m + kPack < L;
                float w[2 * kPack];
                load_pack<FAR_MODE>(a.far, fbase + (long long)(m / kPack) * (kPack * kLanes), w);
                if (two) load_pack<FAR_MODE>(a.far, fbase + (long long)(m / kPack + 1) * (kPack * kLanes), w + kPack);
                else
#pragma unroll
                    for (int u = kPack; u < 2 * kPack; ++u) w[u] = 0.0f;
                const int4 oa = __ldg(tmpl4 + m / kPack);
                const int4 ob = two ? __ldg(tmpl4 + m / kPack + 1) : make_int4(0, 0, 0, 0);
                const int o[2 * kPack] = {oa.x, oa.y, oa.z, oa.w, ob.x, ob.y, ob.z, ob.w};
                if constexpr (OP == Op::Adjoint) {
                    float v[2 * kPack];
#pragma unroll
                    for (int u = 0; u < 2 * kPack; ++u) v[u] = __ldg(a.in + min(max(s + o[u], 0), n_vox - 1));
#pragma unroll
                    for (int u = 0; u < 2 * kPack; ++u) acc += (live && w[u] > 0.0f) ? w[u] * v[u] : 0.0f;
                } else {
#pragma unroll
                    for (int u = 0; u < 2 * kPack; ++u)
                        if (live && w[u] > 0.0f) deposit(s + o[u], w[u]);
                }
            }
            fbase += (long long)L * kLanes;
        }
    }

    if constexpr (OP == Op::Norm) {
        if (valid) a.W[src] = acc;
    } else if constexpr (OP == Op::Layout) {
        if (lane == 0) a.group_total[group] = (long long)acc * kLanes;
    } else if constexpr (OP == Op::Adjoint) {
        if (live) a.out[s] = acc / __ldg(a.W + src);  // prc.cu:266
    } else if constexpr (OP == Op::Count) {
        for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(kFull, cnt, off);
        if (lane == 0) atomicAdd(a.count, cnt);
    }
}

// Ray template: the linear offsets of the post-block steps of each far ray, from the same
// uniform DDA the march performs.
__global__ void template_kernel(const ProjParams p, int* tmpl) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= p.n_rays) return;
    const RayStep R = p.far[r];
    float tx = R.tx, ty = R.ty, tz = R.tz;
    int oi = 0, oj = 0, ok = 0, m = 0;
    int* out = tmpl + (size_t)r * p.tmpl_len;
    for (int step = 0; m < p.tmpl_len && step < 4 * p.tmpl_len; ++step) {
        const bool in_block = abs(oi) <= kNearR && abs(oj) <= kNearR && abs(ok) <= kNearR;
        if (!in_block) out[m++] = (ok * p.g.ny + oj) * p.g.nx + oi;
        const float t_next = fminf(tx, fminf(ty, tz));
        if (t_next == tx) oi += R.di, tx += R.dtx;
        else if (t_next == ty) oj += R.dj, ty += R.dty;
        else ok += R.dk, tz += R.dtz;
    }
}

template <Op OP, bool EXACT, int NEAR_MODE, int FAR_MODE>
cudaError_t launch(const ProjParams& p, const OpArgs& a, cudaStream_t s) {
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    const int blocks = (groups + kWarps - 1) / kWarps;
    if (blocks == 0) return cudaSuccess;
    const size_t smem = NEAR_MODE == kTraceNear && OP != Op::Layout ? kNearSmemBytes : 0;
    auto kernel = project_kernel<OP, EXACT, NEAR_MODE, FAR_MODE>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kernel<<<blocks, kBlock, smem, s>>>(p, a);
    return cudaGetLastError();
}

template <Op OP, bool EXACT>
cudaError_t launch_modes(const ProjParams& p, const OpArgs& a, bool trace_near, cudaStream_t s) {
    if constexpr (OP == Op::Norm || OP == Op::Layout || OP == Op::Count) {
        if (OP == Op::Count && !trace_near && a.near.on())
            return a.near.b16 ? launch<OP, EXACT, kCacheBF16, kMarch>(p, a, s) : launch<OP, EXACT, kCacheF32, kMarch>(p, a, s);
        return launch<OP, EXACT, kTraceNear, kMarch>(p, a, s);
    } else {
        if (trace_near || !a.near.on()) {
            if (a.far.f32) return launch<OP, EXACT, kTraceNear, kFieldF32>(p, a, s);
            if (a.far.b16) return launch<OP, EXACT, kTraceNear, kFieldBF16>(p, a, s);
            return launch<OP, EXACT, kTraceNear, kMarch>(p, a, s);
        }
        if (a.near.b16) {
            if (a.far.b16) return launch<OP, EXACT, kCacheBF16, kFieldBF16>(p, a, s);
            if (a.far.f32) return launch<OP, EXACT, kCacheBF16, kFieldF32>(p, a, s);
            return launch<OP, EXACT, kCacheBF16, kMarch>(p, a, s);
        }
        if (a.far.f32) return launch<OP, EXACT, kCacheF32, kFieldF32>(p, a, s);
        if (a.far.b16) return launch<OP, EXACT, kCacheF32, kFieldBF16>(p, a, s);
        return launch<OP, EXACT, kCacheF32, kMarch>(p, a, s);
    }
}

template <Op OP>
cudaError_t launch_op(const ProjParams& p, const OpArgs& a, bool trace_near, cudaStream_t s) {
    return p.table ? launch_modes<OP, false>(p, a, trace_near, s) : launch_modes<OP, true>(p, a, trace_near, s);
}

}  // namespace

cudaError_t setup_rays(const Grid& g, int n_rays, RayStep* d_far, RayStep* d_near, cudaStream_t s) {
    const int n = n_rays > kNearRays ? n_rays : kNearRays;
    ray_setup_kernel<<<(n + 127) / 128, 128, 0, s>>>(g, n_rays, d_far, d_near);
    return cudaGetLastError();
}

cudaError_t build_template(const ProjParams& p, int* tmpl, cudaStream_t s) {
    template_kernel<<<(p.n_rays + 127) / 128, 128, 0, s>>>(p, tmpl);
    return cudaGetLastError();
}

cudaError_t project(Op op, const ProjParams& p, const OpArgs& a, bool trace_near, cudaStream_t s) {
    switch (op) {
        case Op::Norm: return launch_op<Op::Norm>(p, a, true, s);
        case Op::Forward: return launch_op<Op::Forward>(p, a, trace_near, s);
        case Op::Adjoint: return launch_op<Op::Adjoint>(p, a, trace_near, s);
        case Op::Count: return launch_op<Op::Count>(p, a, trace_near, s);
        case Op::Layout: return launch_op<Op::Layout>(p, a, true, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace prc
