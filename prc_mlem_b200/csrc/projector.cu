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
// here a warp owns 32 consecutive sources (lanes) and all lanes trace the SAME ray k at
// the same time.  Because ray k starts at the same sub-voxel offset with the same direction
// in every source voxel and the grid is uniform, the face-crossing sequence (which axis, and
// the path length dt of each segment) is identical in every lane: it is warp-uniform control
// flow, computed once per ray with prc.cu's own float arithmetic, so the weights are the
// reference's bit for bit.  Only the density along the path differs per lane, which decides
// where each lane stops.  Sources are ordered in 8x2x2 voxel tiles, so the 32 lanes are close
// neighbours: every density read, gather and scatter of a step touches four 32-byte row
// segments, from L1 / L2, where the 10 MB volumes stay resident.  The near block is either traced into a
// per-warp shared-memory tile laid out [offset][lane] (conflict-free, no atomics: each lane
// owns its column) or read from the group-interleaved cache.
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <type_traits>

namespace prc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
#ifndef PRC_PROJ_WARPS
#define PRC_PROJ_WARPS 4
#endif
constexpr int kWarps = PRC_PROJ_WARPS;  // groups per block (default launch)
constexpr int kBlock = kWarps * kLanes;
constexpr int kMaxWarps = 8;  // largest block of a (batched, autotuned) launch
constexpr int kMaxBlock = kMaxWarps * kLanes;
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
// Far-field source: marched rays, the source-major field (adjoint; forward by scatter), or the
// target-major field (forward by gather; the *T modes).
// kFieldBF16H / kFieldBF16TH: the bf16 field gathering a bf16 volume (a.in16) -- inside
// MAP-EM the mixed-precision form keeps the gathered volumes (u = y / W and the EM ratio) in
// bf16, and its forward epilogue writes the ratio as bf16 (a.out16).
// kField24 / kField24T: the 24-bit field (FarField::b24) of PRC_PRECISION_FP24.
enum FarMode : int { kMarch = 0, kFieldF32 = 1, kFieldBF16 = 2, kFieldF32T = 3, kFieldBF16T = 4, kFieldBF16H = 5,
                     kFieldBF16TH = 6, kField24 = 7, kField24T = 8 };
__host__ __device__ constexpr bool target_major(int m) {
    return m == kFieldF32T || m == kFieldBF16T || m == kFieldBF16TH || m == kField24T;
}
__host__ __device__ constexpr bool half_volume(int m) { return m == kFieldBF16H || m == kFieldBF16TH; }
__host__ __device__ constexpr int field_base(int m) {
    return m == kFieldF32 || m == kFieldF32T ? kFieldF32 : (m == kField24 || m == kField24T ? kField24 : kFieldBF16);
}

// ---- stored coefficient field ----------------------------------------------------------------
// Stream of one group: template row 0 is the near block (125 offsets, padded to kNearRow
// steps), rows 1..n_rays the far rays after they leave the block.  Row k contributes len[G][k]
// steps (a multiple of kPack, zero for rays no lane deposits on).  kPack consecutive steps of
// one lane are stored together, so a "pack" (kPack steps x 32 lanes) is one vector load per
// lane, and a group's packs are contiguous in stream order.  desc[pack] holds the element
// offset of the pack's first step in the template, so every pack can be addressed without
// walking the stream.
constexpr int kPack = 4;
constexpr int kNearRow = 128;  // 125 block offsets rounded up to whole packs
// TMA ring of the fp32 and 24-bit field streams: kStages chunks of kChunk bytes per warp.  The bf16 form
// loads its vectors directly and keeps the reservation only for the L1 / shared-memory split it
// gives (launched without it, with the largest L1, it measured 1.7-2x slower).
constexpr int kStages = 2;
constexpr int kChunk = 2048;
constexpr size_t kFieldSmemPerWarp = size_t(kStages) * kChunk;
constexpr size_t kFieldSmemBytes = size_t(kWarps) * kFieldSmemPerWarp;
// try_wait rounds before a bounded mbarrier wait gives up (each round is a bounded hardware wait).
constexpr int kWaitRounds = 1 << 20;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbarrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 1D bulk copy global -> this CTA's shared memory, completion counted on an mbarrier.
// Source and destination are 16-byte aligned and bytes is a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int rounds = kWaitRounds) {
    for (int i = 0; i < rounds; ++i) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// An 8-byte vector of the bf16 field, read once per projection: loaded without allocating in
// L1, which keeps L1 for the volume being gathered.
__device__ __forceinline__ uint2 ld_stream(const uint2* q) {
    uint2 x;
    asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(x.x), "=r"(x.y) : "l"(q));
    return x;
}


__device__ __forceinline__ int near_offset(const ProjParams& p, int q) {
    const int dx = q % kNearSide - kNearR, dy = q / kNearSide % kNearSide - kNearR,
              dz = q / (kNearSide * kNearSide) - kNearR;
    return (dz * p.g.ny + dy) * p.g.nx + dx;
}

// Element index of (step m of the row whose stream block starts at row_base) for this lane.
__device__ __forceinline__ long long pack_slot(long long row_base, int m, int lane) {
    return row_base + (long long)(m / kPack) * (kPack * kLanes) + lane * kPack + m % kPack;
}

// The 24-bit weight of a non-negative finite w: bits 30..7 of its fp32 pattern (the sign is
// always 0; 8 exponent and 16 mantissa bits) rounded to nearest, ties to even (a carry into the
// exponent gives the next binade's value, as it should).  Relative error at most 2^-17.
// Stream layout: every pack (4 steps x 32 lanes, 128 entries) is 384 bytes, the upper 16 bits of
// its 128 values (256 bytes, entry order: lane L's four at 8 L) and then their low bytes (128
// bytes, lane L's four at 256 + 4 L), so a lane loads one 8-byte and one 4-byte vector per pack.
__device__ __forceinline__ unsigned bits24(float w) {
    const unsigned u = __float_as_uint(w);
    return (u + 0x3Fu + ((u >> 7) & 1u)) >> 7;
}
__device__ __forceinline__ float round24(float w) { return __uint_as_float(bits24(w) << 7); }
__device__ __forceinline__ float load24(const unsigned char* b, long long e) {
    const unsigned char* pack = b + (e >> 7) * 384;
    const int i = (int)(e & 127);
    const unsigned hi = *reinterpret_cast<const unsigned short*>(pack + 2 * i), lo = pack[256 + i];
    return __uint_as_float(((hi << 8) | lo) << 7);
}
__device__ __forceinline__ void store24(unsigned char* b, long long e, unsigned v) {
    unsigned char* pack = b + (e >> 7) * 384;
    const int i = (int)(e & 127);
    *reinterpret_cast<unsigned short*>(pack + 2 * i) = (unsigned short)(v >> 8);
    pack[256 + i] = (unsigned char)v;
}
// The four weights of one lane's pack: hi = their upper 16-bit halves (two per word), lo = their
// low bytes.  Each weight's three bytes go to the top of a word, then one bit down (bits 30..7).
__device__ __forceinline__ void decode24(uint2 hi, unsigned lo, float* w) {
    w[0] = __uint_as_float((__byte_perm(hi.x, lo, 0x1044) & 0xFFFFFF00u) >> 1);
    w[1] = __uint_as_float((__byte_perm(hi.x, lo, 0x3255) & 0xFFFFFF00u) >> 1);
    w[2] = __uint_as_float((__byte_perm(hi.y, lo, 0x1066) & 0xFFFFFF00u) >> 1);
    w[3] = __uint_as_float((__byte_perm(hi.y, lo, 0x3277) & 0xFFFFFF00u) >> 1);
}

template <int FAR_MODE>
__device__ __forceinline__ void store_weight(const FarField& f, long long e, float w) {
    if constexpr (FAR_MODE == kFieldF32) f.f32[e] = w;
    else if constexpr (FAR_MODE == kField24) store24(f.b24, e, bits24(w));
    else f.b16[e] = __float2bfloat16_rn(w);
}

// Near block of one lane, traced one direction octant at a time.  A near ray whose direction
// has signs (sx, sy, sz) only visits block offsets (sx a, sy b, sz c) with a, b, c in {0, 1, 2}
// before it leaves the block, so the rays of one octant deposit into 27 offsets: a 27 x 32
// shared-memory tile per warp, added to this lane's column of the fp32 accumulator acc
// ([125 offsets] with stride 32) after each octant.  Rays keep increasing index within an octant.
template <bool EXACT>
__device__ __forceinline__ void trace_near_octants(const ProjParams& p, bool live, int s, int vx, int vy, int vz,
                                                   int warp, int lane, unsigned char* dyn_smem, float* acc) {
    float* tile = reinterpret_cast<float*>(dyn_smem) + warp * (27 * kLanes);
    for (int q = 0; q < kNear; ++q) acc[q * kLanes] = 0.0f;
    for (int o = 0; o < 8; ++o) {
        const int sx = (o & 1) ? 1 : -1, sy = (o & 2) ? 1 : -1, sz = (o & 4) ? 1 : -1;
        for (int j = 0; j < 27; ++j) tile[j * kLanes + lane] = 0.0f;
        const int r0 = __ldg(p.near_start + o), r1 = __ldg(p.near_start + o + 1);
        for (int i = r0; i < r1; ++i) {
            const RayStep R = p.near[__ldg(p.near_order + i)];
            march<true, EXACT>(p, R, live, s, vx, vy, vz, [&](int, float w, int q, int) {
                const int a = abs(q % kNearSide - kNearR), b = abs(q / kNearSide % kNearSide - kNearR),
                          c = abs(q / (kNearSide * kNearSide) - kNearR);
                tile[((c * 3 + b) * 3 + a) * kLanes + lane] += w;
            });
        }
        for (int j = 0; j < 27; ++j) {
            const int dx = sx * (j % 3), dy = sy * (j / 3 % 3), dz = sz * (j / 9);
            acc[(((dz + kNearR) * kNearSide + dy + kNearR) * kNearSide + dx + kNearR) * kLanes] += tile[j * kLanes + lane];
        }
    }
}

// Stable grouping of the near rays by direction octant (one thread; 2048 rays, setup only).
__global__ void order_near_kernel(const RayStep* near, short* order, int* start) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int count[8] = {};
    for (int r = 0; r < kNearRays; ++r) ++count[(near[r].di > 0) | (near[r].dj > 0) << 1 | (near[r].dk > 0) << 2];
    int pos[8];
    start[0] = 0;
    for (int o = 0; o < 8; ++o) start[o + 1] = start[o] + count[o], pos[o] = start[o];
    for (int r = 0; r < kNearRays; ++r)
        order[pos[(near[r].di > 0) | (near[r].dj > 0) << 1 | (near[r].dk > 0) << 2]++] = (short)r;
}

// One warp per group of 32 consecutive sources.  NEAR_MODE says where the 5x5x5 weights come
// from when the far rays are marched; FAR_MODE selects marching or the stored field (which
// then also holds the near block).  Norm always marches and writes W, and the near cache or
// the stored field when they are allocated; Layout marches to size the field.
// The work of one warp (group `group`, warp `warp` of its block): dyn_smem is the block's
// dynamic shared memory (near tiles or field rings are indexed by warp), bars the warp's
// kStages mbarriers.
template <Op OP, bool EXACT, int NEAR_MODE, int FAR_MODE>
__device__ __forceinline__ void project_group(const ProjParams& p, const OpArgs& a, int group, int warp,
                                              unsigned char* dyn_smem, uint64_t* bars) {
    const int lane = threadIdx.x & 31;
    if (group * kLanes >= p.n_active) return;  // the whole warp leaves together
    const int src = group * kLanes + lane;
    const bool valid = src < p.n_active;
    const int s = valid ? __ldg(p.active + src) : 0;
    bool live = valid;
    float scale = 0.0f, acc = 0.0f;
    unsigned long long cnt = 0;
    if constexpr (OP == Op::Forward) {  // prc.cu:244-248
        if (target_major(FAR_MODE)) {
            live = valid;  // gather form: lanes are targets, a.in holds u = f / W
        } else {
            const float fs = valid ? __ldg(a.in + s) : 0.0f, ws = valid ? __ldg(a.W + src) : 0.0f;
            scale = ws > 0.0f ? fs / ws : 0.0f;
            live = valid && scale > 0.0f;
        }
    } else if constexpr (OP == Op::Adjoint) {  // prc.cu:260-264
        const float ws = valid ? __ldg(a.W + src) : 0.0f;
        live = valid && ws > 0.0f;
        if (valid && !live) a.out[s] = 0.0f;
    }
    if (!__any_sync(kFull, live)) return;
    const int nx = p.g.nx, ny = p.g.ny;
    const int vx = s % nx, vy = (s / nx) % ny, vz = s / p.nxy;

    auto deposit = [&](int t, float w) {
        if constexpr (OP == Op::Norm) acc += w;
        else if constexpr (OP == Op::Forward) atomicAdd(a.out + t, scale * w);
        else if constexpr (OP == Op::Adjoint) acc += w * __ldg(a.in + t);
        else cnt += 1;
    };

    if constexpr (FAR_MODE == kMarch) {
        const bool field = OP == Op::Norm && a.far.on();
        const long long gbase = field ? p.src.group_base[group] : 0;
        // Norm: W must sum exactly the weights later projections use, so stored bf16 weights
        // are rounded before they are accumulated.
        const bool near_round = OP == Op::Norm && (a.near.b16 || a.far.b16);
        const bool far_round = OP == Op::Norm && a.far.b16;
        const bool round_24 = OP == Op::Norm && a.far.b24;  // W sums the weights as stored

        // Near block (prc.cu:193-218).
        if constexpr (OP != Op::Layout) {
            float* sum = reinterpret_cast<float*>(dyn_smem) + warp * (kNear * kLanes);
            if constexpr (NEAR_MODE == kTraceNear) {
                if (OP == Op::Norm && a.near_acc) {
                    trace_near_octants<EXACT>(p, live, s, vx, vy, vz, warp, lane, dyn_smem,
                                              a.near_acc + (size_t)group * kNear * kLanes + lane);
                } else {
                    for (int q = 0; q < kNear; ++q) sum[q * kLanes + lane] = 0.0f;
                    for (int r = 0; r < kNearRays; ++r) {
                        const RayStep R = p.near[r];
                        march<true, EXACT>(p, R, live, s, vx, vy, vz,
                                           [&](int, float w, int q, int) { sum[q * kLanes + lane] += w; });
                    }
                }
            }
            // traced near weights of this lane: the shared-memory tile or the octant accumulator
            const bool octants = NEAR_MODE == kTraceNear && OP == Op::Norm && a.near_acc;
            const float* near_sum = octants ? a.near_acc + (size_t)group * kNear * kLanes + lane : sum + lane;
            const size_t cache_base = (size_t)group * kNear * kLanes + lane;
            const float near_scale = (float)p.n_rays / kNearRays;
            for (int q = 0; q < kNear; ++q) {
                const int dx = q % kNearSide - kNearR, dy = q / kNearSide % kNearSide - kNearR,
                          dz = q / (kNearSide * kNearSide) - kNearR;
                float w;
                if constexpr (NEAR_MODE == kTraceNear) {
                    const bool in = (unsigned)(vx + dx) < (unsigned)nx && (unsigned)(vy + dy) < (unsigned)ny &&
                                    (unsigned)(vz + dz) < (unsigned)p.g.nz;
                    w = in ? near_sum[q * kLanes] * near_scale : 0.0f;
                    if constexpr (OP == Op::Norm) {
                        if (near_round) w = __bfloat162float(__float2bfloat16_rn(w));
                        if (round_24) w = round24(w);
                        if (valid && a.near.b16) a.near.b16[cache_base + (size_t)q * kLanes] = __float2bfloat16_rn(w);
                        if (valid && a.near.f32) a.near.f32[cache_base + (size_t)q * kLanes] = w;
                        if (field && valid) {
                            if (a.far.f32) store_weight<kFieldF32>(a.far, pack_slot(gbase, q, lane), w);
                            else if (a.far.b24) store_weight<kField24>(a.far, pack_slot(gbase, q, lane), w);
                            else store_weight<kFieldBF16>(a.far, pack_slot(gbase, q, lane), w);
                        }
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
        long long rbase = gbase + (long long)kNearRow * kLanes;  // Norm: stream block of ray r
        if constexpr (OP == Op::Layout) {
            if (lane == 0) a.len[(size_t)group * p.n_rows] = kNearRow;
            acc = (float)kNearRow;
        }
        for (int r = 0; r < p.n_rays; ++r) {
            const RayStep R = p.far[r];
            if constexpr (OP == Op::Layout) {
                int last = -1;
                march<false, EXACT>(p, R, live, s, vx, vy, vz, [&](int, float, int, int m) { last = m; });
                const int L = (__reduce_max_sync(kFull, last + 1) + kPack - 1) / kPack * kPack;
                if (lane == 0) a.len[(size_t)group * p.n_rows + 1 + r] = (unsigned short)L;
                acc += (float)L;  // exact: totals stay far below 2^24 per group
            } else if constexpr (OP == Op::Norm) {
                march<false, EXACT>(p, R, live, s, vx, vy, vz, [&](int, float w, int, int m) {
                    if (far_round) w = __bfloat162float(__float2bfloat16_rn(w));
                    if (round_24) w = round24(w);
                    acc += w;
                    if (field) {
                        if (a.far.f32) store_weight<kFieldF32>(a.far, pack_slot(rbase, m, lane), w);
                        else if (a.far.b24) store_weight<kField24>(a.far, pack_slot(rbase, m, lane), w);
                        else store_weight<kFieldBF16>(a.far, pack_slot(rbase, m, lane), w);
                    }
                });
                if (field) rbase += (long long)p.src.len[(size_t)group * p.n_rows + 1 + r] * kLanes;
            } else {
                march<false, EXACT>(p, R, live, s, vx, vy, vz, [&](int t, float w, int, int) { deposit(t, w); });
            }
        }
    } else {
        // Stored field.  fp32 and 24-bit: streamed by TMA -- lane 0 keeps kStages bulk copies of kChunk bytes in
        // flight into this warp's shared-memory ring (cp.async.bulk, completion counted by an
        // mbarrier), so the weights arrive as contiguous DRAM bursts without holding
        // registers.  A chunk is consumed in batches of kBatch packs: the packs' template
        // offsets (one int4 broadcast each, addressed by the pack descriptors), the weights
        // from shared memory, then one predicated gather per nonzero weight -- zero padding
        // costs no memory traffic -- or one scatter per nonzero weight without the
        // target-major copy.  Entries of lanes that are not sources are zero by construction.
        // The template offsets are fetched one batch ahead and the descriptors two batches
        // ahead, so the descriptor -> template -> gather chain exposes one memory latency per
        // batch instead of three.
        constexpr bool kGatherT = OP == Op::Forward && target_major(FAR_MODE);
        constexpr int kBase = field_base(FAR_MODE);  // kFieldF32 / kFieldBF16
        constexpr int kElem = kBase == kFieldF32 ? 4 : (kBase == kField24 ? 3 : 2);
        constexpr int kPackBytes = kPack * kLanes * kElem;
#ifndef PRC_FIELD_BATCH
#define PRC_FIELD_BATCH 4
#endif
        constexpr int kBatch = PRC_FIELD_BATCH;  // packs per batch: 16 steps in flight per lane
        // whole batches per ring chunk (24-bit packs of 384 bytes: 4 per 1536-byte chunk)
        constexpr int kPacksPerChunk = kChunk / kPackBytes / kBatch * kBatch;
        constexpr int kChunkBytes = kPacksPerChunk * kPackBytes;
        static_assert(kPacksPerChunk > 0 && kChunkBytes % 16 == 0, "bulk copies of whole 16-byte units");
        const StreamLayout& lay = kGatherT ? p.tgt : p.src;
        const FarField& fld = kGatherT ? a.farT : a.far;
        const int* tmpl = kGatherT ? p.tmpl_neg : p.tmpl;
        const long long e0 = lay.group_base[group], e1 = lay.group_base[group + 1];
        const int* desc = lay.desc + e0 / (kPack * kLanes);
        const int n_packs = (int)((e1 - e0) / (kPack * kLanes));
        // Gathered voxel: source + offset (adjoint) or target - offset (forward).  A 32-bit index
        // (one wide multiply-add per address); the sum wraps only on padding steps (w = 0),
        // whose loads are predicated off, since voxel indices stay below INT_MAX.
        auto gather_index = [&](int o) { return (int)((unsigned)s + (unsigned)o); };
        // the gathered value: the fp32 volume, or the bf16 one of PRC_PRECISION_BF16_VOLUMES
        auto gather = [&](int o) {
            if constexpr (half_volume(FAR_MODE)) return __bfloat162float(__ldg(a.in16 + gather_index(o)));
            else return __ldg(a.in + gather_index(o));
        };
        if constexpr (kBase == kFieldBF16) {
            // bf16 form: each lane loads its own 8-byte vectors straight from HBM (a warp's loads
            // of one pack coalesce into 256 contiguous bytes) one batch ahead of their use.  This
            // form is bound by L1 wavefronts, not bytes, and skipping the shared-memory ring
            // (its copies in and its reads out) measured 5 % faster than the TMA stream.  (The
            // 24-bit form loaded the same way, with a second 4-byte vector per pack, measured
            // within 1.5 % of its TMA stream and is streamed like fp32.)
            const uint2* vec = reinterpret_cast<const uint2*>(fld.b16) + e0 / kPack + lane;
            auto load_vec = [&](int P) {
                uint2 x = make_uint2(0u, 0u);
                if (P < n_packs) x = ld_stream(vec + (size_t)P * kLanes);
                return x;
            };
            auto desc_at = [&](int P) { return P < n_packs ? __ldg(desc + P) : 0; };
            int4 tn[kBatch];
            uint2 wn[kBatch];
            int dq[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) wn[k] = load_vec(k);
#pragma unroll
            for (int k = 0; k < kBatch; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + desc_at(k)));
#pragma unroll
            for (int k = 0; k < kBatch; ++k) dq[k] = desc_at(kBatch + k);
            for (int P0 = 0; P0 < n_packs; P0 += kBatch) {
                int o[kBatch * kPack];
                float w[kBatch * kPack];
                int4 tc[kBatch];
                uint2 wc[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; ++k) tc[k] = tn[k], wc[k] = wn[k];
#pragma unroll
                for (int k = 0; k < kBatch; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + dq[k]));
#pragma unroll
                for (int k = 0; k < kBatch; ++k) wn[k] = load_vec(P0 + kBatch + k);
#pragma unroll
                for (int k = 0; k < kBatch; ++k) dq[k] = desc_at(P0 + 2 * kBatch + k);
#pragma unroll
                for (int k = 0; k < kBatch; ++k) {
                    o[k * kPack] = tc[k].x, o[k * kPack + 1] = tc[k].y, o[k * kPack + 2] = tc[k].z, o[k * kPack + 3] = tc[k].w;
                    w[k * kPack] = __uint_as_float(wc[k].x << 16), w[k * kPack + 1] = __uint_as_float(wc[k].x & 0xffff0000u);
                    w[k * kPack + 2] = __uint_as_float(wc[k].y << 16), w[k * kPack + 3] = __uint_as_float(wc[k].y & 0xffff0000u);
                }
                if constexpr (OP == Op::Adjoint || kGatherT) {
                    float v[kBatch * kPack];
#pragma unroll
                    for (int u = 0; u < kBatch * kPack; ++u) v[u] = w[u] > 0.0f ? gather(o[u]) : 0.0f;
#pragma unroll
                    for (int u = 0; u < kBatch * kPack; ++u) acc = fmaf(w[u], v[u], acc);
                } else {
#pragma unroll
                    for (int u = 0; u < kBatch * kPack; ++u)
                        if (live && w[u] > 0.0f) deposit(s + o[u], w[u]);
                }
            }
        } else {
            unsigned char* ring = dyn_smem + (size_t)warp * kStages * kChunk;
            // a group's stream starts at a multiple of 128 entries: 16-byte aligned in every format
            const char* src_bytes = (kBase == kFieldF32 ? reinterpret_cast<const char*>(fld.f32)
                                     : kBase == kField24 ? reinterpret_cast<const char*>(fld.b24)
                                                         : reinterpret_cast<const char*>(fld.b16)) + e0 * kElem;
            const long long total = (e1 - e0) * kElem;
            const int n_chunks = (n_packs + kPacksPerChunk - 1) / kPacksPerChunk;
            auto issue = [&](int c) {  // lane 0 only
                const int stage = c % kStages;
                const unsigned bytes = (unsigned)min((long long)kChunkBytes, total - (long long)c * kChunkBytes);
                mbar_expect_tx(&bars[stage], bytes);
                bulk_copy_g2s(ring + stage * kChunk, src_bytes + (long long)c * kChunkBytes, bytes, &bars[stage]);
            };
            if (lane == 0) {
                for (int k = 0; k < kStages; ++k) mbar_init(&bars[k], 1);
                fence_mbarrier_init();
                for (int c = 0; c < n_chunks && c < kStages; ++c) issue(c);
            }
            __syncwarp();
            static_assert(kPacksPerChunk % kBatch == 0, "batches stay inside a chunk");
            auto desc_at = [&](int P) { return P < n_packs ? __ldg(desc + P) : 0; };
            int4 tn[kBatch];
            int dq[kBatch];
    #pragma unroll
            for (int k = 0; k < kBatch; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + desc_at(k)));
    #pragma unroll
            for (int k = 0; k < kBatch; ++k) dq[k] = desc_at(kBatch + k);
            bool ok = true;
            for (int c = 0; c < n_chunks; ++c) {
                const int packs = min(kPacksPerChunk, n_packs - c * kPacksPerChunk);
                const int stage = c % kStages;
                if (!mbar_wait_bounded(&bars[stage], (c / kStages) & 1)) {
                    ok = false;
                    break;
                }
                const unsigned char* chunk = ring + stage * kChunk;
                for (int b = 0; b < packs; b += kBatch) {
                    const int P0 = c * kPacksPerChunk + b;
                    int o[kBatch * kPack];
                    float w[kBatch * kPack];
                    int4 tc[kBatch];
    #pragma unroll
                    for (int k = 0; k < kBatch; ++k) tc[k] = tn[k];
    #pragma unroll
                    for (int k = 0; k < kBatch; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + dq[k]));
    #pragma unroll
                    for (int k = 0; k < kBatch; ++k) dq[k] = desc_at(P0 + 2 * kBatch + k);
    #pragma unroll
                    for (int k = 0; k < kBatch; ++k) {
                        const bool here = b + k < packs;
                        const int4 t = tc[k];
                        o[k * kPack] = t.x, o[k * kPack + 1] = t.y, o[k * kPack + 2] = t.z, o[k * kPack + 3] = t.w;
                        if constexpr (kBase == kFieldF32) {
                            const float4 x = here ? reinterpret_cast<const float4*>(chunk + (b + k) * kPackBytes)[lane]
                                                  : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                            w[k * kPack] = x.x, w[k * kPack + 1] = x.y, w[k * kPack + 2] = x.z, w[k * kPack + 3] = x.w;
                        } else if constexpr (kBase == kField24) {
                            const unsigned char* q = chunk + (b + k) * kPackBytes;
                            decode24(here ? reinterpret_cast<const uint2*>(q)[lane] : make_uint2(0u, 0u),
                                     here ? reinterpret_cast<const unsigned*>(q + 256)[lane] : 0u, w + k * kPack);
                        } else {
                            const uint2 x = here ? reinterpret_cast<const uint2*>(chunk + (b + k) * kPackBytes)[lane]
                                                 : make_uint2(0u, 0u);
                            w[k * kPack] = __uint_as_float(x.x << 16), w[k * kPack + 1] = __uint_as_float(x.x & 0xffff0000u);
                            w[k * kPack + 2] = __uint_as_float(x.y << 16), w[k * kPack + 3] = __uint_as_float(x.y & 0xffff0000u);
                        }
                    }
                    if constexpr (OP == Op::Adjoint || kGatherT) {
                        float v[kBatch * kPack];
    #pragma unroll
                        for (int u = 0; u < kBatch * kPack; ++u) v[u] = w[u] > 0.0f ? gather(o[u]) : 0.0f;
    #pragma unroll
                        for (int u = 0; u < kBatch * kPack; ++u) acc = fmaf(w[u], v[u], acc);
                    } else {
    #pragma unroll
                        for (int u = 0; u < kBatch * kPack; ++u)
                            if (live && w[u] > 0.0f) deposit(s + o[u], w[u]);
                    }
                }
                __syncwarp();
                if (lane == 0 && c + kStages < n_chunks) {
                    fence_proxy_async();  // this stage's reads precede the copy that overwrites it
                    issue(c + kStages);
                }
            }
            if (!ok) {
                // A copy did not complete in time: report it, and give the copies still in flight
                // a bounded chance to land before this warp's shared memory is released.
                if (lane == 0) {
                    atomicOr(a.error, 1u);
                    for (int k = 0; k < kStages; ++k) {
                        mbar_wait_bounded(&bars[k], 0);
                        mbar_wait_bounded(&bars[k], 1);
                    }
                }
                __syncwarp();
            }
        }
    }

    if constexpr (OP == Op::Norm) {
        if (valid) a.W[src] = acc;
    } else if constexpr (OP == Op::Layout) {
        if (lane == 0) a.group_total[group] = (long long)acc * kLanes;
    } else if constexpr (OP == Op::Adjoint) {
        if (live) a.out[s] = acc / __ldg(a.W + src);  // prc.cu:266
    } else if constexpr (OP == Op::Forward) {
        if (target_major(FAR_MODE) && valid) {
            // inside MAP-EM the EM ratio of the tissue voxel is taken here (prc.cu:270-274)
            if constexpr (half_volume(FAR_MODE))
                a.out16[s] = __float2bfloat16_rn(__ldg(a.ratio_g + s) / fmaxf(acc, __ldg(a.ratio_eps)));
            else
                a.out[s] = a.ratio_g ? __ldg(a.ratio_g + s) / fmaxf(acc, __ldg(a.ratio_eps)) : acc;
        }
    } else if constexpr (OP == Op::Count) {
        for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(kFull, cnt, off);
        if (lane == 0) atomicAdd(a.count, cnt);
    }
}

// Each warp handles exactly one group per launch, so the mbarriers of its ring are initialised
// once and never reused: walking several groups per warp would need mbarrier.inval and a
// fence.proxy.async before re-initialising them and refilling stages the warp has read.
template <Op OP, bool EXACT, int NEAR_MODE, int FAR_MODE>
__global__ void __launch_bounds__(kMaxBlock) project_kernel(const ProjParams p, const OpArgs a) {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    __shared__ uint64_t field_bars[kMaxWarps][kStages];
    const int warp = threadIdx.x >> 5;
    project_group<OP, EXACT, NEAR_MODE, FAR_MODE>(p, a, blockIdx.x * (blockDim.x >> 5) + warp, warp, dyn_smem,
                                                  field_bars[warp]);
}

template <Op OP, int FAR_MODE>
__device__ __forceinline__ void project_frames_group(const ProjParams& p, const OpArgs& a, const FrameArgs& fr,
                                                     int group, int warp, unsigned char* dyn_smem, uint64_t* bars);

// Batched launch over many volumes: block b belongs to the item (volume) whose first_block is
// the largest one <= b; every item carries its own parameters and projector form.
template <Op OP>
__global__ void __launch_bounds__(kMaxBlock) project_batch_kernel(const BatchItem* items, int n_items) {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    __shared__ uint64_t field_bars[kMaxWarps][kStages];
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first_block <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const ProjParams p = items[lo].p;
    const OpArgs a = items[lo].a;
    const int mode = items[lo].mode;
    const int warp = threadIdx.x >> 5;
    const int group = ((int)blockIdx.x - items[lo].first_block) * (blockDim.x >> 5) + warp;
    uint64_t* bars = field_bars[warp];
    switch (mode) {
        case kBatchTraceMarch: project_group<OP, false, kTraceNear, kMarch>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchCacheF32March: project_group<OP, false, kCacheF32, kMarch>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchCacheBF16March: project_group<OP, false, kCacheBF16, kMarch>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchFieldF32: project_group<OP, false, kTraceNear, kFieldF32>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchFieldBF16: project_group<OP, false, kTraceNear, kFieldBF16>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchFieldF32T: project_group<OP, false, kTraceNear, kFieldF32T>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchFieldBF16T: project_group<OP, false, kTraceNear, kFieldBF16T>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchField24: project_group<OP, false, kTraceNear, kField24>(p, a, group, warp, dyn_smem, bars); break;
        case kBatchField24T: project_group<OP, false, kTraceNear, kField24T>(p, a, group, warp, dyn_smem, bars); break;
        default:
            if constexpr (OP == Op::Forward) {
                if (mode == kBatchFramesF32T) project_frames_group<OP, kFieldF32T>(p, a, items[lo].fr, group, warp, dyn_smem, bars);
                else if (mode == kBatchFramesBF16T) project_frames_group<OP, kFieldBF16T>(p, a, items[lo].fr, group, warp, dyn_smem, bars);
                else if (mode == kBatchFrames24T) project_frames_group<OP, kField24T>(p, a, items[lo].fr, group, warp, dyn_smem, bars);
            } else if constexpr (OP == Op::Adjoint) {
                if (mode == kBatchFramesF32) project_frames_group<OP, kFieldF32>(p, a, items[lo].fr, group, warp, dyn_smem, bars);
                else if (mode == kBatchFramesBF16) project_frames_group<OP, kFieldBF16>(p, a, items[lo].fr, group, warp, dyn_smem, bars);
                else if (mode == kBatchFrames24) project_frames_group<OP, kField24>(p, a, items[lo].fr, group, warp, dyn_smem, bars);
            }
            break;
    }
}

// Up to four frames through one stored field: the gather forms only -- the adjoint over the
// source-major field and the forward over the target-major one (lanes are targets, the gathered
// volume holds each frame's u = f / W).  The gathered volumes are interleaved, fr.in4[t] = the
// four frames' values of voxel t, so ONE 16-byte gather per lane and step fetches every frame:
// the same cache lines, hence the same L1 wavefronts, as one frame's 4-byte gather (the L1 data
// pipe is what bounds these kernels).  The stream is consumed exactly as project_group consumes
// it (the bf16 vectors loaded by the lanes, the fp32 and 24-bit packs through the per-warp TMA
// ring); each pack's weights, template offsets and w > 0 predicates serve all four frames.  One
// pack per batch keeps 16 gathered values in flight per lane, as the single-volume kernel.  Each
// frame accumulates its terms in stream order with fmaf, as project_group does, so every frame
// equals its single-volume projection bit for bit.  Slots fr.n..3 are padding (gathered zeros,
// nothing written).
template <Op OP, int FAR_MODE>
__device__ __forceinline__ void project_frames_group(const ProjParams& p, const OpArgs& a, const FrameArgs& fr,
                                                     int group, int warp, unsigned char* dyn_smem, uint64_t* bars) {
    static_assert(OP == Op::Adjoint ? !target_major(FAR_MODE) : (OP == Op::Forward && target_major(FAR_MODE)),
                  "gather forms only");
    static_assert(!half_volume(FAR_MODE) && FAR_MODE != kMarch, "fp32 volumes through a stored field");
    constexpr int NF = kMaxFrames;  // the interleaved width: one float4 per voxel
    static_assert(NF == 4, "frames are interleaved four to a 16-byte vector");
    const int lane = threadIdx.x & 31;
    if (group * kLanes >= p.n_active) return;  // the whole warp leaves together
    const int src = group * kLanes + lane;
    const bool valid = src < p.n_active;
    const int s = valid ? __ldg(p.active + src) : 0;
    bool live = valid;
    if constexpr (OP == Op::Adjoint) {  // prc.cu:260-264
        const float ws = valid ? __ldg(a.W + src) : 0.0f;
        live = valid && ws > 0.0f;
        if (valid && !live)
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < fr.n) fr.out[f][s] = 0.0f;
    }
    if (!__any_sync(kFull, live)) return;

    constexpr bool kT = target_major(FAR_MODE);
    constexpr int kBase = field_base(FAR_MODE);
    constexpr int kElem = kBase == kFieldF32 ? 4 : (kBase == kField24 ? 3 : 2);
    constexpr int kPackBytes = kPack * kLanes * kElem;
    constexpr int kB = 1;  // packs per batch: 4 steps x 4 frames of gathered values in flight
    constexpr int kPacksPerChunk = kChunk / kPackBytes / kB * kB;
    constexpr int kChunkBytes = kPacksPerChunk * kPackBytes;
    static_assert(kPacksPerChunk > 0 && kChunkBytes % 16 == 0, "bulk copies of whole 16-byte units");
    const StreamLayout& lay = kT ? p.tgt : p.src;
    const FarField& fld = kT ? a.farT : a.far;
    const int* tmpl = kT ? p.tmpl_neg : p.tmpl;
    const long long e0 = lay.group_base[group], e1 = lay.group_base[group + 1];
    const int* desc = lay.desc + e0 / (kPack * kLanes);
    const int n_packs = (int)((e1 - e0) / (kPack * kLanes));
    auto desc_at = [&](int P) { return P < n_packs ? __ldg(desc + P) : 0; };
    float acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f] = 0.0f;
    // One batch: kB packs of template offsets tc and weights w (a zero weight is padding: no load).
    auto consume = [&](const int4* tc, const float* w) {
        int idx[kB * kPack];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
            idx[k * kPack] = (int)((unsigned)s + (unsigned)tc[k].x), idx[k * kPack + 1] = (int)((unsigned)s + (unsigned)tc[k].y);
            idx[k * kPack + 2] = (int)((unsigned)s + (unsigned)tc[k].z), idx[k * kPack + 3] = (int)((unsigned)s + (unsigned)tc[k].w);
        }
        float4 v[kB * kPack];
#pragma unroll
        for (int u = 0; u < kB * kPack; ++u)
            v[u] = w[u] > 0.0f ? __ldg(fr.in4 + idx[u]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int u = 0; u < kB * kPack; ++u) {
            acc[0] = fmaf(w[u], v[u].x, acc[0]);
            acc[1] = fmaf(w[u], v[u].y, acc[1]);
            acc[2] = fmaf(w[u], v[u].z, acc[2]);
            acc[3] = fmaf(w[u], v[u].w, acc[3]);
        }
    };

    if constexpr (kBase == kFieldBF16) {
        const uint2* vec = reinterpret_cast<const uint2*>(fld.b16) + e0 / kPack + lane;
        auto load_vec = [&](int P) {
            uint2 x = make_uint2(0u, 0u);
            if (P < n_packs) x = ld_stream(vec + (size_t)P * kLanes);
            return x;
        };
        int4 tn[kB];
        uint2 wn[kB];
        int dq[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) wn[k] = load_vec(k);
#pragma unroll
        for (int k = 0; k < kB; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + desc_at(k)));
#pragma unroll
        for (int k = 0; k < kB; ++k) dq[k] = desc_at(kB + k);
        for (int P0 = 0; P0 < n_packs; P0 += kB) {
            float w[kB * kPack];
            int4 tc[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                tc[k] = tn[k];
                w[k * kPack] = __uint_as_float(wn[k].x << 16), w[k * kPack + 1] = __uint_as_float(wn[k].x & 0xffff0000u);
                w[k * kPack + 2] = __uint_as_float(wn[k].y << 16), w[k * kPack + 3] = __uint_as_float(wn[k].y & 0xffff0000u);
            }
#pragma unroll
            for (int k = 0; k < kB; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + dq[k]));
#pragma unroll
            for (int k = 0; k < kB; ++k) wn[k] = load_vec(P0 + kB + k);
#pragma unroll
            for (int k = 0; k < kB; ++k) dq[k] = desc_at(P0 + 2 * kB + k);
            consume(tc, w);
        }
    } else {
        unsigned char* ring = dyn_smem + (size_t)warp * kStages * kChunk;
        // a group's stream starts at a multiple of 128 entries: 16-byte aligned in every format
        const char* src_bytes = (kBase == kFieldF32 ? reinterpret_cast<const char*>(fld.f32)
                                                    : reinterpret_cast<const char*>(fld.b24)) + e0 * kElem;
        const long long total = (e1 - e0) * kElem;
        const int n_chunks = (n_packs + kPacksPerChunk - 1) / kPacksPerChunk;
        auto issue = [&](int c) {  // lane 0 only
            const int stage = c % kStages;
            const unsigned bytes = (unsigned)min((long long)kChunkBytes, total - (long long)c * kChunkBytes);
            mbar_expect_tx(&bars[stage], bytes);
            bulk_copy_g2s(ring + stage * kChunk, src_bytes + (long long)c * kChunkBytes, bytes, &bars[stage]);
        };
        if (lane == 0) {
            for (int k = 0; k < kStages; ++k) mbar_init(&bars[k], 1);
            fence_mbarrier_init();
            for (int c = 0; c < n_chunks && c < kStages; ++c) issue(c);
        }
        __syncwarp();
        int4 tn[kB];
        int dq[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + desc_at(k)));
#pragma unroll
        for (int k = 0; k < kB; ++k) dq[k] = desc_at(kB + k);
        bool ok = true;
        for (int c = 0; c < n_chunks; ++c) {
            const int packs = min(kPacksPerChunk, n_packs - c * kPacksPerChunk);
            const int stage = c % kStages;
            if (!mbar_wait_bounded(&bars[stage], (c / kStages) & 1)) {
                ok = false;
                break;
            }
            const unsigned char* chunk = ring + stage * kChunk;
            for (int b = 0; b < packs; b += kB) {
                const int P0 = c * kPacksPerChunk + b;
                float w[kB * kPack];
                int4 tc[kB];
#pragma unroll
                for (int k = 0; k < kB; ++k) tc[k] = tn[k];
#pragma unroll
                for (int k = 0; k < kB; ++k) tn[k] = __ldg(reinterpret_cast<const int4*>(tmpl + dq[k]));
#pragma unroll
                for (int k = 0; k < kB; ++k) dq[k] = desc_at(P0 + 2 * kB + k);
#pragma unroll
                for (int k = 0; k < kB; ++k) {
                    const bool here = b + k < packs;
                    if constexpr (kBase == kFieldF32) {
                        const float4 x = here ? reinterpret_cast<const float4*>(chunk + (b + k) * kPackBytes)[lane]
                                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        w[k * kPack] = x.x, w[k * kPack + 1] = x.y, w[k * kPack + 2] = x.z, w[k * kPack + 3] = x.w;
                    } else {
                        const unsigned char* q = chunk + (b + k) * kPackBytes;
                        decode24(here ? reinterpret_cast<const uint2*>(q)[lane] : make_uint2(0u, 0u),
                                 here ? reinterpret_cast<const unsigned*>(q + 256)[lane] : 0u, w + k * kPack);
                    }
                }
                consume(tc, w);
            }
            __syncwarp();
            if (lane == 0 && c + kStages < n_chunks) {
                fence_proxy_async();  // this stage's reads precede the copy that overwrites it
                issue(c + kStages);
            }
        }
        if (!ok) {
            // A copy did not complete in time: report it, and give the copies still in flight
            // a bounded chance to land before this warp's shared memory is released.
            if (lane == 0) {
                atomicOr(a.error, 1u);
                for (int k = 0; k < kStages; ++k) {
                    mbar_wait_bounded(&bars[k], 0);
                    mbar_wait_bounded(&bars[k], 1);
                }
            }
            __syncwarp();
        }
    }

    if constexpr (OP == Op::Adjoint) {
        if (live) {
            const float ws = __ldg(a.W + src);
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < fr.n) fr.out[f][s] = acc[f] / ws;  // prc.cu:266
        }
    } else if (valid) {
        float r[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f)  // inside MAP-EM the EM ratio (prc.cu:270-274)
            r[f] = f >= fr.n ? 0.0f
                             : (fr.ratio_g[f] ? __ldg(fr.ratio_g[f] + s) / fmaxf(acc[f], __ldg(fr.ratio_eps[f])) : acc[f]);
        if (fr.out4) {
            fr.out4[s] = make_float4(r[0], r[1], r[2], r[3]);
        } else {
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < fr.n) fr.out[f][s] = r[f];
        }
    }
}

// 64 registers at most (four 256-thread blocks per SM), as the single-volume stream kernel.
template <Op OP, int FAR_MODE>
__global__ void __launch_bounds__(kMaxBlock, 4) project_frames_kernel(const ProjParams p, const OpArgs a,
                                                                      const FrameArgs fr) {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    __shared__ uint64_t field_bars[kMaxWarps][kStages];
    const int warp = threadIdx.x >> 5;
    project_frames_group<OP, FAR_MODE>(p, a, fr, blockIdx.x * (blockDim.x >> 5) + warp, warp, dyn_smem,
                                       field_bars[warp]);
}

// Template rows: row 0 the near block's 125 offsets (then zeros), rows 1..n_rays the offsets of
// the post-block steps of each far ray, from the same uniform DDA the march performs.
__global__ void template_kernel(const ProjParams p, int* tmpl) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0)
        for (int q = 0; q < p.tmpl_len; ++q) tmpl[q] = q < kNear ? near_offset(p, q) : 0;
    if (r >= p.n_rays) return;
    const RayStep R = p.far[r];
    float tx = R.tx, ty = R.ty, tz = R.tz;
    int oi = 0, oj = 0, ok = 0, m = 0;
    int* out = tmpl + (size_t)(r + 1) * p.tmpl_len;
    for (int step = 0; m < p.tmpl_len && step < 4 * p.tmpl_len; ++step) {
        const bool in_block = abs(oi) <= kNearR && abs(oj) <= kNearR && abs(ok) <= kNearR;
        if (!in_block) out[m++] = (ok * p.g.ny + oj) * p.g.nx + oi;
        const float t_next = fminf(tx, fminf(ty, tz));
        if (t_next == tx) oi += R.di, tx += R.dtx;
        else if (t_next == ty) oj += R.dj, ty += R.dty;
        else ok += R.dk, tz += R.dtz;
    }
}

// Pack descriptors of every group: the template element offset of each pack's first step.
__global__ void desc_kernel(const ProjParams p, const StreamLayout l, int* desc) {
    const int group = blockIdx.x * blockDim.x + threadIdx.x;
    if (group * kLanes >= p.n_active) return;
    const unsigned short* len = l.len + (size_t)group * p.n_rows;
    int* out = desc + l.group_base[group] / (kPack * kLanes);
    for (int row = 0; row < p.n_rows; ++row)
        for (int m = 0; m < len[row]; m += kPack) *out++ = row * p.tmpl_len + m;
}

// Walks every stored source-major entry w > 0 of a group (lane = source s, template row k,
// step m, target t = s + o).  FILL = false: raises len_t32[group(t)][k] to cover step m.
// FILL = true: copies w into the target-major field at (group(t), row k, step m, lane(t)).
template <bool FILL, int FAR_MODE>
__global__ void __launch_bounds__(kBlock) transpose_kernel(const ProjParams p, const FarField far, const FarField farT,
                                                           int* len_t32, const int* row_base_t) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int group = blockIdx.x * kWarps + warp;
    if (group * kLanes >= p.n_active) return;
    const int src = group * kLanes + lane;
    const bool valid = src < p.n_active;
    const int s = valid ? p.active[src] : 0;
    const unsigned short* len = p.src.len + (size_t)group * p.n_rows;
    long long row_base = p.src.group_base[group];
    for (int k = 0; k < p.n_rows; ++k) {
        const int L = len[k];
        for (int m = 0; m < L; ++m) {
            const long long e = pack_slot(row_base, m, lane);
            float w = 0.0f;
            if (valid) {
                if constexpr (FAR_MODE == kFieldF32) w = far.f32[e];
                else if constexpr (FAR_MODE == kField24) w = load24(far.b24, e);
                else w = __bfloat162float(far.b16[e]);
            }
            const bool dep = valid && w > 0.0f;
            int tsrc = -1;
            if (dep) tsrc = p.vox2src[s + p.tmpl[(size_t)k * p.tmpl_len + m]];
            if constexpr (!FILL) {
                const int key = dep ? (tsrc >> 5) : -1;
                const unsigned same = __match_any_sync(kFull, key);
                if (dep && lane == __ffs(same) - 1) atomicMax(len_t32 + (size_t)key * p.n_rows + k, m + 1);
            } else {
                if (dep) {
                    const int tg = tsrc >> 5, tl = tsrc & 31;
                    const long long et = pack_slot(p.tgt.group_base[tg] + row_base_t[(size_t)tg * p.n_rows + k], m, tl);
                    if constexpr (FAR_MODE == kFieldF32) farT.f32[et] = far.f32[e];
                    else if constexpr (FAR_MODE == kField24) store24(farT.b24, et, bits24(w));  // w is exact in 24 bits
                    else farT.b16[et] = far.b16[e];
                }
            }
        }
        row_base += (long long)L * kLanes;
    }
}

__global__ void forward_prep_kernel(const int* __restrict__ vox2src, const float* __restrict__ W,
                                    const float* __restrict__ f, float* __restrict__ u, float* __restrict__ out,
                                    size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int src = vox2src[i];
        float scale = 0.0f;
        if (src >= 0) {
            const float ws = W[src], fs = f[i];
            scale = ws > 0.0f ? fs / ws : 0.0f;  // prc.cu:246
        } else {
            out[i] = 0.0f;
        }
        u[i] = scale > 0.0f ? scale : 0.0f;
    }
}

// forward_prep with the Biggs-Andrews prediction of the same voxels folded in: one pass reads f
// and prev, writes y, and prepares u = y / W for the gather (four voxels per step when every
// pointer is 16-byte aligned; each voxel computed by the same expressions either way).
__global__ void forward_prep_extrapolate_kernel(const int* __restrict__ vox2src, const float* __restrict__ W,
                                                const float* __restrict__ f, const float* __restrict__ prev,
                                                const float* __restrict__ lambda_p, float* __restrict__ y,
                                                float* __restrict__ u, float* __restrict__ out, size_t n) {
    const float lambda = __ldg(lambda_p);
    auto one = [&](size_t i, float fi, float pi, int src, float& yi, float& ui) {
        yi = fmaxf(fi + lambda * (fi - pi), 0.5f * fi);  // prc.cu:320
        float scale = 0.0f;
        if (src >= 0) {
            const float ws = __ldg(W + src);
            scale = ws > 0.0f ? yi / ws : 0.0f;  // prc.cu:246
        } else {
            out[i] = 0.0f;
        }
        ui = scale > 0.0f ? scale : 0.0f;
    };
    const bool vec = ((uintptr_t)f | (uintptr_t)prev | (uintptr_t)y | (uintptr_t)u | (uintptr_t)vox2src) % 16 == 0;
    const size_t n4 = vec ? n / 4 : 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n4; q += stride) {
        const float4 a = reinterpret_cast<const float4*>(f)[q], b = reinterpret_cast<const float4*>(prev)[q];
        const int4 s4 = reinterpret_cast<const int4*>(vox2src)[q];
        float4 yv, uv;
        one(4 * q, a.x, b.x, s4.x, yv.x, uv.x);
        one(4 * q + 1, a.y, b.y, s4.y, yv.y, uv.y);
        one(4 * q + 2, a.z, b.z, s4.z, yv.z, uv.z);
        one(4 * q + 3, a.w, b.w, s4.w, yv.w, uv.w);
        reinterpret_cast<float4*>(y)[q] = yv;
        reinterpret_cast<float4*>(u)[q] = uv;
    }
    for (size_t i = 4 * n4 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        float yi, ui;
        one(i, f[i], prev[i], vox2src[i], yi, ui);
        y[i] = yi;
        u[i] = ui;
    }
}

// The preparation of the mixed-precision form: the same prediction (PREDICT) and u = y / W, with
// u rounded to bf16 for the bf16 gather.  Every voxel's expressions are those of
// forward_prep_extrapolate_kernel; u16 is 0 off the support.
template <bool PREDICT>
__global__ void forward_prep_half_kernel(const int* __restrict__ vox2src, const float* __restrict__ W,
                                         const float* __restrict__ f, const float* __restrict__ prev,
                                         const float* __restrict__ lambda_p, float* __restrict__ y,
                                         __nv_bfloat16* __restrict__ u16, size_t n) {
    const float lambda = PREDICT ? __ldg(lambda_p) : 0.0f;
    auto one = [&](float fi, float pi, int src, float& yi) {
        yi = PREDICT ? fmaxf(fi + lambda * (fi - pi), 0.5f * fi) : fi;  // prc.cu:320
        float scale = 0.0f;
        if (src >= 0) {
            const float ws = __ldg(W + src);
            scale = ws > 0.0f ? yi / ws : 0.0f;  // prc.cu:246
        }
        return __float2bfloat16_rn(scale > 0.0f ? scale : 0.0f);
    };
    const bool vec = ((uintptr_t)f | (uintptr_t)prev | (uintptr_t)y | (uintptr_t)vox2src) % 16 == 0 &&
                     (uintptr_t)u16 % 8 == 0;
    const size_t n4 = vec ? n / 4 : 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n4; q += stride) {
        const float4 a = reinterpret_cast<const float4*>(f)[q];
        const float4 b = PREDICT ? reinterpret_cast<const float4*>(prev)[q] : a;
        const int4 s4 = reinterpret_cast<const int4*>(vox2src)[q];
        float4 yv;
        __nv_bfloat162 lo, hi;
        lo.x = one(a.x, b.x, s4.x, yv.x);
        lo.y = one(a.y, b.y, s4.y, yv.y);
        hi.x = one(a.z, b.z, s4.z, yv.z);
        hi.y = one(a.w, b.w, s4.w, yv.w);
        if (PREDICT) reinterpret_cast<float4*>(y)[q] = yv;
        uint2 packed;
        packed.x = *reinterpret_cast<const unsigned*>(&lo);
        packed.y = *reinterpret_cast<const unsigned*>(&hi);
        reinterpret_cast<uint2*>(u16)[q] = packed;
    }
    for (size_t i = 4 * n4 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        float yi;
        u16[i] = one(f[i], PREDICT ? prev[i] : f[i], vox2src[i], yi);
        if (PREDICT) y[i] = yi;
    }
}

// ---- radial surrogate ------------------------------------------------------------------------
// kWaterBins equal bins up to the cutoff, the rest equal up to 3.85 x cutoff.  A surrogate field
// stores the water bins of a ray (whole packs of 4 steps).
constexpr int kWaterBins = 12;
static_assert(kWaterBins % 4 == 0 && kWaterBins < kRadialBins, "the water bins fill whole packs");
__device__ __forceinline__ float radial_edge(int b, float cutoff) {
    return b <= kWaterBins ? cutoff * b / kWaterBins
                           : cutoff * (1.0f + 2.85f * (b - kWaterBins) / (kRadialBins - kWaterBins));
}
__device__ __forceinline__ int radial_bin(float t, float cutoff) {
    int b = t < cutoff ? (int)(t / cutoff * kWaterBins)
                       : kWaterBins + (int)((t / cutoff - 1.0f) / 2.85f * (kRadialBins - kWaterBins));
    return b < 0 ? 0 : (b > kRadialBins - 1 ? kRadialBins - 1 : b);
}

// Per far ray: the bin of every post-block step, and for every bin the step whose midpoint is
// closest to the bin centre (its target offset, plain and packed by component).
__global__ void radial_setup_kernel(const ProjParams p, RadialTables tab) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= p.n_rays) return;
    const RayStep R = p.far[r];
    float tx = R.tx, ty = R.ty, tz = R.tz, t = 0.0f;
    int oi = 0, oj = 0, ok = 0, m = 0;
    float best[kRadialBins];
    int best_off[kRadialBins], best_xyz[kRadialBins];
    for (int b = 0; b < kRadialBins; ++b) best[b] = 3.0e38f, best_off[b] = 0, best_xyz[b] = 512 | (512 << 10) | (512 << 20);
    const float cutoff = p.g.cutoff;
    for (int step = 0; m < p.tmpl_len && step < 4 * p.tmpl_len; ++step) {
        const bool in_block = abs(oi) <= kNearR && abs(oj) <= kNearR && abs(ok) <= kNearR;
        const float t_next = fminf(tx, fminf(ty, tz));
        if (!in_block) {
            const float mid = 0.5f * (t + t_next);
            tab.bin_of[(size_t)r * p.tmpl_len + m] = (unsigned char)radial_bin(mid, cutoff);
            for (int b = 0; b < kRadialBins; ++b) {
                const float centre = 0.5f * (radial_edge(b, cutoff) + radial_edge(b + 1, cutoff));
                if (fabsf(mid - centre) < best[b] && abs(oi) < 512 && abs(oj) < 512 && abs(ok) < 512) {
                    best[b] = fabsf(mid - centre);
                    best_off[b] = (ok * p.g.ny + oj) * p.g.nx + oi;
                    best_xyz[b] = (oi + 512) | ((oj + 512) << 10) | ((ok + 512) << 20);
                }
            }
            ++m;
        }
        t = t_next;
        if (t_next == tx) oi += R.di, tx += R.dtx;
        else if (t_next == ty) oj += R.dj, ty += R.dty;
        else ok += R.dk, tz += R.dtz;
    }
    for (int b = 0; b < kRadialBins; ++b) {
        tab.offset[r * kRadialBins + b] = best_off[b];
        tab.xyz[r * kRadialBins + b] = best_xyz[b];
    }
}

template <bool EXACT>
__global__ void __launch_bounds__(kBlock) radial_kernel_kernel(ProjParams p, const RadialTables tab, const int* src,
                                                               int n_src, int warps_per_volume, float* out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * kWarps + warp;
    if (w * kLanes >= n_src) return;
    p.rho += (size_t)(w / warps_per_volume) * p.nxy * p.g.nz;
    const int i = w * kLanes + lane;
    const int s = src[i];
    const int vx = s % p.g.nx, vy = (s / p.g.nx) % p.g.ny, vz = s / p.nxy;
    for (int r = 0; r < p.n_rays; ++r) {
        float c[kRadialBins];
#pragma unroll
        for (int b = 0; b < kRadialBins; ++b) c[b] = 0.0f;
        const unsigned char* bins = tab.bin_of + (size_t)r * p.tmpl_len;
        march<false, EXACT>(p, p.far[r], true, s, vx, vy, vz, [&](int, float wdep, int, int m) {
            const int b = bins[m];
#pragma unroll
            for (int k = 0; k < kRadialBins; ++k)
                if (k == b) c[k] += wdep;
        });
        float4* o = reinterpret_cast<float4*>(out + ((size_t)i * p.n_rays + r) * kRadialBins);
#pragma unroll
        for (int k = 0; k < kRadialBins / 4; ++k) o[k] = make_float4(c[4 * k], c[4 * k + 1], c[4 * k + 2], c[4 * k + 3]);
    }
}

// Surrogate field fill (see engine.h); the near block exactly as the Norm pass traces it, then
// every far ray either marched exactly (a ray the judge sent back, stored in its exact row as
// the Norm pass stores it) or as its radial water bins.  The rows go in stream order: all exact
// rows 1..n_rays, then all radial rows; a row the group does not use has length 0.
template <bool EXACT, int FAR_MODE>
__global__ void __launch_bounds__(kBlock) surrogate_fill_kernel(const ProjParams p, const OpArgs a,
                                                                const RadialTables tab, const __nv_bfloat16* coef,
                                                                const unsigned char* support,
                                                                const unsigned char* fallback_rays, int water_bins) {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int group = blockIdx.x * kWarps + warp;
    if (group * kLanes >= p.n_active) return;
    const int src = group * kLanes + lane;
    const bool valid = src < p.n_active;
    const int s = valid ? p.active[src] : 0;
    const int nx = p.g.nx, ny = p.g.ny, nz = p.g.nz;
    const int vx = s % nx, vy = (s / nx) % ny, vz = s / p.nxy;
    const FarField& f = a.far;
    const long long gbase = p.src.group_base[group];
    const unsigned char* fb = fallback_rays + (size_t)group * p.n_rays;
    const unsigned short* len = p.src.len + (size_t)group * p.n_rows;
    float acc = 0.0f;
    const float* near_sum;
    if (a.near_acc) {
        float* acc_col = a.near_acc + (size_t)group * kNear * kLanes + lane;
        trace_near_octants<EXACT>(p, valid, s, vx, vy, vz, warp, lane, dyn_smem, acc_col);
        near_sum = acc_col;
    } else {
        float* sum = reinterpret_cast<float*>(dyn_smem) + warp * (kNear * kLanes);
        for (int q = 0; q < kNear; ++q) sum[q * kLanes + lane] = 0.0f;
        for (int r = 0; r < kNearRays; ++r)
            march<true, EXACT>(p, p.near[r], valid, s, vx, vy, vz,
                               [&](int, float w, int q, int) { sum[q * kLanes + lane] += w; });
        near_sum = sum + lane;
    }
    const float near_scale = (float)p.n_rays / kNearRays;
    for (int q = 0; q < kNear; ++q) {
        const int dx = q % kNearSide - kNearR, dy = q / kNearSide % kNearSide - kNearR,
                  dz = q / (kNearSide * kNearSide) - kNearR;
        const bool in = (unsigned)(vx + dx) < (unsigned)nx && (unsigned)(vy + dy) < (unsigned)ny &&
                        (unsigned)(vz + dz) < (unsigned)nz;
        float w = in ? near_sum[q * kLanes] * near_scale : 0.0f;
        if (FAR_MODE == kFieldBF16) w = __bfloat162float(__float2bfloat16_rn(w));
        acc += w;
        if (valid) store_weight<FAR_MODE>(f, pack_slot(gbase, q, lane), w);
    }
    long long rbase = gbase + (long long)kNearRow * kLanes;
    for (int r = 0; r < p.n_rays; ++r) {  // exact rows (prc.cu:220-226 as the Norm pass marches them)
        if (fb[r]) {
            march<false, EXACT>(p, p.far[r], valid, s, vx, vy, vz, [&](int, float w, int, int m) {
                if (FAR_MODE == kFieldBF16) w = __bfloat162float(__float2bfloat16_rn(w));
                acc += w;
                store_weight<FAR_MODE>(f, pack_slot(rbase, m, lane), w);
            });
        }
        rbase += (long long)len[1 + r] * kLanes;
    }
    for (int r = 0; r < p.n_rays; ++r) {  // radial rows
        if (!fb[r]) {
            for (int b = 0; b < water_bins; ++b) {
                const int xyz = tab.xyz[r * kRadialBins + b];
                const int dx = (xyz & 1023) - 512, dy = ((xyz >> 10) & 1023) - 512, dz = ((xyz >> 20) & 1023) - 512;
                const bool in = (unsigned)(vx + dx) < (unsigned)nx && (unsigned)(vy + dy) < (unsigned)ny &&
                                (unsigned)(vz + dz) < (unsigned)nz;
                float w = 0.0f;
                if (valid && in && support[s + tab.offset[r * kRadialBins + b]])
                    w = fmaxf(__bfloat162float(coef[(size_t)src * (p.n_rays * kRadialBins) + r * kRadialBins + b]), 0.0f);
                if (FAR_MODE == kFieldBF16) w = __bfloat162float(__float2bfloat16_rn(w));
                acc += w;
                if (valid) store_weight<FAR_MODE>(f, pack_slot(rbase, b, lane), w);
            }
        }
        rbase += (long long)len[1 + p.n_rays + r] * kLanes;
    }
    if (valid) a.W[src] = acc;
}

// Rows 1 + n_rays + r of the template: the 16 bin offsets of far ray r (rows 0..n_rays are the
// near block and the exact ray steps, from template_kernel).
__global__ void surrogate_template_kernel(const ProjParams p, const int* offset, int* tmpl) {
    const int r = blockIdx.x;
    for (int j = threadIdx.x; j < p.tmpl_len; j += blockDim.x)
        tmpl[(size_t)(1 + p.n_rays + r) * p.tmpl_len + j] = j < kRadialBins ? offset[r * kRadialBins + j] : 0;
}

// The interleaved input of a frame pass: per voxel and frame the expressions of
// forward_prep_kernel (PREDICT false: y = f) or forward_prep_extrapolate_kernel (PREDICT true),
// the frames' u = y / W stored side by side in one 16-byte vector (zeros in the unused slots).
template <bool PREDICT>
__global__ void frame_prep_kernel(const int* __restrict__ vox2src, const float* __restrict__ W, const FramePrep fp,
                                  float4* __restrict__ u4, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int src = vox2src[i];
        const float ws = src >= 0 ? __ldg(W + src) : 0.0f;
        float u[kMaxFrames];
#pragma unroll
        for (int k = 0; k < kMaxFrames; ++k) {
            u[k] = 0.0f;
            if (k >= fp.n) continue;
            const float fi = fp.f[k][i];
            float yi = fi;
            if constexpr (PREDICT) {
                const float lambda = __ldg(fp.lambda[k]), pi = fp.prev[k][i];
                yi = fmaxf(fi + lambda * (fi - pi), 0.5f * fi);  // prc.cu:320
                fp.y[k][i] = yi;
            }
            float scale = 0.0f;
            if (src >= 0) scale = ws > 0.0f ? yi / ws : 0.0f;  // prc.cu:246
            else fp.out[k][i] = 0.0f;
            u[k] = scale > 0.0f ? scale : 0.0f;
        }
        u4[i] = make_float4(u[0], u[1], u[2], u[3]);
    }
}

// The frames' volumes fp.f[k] side by side, one 16-byte vector per voxel.
__global__ void frame_pack_kernel(const FramePrep fp, float4* __restrict__ v4, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v[kMaxFrames];
#pragma unroll
        for (int k = 0; k < kMaxFrames; ++k) v[k] = k < fp.n ? __ldg(fp.f[k] + i) : 0.0f;
        v4[i] = make_float4(v[0], v[1], v[2], v[3]);
    }
}

__global__ void forward_prep_batch_kernel(const PrepItem* items) {
    const PrepItem it = items[blockIdx.y];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < it.n; i += (long long)gridDim.x * blockDim.x) {
        if (!it.gather) {
            it.out[i] = 0.0f;
            continue;
        }
        const int src = it.vox2src[i];
        float scale = 0.0f;
        if (src >= 0) {
            const float ws = it.W[src], fs = it.f[i];
            scale = ws > 0.0f ? fs / ws : 0.0f;  // prc.cu:246
        } else {
            it.out[i] = 0.0f;
        }
        const float u = scale > 0.0f ? scale : 0.0f;
        if (it.u4) reinterpret_cast<float*>(it.u4)[4 * i + it.slot] = u;
        else it.u[i] = u;
    }
}

template <Op OP, bool EXACT, int NEAR_MODE, int FAR_MODE>
cudaError_t launch(const ProjParams& p, const OpArgs& a, cudaStream_t s) {
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    const int blocks = (groups + kWarps - 1) / kWarps;
    if (blocks == 0) return cudaSuccess;
    size_t smem = 0;
    // the stored field's ring (the near block is in the field)
    if (FAR_MODE != kMarch) smem = kFieldSmemBytes;
    else if (NEAR_MODE == kTraceNear && OP != Op::Layout)
        smem = OP == Op::Norm && a.near_acc ? size_t(kWarps) * 27 * kLanes * sizeof(float) : kNearSmemBytes;
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
        if constexpr (OP == Op::Forward || OP == Op::Adjoint) {
            if (a.in16) {  // bf16 volumes inside MAP-EM (the bf16 field only)
                if (OP == Op::Forward && a.farT.b16 && a.out16) return launch<OP, EXACT, kTraceNear, kFieldBF16TH>(p, a, s);
                if (OP == Op::Adjoint && a.far.b16) return launch<OP, EXACT, kTraceNear, kFieldBF16H>(p, a, s);
                return cudaErrorInvalidValue;
            }
        }
        if (OP == Op::Forward && a.farT.f32) return launch<OP, EXACT, kTraceNear, kFieldF32T>(p, a, s);
        if (OP == Op::Forward && a.farT.b24) return launch<OP, EXACT, kTraceNear, kField24T>(p, a, s);
        if (OP == Op::Forward && a.farT.b16) return launch<OP, EXACT, kTraceNear, kFieldBF16T>(p, a, s);
        if (a.far.f32) return launch<OP, EXACT, kTraceNear, kFieldF32>(p, a, s);
        if (a.far.b24) return launch<OP, EXACT, kTraceNear, kField24>(p, a, s);
        if (a.far.b16) return launch<OP, EXACT, kTraceNear, kFieldBF16>(p, a, s);
        if (trace_near || !a.near.on()) return launch<OP, EXACT, kTraceNear, kMarch>(p, a, s);
        if (a.near.b16) return launch<OP, EXACT, kCacheBF16, kMarch>(p, a, s);
        return launch<OP, EXACT, kCacheF32, kMarch>(p, a, s);
    }
}

template <Op OP>
cudaError_t launch_op(const ProjParams& p, const OpArgs& a, bool trace_near, cudaStream_t s) {
    return p.table ? launch_modes<OP, false>(p, a, trace_near, s) : launch_modes<OP, true>(p, a, trace_near, s);
}

}  // namespace

cudaError_t order_near_rays(const RayStep* d_near, short* d_order, int* d_start, cudaStream_t s) {
    order_near_kernel<<<1, 32, 0, s>>>(d_near, d_order, d_start);
    return cudaGetLastError();
}

cudaError_t setup_rays(const Grid& g, int n_rays, RayStep* d_far, RayStep* d_near, cudaStream_t s) {
    const int n = n_rays > kNearRays ? n_rays : kNearRays;
    ray_setup_kernel<<<(n + 127) / 128, 128, 0, s>>>(g, n_rays, d_far, d_near);
    return cudaGetLastError();
}

__global__ void negate_kernel(const int* in, int* out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = -in[i];
}

cudaError_t build_template(const ProjParams& p, int* tmpl, int* tmpl_neg, cudaStream_t s) {
    template_kernel<<<(p.n_rays + 128) / 128, 128, 0, s>>>(p, tmpl);
    negate_kernel<<<256, 256, 0, s>>>(tmpl, tmpl_neg, (size_t)p.n_rows * p.tmpl_len);
    return cudaGetLastError();
}

cudaError_t build_descriptors(const ProjParams& p, const StreamLayout& l, int* desc, cudaStream_t s) {
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    if (groups == 0) return cudaSuccess;
    desc_kernel<<<(groups + 127) / 128, 128, 0, s>>>(p, l, desc);
    return cudaGetLastError();
}

cudaError_t transpose_lengths(const ProjParams& p, const FarField& far, int* len_t32, cudaStream_t s) {
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    if (groups == 0) return cudaSuccess;
    if (far.f32) transpose_kernel<false, kFieldF32><<<(groups + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, far, FarField{}, len_t32, nullptr);
    else if (far.b24) transpose_kernel<false, kField24><<<(groups + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, far, FarField{}, len_t32, nullptr);
    else transpose_kernel<false, kFieldBF16><<<(groups + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, far, FarField{}, len_t32, nullptr);
    return cudaGetLastError();
}

cudaError_t transpose_fill(const ProjParams& p, const FarField& far, const FarField& farT, const int* row_base_t,
                           cudaStream_t s) {
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    if (groups == 0) return cudaSuccess;
    if (far.f32) transpose_kernel<true, kFieldF32><<<(groups + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, far, farT, nullptr, row_base_t);
    else if (far.b24) transpose_kernel<true, kField24><<<(groups + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, far, farT, nullptr, row_base_t);
    else transpose_kernel<true, kFieldBF16><<<(groups + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, far, farT, nullptr, row_base_t);
    return cudaGetLastError();
}

cudaError_t forward_prep(const ProjParams& p, const float* W, const float* f, float* u, float* out, cudaStream_t s) {
    const size_t n = (size_t)p.nxy * p.g.nz;
    forward_prep_kernel<<<592, 256, 0, s>>>(p.vox2src, W, f, u, out, n);
    return cudaGetLastError();
}

cudaError_t forward_prep_extrapolate(const ProjParams& p, const float* W, const float* f, const float* prev,
                                     const float* lambda, float* y, float* u, float* out, cudaStream_t s) {
    const size_t n = (size_t)p.nxy * p.g.nz;
    forward_prep_extrapolate_kernel<<<592, 256, 0, s>>>(p.vox2src, W, f, prev, lambda, y, u, out, n);
    return cudaGetLastError();
}

cudaError_t forward_prep_half(const ProjParams& p, const float* W, const float* f, const float* prev,
                              const float* lambda, float* y, __nv_bfloat16* u16, cudaStream_t s) {
    const size_t n = (size_t)p.nxy * p.g.nz;
    if (lambda) forward_prep_half_kernel<true><<<592, 256, 0, s>>>(p.vox2src, W, f, prev, lambda, y, u16, n);
    else forward_prep_half_kernel<false><<<592, 256, 0, s>>>(p.vox2src, W, f, prev, lambda, y, u16, n);
    return cudaGetLastError();
}

int near_row_steps() { return kNearRow; }

size_t batch_smem_per_warp(int mode) {
    if (mode == kBatchTraceMarch) return (size_t)kNear * kLanes * sizeof(float);
    if (mode >= kBatchFieldF32) return kFieldSmemPerWarp;  // the field and frames modes
    return 0;
}

// The bounded-wait path of the field stream exercised on purpose: one thread waits on an
// mbarrier that nothing completes (a transaction count that no copy delivers), gives up after
// `rounds` try_wait rounds, raises the error flag like a field-stream warp does, and returns.
__global__ void wait_selftest_kernel(int rounds, unsigned int* error) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_mbarrier_init();
    mbar_expect_tx(&bar, 16);  // arrival done, 16 bytes expected that never come
    if (!mbar_wait_bounded(&bar, 0, rounds)) atomicOr(error, 1u);
}

cudaError_t wait_selftest(int rounds, unsigned int* error, cudaStream_t s) {
    wait_selftest_kernel<<<1, 32, 0, s>>>(rounds, error);
    return cudaGetLastError();
}

cudaError_t project_batch(Op op, const BatchItem* d_items, int n_items, int total_blocks, int warps, size_t smem,
                          cudaStream_t s) {
    if (total_blocks == 0 || n_items == 0) return cudaSuccess;
    if (warps < 1 || warps > kMaxWarps) return cudaErrorInvalidValue;
    auto go = [&](auto kernel) {
        if (smem > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        kernel<<<total_blocks, warps * kLanes, smem, s>>>(d_items, n_items);
        return cudaGetLastError();
    };
    if (op == Op::Forward) return go(project_batch_kernel<Op::Forward>);
    if (op == Op::Adjoint) return go(project_batch_kernel<Op::Adjoint>);
    return cudaErrorInvalidValue;
}

cudaError_t frame_prep(const ProjParams& p, const float* W, const FramePrep& fp, bool predict, float4* u4,
                       cudaStream_t s) {
    if (fp.n < 2 || fp.n > kMaxFrames) return cudaErrorInvalidValue;
    const size_t n = (size_t)p.nxy * p.g.nz;
    if (predict) frame_prep_kernel<true><<<592, 256, 0, s>>>(p.vox2src, W, fp, u4, n);
    else frame_prep_kernel<false><<<592, 256, 0, s>>>(p.vox2src, W, fp, u4, n);
    return cudaGetLastError();
}

cudaError_t frame_pack(const float* const* in, int n_frames, size_t voxels, float4* v4, cudaStream_t s) {
    if (n_frames < 2 || n_frames > kMaxFrames) return cudaErrorInvalidValue;
    FramePrep fp;
    fp.n = n_frames;
    for (int k = 0; k < n_frames; ++k) fp.f[k] = in[k];
    frame_pack_kernel<<<592, 256, 0, s>>>(fp, v4, voxels);
    return cudaGetLastError();
}

namespace {
template <Op OP, int FAR_MODE>
cudaError_t launch_frames(const ProjParams& p, const OpArgs& a, const FrameArgs& fr, cudaStream_t s) {
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    const int blocks = (groups + kWarps - 1) / kWarps;
    if (blocks == 0) return cudaSuccess;
    auto go = [&](auto kernel) {
        if (kFieldSmemBytes > 48 * 1024) {
            const cudaError_t e =
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFieldSmemBytes);
            if (e != cudaSuccess) return e;
        }
        kernel<<<blocks, kBlock, kFieldSmemBytes, s>>>(p, a, fr);
        return cudaGetLastError();
    };
    if (fr.n < 2 || fr.n > kMaxFrames || !fr.in4) return cudaErrorInvalidValue;
    return go(project_frames_kernel<OP, FAR_MODE>);
}
}  // namespace

cudaError_t project_frames(Op op, const ProjParams& p, const OpArgs& a, const FrameArgs& fr, cudaStream_t s) {
    if (fr.n < 1 || fr.n > kMaxFrames) return cudaErrorInvalidValue;
    for (int f = 0; f < fr.n; ++f) {
        const bool out_ok = fr.out[f] || (fr.n > 1 && op == Op::Forward && fr.out4);
        if (!out_ok || (fr.ratio_g[f] && !fr.ratio_eps[f]) || (fr.n == 1 && !fr.in[0])) return cudaErrorInvalidValue;
    }
    if (fr.n == 1) {  // one frame: the single-volume kernel (same stream, same accumulation order)
        if (op == Op::Forward ? !a.farT.on() : !a.far.on()) return cudaErrorInvalidValue;
        OpArgs b = a;
        b.in = fr.in[0];
        b.out = fr.out[0];
        b.ratio_g = fr.ratio_g[0];
        b.ratio_eps = fr.ratio_eps[0];
        b.in16 = nullptr;
        b.out16 = nullptr;
        return project(op, p, b, false, s);
    }
    if (op == Op::Forward) {
        if (a.farT.f32) return launch_frames<Op::Forward, kFieldF32T>(p, a, fr, s);
        if (a.farT.b24) return launch_frames<Op::Forward, kField24T>(p, a, fr, s);
        if (a.farT.b16) return launch_frames<Op::Forward, kFieldBF16T>(p, a, fr, s);
    } else if (op == Op::Adjoint) {
        if (a.far.f32) return launch_frames<Op::Adjoint, kFieldF32>(p, a, fr, s);
        if (a.far.b24) return launch_frames<Op::Adjoint, kField24>(p, a, fr, s);
        if (a.far.b16) return launch_frames<Op::Adjoint, kFieldBF16>(p, a, fr, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t forward_prep_batch(const PrepItem* d_items, int n_items, cudaStream_t s) {
    if (n_items == 0) return cudaSuccess;
    forward_prep_batch_kernel<<<dim3(128, n_items), 256, 0, s>>>(d_items);
    return cudaGetLastError();
}
int radial_water_bins() { return kWaterBins; }

cudaError_t build_radial_tables(const ProjParams& p, const RadialTables& t, cudaStream_t s) {
    radial_setup_kernel<<<(p.n_rays + 127) / 128, 128, 0, s>>>(p, t);
    return cudaGetLastError();
}

cudaError_t radial_kernels(const ProjParams& p, const RadialTables& t, const int* src, int n_src,
                           int warps_per_volume, float* out, cudaStream_t s) {
    const int warps = n_src / kLanes;
    if (warps == 0) return cudaSuccess;
    if (p.table) radial_kernel_kernel<false><<<(warps + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, t, src, n_src, warps_per_volume, out);
    else radial_kernel_kernel<true><<<(warps + kWarps - 1) / kWarps, kBlock, 0, s>>>(p, t, src, n_src, warps_per_volume, out);
    return cudaGetLastError();
}

cudaError_t surrogate_fill(const ProjParams& p, const OpArgs& a, const RadialTables& t, const __nv_bfloat16* coef,
                           const unsigned char* support, const unsigned char* fallback_rays, int water_bins,
                           cudaStream_t s) {
    if (a.far.b24) return cudaErrorInvalidValue;  // surrogate fields hold fp32 or bf16 weights
    const int groups = (p.n_active + kLanes - 1) / kLanes;
    if (groups == 0) return cudaSuccess;
    const int blocks = (groups + kWarps - 1) / kWarps;
    const size_t smem = a.near_acc ? size_t(kWarps) * 27 * kLanes * sizeof(float) : kNearSmemBytes;
    auto launch_fill = [&](auto kernel) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kernel<<<blocks, kBlock, smem, s>>>(p, a, t, coef, support, fallback_rays, water_bins);
        return cudaGetLastError();
    };
    if (a.far.f32) return p.table ? launch_fill(surrogate_fill_kernel<false, kFieldF32>) : launch_fill(surrogate_fill_kernel<true, kFieldF32>);
    return p.table ? launch_fill(surrogate_fill_kernel<false, kFieldBF16>) : launch_fill(surrogate_fill_kernel<true, kFieldBF16>);
}

cudaError_t build_surrogate_template(const ProjParams& p, const RadialTables& t, int* tmpl, int* tmpl_neg,
                                     cudaStream_t s) {
    template_kernel<<<(p.n_rays + 128) / 128, 128, 0, s>>>(p, tmpl);
    surrogate_template_kernel<<<p.n_rays, 128, 0, s>>>(p, t.offset, tmpl);
    negate_kernel<<<256, 256, 0, s>>>(tmpl, tmpl_neg, (size_t)p.n_rows * p.tmpl_len);
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
