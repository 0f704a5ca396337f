// prc_abi.cu -- the C ABI of include/prc_b200.h: one handle per density map, owning every
// device allocation, its stream, the projector state (Projector, prc.cu:403-450) and the
// MAP-EM state of main() (prc.cu:659-711).
#include "../../include/prc_b200.h"
#include "engine.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

using namespace prc;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define PRC_CUDA(call)                                                                              \
    do {                                                                                            \
        const cudaError_t err_ = (call);                                                            \
        if (err_ != cudaSuccess)                                                                    \
            return fail(err_ == cudaErrorMemoryAllocation ? PRC_ERR_MEMORY : PRC_ERR_CUDA,          \
                        std::string("CUDA error '") + cudaGetErrorString(err_) + "' in " + #call); \
    } while (0)

}  // namespace

void prc::set_last_error(const std::string& msg) { g_last_error = msg; }

// One density map's projector and MAP-EM state.  A batch frame of the same study copies its
// owner's handle (borrow_projector) and then resets what a handle owns (stream, allocations,
// u, scratch, MAP-EM and frame state, timing events): a member added here that a handle owns
// must be reset there as well, or the copy would share it.
struct prc_handle {
    Grid g{};
    RangeModel model;
    prc_options opts{};
    size_t n = 0;  // voxels
    int n_active = 0;
    int n_groups = 0;
    cudaStream_t stream = nullptr;
    int device = 0;

    // projector state
    float* rho = nullptr;
    unsigned char* support = nullptr;
    int* active = nullptr;
    float* W = nullptr;
    float* table = nullptr;
    RayStep* far = nullptr;
    RayStep* near_rays = nullptr;
    short* near_order = nullptr;
    int* near_start = nullptr;
    NearCache cache;
    FarField far_field;
    int* tmpl = nullptr;
    int* tmpl_neg = nullptr;
    unsigned short* len = nullptr;
    long long* group_base = nullptr;
    long long* group_total = nullptr;
    int* desc = nullptr;
    // target-major copy of the field (forward projection as a gather)
    FarField far_t;
    unsigned short* len_t = nullptr;
    long long* group_base_t = nullptr;
    int* desc_t = nullptr;
    int* vox2src = nullptr;
    float* u = nullptr;  // f / W volume for the gather form of the forward projection
    int64_t far_t_entries = 0;
    int64_t surrogate_fallbacks = 0;
    char isotope[8] = {};
    int64_t far_entries = 0;
    int cache_mode = PRC_CACHE_NONE;
    bool trace_near = false;
    ProjParams params{};
    unsigned long long* counter = nullptr;
    unsigned int* error = nullptr;  // device flag raised by a kernel that gave up a bounded wait
    float* scratch = nullptr;      // input volume of the host-memory forms
    float* scratch_out = nullptr;  // output volume of the host-memory operator forms

    // MAP-EM state
    float* g_em = nullptr;
    float* geo_w = nullptr;  // the RDP's 27 neighbour distance weights
    // PRC_PRECISION_BF16_VOLUMES: the gathered volumes of MAP-EM in bf16 (u = y / W, the EM ratio)
    __nv_bfloat16* u16 = nullptr;
    __nv_bfloat16* ratio16 = nullptr;
    float* vol[5] = {};  // f, prev, y, h_prev, est (rotated by pointer swaps)
    float *f = nullptr, *prev = nullptr, *y = nullptr, *h_prev = nullptr, *est = nullptr;
    EmScalars* scalars = nullptr;
    Reduction red{};
    bool em_started = false;
    // Frames sharing this projector (prc_*_frames): each frame's MAP-EM volumes, its u = f / W
    // volume for the forward gather, its FP64 scalars and reduction scratch.  Grown on demand.
    struct Frame {
        float* g = nullptr;
        float* vol[5] = {};  // f, prev, y, h_prev, est (rotated by pointer swaps)
        float* u = nullptr;
        EmScalars* scalars = nullptr;
        Reduction red{};
    };
    std::vector<Frame> frames;
    std::vector<float4*> frame_u4, frame_r4;  // per group of four frames: interleaved u and EM ratio
    int64_t bytes = 0;
    int64_t launches = 0;  // kernels this handle's entry points have enqueued (prc_launch_count)
    int tile = PRC_TILE_AUTO;  // source tile in effect (PRC_TILE_*)

    std::vector<void*> allocations;
    // projection timing (prc_timing): start/end event pairs of forward and adjoint launches
    bool timing = false;
    std::vector<cudaEvent_t> events[2];
    size_t events_used[2] = {0, 0};

    template <class T>
    cudaError_t alloc(T** p, size_t count) {
        void* v = nullptr;
        const cudaError_t e = cudaMalloc(&v, count * sizeof(T) > 0 ? count * sizeof(T) : 1);
        if (e != cudaSuccess) return e;
        allocations.push_back(v);
        bytes += (int64_t)(count * sizeof(T));
        *p = static_cast<T*>(v);
        return cudaMemsetAsync(v, 0, count * sizeof(T), stream);
    }

    cudaStream_t pick(void* s) const { return s ? static_cast<cudaStream_t>(s) : stream; }

    EmVolumes em_volumes() const { return EmVolumes{n, support, scalars, red}; }

    OpArgs op_args() const {
        OpArgs a;
        a.W = W;
        a.near = cache;
        a.far = far_field;
        a.farT = far_t;
        a.error = error;
        return a;
    }
};

// The tile of handles that are not tuned (see choose_tile).
static constexpr int kDefaultTile = PRC_TILE_8x2x2;

// (x, y, z) extent of a PRC_TILE_* source tile; every shape holds 32 voxels.
static const int* tile_dims(int tile) {
    static const int dims[][3] = {{8, 2, 2}, {8, 2, 2}, {16, 2, 1}, {32, 1, 1}, {4, 4, 2}, {16, 1, 2}};
    return dims[tile >= 0 && tile <= PRC_TILE_16x1x2 ? tile : 0];
}

// Reads and clears the device error flag; a raised flag means a kernel gave up a bounded wait.
static int check_device_error(prc_handle* h) {
    unsigned int flag = 0;
    PRC_CUDA(cudaMemcpyAsync(&flag, h->error, sizeof(flag), cudaMemcpyDeviceToHost, h->stream));
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    if (flag) {
        PRC_CUDA(cudaMemsetAsync(h->error, 0, sizeof(flag), h->stream));
        return fail(PRC_ERR_CUDA, "a stored-field copy did not complete within its bounded wait");
    }
    return PRC_OK;
}

extern "C" {

void prc_default_options(prc_options* o) {
    if (!o) return;
    o->rays = 128;
    o->support_rho = 0.05f;
    o->air_cap_mm = 50.0f;
    o->exact_range = 0;
    o->cache = PRC_CACHE_FULL;
    o->precision = PRC_PRECISION_FP32;
    o->tile = PRC_TILE_AUTO;
}

int prc_isotope_count(void) { return kNumIsotopes; }

const char* prc_isotope_name(int i) { return i >= 0 && i < kNumIsotopes ? kIsotopeTable[i].name : nullptr; }

int prc_isotope_cutoff(const char* isotope, float* cutoff_mm) {
    RangeModel m;
    if (!isotope || !m.resolve(isotope)) return fail(PRC_ERR_ISOTOPE, std::string("Unknown isotope ") + (isotope ? isotope : "(null)"));
    if (cutoff_mm) *cutoff_mm = m.cutoff;
    return PRC_OK;
}

const char* prc_last_error(void) { return g_last_error.c_str(); }

int prc_host_alloc(size_t bytes, void** ptr) {
    if (!ptr) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *ptr = nullptr;
    const cudaError_t e = cudaMallocHost(ptr, bytes > 0 ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return fail(PRC_ERR_MEMORY, std::string("cudaMallocHost failed: ") + cudaGetErrorString(e));
    }
    return PRC_OK;
}

void prc_host_free(void* ptr) {
    if (ptr) cudaFreeHost(ptr);
}

void prc_destroy(prc_handle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : h->allocations) cudaFree(p);
    for (auto& pool : h->events)
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

// The target-major copy of the stored field: per target group and template row, the longest
// step any contributing source reaches, prefix sums, then a copy of every weight.  Optional:
// without it (not enough memory) the forward projection scatters with atomics instead.
// The normalisation pass, with its near blocks traced octant by octant into a temporary fp32
// accumulator when one can be had (smaller shared-memory tiles, more warps per SM); otherwise
// into the full per-warp tile.
static float* near_accumulator(prc_handle* h) {
    float* acc = nullptr;
    if (cudaMalloc(&acc, (size_t)h->n_groups * kNear * kLanes * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return acc;
}
static void release_accumulator(prc_handle* h, float* acc) {
    if (!acc) return;
    cudaStreamSynchronize(h->stream);
    cudaFree(acc);
}

static int run_norm(prc_handle* h, OpArgs a) {
    a.near_acc = near_accumulator(h);
    const cudaError_t e = project(Op::Norm, h->params, a, true, h->stream);
    release_accumulator(h, a.near_acc);
    PRC_CUDA(e);
    return PRC_OK;
}

static int build_target_major(prc_handle* h, const std::vector<int>& active, size_t elem) {
    ProjParams& p = h->params;
    const size_t rows = (size_t)h->n_groups * p.n_rows;
    std::vector<int> v2s(h->n, -1);
    for (size_t i = 0; i < active.size(); ++i) v2s[active[i]] = (int)i;
    PRC_CUDA(h->alloc(&h->vox2src, h->n));
    PRC_CUDA(cudaMemcpyAsync(h->vox2src, v2s.data(), h->n * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    p.vox2src = h->vox2src;
    int* len32 = nullptr;
    PRC_CUDA(cudaMalloc(&len32, rows * sizeof(int)));
    struct Free {
        int* p;
        ~Free() { cudaFree(p); }
    } free_len32{len32};
    PRC_CUDA(cudaMemsetAsync(len32, 0, rows * sizeof(int), h->stream));
    PRC_CUDA(transpose_lengths(p, h->far_field, len32, h->stream));
    std::vector<int> l32(rows);
    PRC_CUDA(cudaMemcpyAsync(l32.data(), len32, rows * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    std::vector<unsigned short> lt(rows);
    std::vector<int> row_base(rows);
    std::vector<long long> gbase(h->n_groups + 1);
    long long run = 0;
    for (int g = 0; g < h->n_groups; ++g) {
        gbase[g] = run;
        int within = 0;
        for (int k = 0; k < p.n_rows; ++k) {
            const size_t i = (size_t)g * p.n_rows + k;
            const int L = (l32[i] + 3) / 4 * 4;
            lt[i] = (unsigned short)L;
            row_base[i] = within;
            within += L * kLanes;
        }
        run += within;
    }
    gbase[h->n_groups] = run;
    size_t free_b = 0, total_b = 0;
    PRC_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t desc_count = (size_t)(run / (4 * kLanes));
    // keep room for the MAP-EM volumes and the transient row offsets
    if ((size_t)run * elem + desc_count * 4 + rows * 6 + 16 * h->n * 4 > free_b) return PRC_OK;
    cudaError_t e = elem == 2   ? h->alloc(&h->far_t.b16, (size_t)run)
                    : elem == 3 ? h->alloc(&h->far_t.b24, (size_t)run * 3)
                                : h->alloc(&h->far_t.f32, (size_t)run);
    if (e == cudaSuccess) e = h->alloc(&h->desc_t, desc_count);
    if (e == cudaSuccess) e = h->alloc(&h->len_t, rows);
    if (e == cudaSuccess) e = h->alloc(&h->group_base_t, (size_t)h->n_groups + 1);
    if (e == cudaSuccess) e = h->alloc(&h->u, h->n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        h->far_t = FarField{};
        return PRC_OK;  // the forward keeps its scatter form
    }
    int* d_row_base = nullptr;
    PRC_CUDA(cudaMalloc(&d_row_base, rows * sizeof(int)));
    Free free_rb{d_row_base};
    PRC_CUDA(cudaMemcpyAsync(h->len_t, lt.data(), rows * sizeof(unsigned short), cudaMemcpyHostToDevice, h->stream));
    PRC_CUDA(cudaMemcpyAsync(h->group_base_t, gbase.data(), gbase.size() * sizeof(long long), cudaMemcpyHostToDevice,
                             h->stream));
    PRC_CUDA(cudaMemcpyAsync(d_row_base, row_base.data(), rows * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    p.tgt.len = h->len_t;
    p.tgt.group_base = h->group_base_t;
    PRC_CUDA(build_descriptors(p, p.tgt, h->desc_t, h->stream));
    p.tgt.desc = h->desc_t;
    PRC_CUDA(transpose_fill(p, h->far_field, h->far_t, d_row_base, h->stream));
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    h->far_t_entries = run;
    return PRC_OK;
}

static int create_impl(prc_handle* h, const float* density_host, prc_net* net = nullptr, bool surrogate = false,
                       float target_scale = 1.0f, float fallback_nrmse = 0.0f, int64_t* fallbacks = nullptr,
                       bool batch_member = false);

// The surrogate field (prc_create_surrogate).  Same stream format as the stored field; the
// template has 1 + 2 n_rays rows: the near block, the exact steps of every far ray, and the 16
// radial bins of every far ray.  The tracer judges every (source, far ray); a ray that some
// source of a 32-source group represents poorly keeps its exact steps for the whole group (the
// fallback), every other ray of the group stores the radial coefficients of its water range
// (12 bins: the judge sends every ray with mass beyond it back).  One fill pass
// (surrogate_fill) traces the near block, marches the fallback rays and writes the bins.
static int build_surrogate_field(prc_handle* h, prc_net* net, float target_scale, float fallback_nrmse,
                                 int64_t* fallbacks) {
    ProjParams& p = h->params;
    const Grid& g = h->g;
    if (h->opts.precision == PRC_PRECISION_FP24)
        return fail(PRC_ERR_ARGUMENT, "surrogate fields hold fp32 or bf16 weights (not PRC_PRECISION_FP24)");
    const bool bf16 = h->opts.precision != PRC_PRECISION_FP32;
    const int n_rays = h->opts.rays;
    const int march_len = (int)(((long long)g.nx + g.ny + g.nz + 6) / 4 * 4);
    if (march_len >= 65535) return fail(PRC_ERR_LIMIT, "volume too large for the surrogate field");
    RadialTables tab;
    PRC_CUDA(h->alloc(&tab.bin_of, (size_t)n_rays * march_len));
    PRC_CUDA(h->alloc(&tab.offset, (size_t)n_rays * kRadialBins));
    PRC_CUDA(h->alloc(&tab.xyz, (size_t)n_rays * kRadialBins));
    ProjParams pm = p;
    pm.tmpl_len = march_len;
    PRC_CUDA(build_radial_tables(pm, tab, h->stream));
    __nv_bfloat16* coef = nullptr;
    const size_t n_coef = (size_t)h->n_active * n_rays * kRadialBins;
    PRC_CUDA(cudaMalloc(&coef, n_coef * sizeof(__nv_bfloat16)));
    struct FreeDev {
        void* p;
        ~FreeDev() { cudaFree(p); }
    } free_coef{coef};
    static const char* kIsos[3] = {"18F", "68Ga", "82Rb"};
    int iso = -1;
    for (int i = 0; i < 3; ++i)
        if (std::strcmp(h->isotope, kIsos[i]) == 0) iso = i;
    if (net && (iso < 0 || n_rays != 128))
        return fail(PRC_ERR_ARGUMENT, "the surrogate network covers 18F, 68Ga and 82Rb with 128 far rays");
    if (net) {
        const int rc = surrogate_infer(net, h->rho, g.nx, g.ny, g.nz, iso, h->active, h->n_active,
                                       1.0f / target_scale, coef, h->stream);
        if (rc != PRC_OK) return rc;
    }
    // The tracer: judge of the predictions, ray by ray, and the coefficients themselves without a
    // network.  Rays with more than kBeyondShare of their mass beyond the water range fall back.
    unsigned char* flags = nullptr;  // [n_active][n_rays]
    PRC_CUDA(cudaMalloc(&flags, (size_t)h->n_active * n_rays));
    FreeDev free_flags{flags};
    PRC_CUDA(cudaMemsetAsync(flags, 0, (size_t)h->n_active * n_rays, h->stream));
    {
        const int chunk = 65536;  // sources per traced batch (multiple of 32)
        float* traced = nullptr;
        int* srcs = nullptr;
        PRC_CUDA(cudaMalloc(&traced, (size_t)chunk * n_rays * kRadialBins * sizeof(float)));
        FreeDev free_traced{traced};
        PRC_CUDA(cudaMalloc(&srcs, (size_t)chunk * sizeof(int)));
        FreeDev free_srcs{srcs};
        std::vector<int> host_src(chunk);
        std::vector<int> act(h->n_active);
        PRC_CUDA(cudaMemcpy(act.data(), h->active, act.size() * sizeof(int), cudaMemcpyDeviceToHost));
        for (int first = 0; first < h->n_active; first += chunk) {
            const int n = std::min(chunk, h->n_active - first);
            const int padded = (n + kLanes - 1) / kLanes * kLanes;
            for (int i = 0; i < padded; ++i) host_src[i] = act[first + std::min(i, n - 1)];
            PRC_CUDA(cudaMemcpyAsync(srcs, host_src.data(), padded * sizeof(int), cudaMemcpyHostToDevice, h->stream));
            PRC_CUDA(radial_kernels(pm, tab, srcs, padded, 1 << 30, traced, h->stream));
            // without the judge (fallback_nrmse == 0) a network's prediction is kept wherever
            // its ray stays within the water range
            PRC_CUDA(surrogate_judge(coef, traced, n, n_rays, first, net ? (fallback_nrmse > 0.0f ? fallback_nrmse : 1e30f) : -1.0f,
                                     kBeyondShare, radial_water_bins(), h->active, tab.xyz, g.nx, g.ny, g.nz, flags,
                                     h->stream));
            PRC_CUDA(cudaStreamSynchronize(h->stream));
        }
    }
    // a group keeps a ray exact when any of its sources needs it
    std::vector<unsigned char> src_flags((size_t)h->n_active * n_rays);
    PRC_CUDA(cudaMemcpy(src_flags.data(), flags, src_flags.size(), cudaMemcpyDeviceToHost));
    std::vector<unsigned char> ray_fb((size_t)h->n_groups * n_rays, 0);
    for (int i = 0; i < h->n_active; ++i)
        for (int r = 0; r < n_rays; ++r)
            if (src_flags[(size_t)i * n_rays + r]) ray_fb[(size_t)(i / kLanes) * n_rays + r] = 1;
    int64_t fb_pairs = 0;  // (source, far ray) pairs on exact weights
    for (int gi = 0; gi < h->n_groups; ++gi) {
        const int lanes = std::min(kLanes, h->n_active - gi * kLanes);
        for (int r = 0; r < n_rays; ++r) fb_pairs += ray_fb[(size_t)gi * n_rays + r] ? lanes : 0;
    }
    h->surrogate_fallbacks = fb_pairs;
    if (fallbacks) *fallbacks = fb_pairs;
    unsigned char* d_ray_fb = nullptr;
    PRC_CUDA(h->alloc(&d_ray_fb, ray_fb.size()));
    PRC_CUDA(cudaMemcpyAsync(d_ray_fb, ray_fb.data(), ray_fb.size(), cudaMemcpyHostToDevice, h->stream));

    // Stream layout: the exact lengths of a layout pass for fallback rays, the water bins
    // otherwise.
    p.n_rows = 1 + 2 * n_rays;
    p.tmpl_len = std::max(near_row_steps(), march_len);
    const size_t rows = (size_t)h->n_groups * p.n_rows;
    PRC_CUDA(h->alloc(&h->len, rows));
    PRC_CUDA(h->alloc(&h->group_total, h->n_groups));
    PRC_CUDA(h->alloc(&h->tmpl, (size_t)p.n_rows * p.tmpl_len));
    PRC_CUDA(h->alloc(&h->tmpl_neg, (size_t)p.n_rows * p.tmpl_len));
    p.tmpl = h->tmpl;
    p.tmpl_neg = h->tmpl_neg;
    PRC_CUDA(build_surrogate_template(p, tab, h->tmpl, h->tmpl_neg, h->stream));
    OpArgs la = h->op_args();
    la.len = h->len;
    la.group_total = h->group_total;
    PRC_CUDA(project(Op::Layout, p, la, true, h->stream));
    std::vector<unsigned short> len(rows);
    PRC_CUDA(cudaMemcpyAsync(len.data(), h->len, rows * sizeof(unsigned short), cudaMemcpyDeviceToHost, h->stream));
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    const int water_bins = radial_water_bins();
    std::vector<long long> base(h->n_groups + 1);
    long long run = 0;
    for (int gi = 0; gi < h->n_groups; ++gi) {
        unsigned short* l = &len[(size_t)gi * p.n_rows];
        l[0] = (unsigned short)near_row_steps();
        for (int r = 0; r < n_rays; ++r) {
            const bool exact = ray_fb[(size_t)gi * n_rays + r];
            if (!exact) l[1 + r] = 0;
            l[1 + n_rays + r] = exact ? 0 : (unsigned short)water_bins;
        }
        base[gi] = run;
        for (int k = 0; k < p.n_rows; ++k) run += (long long)l[k] * kLanes;
    }
    base[h->n_groups] = run;
    PRC_CUDA(h->alloc(&h->group_base, base.size()));
    PRC_CUDA(h->alloc(&h->desc, (size_t)(run / (4 * kLanes))));
    PRC_CUDA(bf16 ? h->alloc(&h->far_field.b16, (size_t)run) : h->alloc(&h->far_field.f32, (size_t)run));
    PRC_CUDA(cudaMemcpyAsync(h->len, len.data(), rows * sizeof(unsigned short), cudaMemcpyHostToDevice, h->stream));
    PRC_CUDA(cudaMemcpyAsync(h->group_base, base.data(), base.size() * sizeof(long long), cudaMemcpyHostToDevice,
                             h->stream));
    p.src.len = h->len;
    p.src.group_base = h->group_base;
    PRC_CUDA(build_descriptors(p, p.src, h->desc, h->stream));
    p.src.desc = h->desc;
    {
        OpArgs fa = h->op_args();
        fa.near_acc = near_accumulator(h);  // the near blocks, octant by octant
        const cudaError_t e = surrogate_fill(p, fa, tab, coef, h->support, d_ray_fb, water_bins, h->stream);
        release_accumulator(h, fa.near_acc);
        PRC_CUDA(e);
    }
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    h->far_entries = run;
    h->cache_mode = PRC_CACHE_SOURCE_MAJOR;
    h->trace_near = false;
    return PRC_OK;
}

static int create_impl(prc_handle* h, const float* density_host, prc_net* net, bool surrogate, float target_scale,
                       float fallback_nrmse, int64_t* fallbacks, bool batch_member) {
    const Grid& g = h->g;
    // Host-side clamp, support and source list (prc.cu:598-613).
    std::vector<float> rho(h->n);
    std::vector<unsigned char> support(h->n);
    std::vector<int> active;
    active.reserve(h->n / 2);
    for (size_t i = 0; i < h->n; ++i) {
        const float r = density_host[i];
        if (!std::isfinite(r)) {
            char msg[96];
            snprintf(msg, sizeof(msg), "Non-finite density at voxel %zu", i);
            return fail(PRC_ERR_NONFINITE, msg);
        }
        rho[i] = r > kMinDensity ? r : kMinDensity;
        support[i] = rho[i] >= g.support_rho;
    }
    // Source order: tiles of kTileX x kTileY x kTileZ voxels, x fastest inside a tile.  A warp
    // handles 32 consecutive sources.  Compact tiles give its lanes similar ray lengths (less
    // zero padding in the stored field), long rows make every gather of a step touch fewer
    // cache lines; the order changes no result: every source keeps its own weights and
    // summation order.
    if (h->tile == PRC_TILE_AUTO) h->tile = kDefaultTile;
    const int kTileX = tile_dims(h->tile)[0], kTileY = tile_dims(h->tile)[1], kTileZ = tile_dims(h->tile)[2];
    for (int z0 = 0; z0 < g.nz; z0 += kTileZ)
        for (int y0 = 0; y0 < g.ny; y0 += kTileY)
            for (int x0 = 0; x0 < g.nx; x0 += kTileX)
                for (int z = z0; z < std::min(z0 + kTileZ, g.nz); ++z)
                    for (int y = y0; y < std::min(y0 + kTileY, g.ny); ++y)
                        for (int x = x0; x < std::min(x0 + kTileX, g.nx); ++x) {
                            const size_t i = ((size_t)z * g.ny + y) * g.nx + x;
                            if (support[i]) active.push_back((int)i);
                        }
    h->n_active = (int)active.size();
    h->n_groups = (h->n_active + kLanes - 1) / kLanes;

    PRC_CUDA(cudaGetDevice(&h->device));
    PRC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    PRC_CUDA(h->alloc(&h->rho, h->n));
    PRC_CUDA(h->alloc(&h->support, h->n));
    PRC_CUDA(h->alloc(&h->active, h->n_active));
    PRC_CUDA(h->alloc(&h->W, h->n_active));
    PRC_CUDA(h->alloc(&h->far, h->opts.rays));
    PRC_CUDA(h->alloc(&h->near_rays, kNearRays));
    PRC_CUDA(h->alloc(&h->near_order, kNearRays));
    PRC_CUDA(h->alloc(&h->near_start, 9));
    PRC_CUDA(h->alloc(&h->counter, 1));
    PRC_CUDA(h->alloc(&h->error, 1));
    PRC_CUDA(cudaMemcpyAsync(h->rho, rho.data(), h->n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    PRC_CUDA(cudaMemcpyAsync(h->support, support.data(), h->n, cudaMemcpyHostToDevice, h->stream));
    if (h->n_active)
        PRC_CUDA(cudaMemcpyAsync(h->active, active.data(), active.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 h->stream));

    ProjParams& p = h->params;
    p.g = g;
    p.nxy = g.nx * g.ny;
    p.n_active = h->n_active;
    p.n_rays = h->opts.rays;
    p.rho = h->rho;
    p.active = h->active;
    p.far = h->far;
    p.near = h->near_rays;
    p.near_order = h->near_order;
    p.near_start = h->near_start;
    p.n_branch = h->model.n;
    for (int b = 0; b < 3; ++b) p.br[b] = h->model.br[b];
    if (!h->opts.exact_range) {  // prc.cu:625-633
        const std::vector<float> table = h->model.table();
        PRC_CUDA(h->alloc(&h->table, table.size()));
        PRC_CUDA(cudaMemcpyAsync(h->table, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice,
                                 h->stream));
        p.table = h->table;
        p.table_scale = h->model.table_scale();
    }
    PRC_CUDA(setup_rays(g, h->opts.rays, h->far, h->near_rays, h->stream));
    PRC_CUDA(order_near_rays(h->near_rays, h->near_order, h->near_start, h->stream));

    const bool bf16 = h->opts.precision == PRC_PRECISION_BF16 || h->opts.precision == PRC_PRECISION_BF16_VOLUMES;
    const bool fp24 = h->opts.precision == PRC_PRECISION_FP24;  // the stored field only
    const size_t elem = bf16 ? 2 : (fp24 ? 3 : 4);
    h->trace_near = true;
    if (surrogate) {
        int rc = build_surrogate_field(h, net, target_scale, fallback_nrmse, fallbacks);
        if (rc != PRC_OK) return rc;
        rc = build_target_major(h, active, elem);
        if (rc != PRC_OK) return rc;
        if (h->far_t.on()) h->cache_mode = PRC_CACHE_FULL;
        PRC_CUDA(cudaStreamSynchronize(h->stream));
        return check_device_error(h);
    }
    // Stored coefficient field (near block + far rays): size it with a layout pass, then let
    // the Norm pass fill it.  Template rows hold every step a ray can take inside the image
    // plus the padding of the last pack, in whole int4s.
    const long long tmpl_len =
        std::max<long long>(near_row_steps(), ((long long)g.nx + g.ny + g.nz + 3 + 3) / 4 * 4);
    const bool want_field = h->opts.cache == PRC_CACHE_FULL || h->opts.cache == PRC_CACHE_SOURCE_MAJOR;
    if (want_field && h->n_groups && tmpl_len < 65535) {
        p.tmpl_len = (int)tmpl_len;
        p.n_rows = h->opts.rays + 1;
        PRC_CUDA(h->alloc(&h->tmpl, (size_t)p.n_rows * tmpl_len));
        PRC_CUDA(h->alloc(&h->tmpl_neg, (size_t)p.n_rows * tmpl_len));
        PRC_CUDA(h->alloc(&h->len, (size_t)h->n_groups * p.n_rows));
        PRC_CUDA(h->alloc(&h->group_total, h->n_groups));
        PRC_CUDA(h->alloc(&h->group_base, (size_t)h->n_groups + 1));
        p.tmpl = h->tmpl;
        p.tmpl_neg = h->tmpl_neg;
        PRC_CUDA(build_template(p, h->tmpl, h->tmpl_neg, h->stream));
        OpArgs la = h->op_args();
        la.len = h->len;
        la.group_total = h->group_total;
        PRC_CUDA(project(Op::Layout, p, la, true, h->stream));
        std::vector<long long> totals(h->n_groups);
        PRC_CUDA(cudaMemcpyAsync(totals.data(), h->group_total, totals.size() * sizeof(long long),
                                 cudaMemcpyDeviceToHost, h->stream));
        PRC_CUDA(cudaStreamSynchronize(h->stream));
        long long run = 0;
        for (long long& t : totals) {
            const long long v = t;
            t = run;
            run += v;
        }
        totals.push_back(run);  // group_base[n_groups]: end of the last group
        size_t free_b = 0, total_b = 0;
        PRC_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t desc_count = (size_t)(run / (4 * kLanes));
        if ((size_t)run * elem + desc_count * 4 <= free_b / 2) {
            cudaError_t e = bf16   ? h->alloc(&h->far_field.b16, (size_t)run)
                            : fp24 ? h->alloc(&h->far_field.b24, (size_t)run * 3)
                                   : h->alloc(&h->far_field.f32, (size_t)run);
            if (e == cudaSuccess) e = h->alloc(&h->desc, desc_count);
            if (e == cudaSuccess) {
                PRC_CUDA(cudaMemcpyAsync(h->group_base, totals.data(), totals.size() * sizeof(long long),
                                         cudaMemcpyHostToDevice, h->stream));
                p.src.len = h->len;
                p.src.group_base = h->group_base;
                PRC_CUDA(build_descriptors(p, p.src, h->desc, h->stream));
                p.src.desc = h->desc;
                h->far_entries = run;
                h->cache_mode = PRC_CACHE_SOURCE_MAJOR;
                h->trace_near = false;
            } else {
                cudaGetLastError();  // optional: fall back to the near cache
            }
        }
    }
    // Near cache when the field is off and it fits in a quarter of free memory (prc.cu:411-419).
    if (h->cache_mode == PRC_CACHE_NONE && h->opts.cache >= PRC_CACHE_NEAR && h->n_groups) {
        size_t free_b = 0, total_b = 0;
        PRC_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t entries = (size_t)h->n_groups * kNear * kLanes;
        // a batch member keeps a near cache whenever it fits: retracing 2048 near rays per
        // source every pass would dominate the whole batch
        const size_t limit = batch_member ? (free_b > ((size_t)1 << 30) ? free_b - ((size_t)1 << 30) : 0) : free_b / 4;
        if (entries * (bf16 ? 2 : 4) <= limit) {  // the near cache is fp32 unless bf16
            cudaError_t e = bf16 ? h->alloc(&h->cache.b16, entries) : h->alloc(&h->cache.f32, entries);
            if (e == cudaSuccess) h->trace_near = false, h->cache_mode = PRC_CACHE_NEAR;
            else cudaGetLastError();  // optional: fall back to retracing
        }
    }
    if (const int rc = run_norm(h, h->op_args()); rc != PRC_OK) return rc;
    if (h->cache_mode == PRC_CACHE_SOURCE_MAJOR && h->opts.cache == PRC_CACHE_FULL) {
        const int rc = build_target_major(h, active, elem);
        if (rc != PRC_OK) return rc;
        if (h->far_t.on()) h->cache_mode = PRC_CACHE_FULL;
    }
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    return check_device_error(h);
}

static int create_handle(const prc_geometry* geo, const char* isotope, const prc_options* opts_in,
                         const float* density_host, prc_net* net, bool surrogate, float target_scale,
                         float fallback_nrmse, int64_t* fallbacks, prc_handle** out, bool batch_member) {
    if (!out) return fail(PRC_ERR_ARGUMENT, "Invalid argument: null handle pointer");
    *out = nullptr;
    if (!geo || !density_host) return fail(PRC_ERR_ARGUMENT, "Invalid argument: null geometry or density");
    prc_options o;
    prc_default_options(&o);
    if (opts_in) o = *opts_in;
    // prc.cu:540-551
    if (geo->nx <= 0 || geo->ny <= 0 || geo->nz <= 0 || !(geo->dx > 0) || !(geo->dy > 0) || !(geo->dz > 0) ||
        !std::isfinite(geo->dx) || !std::isfinite(geo->dy) || !std::isfinite(geo->dz) || o.rays < 2 ||
        (o.rays & 1) || o.rays > INT_MAX - 31 || !(o.support_rho >= 0) || !(o.air_cap_mm > 0) ||
        !std::isfinite(o.support_rho) || !std::isfinite(o.air_cap_mm) ||
        o.precision < PRC_PRECISION_FP32 || o.precision > PRC_PRECISION_FP24 || o.cache < PRC_CACHE_NONE ||
        o.cache > PRC_CACHE_SOURCE_MAJOR || o.tile < PRC_TILE_AUTO || o.tile > PRC_TILE_16x1x2 ||
        !(target_scale > 0) || !(fallback_nrmse >= 0))
        return fail(PRC_ERR_ARGUMENT, "Invalid geometry or solver parameters");
    if (geo->nx > INT_MAX / geo->ny || geo->nx * geo->ny > INT_MAX / geo->nz)
        return fail(PRC_ERR_LIMIT, "Volume exceeds the INT_MAX voxel index limit");
    prc_handle* h = new prc_handle();
    if (!h->model.resolve(isotope ? isotope : "")) {
        delete h;
        return fail(PRC_ERR_ISOTOPE, std::string("Unknown isotope ") + (isotope ? isotope : "(null)"));
    }
    std::strncpy(h->isotope, isotope, sizeof(h->isotope) - 1);
    h->opts = o;
    h->tile = o.tile;
    h->g = Grid{geo->nx, geo->ny, geo->nz, geo->dx, geo->dy, geo->dz, h->model.cutoff, o.support_rho, o.air_cap_mm};
    h->n = (size_t)geo->nx * geo->ny * geo->nz;
    const int rc = create_impl(h, density_host, net, surrogate, target_scale, fallback_nrmse, fallbacks, batch_member);
    if (rc != PRC_OK) {
        const std::string msg = g_last_error;
        prc_destroy(h);
        g_last_error = msg;
        return rc;
    }
    *out = h;
    return PRC_OK;
}


// ---- source-tile autotuner (PRC_TILE_AUTO) ---------------------------------------------------
// The tile shape trades the field's zero padding (compact tiles: the 32 lanes of a group stop
// their rays at similar steps) against the cache lines every gather of a step touches (long
// rows).  Which wins depends on the grid, the isotope's range and the stored precision, so the
// tuner (prc_tune_tile; every frame configuration of a batch) builds the stored field with every
// candidate shape on the central slab of at most kTuneSlices z-slices of the density (the same
// rays, ranges and tissue mix at a fraction of the build time), times one forward and one
// adjoint projection with CUDA events after a warm-up pair, and keeps the fastest; handles
// created with PRC_TILE_AUTO take the remembered choice of their configuration, or kDefaultTile
// when it was never tuned.  Forms without a stored field (near cache, traced) and surrogate
// fields take kDefaultTile.
static constexpr int kTileCandidates[] = {PRC_TILE_8x2x2, PRC_TILE_16x2x1, PRC_TILE_32x1x1};
static constexpr int kTuneSlices = 32;
static std::mutex g_tile_mutex;
static std::map<std::string, int> g_tile_choice;

static std::string tile_key(const prc_geometry* geo, const char* isotope, const prc_options& o) {
    char key[256];
    snprintf(key, sizeof(key), "%d %d %d %a %a %a %s %d %a %a %d %d %d", geo->nx, geo->ny, geo->nz, geo->dx, geo->dy,
             geo->dz, isotope ? isotope : "", o.rays, o.support_rho, o.air_cap_mm, o.exact_range, o.cache,
             o.precision);
    return key;
}

// Device milliseconds of one forward and one adjoint projection of the handle (after a warm-up
// pair), on zero volumes: the gathers run whatever the values.
static int time_projection_pair(prc_handle* h, float* ms) {
    float *in = nullptr, *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct Cleanup {
        float*& in;
        float*& out;
        cudaEvent_t& e0;
        cudaEvent_t& e1;
        ~Cleanup() {
            if (in) cudaFree(in);
            if (out) cudaFree(out);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } cleanup{in, out, e0, e1};
    PRC_CUDA(cudaMalloc(&in, h->n * sizeof(float)));
    PRC_CUDA(cudaMalloc(&out, h->n * sizeof(float)));
    PRC_CUDA(cudaMemsetAsync(in, 0, h->n * sizeof(float), h->stream));
    PRC_CUDA(cudaEventCreate(&e0));
    PRC_CUDA(cudaEventCreate(&e1));
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) PRC_CUDA(cudaEventRecord(e0, h->stream));
        int rc = prc_forward(h, in, out, h->stream);
        if (rc == PRC_OK) rc = prc_adjoint(h, in, out, h->stream);
        if (rc != PRC_OK) return rc;
    }
    PRC_CUDA(cudaEventRecord(e1, h->stream));
    PRC_CUDA(cudaEventSynchronize(e1));
    PRC_CUDA(cudaEventElapsedTime(ms, e0, e1));
    return check_device_error(h);
}

// The remembered choice of a configuration (tune = false) or, when there is none, the tuner's
// (tune = true) or kDefaultTile.
static int choose_tile(const prc_geometry* geo, const char* isotope, const prc_options& o, const float* density_host,
                       bool surrogate, bool tune) {
    if (surrogate || (o.cache != PRC_CACHE_FULL && o.cache != PRC_CACHE_SOURCE_MAJOR)) return kDefaultTile;
    const std::string key = tile_key(geo, isotope, o);
    {
        std::lock_guard<std::mutex> lock(g_tile_mutex);
        const auto it = g_tile_choice.find(key);
        if (it != g_tile_choice.end()) return it->second;
    }
    if (!tune) return kDefaultTile;
    prc_geometry slab = *geo;
    const float* slab_density = density_host;
    if (geo->nz > kTuneSlices) {
        slab.nz = kTuneSlices;
        slab_density += (size_t)(geo->nz - kTuneSlices) / 2 * geo->nx * geo->ny;
    }
    int best = kDefaultTile;
    float best_ms = 0.0f;
    for (const int cand : kTileCandidates) {
        prc_options oc = o;
        oc.tile = cand;
        prc_handle* h = nullptr;
        if (create_handle(&slab, isotope, &oc, slab_density, nullptr, false, 1.0f, 0.0f, nullptr, &h, false) != PRC_OK)
            continue;  // e.g. not enough memory for this shape's field: not a candidate
        float ms = 0.0f;
        const bool field = h->far_field.on();
        const int rc = field ? time_projection_pair(h, &ms) : PRC_ERR_STATE;
        prc_destroy(h);
        if (!field) break;  // no stored field: the shape does not matter
        if (rc == PRC_OK && (best_ms == 0.0f || ms < best_ms)) best = cand, best_ms = ms;
    }
    g_last_error.clear();
    std::lock_guard<std::mutex> lock(g_tile_mutex);
    g_tile_choice[key] = best;
    return best;
}

static int create_common(const prc_geometry* geo, const char* isotope, const prc_options* opts_in,
                         const float* density_host, prc_net* net, bool surrogate, float target_scale,
                         float fallback_nrmse, int64_t* fallbacks, prc_handle** out, bool batch_member = false) {
    prc_options o;
    prc_default_options(&o);
    if (opts_in) o = *opts_in;
    if (o.tile == PRC_TILE_AUTO && geo && density_host && out && o.cache >= PRC_CACHE_NONE &&
        o.cache <= PRC_CACHE_SOURCE_MAJOR) {
        RangeModel m;
        if (m.resolve(isotope ? isotope : ""))
            o.tile = choose_tile(geo, isotope, o, density_host, surrogate, batch_member);
    }
    return create_handle(geo, isotope, &o, density_host, net, surrogate, target_scale, fallback_nrmse, fallbacks, out,
                         batch_member);
}

int prc_tune_tile(const prc_geometry* geo, const char* isotope, const prc_options* opts_in, const float* density_host,
                  int* tile) {
    if (!geo || !density_host || !tile) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    prc_options o;
    prc_default_options(&o);
    if (opts_in) o = *opts_in;
    RangeModel m;
    if (!m.resolve(isotope ? isotope : "")) return fail(PRC_ERR_ISOTOPE, std::string("Unknown isotope ") + (isotope ? isotope : "(null)"));
    if (o.cache < PRC_CACHE_NONE || o.cache > PRC_CACHE_SOURCE_MAJOR)
        return fail(PRC_ERR_ARGUMENT, "Invalid geometry or solver parameters");
    *tile = choose_tile(geo, isotope, o, density_host, false, true);
    return PRC_OK;
}

int prc_create(const prc_geometry* geo, const char* isotope, const prc_options* opts, const float* density_host,
               prc_handle** out) {
    return create_common(geo, isotope, opts, density_host, nullptr, false, 1.0f, 0.0f, nullptr, out);
}

int prc_create_surrogate(const prc_geometry* geo, const char* isotope, const prc_options* opts,
                         const float* density_host, prc_net* net, float target_scale, float fallback_nrmse,
                         int64_t* fallbacks, prc_handle** out) {
    return create_common(geo, isotope, opts, density_host, net, true, target_scale, fallback_nrmse, fallbacks, out);
}

int prc_cache_mode(const prc_handle* h, int* mode, int64_t* source_major_entries, int64_t* target_major_entries) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (mode) *mode = h->cache_mode;
    if (source_major_entries) *source_major_entries = h->far_entries;
    if (target_major_entries) *target_major_entries = h->far_t_entries;
    return PRC_OK;
}

int prc_active_count(const prc_handle* h, int64_t* n) {
    if (!h || !n) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *n = h->n_active;
    return PRC_OK;
}

int prc_cutoff(const prc_handle* h, float* c) {
    if (!h || !c) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *c = h->g.cutoff;
    return PRC_OK;
}

int prc_device_bytes(const prc_handle* h, int64_t* b) {
    if (!h || !b) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *b = h->bytes;
    return PRC_OK;
}

void* prc_stream(const prc_handle* h) { return h ? (void*)h->stream : nullptr; }

// Records the next event of pool `kind` (0 forward, 1 adjoint) when timing is on; events come
// in start / end pairs around each projection launch.
static cudaError_t timing_mark(prc_handle* h, int kind, cudaStream_t s) {
    if (!h->timing) return cudaSuccess;
    std::vector<cudaEvent_t>& pool = h->events[kind];
    if (h->events_used[kind] == pool.size()) {
        cudaEvent_t e = nullptr;
        const cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) return err;
        pool.push_back(e);
    }
    return cudaEventRecord(pool[h->events_used[kind]++], s);
}

int prc_timing(prc_handle* h, int enable) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (enable) h->events_used[0] = h->events_used[1] = 0;
    h->timing = enable != 0;
    return PRC_OK;
}

int prc_timing_read(prc_handle* h, double* forward_ms, int64_t* n_forward, double* adjoint_ms, int64_t* n_adjoint) {
    if (!h || !forward_ms || !n_forward || !adjoint_ms || !n_adjoint) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    double* total[2] = {forward_ms, adjoint_ms};
    int64_t* count[2] = {n_forward, n_adjoint};
    for (int kind = 0; kind < 2; ++kind) {
        *total[kind] = 0.0;
        *count[kind] = (int64_t)(h->events_used[kind] / 2);
        for (size_t i = 0; i + 1 < h->events_used[kind]; i += 2) {
            PRC_CUDA(cudaEventSynchronize(h->events[kind][i + 1]));
            float ms = 0.0f;
            PRC_CUDA(cudaEventElapsedTime(&ms, h->events[kind][i], h->events[kind][i + 1]));
            *total[kind] += ms;
        }
    }
    return PRC_OK;
}

int prc_forward(prc_handle* h, const float* d_in, float* d_out, void* stream) {
    if (!h || !d_in || !d_out) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    const cudaStream_t s = h->pick(stream);
    OpArgs a = h->op_args();
    a.in = d_in;
    a.out = d_out;
    if (h->far_t.on()) {  // gather form: u = f / W, then out[t] = sum_k T_tk u[t - o_k]
        PRC_CUDA(forward_prep(h->params, h->W, d_in, h->u, d_out, s));
        ++h->launches;
        a.in = h->u;
    } else {
        PRC_CUDA(cudaMemsetAsync(d_out, 0, h->n * sizeof(float), s));
    }
    PRC_CUDA(timing_mark(h, 0, s));
    PRC_CUDA(project(Op::Forward, h->params, a, h->trace_near, s));
    ++h->launches;
    PRC_CUDA(timing_mark(h, 0, s));
    return PRC_OK;
}

int prc_adjoint(prc_handle* h, const float* d_in, float* d_out, void* stream) {
    if (!h || !d_in || !d_out) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    OpArgs a = h->op_args();
    a.in = d_in;
    a.out = d_out;
    const cudaStream_t s = h->pick(stream);
    PRC_CUDA(timing_mark(h, 1, s));
    PRC_CUDA(project(Op::Adjoint, h->params, a, h->trace_near, s));
    ++h->launches;
    PRC_CUDA(timing_mark(h, 1, s));
    return PRC_OK;
}

// PRC_PRECISION_BF16_VOLUMES keeps the volumes MAP-EM gathers in bf16 as well: with the bf16 field
// in both majors (the forward is a gather whose epilogue takes the ratio).
static bool half_volumes(const prc_handle* h) {
    return h->opts.precision == PRC_PRECISION_BF16_VOLUMES && h->far_t.b16 && h->far_field.b16;
}

static int ensure_em(prc_handle* h) {
    if (!h->g_em) {
        PRC_CUDA(h->alloc(&h->g_em, h->n));
        for (float*& v : h->vol) PRC_CUDA(h->alloc(&v, h->n));
        PRC_CUDA(h->alloc(&h->scalars, 1));
        PRC_CUDA(h->alloc(&h->red.partials, (size_t)kReduceBlocks * 4));
        PRC_CUDA(h->alloc(&h->red.counter, 1));
        PRC_CUDA(h->alloc(&h->geo_w, 27));
        PRC_CUDA(em_geometry_weights(h->g, h->geo_w, h->stream));
    }
    // (a batch adds its target-major copies after this first call, so checked every time)
    if (half_volumes(h) && !h->u16) {
        PRC_CUDA(h->alloc(&h->u16, h->n));
        PRC_CUDA(h->alloc(&h->ratio16, h->n));
    }
    return PRC_OK;
}

// Device address of a float member of the handle's device-resident EmScalars.
static const float* scalar_field(const prc_handle* h, size_t offset) {
    return reinterpret_cast<const float*>(reinterpret_cast<const char*>(h->scalars) + offset);
}

static int em_begin_impl(prc_handle* h, const float* d_g, bool initialize, cudaStream_t s) {
    if (h->n_active == 0) return fail(PRC_ERR_NO_ACTIVITY, "No tissue voxels: nothing to do");
    int rc = ensure_em(h);
    if (rc != PRC_OK) return rc;
    h->f = h->vol[0], h->prev = h->vol[1], h->y = h->vol[2], h->h_prev = h->vol[3], h->est = h->vol[4];
    // the history buffers start at zero (prc.cu:661-665): prev, y and h_prev
    PRC_CUDA(cudaMemsetAsync(h->prev, 0, h->n * sizeof(float), s));
    PRC_CUDA(cudaMemsetAsync(h->y, 0, h->n * sizeof(float), s));
    PRC_CUDA(cudaMemsetAsync(h->h_prev, 0, h->n * sizeof(float), s));
    PRC_CUDA(em_begin(h->em_volumes(), d_g, h->g_em, h->f, h->n_active, initialize, s));
    h->launches += initialize ? 3 : 1;
    h->em_started = true;
    return PRC_OK;
}

int prc_em_begin(prc_handle* h, const float* d_g, void* stream) {
    if (!h || !d_g) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    return em_begin_impl(h, d_g, true, h->pick(stream));
}

int prc_em_iterate(prc_handle* h, int n_iter, float beta, float gamma, int accelerate, void* stream) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (!h->em_started) return fail(PRC_ERR_STATE, "prc_em_iterate called before prc_em_begin");
    if (n_iter < 0 || !(beta >= 0) || !(gamma >= 0) || !std::isfinite(beta) || !std::isfinite(gamma))
        return fail(PRC_ERR_ARGUMENT, "Invalid geometry or solver parameters");
    const cudaStream_t s = h->pick(stream);
    const EmVolumes v = h->em_volumes();
    // With the target-major field the forward projection is a gather whose preparation pass
    // also makes the Biggs-Andrews prediction and whose epilogue takes the EM ratio, so an
    // iteration is five launches: prep(+extrapolate), forward(+ratio), adjoint, RDP update,
    // finish.  The scatter and traced forms keep the separate extrapolate and ratio passes.
    const bool fused = h->far_t.on();
    const bool half = half_volumes(h);
    for (int it = 0; it < n_iter; ++it) {  // prc.cu:675-700
        const float* start = h->f;
        if (fused) {
            const float* lambda = accelerate ? scalar_field(h, offsetof(EmScalars, lambda)) : nullptr;
            if (half) {
                PRC_CUDA(forward_prep_half(h->params, h->W, h->f, h->prev, lambda, h->y, h->u16, s));
            } else if (accelerate) {
                PRC_CUDA(forward_prep_extrapolate(h->params, h->W, h->f, h->prev, lambda, h->y, h->u, h->est, s));
            } else {
                PRC_CUDA(forward_prep(h->params, h->W, h->f, h->u, h->est, s));
            }
            if (accelerate) start = h->y;
            ++h->launches;
            OpArgs a = h->op_args();
            a.in = h->u;
            a.out = h->est;
            if (half) a.in16 = h->u16, a.out16 = h->ratio16;
            a.ratio_g = h->g_em;
            a.ratio_eps = scalar_field(h, offsetof(EmScalars, eps));
            PRC_CUDA(timing_mark(h, 0, s));
            PRC_CUDA(project(Op::Forward, h->params, a, h->trace_near, s));
            PRC_CUDA(timing_mark(h, 0, s));
            ++h->launches;
        } else {
            if (accelerate) {
                PRC_CUDA(em_extrapolate(v, h->f, h->prev, h->y, s));
                ++h->launches;
                start = h->y;
            }
            const int rc = prc_forward(h, start, h->est, s);
            if (rc != PRC_OK) return rc;
            PRC_CUDA(em_ratio(v, h->g_em, h->est, s));
            ++h->launches;
        }
        if (half) {  // the adjoint gathers the bf16 ratio
            OpArgs a = h->op_args();
            a.in16 = h->ratio16;
            a.out = h->prev;  // prediction has consumed prev
            PRC_CUDA(timing_mark(h, 1, s));
            PRC_CUDA(project(Op::Adjoint, h->params, a, h->trace_near, s));
            PRC_CUDA(timing_mark(h, 1, s));
            ++h->launches;
        } else {
            const int rc = prc_adjoint(h, h->est, h->prev, s);  // prediction has consumed prev
            if (rc != PRC_OK) return rc;
        }
        // est is 0 off the support, which is what the update leaves there: every MAP-EM volume
        // starts at 0 there and no pass writes anything but 0 off the support
        PRC_CUDA(em_update_active(v, h->g, h->active, h->n_active, h->geo_w, start, h->prev, h->est, beta, gamma, s));
        ++h->launches;
        if (beta > 0.0f || accelerate) {
            PRC_CUDA(em_finish(v, h->est, accelerate ? h->y : nullptr, h->h_prev, beta > 0.0f, s));
            ++h->launches;
        }
        if (accelerate) {
            std::swap(h->y, h->h_prev);
            std::swap(h->prev, h->f);
        }
        std::swap(h->f, h->est);
    }
    return PRC_OK;
}

int prc_em_estimate(prc_handle* h, float* d_out, void* stream) {
    if (!h || !d_out) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (!h->em_started) return fail(PRC_ERR_STATE, "prc_em_estimate called before prc_em_begin");
    PRC_CUDA(cudaMemcpyAsync(d_out, h->f, h->n * sizeof(float), cudaMemcpyDeviceToDevice, h->pick(stream)));
    return PRC_OK;
}

int prc_em_run(prc_handle* h, const float* d_g, float* d_out, int iterations, float beta, float gamma,
               int accelerate, void* stream) {
    if (!h || !d_g || !d_out) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (iterations < 0) return fail(PRC_ERR_ARGUMENT, "Invalid geometry or solver parameters");
    const cudaStream_t s = h->pick(stream);
    int rc = em_begin_impl(h, d_g, iterations > 0, s);
    if (rc == PRC_OK) rc = prc_em_iterate(h, iterations, beta, gamma, accelerate, s);
    if (rc == PRC_OK) rc = prc_em_estimate(h, d_out, s);
    return rc;
}

static int ensure_scratch(prc_handle* h) {
    if (!h->scratch) PRC_CUDA(h->alloc(&h->scratch, h->n));
    if (!h->scratch_out) PRC_CUDA(h->alloc(&h->scratch_out, h->n));
    return PRC_OK;
}

int prc_em_run_host(prc_handle* h, const float* g_host, float* out_host, int iterations, float beta, float gamma,
                    int accelerate) {
    if (!h || !g_host || !out_host) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    int rc = ensure_scratch(h);
    if (rc != PRC_OK) return rc;
    PRC_CUDA(cudaMemcpyAsync(h->scratch, g_host, h->n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    rc = prc_em_run(h, h->scratch, h->scratch, iterations, beta, gamma, accelerate, h->stream);
    if (rc != PRC_OK) return rc;
    PRC_CUDA(cudaMemcpyAsync(out_host, h->scratch, h->n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return check_device_error(h);
}

int prc_em_begin_host(prc_handle* h, const float* g_host) {
    if (!h || !g_host) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    int rc = ensure_scratch(h);
    if (rc != PRC_OK) return rc;
    PRC_CUDA(cudaMemcpyAsync(h->scratch, g_host, h->n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    rc = em_begin_impl(h, h->scratch, true, h->stream);
    if (rc != PRC_OK) return rc;
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    return PRC_OK;
}

int prc_em_estimate_host(prc_handle* h, float* out_host) {
    if (!h || !out_host) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (!h->em_started) return fail(PRC_ERR_STATE, "prc_em_estimate_host called before prc_em_begin");
    PRC_CUDA(cudaMemcpyAsync(out_host, h->f, h->n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    return PRC_OK;
}

int prc_forward_host(prc_handle* h, const float* in_host, float* out_host) {
    if (!h || !in_host || !out_host) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    int rc = ensure_scratch(h);
    if (rc != PRC_OK) return rc;
    float* in = h->scratch;
    float* out = h->scratch_out;
    PRC_CUDA(cudaMemcpyAsync(in, in_host, h->n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    rc = prc_forward(h, in, out, h->stream);
    if (rc != PRC_OK) return rc;
    PRC_CUDA(cudaMemcpyAsync(out_host, out, h->n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return check_device_error(h);
}

int prc_adjoint_host(prc_handle* h, const float* in_host, float* out_host) {
    if (!h || !in_host || !out_host) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    int rc = ensure_scratch(h);
    if (rc != PRC_OK) return rc;
    float* in = h->scratch;
    float* out = h->scratch_out;
    PRC_CUDA(cudaMemcpyAsync(in, in_host, h->n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    PRC_CUDA(cudaMemsetAsync(out, 0, h->n * sizeof(float), h->stream));
    rc = prc_adjoint(h, in, out, h->stream);
    if (rc != PRC_OK) return rc;
    PRC_CUDA(cudaMemcpyAsync(out_host, out, h->n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    return check_device_error(h);
}

// ---- frames that share this projector --------------------------------------------------------
// The frames of one dynamic study share the density map, isotope and grid, hence the operator:
// with the stored field the frames go through the projections in groups of up to kMaxFrames,
// each group one pass over the field gathering an interleaved volume (four frames per voxel).
// A group of one frame takes the single-volume kernels.
static int ensure_frames(prc_handle* h, int n_frames) {
    while ((int)h->frames.size() < n_frames) {
        prc_handle::Frame fr;
        PRC_CUDA(h->alloc(&fr.g, h->n));
        for (float*& v : fr.vol) PRC_CUDA(h->alloc(&v, h->n));
        PRC_CUDA(h->alloc(&fr.u, h->n));
        PRC_CUDA(h->alloc(&fr.scalars, 1));
        PRC_CUDA(h->alloc(&fr.red.partials, (size_t)kReduceBlocks * 4));
        PRC_CUDA(h->alloc(&fr.red.counter, 1));
        h->frames.push_back(fr);
    }
    while ((int)h->frame_u4.size() < (n_frames + kMaxFrames - 1) / kMaxFrames) {
        float4 *u4 = nullptr, *r4 = nullptr;
        PRC_CUDA(h->alloc(&u4, h->n));
        PRC_CUDA(h->alloc(&r4, h->n));
        h->frame_u4.push_back(u4);
        h->frame_r4.push_back(r4);
    }
    return PRC_OK;
}

static int check_frames(int n_frames, const float* const* in, const void* out) {
    if (n_frames < 1 || !in || !out) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    for (int i = 0; i < n_frames; ++i)
        if (!in[i] || !static_cast<float* const*>(out)[i]) return fail(PRC_ERR_ARGUMENT, "Invalid argument: null frame volume");
    return PRC_OK;
}

// One projection pass of frames [first, first + k).
static int frame_pass(prc_handle* h, Op op, const FrameArgs& fr, cudaStream_t s) {
    const int kind = op == Op::Forward ? 0 : 1;
    PRC_CUDA(timing_mark(h, kind, s));
    PRC_CUDA(project_frames(op, h->params, h->op_args(), fr, s));
    PRC_CUDA(timing_mark(h, kind, s));
    ++h->launches;
    return PRC_OK;
}

int prc_forward_frames(prc_handle* h, int n_frames, const float* const* d_in, float* const* d_out, void* stream) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (const int rc = check_frames(n_frames, d_in, d_out); rc != PRC_OK) return rc;
    const cudaStream_t s = h->pick(stream);
    if (!h->far_t.on()) {  // no target-major field: one projection per frame
        for (int i = 0; i < n_frames; ++i)
            if (const int rc = prc_forward(h, d_in[i], d_out[i], s); rc != PRC_OK) return rc;
        return PRC_OK;
    }
    if (const int rc = ensure_frames(h, n_frames); rc != PRC_OK) return rc;
    for (int first = 0; first < n_frames; first += kMaxFrames) {
        const int k = std::min(kMaxFrames, n_frames - first);
        if (k == 1) {
            if (const int rc = prc_forward(h, d_in[first], d_out[first], s); rc != PRC_OK) return rc;
            continue;
        }
        float4* u4 = h->frame_u4[first / kMaxFrames];
        FramePrep fp;  // u = f / W interleaved, out = 0 off the support
        FrameArgs fr;
        fp.n = fr.n = k;
        for (int f = 0; f < k; ++f) fp.f[f] = d_in[first + f], fp.out[f] = d_out[first + f], fr.out[f] = d_out[first + f];
        PRC_CUDA(frame_prep(h->params, h->W, fp, false, u4, s));
        ++h->launches;
        fr.in4 = u4;
        if (const int rc = frame_pass(h, Op::Forward, fr, s); rc != PRC_OK) return rc;
    }
    return PRC_OK;
}

int prc_adjoint_frames(prc_handle* h, int n_frames, const float* const* d_in, float* const* d_out, void* stream) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (const int rc = check_frames(n_frames, d_in, d_out); rc != PRC_OK) return rc;
    const cudaStream_t s = h->pick(stream);
    if (!h->far_field.on()) {
        for (int i = 0; i < n_frames; ++i)
            if (const int rc = prc_adjoint(h, d_in[i], d_out[i], s); rc != PRC_OK) return rc;
        return PRC_OK;
    }
    if (const int rc = ensure_frames(h, n_frames); rc != PRC_OK) return rc;
    for (int first = 0; first < n_frames; first += kMaxFrames) {
        const int k = std::min(kMaxFrames, n_frames - first);
        if (k == 1) {
            if (const int rc = prc_adjoint(h, d_in[first], d_out[first], s); rc != PRC_OK) return rc;
            continue;
        }
        float4* v4 = h->frame_r4[first / kMaxFrames];
        PRC_CUDA(frame_pack(d_in + first, k, h->n, v4, s));
        ++h->launches;
        FrameArgs fr;
        fr.n = k;
        fr.in4 = v4;
        for (int f = 0; f < k; ++f) fr.out[f] = d_out[first + f];
        if (const int rc = frame_pass(h, Op::Adjoint, fr, s); rc != PRC_OK) return rc;
    }
    return PRC_OK;
}

int prc_em_run_frames(prc_handle* h, int n_frames, const float* const* d_g, float* const* d_out, int iterations,
                      float beta, float gamma, int accelerate, void* stream) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    if (const int rc = check_frames(n_frames, d_g, d_out); rc != PRC_OK) return rc;
    if (iterations < 0 || !(beta >= 0) || !(gamma >= 0) || !std::isfinite(beta) || !std::isfinite(gamma))
        return fail(PRC_ERR_ARGUMENT, "Invalid geometry or solver parameters");
    const cudaStream_t s = h->pick(stream);
    if (!h->far_t.on() || !h->far_field.on() || half_volumes(h)) {  // one correction per frame
        for (int i = 0; i < n_frames; ++i)
            if (const int rc = prc_em_run(h, d_g[i], d_out[i], iterations, beta, gamma, accelerate, s); rc != PRC_OK)
                return rc;
        return PRC_OK;
    }
    if (h->n_active == 0) return fail(PRC_ERR_NO_ACTIVITY, "No tissue voxels: nothing to do");
    if (const int rc = ensure_em(h); rc != PRC_OK) return rc;  // the RDP's distance weights
    if (const int rc = ensure_frames(h, n_frames); rc != PRC_OK) return rc;
    const int n = n_frames;
    // Every frame runs prc_em_iterate's five-launch iteration (prc.cu:675-700) with its own
    // volumes and FP64 scalars; the preparation and the two projections are shared per group.
    std::vector<float*> f(n), prev(n), y(n), hp(n), est(n);
    std::vector<const float*> start(n);
    std::vector<EmVolumes> v(n);
    auto scalar = [](const EmScalars* sc, size_t off) {
        return reinterpret_cast<const float*>(reinterpret_cast<const char*>(sc) + off);
    };
    for (int i = 0; i < n; ++i) {
        const prc_handle::Frame& fr = h->frames[i];
        f[i] = fr.vol[0], prev[i] = fr.vol[1], y[i] = fr.vol[2], hp[i] = fr.vol[3], est[i] = fr.vol[4];
        v[i] = EmVolumes{h->n, h->support, fr.scalars, fr.red};
        for (float* p : {prev[i], y[i], hp[i]}) PRC_CUDA(cudaMemsetAsync(p, 0, h->n * sizeof(float), s));
        PRC_CUDA(em_begin(v[i], d_g[i], fr.g, f[i], h->n_active, iterations > 0, s));
        h->launches += iterations > 0 ? 3 : 1;
    }
    for (int it = 0; it < iterations; ++it) {
        // forward preparation (with the prediction), forward gather with the ratio, adjoint gather
        for (int first = 0; first < n; first += kMaxFrames) {
            const int k = std::min(kMaxFrames, n - first);
            const prc_handle::Frame* fr0 = &h->frames[first];
            FrameArgs fwd, adj;
            fwd.n = adj.n = k;
            if (k == 1) {  // the single-volume kernels: u and the ratio in the frame's own volumes
                const int i = first;
                if (accelerate) {
                    PRC_CUDA(forward_prep_extrapolate(h->params, h->W, f[i], prev[i],
                                                      scalar(fr0->scalars, offsetof(EmScalars, lambda)), y[i], fr0->u,
                                                      est[i], s));
                } else {
                    PRC_CUDA(forward_prep(h->params, h->W, f[i], fr0->u, est[i], s));
                }
                fwd.in[0] = fr0->u, fwd.out[0] = est[i];
                adj.in[0] = est[i], adj.out[0] = prev[i];
            } else {
                float4 *u4 = h->frame_u4[first / kMaxFrames], *r4 = h->frame_r4[first / kMaxFrames];
                FramePrep fp;
                fp.n = k;
                for (int j = 0; j < k; ++j) {
                    const int i = first + j;
                    fp.f[j] = f[i], fp.prev[j] = prev[i], fp.y[j] = y[i], fp.out[j] = est[i];
                    fp.lambda[j] = scalar(h->frames[i].scalars, offsetof(EmScalars, lambda));
                    adj.out[j] = prev[i];
                }
                PRC_CUDA(frame_prep(h->params, h->W, fp, accelerate != 0, u4, s));
                fwd.in4 = u4, fwd.out4 = r4;  // the ratio, interleaved for the adjoint's gather
                adj.in4 = r4;
            }
            ++h->launches;
            for (int j = 0; j < k; ++j) {
                const int i = first + j;
                fwd.ratio_g[j] = h->frames[i].g;
                fwd.ratio_eps[j] = scalar(h->frames[i].scalars, offsetof(EmScalars, eps));
                start[i] = accelerate ? y[i] : f[i];
            }
            if (const int rc = frame_pass(h, Op::Forward, fwd, s); rc != PRC_OK) return rc;
            if (const int rc = frame_pass(h, Op::Adjoint, adj, s); rc != PRC_OK) return rc;
        }
        // est is 0 off the support (the preparation wrote it), which the update leaves there
        for (int i = 0; i < n; ++i) {
            PRC_CUDA(em_update_active(v[i], h->g, h->active, h->n_active, h->geo_w, start[i], prev[i], est[i], beta,
                                      gamma, s));
            ++h->launches;
            if (beta > 0.0f || accelerate) {
                PRC_CUDA(em_finish(v[i], est[i], accelerate ? y[i] : nullptr, hp[i], beta > 0.0f, s));
                ++h->launches;
            }
            if (accelerate) {
                std::swap(y[i], hp[i]);
                std::swap(prev[i], f[i]);
            }
            std::swap(f[i], est[i]);
        }
    }
    for (int i = 0; i < n; ++i)
        PRC_CUDA(cudaMemcpyAsync(d_out[i], f[i], h->n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    return PRC_OK;
}

int prc_sum(prc_handle* h, const float* d_x, double* sum, void* stream) {
    if (!h || !d_x || !sum) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    int rc = ensure_em(h);
    if (rc != PRC_OK) return rc;
    const cudaStream_t s = h->pick(stream);
    PRC_CUDA(em_sum(h->em_volumes(), d_x, s));
    ++h->launches;
    PRC_CUDA(cudaMemcpyAsync(sum, &h->scalars->sum, sizeof(double), cudaMemcpyDeviceToHost, s));
    PRC_CUDA(cudaStreamSynchronize(s));
    return PRC_OK;
}

int prc_count_deposits(prc_handle* h, int64_t* deposits) {
    if (!h || !deposits) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    PRC_CUDA(cudaMemsetAsync(h->counter, 0, sizeof(unsigned long long), h->stream));
    OpArgs a = h->op_args();
    a.count = h->counter;
    PRC_CUDA(project(Op::Count, h->params, a, h->trace_near, h->stream));
    unsigned long long v = 0;
    PRC_CUDA(cudaMemcpyAsync(&v, h->counter, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    *deposits = (int64_t)v;
    return PRC_OK;
}

int prc_wait_selftest(prc_handle* h, int rounds) {
    if (!h || rounds < 1 || rounds > (1 << 20)) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    PRC_CUDA(wait_selftest(rounds, h->error, h->stream));
    return prc_synchronize(h);
}

int prc_tile(const prc_handle* h, int* tile) {
    if (!h || !tile) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *tile = h->tile;
    return PRC_OK;
}

int prc_launch_count(const prc_handle* h, int64_t* n) {
    if (!h || !n) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *n = h->launches;
    return PRC_OK;
}

int prc_synchronize(prc_handle* h) {
    if (!h) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    PRC_CUDA(cudaStreamSynchronize(h->stream));
    return check_device_error(h);
}

}  // extern "C"

// ================================================================================================
// Batched frames: one handle per frame (each with its own projector form, chosen by memory),
// every MAP-EM phase of every frame in one launch, the whole schedule captured into a CUDA graph.
// ================================================================================================
struct prc_batch {
    std::vector<prc_handle*> frames;
    cudaStream_t stream = nullptr;
    int warps = kWarpsDefault;
    bool tuned = false;
    void* d_tables = nullptr;
    size_t table_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // what the captured graph was built for
    std::vector<const float*> key_g;
    std::vector<float*> key_out;
    int key_iters = -1, key_accel = -1;
    float key_beta = -1.0f, key_gamma = -1.0f;
    static constexpr int kWarpsDefault = 4;
    // Frames sharing one projector with its stored field in both majors go through the
    // projections in chunks of 2..4 (one item of the batched launch each, gathering the
    // interleaved u4 / r4 of the chunk: the forward preparation writes u4, the forward's
    // epilogue the EM ratios r4); chunk_of / slot_of place a frame (-1: its own item).
    std::vector<std::vector<int>> chunks;
    std::vector<float4*> chunk_u4, chunk_r4;
    std::vector<int> chunk_of, slot_of;
};

namespace {

int batch_mode(const prc_handle* h, Op op) {
    if (op == Op::Forward && h->far_t.on())
        return h->far_t.b16 ? kBatchFieldBF16T : (h->far_t.b24 ? kBatchField24T : kBatchFieldF32T);
    if (h->far_field.on()) return h->far_field.b16 ? kBatchFieldBF16 : (h->far_field.b24 ? kBatchField24 : kBatchFieldF32);
    if (!h->trace_near && h->cache.on()) return h->cache.b16 ? kBatchCacheBF16March : kBatchCacheF32March;
    return kBatchTraceMarch;
}

int frames_mode(const prc_handle* h, Op op) {
    if (op == Op::Forward) return h->far_t.b16 ? kBatchFramesBF16T : (h->far_t.b24 ? kBatchFrames24T : kBatchFramesF32T);
    return h->far_field.b16 ? kBatchFramesBF16 : (h->far_field.b24 ? kBatchFrames24 : kBatchFramesF32);
}

void release_graph(prc_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// The enqueued schedule of one batched MAP-EM run, built on the host.
struct BatchPlan {
    std::vector<unsigned char> host;  // all tables, uploaded at once
    struct Launch {
        int kind;  // 0 EM phase, 1 projector, 2 forward prep, 3 memset (frame, buffer), 4 copy-out (frame)
        EmPhase phase;
        Op op;
        size_t offset;  // of its table in `host`
        int n_items;
        int total_blocks;
        size_t smem;
        int frame;
        float* ptr;
    };
    std::vector<Launch> launches;
    template <class T>
    size_t add(const std::vector<T>& v) {
        const size_t off = (host.size() + 255) / 256 * 256;
        host.resize(off + v.size() * sizeof(T));
        std::memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

BatchPlan plan_batch(prc_batch* b, const float* const* d_g, float* const* d_out, int iterations, float beta,
                     float gamma, bool accel, int warps, bool forward_only) {
    BatchPlan plan;
    const int n = (int)b->frames.size();
    struct Bufs {
        float *f, *prev, *y, *h_prev, *est;
    };
    std::vector<Bufs> bufs(n);
    for (int i = 0; i < n; ++i) {
        prc_handle* h = b->frames[i];
        bufs[i] = {h->vol[0], h->vol[1], h->vol[2], h->vol[3], h->vol[4]};
    }
    auto em_items = [&]() {
        std::vector<EmItem> items(n);
        for (int i = 0; i < n; ++i) {
            prc_handle* h = b->frames[i];
            EmItem& it = items[i];
            it.v = h->em_volumes();
            it.grid = h->g;
            it.n_active = h->n_active;
            it.active = h->active;
            it.geo_w = h->geo_w;
            it.g_in = d_g ? d_g[i] : nullptr;
            it.g = h->g_em;
            it.f = bufs[i].f, it.prev = bufs[i].prev, it.y = bufs[i].y, it.h_prev = bufs[i].h_prev,
            it.est = bufs[i].est;
        }
        return items;
    };
    auto em_launch = [&](EmPhase ph, size_t off, int n_items) {
        BatchPlan::Launch l{};
        l.kind = 0, l.phase = ph, l.offset = off, l.n_items = n_items;
        plan.launches.push_back(l);
    };
    // ratio: inside MAP-EM a chunk's forward pass takes its frames' EM ratios in its epilogue,
    // interleaved into the chunk's r4 for the adjoint (those frames skip the Ratio phase)
    auto projector_launch = [&](Op op, const std::vector<const float*>& in, const std::vector<float*>& out,
                                bool ratio) {
        std::vector<BatchItem> items;
        int blocks = 0;
        size_t smem = 0;
        for (int i = 0; i < n; ++i) {
            const int c = b->chunk_of[i];
            if (c >= 0 && b->slot_of[i] != 0) continue;  // the chunk's item is made at its first frame
            prc_handle* h = b->frames[i];
            BatchItem it{};
            it.p = h->params;
            it.a = h->op_args();
            it.a.in = in[i];
            it.a.out = out[i];
            it.mode = batch_mode(h, op);
            if (c >= 0) {  // one pass for the chunk's frames
                const std::vector<int>& fr = b->chunks[c];
                it.mode = frames_mode(h, op);
                it.fr.n = (int)fr.size();
                it.fr.in4 = op == Op::Forward ? b->chunk_u4[c] : b->chunk_r4[c];
                for (size_t j = 0; j < fr.size(); ++j) it.fr.out[j] = out[fr[j]];
                if (op == Op::Forward && ratio) {
                    it.fr.out4 = b->chunk_r4[c];
                    for (size_t j = 0; j < fr.size(); ++j) {
                        const prc_handle* fh = b->frames[fr[j]];
                        it.fr.ratio_g[j] = fh->g_em;
                        it.fr.ratio_eps[j] = reinterpret_cast<const float*>(reinterpret_cast<const char*>(fh->scalars) +
                                                                            offsetof(EmScalars, eps));
                    }
                }
            }
            const int groups = (h->n_active + kLanes - 1) / kLanes;
            it.blocks = (groups + warps - 1) / warps;
            it.first_block = blocks;
            blocks += it.blocks;
            smem = std::max(smem, batch_smem_per_warp(it.mode) * warps);
            items.push_back(it);
        }
        BatchPlan::Launch l{};
        l.kind = 1, l.op = op, l.offset = plan.add(items), l.n_items = (int)items.size(), l.total_blocks = blocks,
        l.smem = smem;
        plan.launches.push_back(l);
    };
    auto forward = [&](const std::vector<const float*>& in, const std::vector<float*>& out, bool ratio) {
        std::vector<PrepItem> prep(n);
        std::vector<const float*> pin(n);
        for (int i = 0; i < n; ++i) {
            prc_handle* h = b->frames[i];
            const bool gather = h->far_t.on();
            prep[i] = PrepItem{h->vox2src, h->W, in[i], h->u, out[i], (long long)h->n, gather ? 1 : 0, 0, nullptr};
            if (b->chunk_of[i] >= 0) prep[i].u4 = b->chunk_u4[b->chunk_of[i]], prep[i].slot = b->slot_of[i];
            pin[i] = gather ? h->u : in[i];
        }
        BatchPlan::Launch l{};
        l.kind = 2, l.offset = plan.add(prep), l.n_items = n;
        plan.launches.push_back(l);
        projector_launch(Op::Forward, pin, out, ratio);
    };
    if (forward_only) {  // one forward projection of every frame (autotuning)
        std::vector<const float*> in(n);
        std::vector<float*> out(n);
        for (int i = 0; i < n; ++i) in[i] = d_g[i], out[i] = b->frames[i]->vol[4];
        forward(in, out, false);
        return plan;
    }
    // initialisation (prc_em_begin for every frame)
    for (int i = 0; i < n; ++i)
        for (float* p : {bufs[i].prev, bufs[i].y, bufs[i].h_prev}) {
            BatchPlan::Launch l{};
            l.kind = 3, l.frame = i, l.ptr = p;
            plan.launches.push_back(l);
        }
    em_launch(EmPhase::Begin, plan.add(em_items()), n);
    for (int it = 0; it < iterations; ++it) {
        const std::vector<EmItem> all = em_items();
        const size_t items = plan.add(all);
        std::vector<EmItem> unchunked;  // the frames whose ratio is a phase of its own
        for (int i = 0; i < n; ++i)
            if (b->chunk_of[i] < 0) unchunked.push_back(all[i]);
        std::vector<const float*> start(n), est_in(n);
        std::vector<float*> est(n), prev(n);
        for (int i = 0; i < n; ++i) {
            start[i] = accel ? bufs[i].y : bufs[i].f;
            est[i] = bufs[i].est;
            est_in[i] = bufs[i].est;
            prev[i] = bufs[i].prev;
        }
        if (accel) em_launch(EmPhase::Extrapolate, items, n);
        forward(start, est, true);
        if (!unchunked.empty()) em_launch(EmPhase::Ratio, plan.add(unchunked), (int)unchunked.size());
        projector_launch(Op::Adjoint, est_in, prev, false);
        em_launch(EmPhase::Update, items, n);
        if (beta > 0.0f || accel) em_launch(EmPhase::Finish, items, n);
        for (int i = 0; i < n; ++i) {  // prc.cu:697-700
            if (accel) {
                std::swap(bufs[i].y, bufs[i].h_prev);
                std::swap(bufs[i].prev, bufs[i].f);
            }
            std::swap(bufs[i].f, bufs[i].est);
        }
    }
    for (int i = 0; i < n; ++i) {
        BatchPlan::Launch l{};
        l.kind = 4, l.frame = i, l.ptr = bufs[i].f;
        plan.launches.push_back(l);
    }
    (void)d_out;
    return plan;
}

// Enqueues the schedule on the batch's stream.  With `timed`, every kernel launch (a MAP-EM
// phase, a batched projection, a forward preparation) is bracketed by a pair of CUDA events
// appended to it; memsets and copies are not.
int enqueue_plan(prc_batch* b, const BatchPlan& plan, float* const* d_out, float beta, float gamma, bool accel,
                 int warps, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* timed = nullptr) {
    const unsigned char* base = static_cast<const unsigned char*>(b->d_tables);
    const int em_blocks = std::max(1, std::min(kReduceBlocks, 4096 / std::max(1, (int)b->frames.size())));
    for (const BatchPlan::Launch& l : plan.launches) {
        cudaError_t e = cudaSuccess;
        const bool kernel = l.kind <= 2;
        if (timed && kernel) {
            std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
            PRC_CUDA(cudaEventCreate(&ev.first));
            PRC_CUDA(cudaEventCreate(&ev.second));
            timed->push_back(ev);
            PRC_CUDA(cudaEventRecord(ev.first, b->stream));
        }
        switch (l.kind) {
            case 0:
                e = em_batch_phase(l.phase, reinterpret_cast<const EmItem*>(base + l.offset), l.n_items, em_blocks, beta,
                                   gamma, accel, b->stream);
                break;
            case 1:
                e = project_batch(l.op, reinterpret_cast<const BatchItem*>(base + l.offset), l.n_items, l.total_blocks,
                                  warps, l.smem, b->stream);
                break;
            case 2:
                e = forward_prep_batch(reinterpret_cast<const PrepItem*>(base + l.offset), l.n_items, b->stream);
                break;
            case 3:
                e = cudaMemsetAsync(l.ptr, 0, b->frames[l.frame]->n * sizeof(float), b->stream);
                break;
            case 4:
                e = cudaMemcpyAsync(d_out[l.frame], l.ptr, b->frames[l.frame]->n * sizeof(float),
                                    cudaMemcpyDeviceToDevice, b->stream);
                break;

        }
        if (e != cudaSuccess) return fail(PRC_ERR_CUDA, std::string("CUDA error '") + cudaGetErrorString(e) +
                                                            "' in the batched MAP-EM schedule");
        if (timed && kernel) PRC_CUDA(cudaEventRecord(timed->back().second, b->stream));
    }
    return PRC_OK;
}

// Frames that repeat an earlier frame's geometry, isotope and density array share its projector.
bool same_projector(const prc_frame& a, const prc_frame& b) {
    const prc_geometry &x = a.geometry, &y = b.geometry;
    return a.density_host && a.density_host == b.density_host && a.isotope && b.isotope &&
           std::strcmp(a.isotope, b.isotope) == 0 && x.nx == y.nx && x.ny == y.ny && x.nz == y.nz && x.dx == y.dx &&
           x.dy == y.dy && x.dz == y.dz;
}

// A handle on another handle's projector: every projector array (density, support, W, stored
// field in both majors, templates, rays) is the owner's, read only; the borrower owns its stream,
// its forward-gather scratch u and, once allocated, its MAP-EM state, and frees only those.
int borrow_projector(const prc_handle* o, prc_handle** out) {
    prc_handle* h = new prc_handle(*o);
    h->allocations.clear();
    h->bytes = 0;
    h->launches = 0;
    h->stream = nullptr;
    h->u = nullptr;
    h->scratch = h->scratch_out = nullptr;
    h->g_em = h->geo_w = nullptr;
    h->u16 = h->ratio16 = nullptr;
    for (float*& v : h->vol) v = nullptr;
    h->f = h->prev = h->y = h->h_prev = h->est = nullptr;
    h->scalars = nullptr;
    h->red = Reduction{};
    h->em_started = false;
    h->frames.clear();
    h->frame_u4.clear();
    h->frame_r4.clear();
    h->timing = false;
    for (auto& pool : h->events) pool.clear();
    h->events_used[0] = h->events_used[1] = 0;
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && o->u) e = h->alloc(&h->u, h->n);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        prc_destroy(h);
        return fail(e == cudaErrorMemoryAllocation ? PRC_ERR_MEMORY : PRC_ERR_CUDA,
                    std::string("CUDA error '") + cudaGetErrorString(e) + "' while sharing a projector");
    }
    *out = h;
    return PRC_OK;
}

int upload_plan(prc_batch* b, const BatchPlan& plan) {
    if (plan.host.size() > b->table_bytes) {
        if (b->d_tables) cudaFree(b->d_tables);
        b->d_tables = nullptr;
        PRC_CUDA(cudaMalloc(&b->d_tables, plan.host.size()));
        b->table_bytes = plan.host.size();
    }
    PRC_CUDA(cudaMemcpyAsync(b->d_tables, plan.host.data(), plan.host.size(), cudaMemcpyHostToDevice, b->stream));
    PRC_CUDA(cudaStreamSynchronize(b->stream));
    return PRC_OK;
}

}  // namespace

extern "C" {

void prc_batch_destroy(prc_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    release_graph(b);
    if (b->d_tables) cudaFree(b->d_tables);
    for (float4* p : b->chunk_u4) cudaFree(p);
    for (float4* p : b->chunk_r4) cudaFree(p);
    for (prc_handle* h : b->frames) prc_destroy(h);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int prc_batch_create(int n_frames, const prc_frame* frames, const prc_options* opts, prc_net* net, float target_scale,
                     float fallback_nrmse, prc_batch** out) {
    if (!out || n_frames <= 0 || !frames) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *out = nullptr;
    if (opts && opts->exact_range) return fail(PRC_ERR_ARGUMENT, "Invalid geometry or solver parameters: batched "
                                                                   "frames use the survival table");
    prc_batch* b = new prc_batch();
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return fail(PRC_ERR_CUDA, "cudaStreamCreate failed");
    }
    static const char* kNet[3] = {"18F", "68Ga", "82Rb"};
    // While the frames build their projectors (each stored field takes at most half of the free
    // memory it sees), hold back what they will still need: every frame's MAP-EM volumes and
    // scratch plus 8 GiB for the caller's data until all are built, and each frame's near cache
    // (estimated for half its voxels) until that frame is built.
    auto hold = [](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return p;
    };
    size_t em_bytes = (size_t)8 << 30;
    std::vector<void*> near_hold(n_frames, nullptr);
    for (int i = 0; i < n_frames; ++i) {
        const prc_geometry& g = frames[i].geometry;
        const size_t n = (size_t)std::max(g.nx, 0) * std::max(g.ny, 0) * std::max(g.nz, 0);
        em_bytes += n * sizeof(float) * 12;
    }
    void* held = hold(em_bytes);
    for (int i = 0; i < n_frames; ++i) {
        const prc_geometry& g = frames[i].geometry;
        const size_t n = (size_t)std::max(g.nx, 0) * std::max(g.ny, 0) * std::max(g.nz, 0);
        near_hold[i] = hold(n / 2 * kNear * sizeof(float));
    }
    // First every frame builds its source-major field (half the memory of both copies) or, when
    // even that does not fit, its near cache; target-major copies are added afterwards.
    prc_options member;
    prc_default_options(&member);
    if (opts) member = *opts;
    const bool want_full = member.cache == PRC_CACHE_FULL;
    if (want_full) member.cache = PRC_CACHE_SOURCE_MAJOR;
    // the frames of one study (the same geometry, isotope and density array) share one projector:
    // frame i borrows frame owner[i]'s once every projector is built
    std::vector<int> owner(n_frames, -1);
    for (int i = 0; i < n_frames; ++i)
        for (int j = 0; j < i && owner[i] < 0; ++j)
            if (owner[j] < 0 && same_projector(frames[i], frames[j])) owner[i] = j;
    for (int i = 0; i < n_frames; ++i) {
        const prc_frame& f = frames[i];
        if (near_hold[i]) cudaFree(near_hold[i]), near_hold[i] = nullptr;
        if (owner[i] >= 0) {
            b->frames.push_back(nullptr);
            continue;
        }
        bool learned = false;
        for (const char* iso : kNet) learned = learned || (net && f.isotope && std::strcmp(f.isotope, iso) == 0);
        prc_handle* h = nullptr;
        const int rc = create_common(&f.geometry, f.isotope, &member, f.density_host, learned ? net : nullptr, learned,
                                     target_scale, fallback_nrmse, nullptr, &h, true);
        if (rc != PRC_OK) {
            const std::string msg = g_last_error;
            if (held) cudaFree(held);
            for (void* p : near_hold)
                if (p) cudaFree(p);
            prc_batch_destroy(b);
            g_last_error = "frame " + std::to_string(i) + ": " + msg;
            return rc;
        }
        b->frames.push_back(h);
    }
    if (held) cudaFree(held);
    for (int i = 0; i < n_frames; ++i) {
        if (!b->frames[i]) continue;
        const int em = ensure_em(b->frames[i]);
        if (em != PRC_OK) {
            const std::string msg = g_last_error;
            prc_batch_destroy(b);
            g_last_error = "frame " + std::to_string(i) + ": " + msg;
            return em;
        }
    }
    if (want_full) {  // target-major copies (forward as a gather), smallest fields first, while they fit
        std::vector<int> order;
        for (int i = 0; i < n_frames; ++i)
            if (b->frames[i]) order.push_back(i);
        std::sort(order.begin(), order.end(),
                  [&](int x, int y) { return b->frames[x]->far_entries < b->frames[y]->far_entries; });
        for (int i : order) {
            prc_handle* h = b->frames[i];
            if (!h->far_field.on()) continue;
            // keep 8 GiB plus every frame's data and result volumes for the caller
            size_t free_b2 = 0, total_b2 = 0;
            if (cudaMemGetInfo(&free_b2, &total_b2) != cudaSuccess) break;
            size_t caller = (size_t)8 << 30;
            for (int k = 0; k < n_frames; ++k)
                caller += 3 * (size_t)frames[k].geometry.nx * frames[k].geometry.ny * frames[k].geometry.nz * sizeof(float);
            const size_t elem_b = h->far_field.b16 ? 2 : (h->far_field.b24 ? 3 : 4);
            const size_t need = (size_t)((double)h->far_entries * elem_b * 1.05) + caller;
            if (free_b2 < need) continue;
            std::vector<int> act(h->n_active);
            if (cudaMemcpy(act.data(), h->active, act.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) break;
            const int rc = build_target_major(h, act, elem_b);
            if (rc != PRC_OK) {
                prc_batch_destroy(b);
                return rc;
            }
            if (h->far_t.on()) h->cache_mode = PRC_CACHE_FULL;
        }
    }
    for (int i = 0; i < n_frames; ++i) {
        if (owner[i] < 0) continue;
        int rc = borrow_projector(b->frames[owner[i]], &b->frames[i]);
        if (rc == PRC_OK) rc = ensure_em(b->frames[i]);
        if (rc != PRC_OK) {
            const std::string msg = g_last_error;
            prc_batch_destroy(b);
            g_last_error = "frame " + std::to_string(i) + ": " + msg;
            return rc;
        }
    }
    // chunks of 2..4 frames on one projector with the stored field in both majors
    b->chunk_of.assign(n_frames, -1);
    b->slot_of.assign(n_frames, -1);
    for (int o = 0; o < n_frames; ++o) {
        if (owner[o] >= 0) continue;
        const prc_handle* h = b->frames[o];
        if (!h->far_t.on() || !h->far_field.on()) continue;
        std::vector<int> list{o};
        for (int i = o + 1; i < n_frames; ++i)
            if (owner[i] == o) list.push_back(i);
        for (size_t k = 0; k + 1 < list.size(); k += kMaxFrames) {
            const size_t m = std::min(list.size() - k, (size_t)kMaxFrames);
            if (m < 2) break;
            float4 *u4 = nullptr, *r4 = nullptr;
            cudaError_t e = cudaMalloc(&u4, h->n * sizeof(float4));
            if (e == cudaSuccess) b->chunk_u4.push_back(u4), e = cudaMalloc(&r4, h->n * sizeof(float4));
            if (e == cudaSuccess) b->chunk_r4.push_back(r4);
            if (e == cudaSuccess) e = cudaMemsetAsync(u4, 0, h->n * sizeof(float4), b->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(r4, 0, h->n * sizeof(float4), b->stream);
            if (e != cudaSuccess) {
                prc_batch_destroy(b);
                return fail(e == cudaErrorMemoryAllocation ? PRC_ERR_MEMORY : PRC_ERR_CUDA,
                            std::string("CUDA error '") + cudaGetErrorString(e) + "' for shared frame passes");
            }
            for (size_t j = 0; j < m; ++j) b->chunk_of[list[k + j]] = (int)b->chunks.size(), b->slot_of[list[k + j]] = (int)j;
            b->chunks.emplace_back(list.begin() + k, list.begin() + k + m);
        }
    }
    if (const cudaError_t e = cudaStreamSynchronize(b->stream); e != cudaSuccess) {
        prc_batch_destroy(b);
        return fail(PRC_ERR_CUDA, std::string("CUDA error '") + cudaGetErrorString(e) + "' in prc_batch_create");
    }
    *out = b;
    return PRC_OK;
}

int prc_batch_em_run(prc_batch* b, const float* const* d_g, float* const* d_out, int iterations, float beta,
                     float gamma, int accelerate) {
    if (!b || !d_g || !d_out || iterations < 1 || !(beta >= 0) || !(gamma >= 0))
        return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    for (prc_handle* h : b->frames)
        if (h->n_active == 0) return fail(PRC_ERR_NO_ACTIVITY, "No tissue voxels in a frame: nothing to do");
    const int n = (int)b->frames.size();
    if (!b->tuned) {
        // autotune the projector's warps per block on one forward projection of every frame
        float best = 3.0e38f;
        int best_w = prc_batch::kWarpsDefault;
        cudaEvent_t e0, e1;
        PRC_CUDA(cudaEventCreate(&e0));
        PRC_CUDA(cudaEventCreate(&e1));
        for (int w : {2, 4, 8}) {
            BatchPlan plan = plan_batch(b, d_g, d_out, 0, beta, gamma, accelerate != 0, w, true);
            int rc = upload_plan(b, plan);
            if (rc == PRC_OK) rc = enqueue_plan(b, plan, d_out, beta, gamma, accelerate != 0, w);  // warm-up
            PRC_CUDA(cudaEventRecord(e0, b->stream));
            if (rc == PRC_OK) rc = enqueue_plan(b, plan, d_out, beta, gamma, accelerate != 0, w);
            PRC_CUDA(cudaEventRecord(e1, b->stream));
            PRC_CUDA(cudaEventSynchronize(e1));
            if (rc != PRC_OK) return rc;
            float ms = 0.0f;
            PRC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) best = ms, best_w = w;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->warps = best_w;
        b->tuned = true;
    }
    const std::vector<const float*> key_g(d_g, d_g + n);
    const std::vector<float*> key_out(d_out, d_out + n);
    const bool same = b->exec && key_g == b->key_g && key_out == b->key_out && b->key_iters == iterations &&
                      b->key_beta == beta && b->key_gamma == gamma && b->key_accel == accelerate;
    if (!same) {
        release_graph(b);
        BatchPlan plan = plan_batch(b, d_g, d_out, iterations, beta, gamma, accelerate != 0, b->warps, false);
        int rc = upload_plan(b, plan);
        if (rc != PRC_OK) return rc;
        PRC_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_plan(b, plan, d_out, beta, gamma, accelerate != 0, b->warps);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
        if (rc != PRC_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        PRC_CUDA(ce);
        b->graph = graph;
        PRC_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->key_g = key_g, b->key_out = key_out, b->key_iters = iterations, b->key_beta = beta;
        b->key_gamma = gamma, b->key_accel = accelerate;
    }
    PRC_CUDA(cudaGraphLaunch(b->exec, b->stream));
    return PRC_OK;
}

int prc_batch_profile(prc_batch* b, const float* const* d_g, float* const* d_out, int iterations, float beta,
                      float gamma, int accelerate, double* graph_ms, double* launches_ms, int* launches) {
    if (!graph_ms || !launches_ms || !launches) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    int rc = prc_batch_em_run(b, d_g, d_out, iterations, beta, gamma, accelerate);  // tuned, captured, warm
    if (rc != PRC_OK) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PRC_CUDA(cudaEventCreate(&e0));
    PRC_CUDA(cudaEventCreate(&e1));
    PRC_CUDA(cudaEventRecord(e0, b->stream));
    PRC_CUDA(cudaGraphLaunch(b->exec, b->stream));
    PRC_CUDA(cudaEventRecord(e1, b->stream));
    PRC_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    PRC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *graph_ms = ms;
    // the same schedule launch by launch (its tables are the graph's, uploaded again unchanged)
    BatchPlan plan = plan_batch(b, d_g, d_out, iterations, beta, gamma, accelerate != 0, b->warps, false);
    rc = upload_plan(b, plan);
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed;
    if (rc == PRC_OK) rc = enqueue_plan(b, plan, d_out, beta, gamma, accelerate != 0, b->warps, &timed);
    double sum = 0.0;
    if (rc == PRC_OK) {
        PRC_CUDA(cudaStreamSynchronize(b->stream));
        for (auto& ev : timed) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, ev.first, ev.second) == cudaSuccess) sum += t;
        }
    }
    for (auto& ev : timed) cudaEventDestroy(ev.first), cudaEventDestroy(ev.second);
    *launches_ms = sum;
    *launches = (int)timed.size();
    return rc;
}

int prc_batch_synchronize(prc_batch* b) {
    if (!b) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    PRC_CUDA(cudaStreamSynchronize(b->stream));
    for (prc_handle* h : b->frames) {
        const int rc = check_device_error(h);
        if (rc != PRC_OK) return rc;
    }
    return PRC_OK;
}

void* prc_batch_stream(const prc_batch* b) { return b ? (void*)b->stream : nullptr; }

int prc_batch_frame(prc_batch* b, int i, prc_handle** out) {
    if (!b || !out || i < 0 || i >= (int)b->frames.size()) return fail(PRC_ERR_ARGUMENT, "Invalid argument");
    *out = b->frames[i];
    return PRC_OK;
}

int prc_batch_warps(const prc_batch* b) { return b ? b->warps : 0; }

}  // extern "C"
