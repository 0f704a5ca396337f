// engine.h -- internal interface between the C ABI (prc_abi.cu) and the kernel files
// (projector.cu, em.cu).  Not installed; the public surface is include/prc_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <string>

#include "range_model.h"

namespace prc {

// Uniform DDA state of one ray, derived once per run from ray(k, n) exactly as prc.cu:138-142
// derives it at the start of every trace: distances [mm] to the first x/y/z voxel faces, the
// distances between consecutive faces and the step signs.  Every source traces a ray k from
// the same sub-voxel offset along the same direction, so this record is shared by all sources.
struct RayStep {
    float tx, ty, tz;
    float dtx, dty, dtz;
    int di, dj, dk;
    int pad;
};

// Layout of a stored field stream (see FarField).
struct StreamLayout {
    const unsigned short* len = nullptr;    // [n_groups][n_rows]: stored steps of row k in group G
    const long long* group_base = nullptr;  // [n_groups + 1]: element offset of group G's stream
    const int* desc = nullptr;              // per pack: template element offset of its first step
};

// Everything a projector kernel needs to know about one volume.
struct ProjParams {
    Grid g;
    int nxy;                 // nx * ny
    int n_active;            // tissue voxels (sources)
    int n_rays;              // far-field rays per source
    const float* rho;        // clamped density, nx*ny*nz
    const int* active;       // linear voxel index of each source, increasing
    const RayStep* far;      // n_rays records
    const RayStep* near;     // kNearRays records
    const short* near_order; // the near rays grouped by direction octant (increasing index in each)
    const int* near_start;   // [9]: first entry of octant o in near_order (o = x+ | y+ << 1 | z+ << 2)
    const float* table;      // kRangeBins + 1 survival samples, or nullptr for analytic
    float table_scale;       // bins per mm
    int n_branch;            // analytic model (used when table == nullptr)
    Branch br[3];
    // Far-field layout (used by the stored field; null until the layout pass has run).
    const int* tmpl;                 // [n_rows][tmpl_len]: linear target offset of step m of row k;
                                     // row 0 is the 5x5x5 block, row 1 + r the post-block steps of
                                     // far ray r (the same for every source)
    const int* tmpl_neg;             // the same offsets negated (target-major gathers: source = t - o)
    int tmpl_len;                    // steps per row: covers every step a ray takes in the image
    int n_rows;                      // n_rays + 1
    StreamLayout src;                // source-major field: group = 32 consecutive sources (8x2x2 tiles)
    StreamLayout tgt;                // target-major field: group = 32 consecutive targets
    const int* vox2src;              // voxel -> source index, -1 off the support
};

// Stored weights ("coefficient field") of near block and far rays: for group G, template row k,
// step m and lane l, the entry group_base[G] + (sum_{k'<k} len[G][k']) * 32 + (m / 4) * 128 +
// l * 4 + m % 4.  Target voxels come from the template, so no index is stored.  The
// source-major field (lane = source s, target s + o) serves the adjoint as a gather; the
// target-major copy of the same weights (lane = target t, source t - o) serves the forward as a
// gather of u = f / W.
struct FarField {
    float* f32 = nullptr;
    __nv_bfloat16* b16 = nullptr;
    // 24-bit weights: bits 30..7 of each (non-negative) fp32 weight rounded to nearest (8 exponent
    // bits, 16 mantissa bits), little-endian, 3 bytes per entry
    unsigned char* b24 = nullptr;
    __host__ __device__ bool on() const { return f32 || b16 || b24; }
};

// Near-field weight cache, group-interleaved: entry (source src, block offset q) lives at
// ((src / 32) * 125 + q) * 32 + src % 32, so the 32 sources of one warp read 128 contiguous
// bytes per offset.  Exactly one of f32 / b16 is non-null when the cache is on.
struct NearCache {
    float* f32 = nullptr;
    __nv_bfloat16* b16 = nullptr;
    __host__ __device__ bool on() const { return f32 || b16; }
};

// Norm: W and the caches.  Forward / Adjoint: the operators.  Count: deposits per projection.
// Layout: per group and ray, the number of post-block steps up to the last deposit of any lane
// (written to len; the per-group totals to a.group_total).
enum class Op : int { Norm = 0, Forward = 1, Adjoint = 2, Count = 3, Layout = 4 };

// Per-launch operands.  Norm writes W (and the cache when it is on); Forward scatters
// f_s / W_s * w_st into out (which must be zeroed first); Adjoint writes out[s] on tissue;
// Count adds the deposit count to *count.
struct OpArgs {
    const float* in = nullptr;   // f (Forward) or the gathered image (Adjoint)
    float* out = nullptr;
    float* W = nullptr;
    NearCache near;
    FarField far;                          // source-major stored field
    FarField farT;                         // target-major stored field (forward as a gather)
    unsigned long long* count = nullptr;
    unsigned int* error = nullptr;         // set non-zero when a stored-field copy timed out
    unsigned short* len = nullptr;         // Layout output
    long long* group_total = nullptr;      // Layout output: entries per group (sum of len * 32)
    // Norm: fp32 accumulator of the traced near block, [group][125 offsets][32 lanes].  When set,
    // the near rays are traced one direction octant at a time into a 27-offset shared-memory tile
    // (3.4 KB per warp instead of 16 KB, so four times the warps fit on an SM).
    float* near_acc = nullptr;
    // Forward gather form inside MAP-EM: when set, the epilogue writes the EM ratio
    // ratio_g[t] / max((A f)_t, *ratio_eps) of every tissue voxel instead of (A f)_t (prc.cu:270-274).
    const float* ratio_g = nullptr;
    const float* ratio_eps = nullptr;
    // bf16 volumes (mixed-precision form inside MAP-EM): the gathered input and the forward's
    // ratio output; only with the bf16 field (the gather of in16 replaces that of in).
    const __nv_bfloat16* in16 = nullptr;
    __nv_bfloat16* out16 = nullptr;
};

// ---- radial surrogate support -----------------------------------------------------------------
// The surrogate summarises the far field of a source by 16 radial bins per far ray: bin b of ray
// r gathers the deposits whose segment midpoint lies at path length t in [e_b, e_{b+1}), with
// 12 equal bins up to the water-equivalent cutoff and 4 equal bins from there to 3.85 x cutoff
// (the range in 0.26 g/cm3 lung).  Each (ray, bin) is deposited at one fixed step of the ray:
// the post-block step whose midpoint is closest to the bin centre.
constexpr int kRadialBins = 16;
struct RadialTables {
    unsigned char* bin_of = nullptr;  // [n_rays][tmpl_len]: bin of post-block step m of ray r
    int* offset = nullptr;            // [n_rays][16]: linear target offset of bin b of ray r
    int* xyz = nullptr;               // the same offset as packed (dx+512) | (dy+512) << 10 | (dz+512) << 20
};
cudaError_t build_radial_tables(const ProjParams& p, const RadialTables& t, cudaStream_t s);
// Traced radial coefficients out[i][r][b] (fp32) of sources src[i] (voxel indices), sources
// 32i..32i+31 all in volume vol_of_warp(i) = (i / 32) / warps_per_volume of rho + vol * volume
// voxels.  n_src must be a multiple of 32.
cudaError_t radial_kernels(const ProjParams& p, const RadialTables& t, const int* src, int n_src,
                           int warps_per_volume, float* out, cudaStream_t s);
// Surrogate field fill: near block traced as in the Norm pass (row 0); far ray r of group G
// exactly traced into row 1 + r where fallback_rays[G * n_rays + r] is set (the Norm pass's
// weights), otherwise its first `water_bins` radial coefficients coef[src][r*16 + b] (bf16) into
// row 1 + n_rays + r, each dropped where its target voxel is outside the image or not tissue;
// W_s = the sum of every stored weight.
cudaError_t surrogate_fill(const ProjParams& p, const OpArgs& a, const RadialTables& t, const __nv_bfloat16* coef,
                           const unsigned char* support, const unsigned char* fallback_rays, int water_bins,
                           cudaStream_t s);
// Template rows of the surrogate field: row 0 the near block, row 1 + r the 16 bin offsets.
cudaError_t build_surrogate_template(const ProjParams& p, const RadialTables& t, int* tmpl, int* tmpl_neg,
                                     cudaStream_t s);

}  // namespace prc
struct prc_net;
namespace prc {
// Whole-volume CNN inference into bf16 coefficients coef[src][2048] (surrogate.cu).
int surrogate_infer(prc_net* net, const float* rho, int nx, int ny, int nz, int iso, const int* active, int n_active,
                    float inv_target_scale, __nv_bfloat16* coef, cudaStream_t s);
// The tracer's judgement of sources [first, first + n_src), ray by ray: a far ray of a source is
// poorly represented when the L2 norm of (stored prediction - traced coefficients) over its 16
// bins exceeds `threshold` times the source's RMS ray norm (the square root of the mean over
// its rays of the traced squared norm; skipped when threshold < 0), or when more than `beyond`
// of its traced mass lies past the water-equivalent cutoff distance (a ray through lung or out
// of the body, where the radial bins are coarse), or (threshold >= 0) when the volume's edge
// cuts it inside the water range (the voxel of its last water bin, from the packed offsets
// bin_xyz of RadialTables::xyz, lies outside the nx x ny x nz volume: a truncated kernel).  The
// stored prediction is zero past the water bins.  Sources are active[first + i].  Without a
// network (threshold < 0) the traced coefficients are copied into coef.  coef and traced hold
// n_rays x 16 bins per source; flags[(first + i) * n_rays + r] is set to 1 for a poorly
// represented ray r of source first + i, 0 otherwise.
cudaError_t surrogate_judge(__nv_bfloat16* coef, const float* traced, int n_src, int n_rays, int first,
                            float threshold, float beyond, int water_bins, const int* active, const int* bin_xyz,
                            int nx, int ny, int nz, unsigned char* flags, cudaStream_t s);
// Radial bins of the water range (12, a multiple of 4): the coefficients a surrogate field stores
// for a far ray.
int radial_water_bins();
// A far ray with more than this share of its traced mass past the water range keeps its exact
// weights in a surrogate field (and trains no network output).
constexpr float kBeyondShare = 0.02f;

// ---- frames that share one stored field (dynamic PET: one density, many activity volumes) ----
// One pass over the stored field projects up to kMaxFrames volumes: every stored weight, its
// template offsets and its predicate are loaded once, and one 16-byte gather of the interleaved
// volume (four frames per voxel) feeds every frame's accumulation.  Per frame the accumulation
// order is the single-volume kernel's, so each frame's result is bit-identical to projecting it
// alone.
constexpr int kMaxFrames = 4;
struct FrameArgs {
    const float* in[kMaxFrames] = {};        // n == 1: the gathered volume (single-volume kernel)
    const float4* in4 = nullptr;             // n >= 2: in4[t] = the frames' gathered values of voxel t
                                             // (u = f / W, or the EM ratio); slots n..3 zero
    float* out[kMaxFrames] = {};             // each frame's result
    float4* out4 = nullptr;                  // forward, n >= 2: results interleaved here instead of out
    const float* ratio_g[kMaxFrames] = {};   // forward inside MAP-EM: write g / max(Af, *eps) (prc.cu:270-274)
    const float* ratio_eps[kMaxFrames] = {};
    int n = 0;                               // frames in this pass, 1..kMaxFrames
};
// Forward (target-major field, a gather of each frame's u) or Adjoint (source-major field) of
// fr.n frames through the stored field of a (fp32, 24-bit or bf16 weights; not the bf16-volume
// form).  cudaErrorInvalidValue when the handle has no such field.
cudaError_t project_frames(Op op, const ProjParams& p, const OpArgs& a, const FrameArgs& fr, cudaStream_t s);
// Interleaving for the frame passes (n frames, 2..4; slots n..3 of every voxel are zero):
// frame_prep: u4 = each frame's y / W (PREDICT: y = the Biggs-Andrews prediction
// max(f + lambda (f - prev), f / 2), written to y[k]; else y = f) on the support, and out[k] = 0
// off it -- per voxel and frame the expressions of forward_prep / forward_prep_extrapolate.
// frame_pack: v4 = the frames' volumes in[k] side by side.
struct FramePrep {
    const float* f[kMaxFrames] = {};
    const float* prev[kMaxFrames] = {};
    const float* lambda[kMaxFrames] = {};
    float* y[kMaxFrames] = {};
    float* out[kMaxFrames] = {};
    int n = 0;
};
cudaError_t frame_prep(const ProjParams& p, const float* W, const FramePrep& fp, bool predict, float4* u4,
                       cudaStream_t s);
cudaError_t frame_pack(const float* const* in, int n, size_t voxels, float4* v4, cudaStream_t s);

// ---- batched projection over many volumes (one launch for all) --------------------------------
enum BatchMode : int {
    kBatchTraceMarch = 0,      // near block and far rays traced every pass
    kBatchCacheF32March = 1,   // near cache (fp32 / bf16), far rays traced
    kBatchCacheBF16March = 2,
    kBatchFieldF32 = 3,        // stored field, source-major (adjoint gather / forward scatter)
    kBatchFieldBF16 = 4,
    kBatchFieldF32T = 5,       // stored field, target-major (forward gather of u = f / W)
    kBatchFieldBF16T = 6,
    kBatchField24 = 7,         // the 24-bit field, source-major and target-major
    kBatchField24T = 8,
    // frames sharing one projector, up to four per item (BatchItem::fr, interleaved volumes)
    kBatchFramesF32 = 9,
    kBatchFramesBF16 = 10,
    kBatchFrames24 = 11,
    kBatchFramesF32T = 12,
    kBatchFramesBF16T = 13,
    kBatchFrames24T = 14
};
struct BatchItem {
    ProjParams p;
    OpArgs a;
    FrameArgs fr;  // kBatchFrames* modes: the frames of this item (fr.in4, fr.out[0..fr.n))
    int mode;
    int first_block;  // blocks [first_block, first_block + blocks) of the launch belong to this item
    int blocks;
    int pad;
};
// Dynamic shared memory per warp a mode needs.
size_t batch_smem_per_warp(int mode);
cudaError_t project_batch(Op op, const BatchItem* d_items, int n_items, int total_blocks, int warps, size_t smem,
                          cudaStream_t s);
// Batched forward preparation: gather items get u = f / W (and 0 off the support of out),
// scatter items get out = 0.  With u4 set, u goes to component `slot` of the interleaved u4
// instead of u (a frame of a shared pass).
struct PrepItem {
    const int* vox2src;
    const float* W;
    const float* f;
    float* u;
    float* out;
    long long n;
    int gather;
    int slot;
    float4* u4;
};
cudaError_t forward_prep_batch(const PrepItem* d_items, int n_items, cudaStream_t s);

// Self-test of the bounded mbarrier wait: a wait that nothing completes, `rounds` rounds.
cudaError_t wait_selftest(int rounds, unsigned int* error, cudaStream_t s);

// Target-major field construction (setup only).
cudaError_t transpose_lengths(const ProjParams& p, const FarField& far, int* len_t32, cudaStream_t s);
cudaError_t transpose_fill(const ProjParams& p, const FarField& far, const FarField& farT, const int* row_base_t,
                           cudaStream_t s);
// u = f / W on the support (0 where that is not positive, as prc.cu:244-248 skips the source)
// and out = 0 off the support: the input of the gather form of the forward projection.
cudaError_t forward_prep(const ProjParams& p, const float* W, const float* f, float* u, float* out, cudaStream_t s);
// The same preparation fused with the Biggs-Andrews prediction (prc.cu:318-321): every voxel's
// y = max(f + lambda (f - prev), f / 2) with lambda = *lambda, then u = y / W on the support.
cudaError_t forward_prep_extrapolate(const ProjParams& p, const float* W, const float* f, const float* prev,
                                     const float* lambda, float* y, float* u, float* out, cudaStream_t s);
// The same with u stored in bf16 (u16) and no `out` (the ratio goes to its own bf16 volume);
// lambda == nullptr: no prediction, y is not written and u = f / W.
cudaError_t forward_prep_half(const ProjParams& p, const float* W, const float* f, const float* prev,
                              const float* lambda, float* y, __nv_bfloat16* u16, cudaStream_t s);

// projector.cu
cudaError_t setup_rays(const Grid& g, int n_rays, RayStep* d_far, RayStep* d_near, cudaStream_t s);
// Groups the near rays by direction octant (order[kNearRays], start[9]); after setup_rays.
cudaError_t order_near_rays(const RayStep* d_near, short* d_order, int* d_start, cudaStream_t s);
// trace_near: retrace the near block (no cache).  Forward / Adjoint / Count read the stored far
// field when a.far is on, and march the far rays otherwise.
cudaError_t project(Op op, const ProjParams& p, const OpArgs& a, bool trace_near, cudaStream_t s);
// Fills the template ([n_rows][tmpl_len] ints) and its negated copy.
cudaError_t build_template(const ProjParams& p, int* tmpl, int* tmpl_neg, cudaStream_t s);
// Fills the pack descriptors (one int per 128 stored entries) of a stream layout.
cudaError_t build_descriptors(const ProjParams& p, const StreamLayout& l, int* desc, cudaStream_t s);

// Stored steps of the near-block row (125 offsets padded to whole packs).
int near_row_steps();

// em.cu ---------------------------------------------------------------------------------------
// Device scalars of one MAP-EM run; all FP64 where the reference accumulates in FP64.
struct EmScalars {
    double support_sum;  // measured counts on the support
    double sum;          // last FP64 volume sum
    float eps;           // 1e-6 * support_sum / n_active (prc.cu:668)
    float floor;         // 1000 * eps (prc.cu:670)
    float lambda;        // Biggs-Andrews step length for the next prediction
    float scale;         // count rescale of the current iteration
    float init_scale;    // count rescale of the initial estimate
    int pad;
};

// Grid-wide FP64 reduction scratch: block partials, and a counter the last block resets.
struct Reduction {
    double* partials;       // kReduceBlocks * 4
    unsigned int* counter;  // one
};
constexpr int kReduceBlocks = 592;  // 148 SMs x 4
constexpr int kEmThreads = 256;

struct EmVolumes {
    size_t n;            // voxels
    const unsigned char* support;
    EmScalars* scalars;
    Reduction red;
};

// g = support ? max(g_in, 0) : 0 and f = g; with `initialize`, also the floor and count rescale.
cudaError_t em_begin(const EmVolumes& v, const float* g_in, float* g, float* f, int n_active, bool initialize,
                     cudaStream_t s);
cudaError_t em_extrapolate(const EmVolumes& v, const float* f, const float* prev, float* y, cudaStream_t s);
cudaError_t em_ratio(const EmVolumes& v, const float* g, float* est, cudaStream_t s);
cudaError_t em_update(const EmVolumes& v, const Grid& grid, const float* start, const float* back, float* next,
                      float beta, float gamma, cudaStream_t s);
// The RDP update over the tissue voxels only (active[0..n_active), any order): the 26
// neighbour distance weights come precomputed from geo_w (em_geometry_weights), and voxels off
// the support are not written -- `next` must already be 0 there (it is: it holds the EM ratio,
// which is 0 off the support).  Same arithmetic per voxel as em_update.
cudaError_t em_update_active(const EmVolumes& v, const Grid& grid, const int* active, int n_active,
                             const float* geo_w, const float* start, const float* back, float* next, float beta,
                             float gamma, cudaStream_t s);
// geo_w[27] = min(dx, dy, dz) / |offset| for every 3x3x3 neighbour offset (0 at the centre),
// with the expression of prc.cu:293-296.
cudaError_t em_geometry_weights(const Grid& grid, float* geo_w, cudaStream_t s);
cudaError_t em_finish(const EmVolumes& v, float* next, float* residual, const float* h_prev, bool use_scale,
                      cudaStream_t s);
cudaError_t em_sum(const EmVolumes& v, const float* x, cudaStream_t s);

// One volume of a batched MAP-EM phase: its scratch and the buffers of the current iteration
// (start = accelerate ? y : f, the adjoint lands in prev, the new estimate in est).
struct EmItem {
    EmVolumes v;
    Grid grid;
    int n_active;
    int pad;
    const int* active;    // the tissue voxels (the RDP update visits only these)
    const float* geo_w;   // the RDP's 27 neighbour distance weights
    const float* g_in;
    float* g;
    float* f;
    float* prev;
    float* y;
    float* h_prev;
    float* est;
};
enum class EmPhase : int { Begin = 0, Extrapolate = 1, Ratio = 2, Update = 3, Finish = 4 };
// One launch (three for Begin) covering every item; blocks per item at most kReduceBlocks.
cudaError_t em_batch_phase(EmPhase phase, const EmItem* d_items, int n_items, int blocks, float beta, float gamma,
                           bool accelerate, cudaStream_t s);
cudaError_t em_mask_copy(const EmVolumes& v, const float* src, float* dst, float fill, cudaStream_t s);

// Sets the message prc_last_error() returns on this thread (for entry points outside prc_abi.cu).
void set_last_error(const std::string& msg);

}  // namespace prc
