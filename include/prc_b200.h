/*
 * prc_b200.h -- C ABI of the B200 positron-range-correction engine (libprc_b200.so).
 *
 * The reference (jlherraiz/PRC_MLEM) exposes its hot path only through the `prc` executable
 * (prc.cu:564-722); inside it the operator seam is `class Projector` (prc.cu:403-450) and the
 * MAP-EM loop of main() (prc.cu:659-711).  This header is that seam as a library: every entry
 * point names the reference code it replaces.  All functions:
 *   - are host-callable, return 0 (PRC_OK) or a PRC_ERR_* code and never exit the process;
 *   - take plain pointers and sizes; "d_" pointers are device (CUDA global memory) arrays of
 *     nx*ny*nz float32 values, X fastest (NumPy shape nz, ny, nx), "host" pointers are host
 *     memory of the same layout;
 *   - take `stream` as a cudaStream_t passed as void*; NULL selects the handle's own stream.
 *     Work is enqueued asynchronously unless the function says it synchronises;
 *   - are not thread-safe on one handle; distinct handles are independent.
 * prc_last_error() returns a message for the most recent failure on the calling thread.
 */
#ifndef PRC_B200_H
#define PRC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PRC_OK = 0,
    PRC_ERR_ARGUMENT = 1,    /* invalid geometry or solver parameter ("Invalid ..." in prc.cu:540-546) */
    PRC_ERR_ISOTOPE = 2,     /* unknown isotope name (prc.cu:570-576) */
    PRC_ERR_NONFINITE = 3,   /* NaN/inf in density or activity (prc.cu:599-602) */
    PRC_ERR_NO_ACTIVITY = 4, /* no activity in the support (prc.cu:619-622) */
    PRC_ERR_CUDA = 5,        /* a CUDA runtime call failed (prc.cu:24-32 exits instead) */
    PRC_ERR_MEMORY = 6,      /* device allocation failed */
    PRC_ERR_STATE = 7,       /* call order violated (e.g. iterate before begin) */
    PRC_ERR_LIMIT = 8        /* voxel count beyond the INT_MAX index limit (prc.cu:547-551) */
};

/* Precision of the projector's stored weights (near cache and far-field coefficient field). */
enum {
    PRC_PRECISION_FP32 = 0,        /* float weights: the reference's numerics */
    PRC_PRECISION_BF16 = 1,        /* bfloat16 stored weights, float accumulation, FP64 global sums */
    PRC_PRECISION_BF16_VOLUMES = 2, /* as PRC_PRECISION_BF16, and inside MAP-EM the volumes the
                                      projections gather (y / W and the EM ratio) in bfloat16 too */
    PRC_PRECISION_FP24 = 3          /* stored-field weights of 24 bits (the non-negative fp32 weight
                                      without its sign bit and rounded to 16 mantissa bits: relative
                                      error <= 2^-17), float near cache,
                                      accumulation and volumes; 3/4 of the fp32 field's bytes.  Not
                                      for surrogate fields. */
};

/* What the projector keeps in device memory between projections.  The reference caches the
 * 5x5x5 near block (prc.cu:411-419) and retraces the far rays in every projection. */
enum {
    PRC_CACHE_NONE = 0, /* retrace near block and far rays every projection (--no-cache-near) */
    PRC_CACHE_NEAR = 1, /* cache the near block, retrace far rays (the reference's default) */
    PRC_CACHE_FULL = 2, /* store every weight (near block and far rays) as a coefficient field
                           indexed by a shared ray template, source-major for the adjoint and
                           target-major for the forward projection (both gathers); falls back to
                           PRC_CACHE_SOURCE_MAJOR, then PRC_CACHE_NEAR, when memory is short */
    PRC_CACHE_SOURCE_MAJOR = 3 /* the source-major field only: half the memory of PRC_CACHE_FULL,
                                  the forward projection scatters with atomics */
};

/* Source tiles of the stored coefficient field: a warp owns 32 tissue voxels taken in tiles
 * of this shape (x fastest inside a tile, tiles in x, y, z order), so every gather of one step
 * touches the rows of one tile shifted by the step's offset.  PRC_TILE_AUTO takes the shape
 * prc_tune_tile chose for the same configuration earlier in the process, or 8x2x2 when it was
 * never tuned; batched frames are tuned per configuration.  The shape changes no result: every
 * source keeps its own weights and summation order. */
enum {
    PRC_TILE_AUTO = 0,
    PRC_TILE_8x2x2 = 1,
    PRC_TILE_16x2x1 = 2,
    PRC_TILE_32x1x1 = 3,
    PRC_TILE_4x4x2 = 4,
    PRC_TILE_16x1x2 = 5
};

/* Volume geometry: positional arguments NX NY NZ DX DY DZ of prc.cu:515-516. */
typedef struct prc_geometry {
    int nx, ny, nz;
    float dx, dy, dz; /* voxel size [mm] */
} prc_geometry;

/* Projector options: --rays, --support-rho, --air-cap-mm, --exact-range, --no-cache-near of
 * prc.cu:452-459, plus the cache mode, the stored-weight precision and the source tile. */
typedef struct prc_options {
    int rays;          /* even far-field rays per source, >= 2 (default 128) */
    float support_rho; /* voxels with density >= support_rho hold activity (default 0.05) */
    float air_cap_mm;  /* a positron that crossed this much sub-support path escaped (default 50) */
    int exact_range;   /* 1: analytic survival instead of the 4097-entry table */
    int cache;         /* PRC_CACHE_* (default PRC_CACHE_FULL) */
    int precision;     /* PRC_PRECISION_* */
    int tile;          /* PRC_TILE_* source tile of the stored field (default PRC_TILE_AUTO) */
} prc_options;

typedef struct prc_handle prc_handle;

/* Fills the reference defaults (prc.cu:456-458). */
void prc_default_options(prc_options* opts);

/* Water-equivalent 99.95 % range cutoff [mm] of an isotope, with the weight fix of
 * prc.cu:577-584 and the bisection of prc.cu:83-91.  Host only, no CUDA call. */
int prc_isotope_cutoff(const char* isotope, float* cutoff_mm);

/* Number of supported isotopes and the name of the i-th one (usage text, prc.cu:482). */
int prc_isotope_count(void);
const char* prc_isotope_name(int i);

/* Builds the projector for one density map (host array, g/cm3): clamps density to >= 1e-3,
 * derives the support and active-source list (prc.cu:598-613), uploads them, and runs the
 * normalisation pass that computes W_s and the near-field cache (Projector::Projector,
 * prc.cu:405-422).  Synchronises.  Rejects non-finite density with PRC_ERR_NONFINITE. */
int prc_create(const prc_geometry* geometry, const char* isotope, const prc_options* opts,
               const float* density_host, prc_handle** out);

/* The same operator with the far field of every source replaced by 128 directions x 16 radial
 * bins of range-kernel coefficients predicted by the learned surrogate `net` (a prc_net* from
 * prc_surrogate.h; NULL = the traced radial kernels of every source, i.e. the surrogate
 * representation without a network) from the density patch around the source.  No
 * counterpart in the reference.  target_scale is the factor the network was trained with.
 * The ray tracer judges every (source, far ray): a ray whose traced mass reaches more than 2%
 * past the water-equivalent range of the bins, with a network every ray the volume's edge cuts
 * inside that range, and (fallback_nrmse > 0) every ray whose predicted coefficients differ
 * from the traced ones by more than fallback_nrmse times the source's RMS ray norm (L2 over
 * the ray's 16 bins) keeps its exact ray-marched weights, for all 32 sources of its stream
 * group; the other rays store the coefficients of the water range.  *fallbacks (optional)
 * receives the number of (source, far ray) pairs on exact weights (out of n_active x rays).
 * The near block is traced exactly.  Forward, adjoint and MAP-EM then work as for prc_create.  Synchronises. */
typedef struct prc_net prc_net;
int prc_create_surrogate(const prc_geometry* geometry, const char* isotope, const prc_options* opts,
                         const float* density_host, prc_net* net, float target_scale, float fallback_nrmse,
                         int64_t* fallbacks, prc_handle** out);

/* The source-tile autotuner (no counterpart in the reference): builds the stored field of the
 * central slab (at most 32 z-slices) of this density with each candidate tile (8x2x2, 16x2x1,
 * 32x1x1), times one forward and one adjoint projection of each with CUDA events, and returns the
 * fastest in *tile.  The choice is remembered for the configuration (grid, spacing, isotope,
 * rays, support, air cap, form) for the rest of the process, so later calls and PRC_TILE_AUTO
 * handles of it cost nothing.  Synchronises. */
int prc_tune_tile(const prc_geometry* geometry, const char* isotope, const prc_options* opts,
                  const float* density_host, int* tile);

/* Releases every device allocation of the handle (Projector::~Projector, prc.cu:423-427). */
void prc_destroy(prc_handle* h);

/* Tissue (active) voxel count and the water-equivalent cutoff of the handle. */
int prc_active_count(const prc_handle* h, int64_t* n_active);
int prc_cutoff(const prc_handle* h, float* cutoff_mm);
/* Bytes of device memory the handle owns. */
int prc_device_bytes(const prc_handle* h, int64_t* bytes);
/* The cache mode in effect (PRC_CACHE_*, after any fall-back) and the entries of the stored
 * field: source-major (used by the adjoint) and target-major (used by the forward projection,
 * which falls back to an atomic scatter over the source-major field when this copy is 0). */
int prc_cache_mode(const prc_handle* h, int* mode, int64_t* source_major_entries, int64_t* target_major_entries);
/* The handle's stream (a cudaStream_t) as void*. */
void* prc_stream(const prc_handle* h);

/* d_out = A d_in, overwritten on every voxel (Projector::forward, prc.cu:430-434). */
int prc_forward(prc_handle* h, const float* d_in, float* d_out, void* stream);

/* d_out[s] = (A^T d_in)[s] on tissue voxels; other voxels are left untouched
 * (Projector::adjoint, prc.cu:436). */
int prc_adjoint(prc_handle* h, const float* d_in, float* d_out, void* stream);

/* Starts a MAP-EM run on measured data d_g: clamps it to >= 0 and zeroes it off the support,
 * computes eps = 1e-6 * sum / n_active, floors the estimate at 1000 eps and rescales it to the
 * measured counts (prc.cu:604-613, 666-672).  All on device; no host synchronisation. */
int prc_em_begin(prc_handle* h, const float* d_g, void* stream);

/* Runs n further MAP-EM iterations (extrapolate, forward, ratio, adjoint, RDP update, count
 * rescale, Biggs-Andrews step length; prc.cu:675-700).  beta >= 0 is the RDP strength, gamma >= 0
 * its edge parameter, accelerate = 0 gives plain MAP-EM (--no-accel).  The step length and the
 * count rescale are computed on device in FP64, so no call synchronises.  The acceleration
 * history carries over between calls, so k calls of n iterations equal one call of k*n. */
int prc_em_iterate(prc_handle* h, int n, float beta, float gamma, int accelerate, void* stream);

/* Copies the current estimate into d_out (all voxels). */
int prc_em_estimate(prc_handle* h, float* d_out, void* stream);

/* prc_em_begin + prc_em_iterate + prc_em_estimate.  iterations == 0 returns the supported,
 * clamped input unchanged, as prc.cu:669 skips initialisation. */
int prc_em_run(prc_handle* h, const float* d_g, float* d_out, int iterations, float beta, float gamma,
               int accelerate, void* stream);

/* The same correction from and to host memory: copies g_host in, runs, copies the estimate
 * back into out_host.  Synchronises. */
int prc_em_run_host(prc_handle* h, const float* g_host, float* out_host, int iterations, float beta,
                    float gamma, int accelerate);

/* Frames of one dynamic study: n_frames volumes that share this handle's density map, isotope
 * and grid, hence its operator.  Each is the reference's single-volume computation run once per
 * frame (prc.cu:430-436 for the projections, prc.cu:659-711 for MAP-EM: main() corrects one
 * volume per process).  With the stored field (PRC_CACHE_FULL in both majors) every projection
 * reads the field once for up to four frames, and each frame's result is bit-identical to the
 * single-volume entry point's on the same input; other forms (and the bf16-volume precision in
 * MAP-EM) run the frames one after another through the single-volume entry points.  d_in / d_g
 * and d_out are arrays of n_frames device pointers to distinct volumes; enqueued on `stream`
 * like the single-volume forms.  After the first call the handle keeps, for reuse, n_frames sets of MAP-EM volumes
 * (7 volumes each) and two interleaved volumes (16 bytes per voxel) per group of four frames;
 * the single-volume MAP-EM state is separate and untouched. */
int prc_forward_frames(prc_handle* h, int n_frames, const float* const* d_in, float* const* d_out, void* stream);
int prc_adjoint_frames(prc_handle* h, int n_frames, const float* const* d_in, float* const* d_out, void* stream);
int prc_em_run_frames(prc_handle* h, int n_frames, const float* const* d_g, float* const* d_out, int iterations,
                      float beta, float gamma, int accelerate, void* stream);

/* prc_em_begin from host memory, and the current estimate copied back to host memory (the
 * checkpoint path of --save-every, prc.cu:705-709).  Synchronise. */
int prc_em_begin_host(prc_handle* h, const float* g_host);
int prc_em_estimate_host(prc_handle* h, float* out_host);

/* Host-memory forms of the two operators (the --mode forward / adjoint paths, prc.cu:648-657).
 * prc_adjoint_host writes every voxel of out_host: A^T in on tissue, 0 elsewhere.  Synchronise. */
int prc_forward_host(prc_handle* h, const float* in_host, float* out_host);
int prc_adjoint_host(prc_handle* h, const float* in_host, float* out_host);

/* FP64 sum of a device volume (device_sum, prc.cu:392-395).  Synchronises. */
int prc_sum(prc_handle* h, const float* d_x, double* sum, void* stream);

/* Number of (source, target) deposits of one projection, near and far (the V of the
 * algorithmic-bytes accounting).  Synchronises. */
int prc_count_deposits(prc_handle* h, int64_t* deposits);

/* FP64 sum of n device floats into *d_sum (device memory), enqueued on `stream` (a
 * cudaStream_t; NULL = the default stream).  It allocates no device memory: no counterpart in
 * the reference; it exists for callers that cannot allocate at the point of the call (services
 * that reserve all device memory at start-up, hot paths that must not pay cudaMalloc's
 * synchronisation, operators inside another framework's allocator).  Its scratch is a
 * file-scope device array of about 512 KiB that every GPU loading the library holds until
 * exit; n is limited to 2^28 elements (PRC_ERR_LIMIT beyond).  The first call on each device
 * looks up that array's device address, and under CUDA's lazy module loading (the default)
 * that lookup is what loads the array onto the device: make one warm-up call per device at
 * start-up, before reserving the rest of device memory and before any stream capture (or run
 * with CUDA_MODULE_LOADING=EAGER); later calls allocate nothing.  A failed lookup is retried by
 * the next call.  All calls share the array: calls that overlap on the GPU (other streams,
 * other threads) race. */
int prc_sum_static(const float* d_x, int64_t n, double* d_sum, void* stream);

/* ---- batched frames (dynamic PET) ---------------------------------------------------------
 * No counterpart in the reference.  Many volumes of different grids and isotopes corrected
 * together: every MAP-EM phase of every frame runs as one launch (the projector's blocks map to
 * (frame, group); the image updates take one grid row per frame, each with its own FP64
 * reductions), and the whole schedule of a run is captured once into a CUDA graph and replayed.
 * Each frame chooses its projector form as prc_create does (stored field while memory lasts,
 * then the near cache); with `net`, frames of 18F, 68Ga and 82Rb use the learned surrogate
 * (prc_create_surrogate with target_scale and fallback_nrmse).  Frames that pass the same
 * density_host pointer with the same geometry and isotope (the frames of one study) share one
 * projector: it is built once, and the later frames hold only their own MAP-EM volumes.  The
 * first run autotunes the projector's warps per block (2, 4 or 8) on one forward projection of
 * every frame. */
typedef struct prc_frame {
    prc_geometry geometry;
    const char* isotope;
    const float* density_host;
} prc_frame;
typedef struct prc_batch prc_batch;
int prc_batch_create(int n_frames, const prc_frame* frames, const prc_options* opts, prc_net* net,
                     float target_scale, float fallback_nrmse, prc_batch** out);
void prc_batch_destroy(prc_batch* b);
/* d_g[i], d_out[i]: device volumes of frame i.  Enqueued on prc_batch_stream(b); a graph is
 * captured on the first call and re-captured when the pointers or parameters change. */
int prc_batch_em_run(prc_batch* b, const float* const* d_g, float* const* d_out, int iterations, float beta,
                     float gamma, int accelerate);
int prc_batch_synchronize(prc_batch* b);
void* prc_batch_stream(const prc_batch* b);
/* The measurement behind the schedule's design (no counterpart in the reference): runs the
 * MAP-EM schedule of prc_batch_em_run with these arguments as one replay of its captured CUDA
 * graph (*graph_ms, device time) and once more launch by launch with CUDA events around every
 * kernel launch (*launches_ms, the sum over its *launches launches).  graph_ms - launches_ms
 * bounds what fusing the phases of an iteration into one persistent kernel could save.
 * Synchronises. */
int prc_batch_profile(prc_batch* b, const float* const* d_g, float* const* d_out, int iterations, float beta,
                      float gamma, int accelerate, double* graph_ms, double* launches_ms, int* launches);

/* The handle of frame i (owned by the batch), and the autotuned warps per block. */
int prc_batch_frame(prc_batch* b, int i, prc_handle** out);
int prc_batch_warps(const prc_batch* b);

/* Projection timing (no counterpart in the reference, whose main() prints only wall-clock
 * totals): while timing is on, every forward and adjoint projection launch of the handle --
 * those inside prc_em_iterate included -- is bracketed by CUDA events on its stream.
 * prc_timing(h, 1) starts a new measurement, prc_timing(h, 0) stops recording; prc_timing_read
 * waits for the recorded events and returns the summed device milliseconds and the number of
 * launches of each kind since the start. */
int prc_timing(prc_handle* h, int enable);
int prc_timing_read(prc_handle* h, double* forward_ms, int64_t* n_forward, double* adjoint_ms, int64_t* n_adjoint);

/* The source tile (PRC_TILE_*) the handle's stored field uses, after any automatic choice. */
int prc_tile(const prc_handle* h, int* tile);

/* Number of kernels the handle's entry points have enqueued since it was created (projections,
 * MAP-EM image updates and reductions; copies and memsets are not counted).  No counterpart in
 * the reference. */
int prc_launch_count(const prc_handle* h, int64_t* n);

/* Waits for all work on the handle's stream; reports PRC_ERR_CUDA if a kernel gave up a
 * bounded wait since the last check. */
int prc_synchronize(prc_handle* h);

/* Failure-detection self-test (no counterpart in the reference): launches a kernel whose
 * mbarrier wait nothing completes, bounded to `rounds` try_wait rounds (1 .. 2^20); the kernel
 * gives up, raises the handle's error flag and returns, so this returns PRC_ERR_CUDA with the
 * bounded-wait message while the CUDA context stays usable. */
int prc_wait_selftest(prc_handle* h, int rounds);

/* Page-locked host memory for image buffers (cudaMallocHost / cudaFreeHost): the host-memory
 * entry points copy from and to it at full PCIe / C2C speed.  No counterpart in the reference,
 * whose host buffers are pageable std::vectors (prc.cu:592, 646). */
int prc_host_alloc(size_t bytes, void** ptr);
void prc_host_free(void* ptr);

/* Message of the most recent failure on this thread ("" if none). */
const char* prc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PRC_B200_H */
