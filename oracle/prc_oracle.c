/*
 * prc_oracle.c -- CPU restatement of the positron-range projector and MAP-EM loop of
 * jlherraiz/PRC_MLEM (prc.cu).  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it as the checker; the product never links it.
 *
 * Parity is pinned two ways: against outputs of the reference executable itself (prc.cu built
 * for sm_100a by oracle/build_ref.sh, run on a B200; fixtures under tests/golden/) and against
 * the reference's own FP64 range quadrature tests/reference.py::kernel (homogeneous water KAT).
 *
 * Every routine exists in two precisions, generated from one body by the REAL macro below:
 *   *_f64 : FP64 arithmetic; survival analytic (table_bins == 0) or from an FP64 table;
 *   *_f32 : float arithmetic mirroring prc.cu's device code (4097-entry float table, fmaf lerp).
 * Citations are prc.cu line numbers.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NEAR_R 2
#define NEAR_SIDE 5
#define NEAR_N 125
#define NEAR_RAYS 2048
#define RANGE_BINS 4096
#define MIN_DENSITY 1.0e-3f

typedef struct {
    int nx, ny, nz;
    float sx, sy, sz;
    float cutoff;       /* water-equivalent cutoff [mm] (prc.cu:97) */
    float support_rho;  /* tissue threshold (prc.cu:98) */
    float air_cap;      /* consecutive sub-support path limit [mm] (prc.cu:99) */
    int n_rays;         /* far-field rays, even */
    int n_branch;
    float br[3][5];     /* w, a, b, c, f per branch, weights already fixed (prc.cu:577-584) */
    int table_bins;     /* f32: ignored (always the 4097-entry float table unless exact);
                           f64: 0 = analytic survival, >0 = FP64 lerp table of that many bins */
    int exact_range;    /* f32 only: analytic float survival instead of the table (prc.cu:75) */
    int threads;        /* OpenMP threads, 0 = default */
} oracle_params;

/* ---------------------------------------------------------------- isotope model (prc.cu:38-91) */
typedef struct { const char* name; int n; float br[3][5]; } iso_entry;
static const iso_entry kIso[] = {
    {"11C", 1, {{1.000f, 0.777f, 0.468f, 0.217f, 0.010f}}},
    {"13N", 1, {{1.000f, 0.537f, 0.347f, 0.193f, 0.050f}}},
    {"15O", 1, {{1.000f, 0.295f, 0.221f, 0.133f, 0.118f}}},
    {"18F", 1, {{1.000f, 1.612f, 0.703f, 0.526f, 0.011f}}},
    {"64Cu", 1, {{1.000f, 1.494f, 0.000f, 0.631f, 0.251f}}},
    {"68Ga", 2, {{0.014f, 1.048f, 0.000f, 0.475f, 0.271f}, {0.986f, 0.289f, 0.137f, 0.159f, 0.322f}}},
    {"82Rb", 2, {{0.136f, 0.191f, 0.084f, 0.114f, 0.408f}, {0.857f, 0.135f, 0.063f, 0.087f, 0.451f}}},
    {"124I", 3, {{0.013f, 1.007f, 0.000f, 0.421f, 0.443f}, {0.515f, 0.412f, 0.000f, 0.210f, 0.458f},
                 {0.471f, 0.241f, 0.000f, 0.150f, 0.369f}}},
};

/* float survival exactly as the host code evaluates it (prc.cu:65-72) */
static float survival_f(const float br[][5], int n, float r) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) {
        const float x = br[i][2] * r, y = br[i][3] * r;
        s += br[i][0] * expf(-(powf(br[i][1] * r, 1.0f + br[i][4]) + x * x * sqrtf(x) + y * y * y * sqrtf(y)));
    }
    return s;
}

static double survival_d(const float br[][5], int n, double r) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) {
        const double x = (double)br[i][2] * r, y = (double)br[i][3] * r;
        s += (double)br[i][0] *
             exp(-(pow((double)br[i][1] * r, 1.0 + (double)br[i][4]) + x * x * sqrt(x) + y * y * y * sqrt(y)));
    }
    return s;
}

/* Looks up an isotope, applies the weight fix (prc.cu:577-584) and the 99.95 % cutoff
 * bisection (prc.cu:83-91, 587).  Returns 0, or -1 for an unknown name. */
int oracle_isotope(const char* name, int* n_branch, float* br15, float* cutoff) {
    for (size_t k = 0; k < sizeof(kIso) / sizeof(kIso[0]); ++k) {
        if (strcmp(name, kIso[k].name) != 0) continue;
        float br[3][5];
        memcpy(br, kIso[k].br, sizeof(br));
        const int n = kIso[k].n;
        float wsum = 0.0f;
        int smallest = 0;
        for (int b = 0; b < n; ++b) {
            wsum += br[b][0];
            if (br[b][0] < br[smallest][0]) smallest = b;
        }
        br[smallest][0] += 1.0f - wsum;
        float lo = 0.0f, hi = 1.0f;
        while (1.0f - survival_f(br, n, hi) < 0.9995f && hi < 256.0f) hi *= 2.0f;
        for (int it = 0; it < 64; ++it) {
            const float mid = 0.5f * (lo + hi);
            if (1.0f - survival_f(br, n, mid) < 0.9995f) lo = mid; else hi = mid;
        }
        *n_branch = n;
        memcpy(br15, br, sizeof(br));
        *cutoff = hi;
        return 0;
    }
    return -1;
}

/* ---------------------------------------------------------------- survival tables */
typedef struct {
    const oracle_params* p;
    float* tf;      /* float table, RANGE_BINS + 1 entries */
    float sf;       /* float bins per mm */
    double* td;     /* double table, bins + 1 entries */
    double sd;
    int bins_d;
} surv_ctx;

static void surv_init(surv_ctx* c, const oracle_params* p, int f32) {
    memset(c, 0, sizeof(*c));
    c->p = p;
    if (f32) {
        if (p->exact_range) return;
        c->sf = RANGE_BINS / p->cutoff;  /* prc.cu:626-628 */
        c->tf = (float*)malloc(sizeof(float) * (RANGE_BINS + 1));
        for (int j = 0; j <= RANGE_BINS; ++j) c->tf[j] = survival_f(p->br, p->n_branch, j / c->sf);
    } else if (p->table_bins > 0) {
        c->bins_d = p->table_bins;
        c->sd = (double)p->table_bins / (double)p->cutoff;
        c->td = (double*)malloc(sizeof(double) * (p->table_bins + 1));
        for (int j = 0; j <= p->table_bins; ++j) c->td[j] = survival_d(p->br, p->n_branch, j / c->sd);
    }
}

static void surv_free(surv_ctx* c) {
    free(c->tf);
    free(c->td);
}

/* prc.cu:74-80 */
static inline float surv_at_f(const surv_ctx* c, float w) {
    if (!c->tf) return survival_f(c->p->br, c->p->n_branch, w);
    const float u = w * c->sf;
    int i = (int)u;
    if (i > RANGE_BINS - 1) i = RANGE_BINS - 1;
    const float lo = c->tf[i], hi = c->tf[i + 1];
    return fmaf(fminf(u - (float)i, 1.0f), hi - lo, lo);
}

static inline double surv_at_d(const surv_ctx* c, double w) {
    if (!c->td) return survival_d(c->p->br, c->p->n_branch, w);
    const double u = w * c->sd;
    int i = (int)u;
    if (i > c->bins_d - 1) i = c->bins_d - 1;
    const double lo = c->td[i], hi = c->td[i + 1];
    double a = u - (double)i;
    if (a > 1.0) a = 1.0;
    return lo + a * (hi - lo);
}

/* ---------------------------------------------------------------- rays (prc.cu:118-129) */
static void ray_f(int k, int n, float* x, float* d) {
    const unsigned m = (unsigned)k >> 1;
    const float sign = (k & 1) ? -1.0f : 1.0f, z = 1.0f - (m + 0.5f) / ((n + 1) >> 1);
    const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z)), to_unit = 2.3283064e-10f;
    const float ph = 2.0f * to_unit * (float)(m * 2654435769u);
    const double a = M_PI * (double)ph;
    const float sn = (float)sin(a), cs = (float)cos(a);
    d[0] = sign * r * cs, d[1] = sign * r * sn, d[2] = sign * z;
    x[0] = sign * (to_unit * (float)(0x80000000u + m * 3518319155u) - 0.5f);
    x[1] = sign * (to_unit * (float)(0x80000000u + m * 2882110345u) - 0.5f);
    x[2] = sign * (to_unit * (float)(0x80000000u + m * 2360945575u) - 0.5f);
}

static void ray_d(int k, int n, double* x, double* d) {
    const unsigned m = (unsigned)k >> 1;
    const double sign = (k & 1) ? -1.0 : 1.0, z = 1.0 - (m + 0.5) / ((n + 1) >> 1);
    const double r = sqrt(fmax(0.0, 1.0 - z * z)), to_unit = 2.3283064365386963e-10; /* 2^-32 */
    const double a = M_PI * 2.0 * to_unit * (double)(uint32_t)(m * 2654435769u);
    d[0] = sign * r * cos(a), d[1] = sign * r * sin(a), d[2] = sign * z;
    x[0] = sign * (to_unit * (double)(uint32_t)(0x80000000u + m * 3518319155u) - 0.5);
    x[1] = sign * (to_unit * (double)(uint32_t)(0x80000000u + m * 2882110345u) - 0.5);
    x[2] = sign * (to_unit * (double)(uint32_t)(0x80000000u + m * 2360945575u) - 0.5);
}

static inline int inside_g(const oracle_params* p, int i, int j, int k) {
    return i >= 0 && i < p->nx && j >= 0 && j < p->ny && k >= 0 && k < p->nz;
}

/* ------------------------------------------------------------ precision-generic body
 * The block below is instantiated twice: REAL=double (suffix _f64) and REAL=float (_f32). */
#define ORACLE_BODY(REAL, SFX, RAY, SURV, FMIN, FMAX, FABS, SQRT)                                   \
                                                                                                    \
/* DDA of prc.cu:134-165.  visit(ctx, t, p) receives the linear target index and the deposit. */  \
typedef void (*visit_fn_##SFX)(void* ctx, long t, REAL p);                                         \
static void trace_##SFX(const oracle_params* g, const surv_ctx* sc, const float* rho, int vx,     \
                        int vy, int vz, const REAL* x, const REAL* d, int near, visit_fn_##SFX vf, \
                        void* ctx) {                                                               \
    const REAL big = (REAL)1.0e30;                                                                 \
    const int di = d[0] > 0 ? 1 : -1, dj = d[1] > 0 ? 1 : -1, dk = d[2] > 0 ? 1 : -1;              \
    REAL tx = d[0] != 0 ? ((REAL)0.5 * di - x[0]) * (REAL)g->sx / d[0] : big,                      \
         dtx = d[0] != 0 ? (REAL)g->sx / FABS(d[0]) : big;                                         \
    REAL ty = d[1] != 0 ? ((REAL)0.5 * dj - x[1]) * (REAL)g->sy / d[1] : big,                      \
         dty = d[1] != 0 ? (REAL)g->sy / FABS(d[1]) : big;                                         \
    REAL tz = d[2] != 0 ? ((REAL)0.5 * dk - x[2]) * (REAL)g->sz / d[2] : big,                      \
         dtz = d[2] != 0 ? (REAL)g->sz / FABS(d[2]) : big;                                         \
    int i = vx, j = vy, k = vz;                                                                    \
    REAL t = 0, w = 0, surv = 1, air = 0;                                                          \
    const REAL cutoff = (REAL)g->cutoff, srho = (REAL)g->support_rho, cap = (REAL)g->air_cap;      \
    for (;;) {                                                                                     \
        const int in_block = abs(i - vx) <= NEAR_R && abs(j - vy) <= NEAR_R && abs(k - vz) <= NEAR_R; \
        if (near && !in_block) return;                                                             \
        const REAL t_next = FMIN(tx, FMIN(ty, tz));                                                \
        const long idx = ((long)k * g->ny + j) * g->nx + i;                                        \
        const REAL r = (REAL)rho[idx];                                                             \
        const REAL w_next = FMIN(w + r * (t_next - t), cutoff);                                    \
        const REAL surv_next = SURV(sc, w_next);                                                   \
        if (r >= srho) {                                                                           \
            air = 0;                                                                               \
            if (in_block == near && surv > surv_next) vf(ctx, idx, surv - surv_next);              \
        } else if ((air += t_next - t) > cap) {                                                    \
            return;                                                                                \
        }                                                                                          \
        if (w_next >= cutoff) return;                                                              \
        t = t_next, w = w_next, surv = surv_next;                                                  \
        if (t_next == tx) i += di, tx += dtx;                                                      \
        else if (t_next == ty) j += dj, ty += dty;                                                 \
        else k += dk, tz += dtz;                                                                   \
        if (!inside_g(g, i, j, k)) return;                                                         \
    }                                                                                              \
}                                                                                                  \
                                                                                                   \
typedef struct { REAL* sum; int vx, vy, vz, nx, ny; } near_ctx_##SFX;                              \
static void near_visit_##SFX(void* c, long t, REAL p) {                                           \
    near_ctx_##SFX* n = (near_ctx_##SFX*)c;                                                        \
    const int i = (int)(t % n->nx), j = (int)((t / n->nx) % n->ny), k = (int)(t / ((long)n->nx * n->ny)); \
    n->sum[((k - n->vz + NEAR_R) * NEAR_SIDE + j - n->vy + NEAR_R) * NEAR_SIDE + i - n->vx + NEAR_R] += p; \
}                                                                                                  \
typedef struct { REAL acc; } sum_ctx_##SFX;                                                        \
static void sum_visit_##SFX(void* c, long t, REAL p) { (void)t; ((sum_ctx_##SFX*)c)->acc += p; }   \
typedef struct { const REAL* in; REAL acc; } gather_ctx_##SFX;                                     \
static void gather_visit_##SFX(void* c, long t, REAL p) {                                          \
    gather_ctx_##SFX* q = (gather_ctx_##SFX*)c;                                                    \
    q->acc += p * q->in[t];                                                                        \
}                                                                                                  \
typedef struct { REAL* out; REAL scale; } scatter_ctx_##SFX;                                       \
static void scatter_visit_##SFX(void* c, long t, REAL p) {                                         \
    scatter_ctx_##SFX* q = (scatter_ctx_##SFX*)c;                                                  \
    const REAL v = q->scale * p;                                                                   \
    _Pragma("omp atomic") q->out[t] += v;                                                          \
}                                                                                                  \
typedef struct { long n; } count_ctx_##SFX;                                                        \
static void count_visit_##SFX(void* c, long t, REAL p) { (void)t; (void)p; ((count_ctx_##SFX*)c)->n++; } \
                                                                                                   \
/* Near-block weights of one source on the far-ray scale (prc.cu:193-218): w[q] for q in 125,   \
 * zero outside the image. */                                                                     \
static void near_weights_##SFX(const oracle_params* g, const surv_ctx* sc, const float* rho,      \
                               int s, REAL* w) {                                                   \
    const int vx = s % g->nx, vy = (s / g->nx) % g->ny, vz = s / (g->nx * g->ny);                  \
    REAL sum[NEAR_N];                                                                              \
    for (int q = 0; q < NEAR_N; ++q) sum[q] = 0;                                                   \
    near_ctx_##SFX nc = {sum, vx, vy, vz, g->nx, g->ny};                                           \
    for (int r = 0; r < NEAR_RAYS; ++r) {                                                          \
        REAL x[3], d[3];                                                                           \
        RAY(r, NEAR_RAYS, x, d);                                                                   \
        trace_##SFX(g, sc, rho, vx, vy, vz, x, d, 1, near_visit_##SFX, &nc);                       \
    }                                                                                              \
    for (int q = 0; q < NEAR_N; ++q) {                                                             \
        const int i = vx + q % NEAR_SIDE - NEAR_R, j = vy + q / NEAR_SIDE % NEAR_SIDE - NEAR_R,    \
                  k = vz + q / (NEAR_SIDE * NEAR_SIDE) - NEAR_R;                                   \
        w[q] = inside_g(g, i, j, k) ? sum[q] * ((REAL)g->n_rays / NEAR_RAYS) : 0;                  \
    }                                                                                              \
}                                                                                                  \
                                                                                                   \
static long near_target_##SFX(const oracle_params* g, int s, int q) {                              \
    const int vx = s % g->nx, vy = (s / g->nx) % g->ny, vz = s / (g->nx * g->ny);                  \
    const int i = vx + q % NEAR_SIDE - NEAR_R, j = vy + q / NEAR_SIDE % NEAR_SIDE - NEAR_R,        \
              k = vz + q / (NEAR_SIDE * NEAR_SIDE) - NEAR_R;                                       \
    if (!inside_g(g, i, j, k)) return -1;                                                          \
    return ((long)k * g->ny + j) * g->nx + i;                                                      \
}                                                                                                  \
                                                                                                   \
static void far_rays_##SFX(const oracle_params* g, const surv_ctx* sc, const float* rho, int s,   \
                           visit_fn_##SFX vf, void* ctx) {                                         \
    const int vx = s % g->nx, vy = (s / g->nx) % g->ny, vz = s / (g->nx * g->ny);                  \
    for (int r = 0; r < g->n_rays; ++r) {                                                          \
        REAL x[3], d[3];                                                                           \
        RAY(r, g->n_rays, x, d);                                                                   \
        trace_##SFX(g, sc, rho, vx, vy, vz, x, d, 0, vf, ctx);                                     \
    }                                                                                              \
}                                                                                                  \
                                                                                                   \
/* NormOp pass (prc.cu:232-237, 420): W and the near cache (n_active x 125). */                   \
void oracle_normalize_##SFX(const oracle_params* g, const float* rho, const int* active,          \
                            int n_active, REAL* W, REAL* near) {                                   \
    surv_ctx sc;                                                                                   \
    surv_init(&sc, g, sizeof(REAL) == 4);                                                          \
    if (g->threads > 0) omp_set_num_threads(g->threads);                                           \
    _Pragma("omp parallel for schedule(dynamic, 16)")                                              \
    for (int src = 0; src < n_active; ++src) {                                                     \
        const int s = active[src];                                                                 \
        REAL* w = near + (size_t)src * NEAR_N;                                                     \
        near_weights_##SFX(g, &sc, rho, s, w);                                                     \
        sum_ctx_##SFX c = {0};                                                                     \
        for (int q = 0; q < NEAR_N; ++q) if (w[q] > 0) c.acc += w[q];                              \
        far_rays_##SFX(g, &sc, rho, s, sum_visit_##SFX, &c);                                       \
        W[src] = c.acc;                                                                            \
    }                                                                                              \
    surv_free(&sc);                                                                                \
}                                                                                                  \
                                                                                                   \
/* ForwardOp (prc.cu:239-254, 430-434): out = A f, overwritten. */                                 \
void oracle_forward_##SFX(const oracle_params* g, const float* rho, const int* active,            \
                          int n_active, const REAL* W, const REAL* near, const REAL* f, REAL* out) { \
    surv_ctx sc;                                                                                   \
    surv_init(&sc, g, sizeof(REAL) == 4);                                                          \
    const long n = (long)g->nx * g->ny * g->nz;                                                    \
    for (long i = 0; i < n; ++i) out[i] = 0;                                                       \
    if (g->threads > 0) omp_set_num_threads(g->threads);                                           \
    _Pragma("omp parallel for schedule(dynamic, 16)")                                              \
    for (int src = 0; src < n_active; ++src) {                                                     \
        const int s = active[src];                                                                 \
        const REAL fs = f[s], ws = W[src];                                                         \
        const REAL scale = ws > 0 ? fs / ws : 0;                                                   \
        if (!(scale > 0)) continue;                                                                \
        scatter_ctx_##SFX c = {out, scale};                                                        \
        for (int q = 0; q < NEAR_N; ++q) {                                                         \
            const long t = near_target_##SFX(g, s, q);                                             \
            const REAL w = near[(size_t)src * NEAR_N + q];                                         \
            if (t >= 0 && w > 0) scatter_visit_##SFX(&c, t, w);                                    \
        }                                                                                          \
        far_rays_##SFX(g, &sc, rho, s, scatter_visit_##SFX, &c);                                   \
    }                                                                                              \
    surv_free(&sc);                                                                                \
}                                                                                                  \
                                                                                                   \
/* AdjointOp (prc.cu:256-267, 436): out[s] = A^T in on tissue voxels only. */                      \
void oracle_adjoint_##SFX(const oracle_params* g, const float* rho, const int* active,            \
                          int n_active, const REAL* W, const REAL* near, const REAL* in, REAL* out) { \
    surv_ctx sc;                                                                                   \
    surv_init(&sc, g, sizeof(REAL) == 4);                                                          \
    if (g->threads > 0) omp_set_num_threads(g->threads);                                           \
    _Pragma("omp parallel for schedule(dynamic, 16)")                                              \
    for (int src = 0; src < n_active; ++src) {                                                     \
        const int s = active[src];                                                                 \
        if (!(W[src] > 0)) { out[s] = 0; continue; }                                               \
        gather_ctx_##SFX c = {in, 0};                                                              \
        for (int q = 0; q < NEAR_N; ++q) {                                                         \
            const long t = near_target_##SFX(g, s, q);                                             \
            const REAL w = near[(size_t)src * NEAR_N + q];                                         \
            if (t >= 0 && w > 0) gather_visit_##SFX(&c, t, w);                                     \
        }                                                                                          \
        far_rays_##SFX(g, &sc, rho, s, gather_visit_##SFX, &c);                                    \
        out[s] = c.acc / W[src];                                                                   \
    }                                                                                              \
    surv_free(&sc);                                                                                \
}                                                                                                  \
                                                                                                   \
/* Number of (source, target) deposits of one projection: near entries with w > 0 plus every far \
 * ray visit.  This is V of the algorithmic-bytes accounting. */                                   \
long oracle_count_deposits_##SFX(const oracle_params* g, const float* rho, const int* active,     \
                                 int n_active, const REAL* near) {                                 \
    surv_ctx sc;                                                                                   \
    surv_init(&sc, g, sizeof(REAL) == 4);                                                          \
    long total = 0;                                                                                \
    if (g->threads > 0) omp_set_num_threads(g->threads);                                           \
    _Pragma("omp parallel for schedule(dynamic, 16) reduction(+ : total)")                         \
    for (int src = 0; src < n_active; ++src) {                                                     \
        const int s = active[src];                                                                 \
        count_ctx_##SFX c = {0};                                                                   \
        for (int q = 0; q < NEAR_N; ++q)                                                           \
            if (near_target_##SFX(g, s, q) >= 0 && near[(size_t)src * NEAR_N + q] > 0) c.n++;     \
        far_rays_##SFX(g, &sc, rho, s, count_visit_##SFX, &c);                                     \
        total += c.n;                                                                              \
    }                                                                                              \
    surv_free(&sc);                                                                                \
    return total;                                                                                  \
}                                                                                                  \
                                                                                                   \
/* update_kernel (prc.cu:279-309): RDP MAP-EM step for every voxel. */                            \
void oracle_update_##SFX(const oracle_params* g, const REAL* f, const REAL* back,                 \
                         const unsigned char* support, REAL* next, REAL beta, REAL gamma, REAL eps) { \
    const long n = (long)g->nx * g->ny * g->nz;                                                    \
    const REAL smin = (REAL)FMIN(g->sx, FMIN(g->sy, g->sz));                                       \
    if (g->threads > 0) omp_set_num_threads(g->threads);                                           \
    _Pragma("omp parallel for schedule(static)")                                                   \
    for (long idx = 0; idx < n; ++idx) {                                                           \
        if (!support[idx]) { next[idx] = 0; continue; }                                            \
        const REAL fj = f[idx], f_em = fj * back[idx];                                             \
        if (beta == 0) { next[idx] = FMAX(f_em, (REAL)0); continue; }                              \
        const int i = (int)(idx % g->nx), j = (int)((idx / g->nx) % g->ny),                        \
                  k = (int)(idx / ((long)g->nx * g->ny));                                          \
        REAL grad = 0, curv = 0;                                                                   \
        for (int dz = -1; dz <= 1; ++dz)                                                           \
            for (int dy = -1; dy <= 1; ++dy)                                                       \
                for (int dx = -1; dx <= 1; ++dx) {                                                 \
                    if (!(dx | dy | dz) || !inside_g(g, i + dx, j + dy, k + dz)) continue;         \
                    const long nb = idx + ((long)dz * g->ny + dy) * g->nx + dx;                    \
                    if (!support[nb]) continue;                                                    \
                    const REAL mx = dx * (REAL)g->sx, my = dy * (REAL)g->sy, mz = dz * (REAL)g->sz; \
                    const REAL w = smin / SQRT(mx * mx + my * my + mz * mz);                       \
                    const REAL fk = f[nb], dd = fj - fk, ad = FABS(dd);                            \
                    const REAL D = fj + fk + gamma * ad + eps, invD = 1 / D;                       \
                    grad += w * dd * (fj + 3 * fk + gamma * ad + 2 * eps) * invD * invD;           \
                    const REAL half_quad = (2 * (fj + fk + eps) + gamma * ad) * invD * invD;       \
                    const REAL hess = 2 * (2 * fk + eps) * (2 * fk + eps) * invD * invD * invD;    \
                    curv += 2 * w * FMAX(half_quad, hess);                                         \
                }                                                                                  \
        const REAL a = beta * curv, B = 1 + beta * (grad - curv * fj);                             \
        const REAL root = SQRT(B * B + 4 * a * f_em);                                              \
        next[idx] = B >= 0 ? (f_em > 0 ? 2 * f_em / (B + root) : 0) : (root - B) / (2 * a);        \
    }                                                                                              \
}                                                                                                  \
                                                                                                   \
static double vsum_##SFX(const REAL* a, long n) {                                                  \
    double s = 0;                                                                                  \
    for (long i = 0; i < n; ++i) s += (double)a[i];                                                \
    return s;                                                                                      \
}                                                                                                  \
static double vdot_##SFX(const REAL* a, const REAL* b, long n) {                                   \
    double s = 0;                                                                                  \
    for (long i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];                                 \
    return s;                                                                                      \
}                                                                                                  \
                                                                                                   \
/* main()'s correction loop (prc.cu:659-711).  img: input after clamping and support masking     \
 * (prc.cu:598-613); out: the corrected estimate.  W and near come from oracle_normalize. */       \
void oracle_correct_##SFX(const oracle_params* g, const float* rho, const int* active,            \
                          int n_active, const unsigned char* support, const REAL* W,               \
                          const REAL* near, const REAL* img, int iterations, float beta_f,         \
                          float gamma_f, int accelerate, REAL* out) {                              \
    const long n = (long)g->nx * g->ny * g->nz;                                                    \
    const REAL beta = (REAL)beta_f, gamma = (REAL)gamma_f;                                         \
    double support_sum = 0;                                                                        \
    for (long i = 0; i < n; ++i) if (support[i]) support_sum += (double)img[i];                    \
    REAL* f = (REAL*)calloc(n, sizeof(REAL));                                                      \
    REAL* prev = (REAL*)calloc(n, sizeof(REAL));                                                   \
    REAL* y = accelerate ? (REAL*)calloc(n, sizeof(REAL)) : NULL;                                  \
    REAL* h_prev = accelerate ? (REAL*)calloc(n, sizeof(REAL)) : NULL;                             \
    REAL* est = (REAL*)calloc(n, sizeof(REAL));                                                    \
    memcpy(f, img, n * sizeof(REAL));                                                              \
    const REAL eps = (REAL)(1.0e-6 * support_sum / n_active);                                      \
    if (iterations > 0) {                                                                          \
        for (long i = 0; i < n; ++i) if (support[i]) f[i] = FMAX(f[i], 1000 * eps);                \
        const REAL scale = (REAL)(support_sum / vsum_##SFX(f, n));                                 \
        for (long i = 0; i < n; ++i) f[i] = f[i] * scale;                                          \
    }                                                                                              \
    REAL lambda = 0;                                                                               \
    for (int it = 1; it <= iterations; ++it) {                                                     \
        const REAL* start = f;                                                                     \
        if (accelerate) {                                                                          \
            for (long i = 0; i < n; ++i) y[i] = FMAX(f[i] + lambda * (f[i] - prev[i]), (REAL)0.5 * f[i]); \
            start = y;                                                                             \
        }                                                                                          \
        oracle_forward_##SFX(g, rho, active, n_active, W, near, start, est);                       \
        for (long i = 0; i < n; ++i) est[i] = support[i] ? img[i] / FMAX(est[i], eps) : 0;         \
        oracle_adjoint_##SFX(g, rho, active, n_active, W, near, est, prev);                        \
        oracle_update_##SFX(g, start, prev, support, est, beta, gamma, eps);                       \
        REAL scale = 1;                                                                            \
        if (beta > 0) {                                                                            \
            const double s = vsum_##SFX(est, n);                                                   \
            if (s > 0) scale = (REAL)(support_sum / s);                                            \
        }                                                                                          \
        if (beta > 0 || accelerate)                                                                \
            for (long i = 0; i < n; ++i) {                                                         \
                const REAL v = est[i] * scale;                                                     \
                est[i] = v;                                                                        \
                if (accelerate) y[i] = v - y[i];                                                   \
            }                                                                                      \
        if (accelerate) {                                                                          \
            const double hh = vdot_##SFX(h_prev, h_prev, n);                                       \
            double l = hh > 0 ? vdot_##SFX(y, h_prev, n) / hh : 0;                                 \
            l = l < 0 ? 0 : (l > 1 ? 1 : l);                                                       \
            lambda = (REAL)l;                                                                      \
            REAL* t = y; y = h_prev; h_prev = t;                                                   \
            t = prev; prev = f; f = t;                                                             \
        }                                                                                          \
        REAL* t = f; f = est; est = t;                                                             \
    }                                                                                              \
    memcpy(out, f, n * sizeof(REAL));                                                              \
    free(f); free(prev); free(y); free(h_prev); free(est);                                         \
}

static inline float fminf_(float a, float b) { return fminf(a, b); }
static inline float fmaxf_(float a, float b) { return fmaxf(a, b); }

ORACLE_BODY(double, f64, ray_d, surv_at_d, fmin, fmax, fabs, sqrt)
ORACLE_BODY(float, f32, ray_f, surv_at_f, fminf_, fmaxf_, fabsf, sqrtf)

/* Survival evaluated as the projector sees it: analytic FP64, FP64 table, or the float table. */
void oracle_survival(const oracle_params* g, int f32, const double* r, double* s, long n) {
    surv_ctx sc;
    surv_init(&sc, g, f32);
    for (long i = 0; i < n; ++i) s[i] = f32 ? (double)surv_at_f(&sc, (float)r[i]) : surv_at_d(&sc, r[i]);
    surv_free(&sc);
}

/* The float table itself (RANGE_BINS + 1 entries), as prc.cu:625-633 builds it. */
void oracle_survival_table_f32(const oracle_params* g, float* table) {
    const float scale = RANGE_BINS / g->cutoff;
    for (int j = 0; j <= RANGE_BINS; ++j) table[j] = survival_f(g->br, g->n_branch, j / scale);
}

void oracle_ray(int f32, int k, int n, double* x, double* d) {
    if (f32) {
        float xf[3], df[3];
        ray_f(k, n, xf, df);
        for (int a = 0; a < 3; ++a) x[a] = xf[a], d[a] = df[a];
    } else {
        ray_d(k, n, x, d);
    }
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
