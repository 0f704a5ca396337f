// range_model.h -- isotope range model, survival lookup and the per-volume geometry record.
//
// The positron survival model S(r) = sum_b w_b exp(-[(a r)^(1+f) + (b r)^2.5 + (c r)^3.5]) and its
// coefficients are those of jlherraiz/PRC_MLEM prc.cu:34-57 (Paneque-Yunta et al., Phys. Med.
// Biol. 70 (2025) 165013, Tables 4-5).  The host-side evaluation below is written so that it
// rounds exactly like prc.cu's host code (plain float expressions, glibc powf/expf/sqrtf), which
// makes the 99.95 % cutoff (prc.cu:83-91) and the 4097-entry float table (prc.cu:625-633)
// bit-identical to the reference's.
#pragma once

#include <cmath>
#include <cstring>
#include <vector>

namespace prc {

constexpr int kRangeBins = 4096;        // table of S on [0, cutoff] (prc.cu:61)
constexpr float kMinDensity = 1.0e-3f;  // density floor (prc.cu:102)
constexpr int kNearR = 2, kNearSide = 5, kNear = 125;  // 5x5x5 near block (prc.cu:103)
constexpr int kNearRays = 2048;         // near-block rays (prc.cu:104)
constexpr int kLanes = 32;              // sources per coherent group (one warp)

struct Branch {
    float w, a, b, c, f;
};

struct Isotope {
    const char* name;
    int n;
    Branch br[3];
};

// prc.cu:47-57
static const Isotope kIsotopeTable[] = {
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
constexpr int kNumIsotopes = sizeof(kIsotopeTable) / sizeof(kIsotopeTable[0]);

// Geometry and tracing limits of one volume (prc.cu:94-100).
struct Grid {
    int nx, ny, nz;
    float sx, sy, sz;   // voxel size [mm]
    float cutoff;       // water-equivalent cutoff [mm]
    float support_rho;  // tissue threshold [g/cm3]
    float air_cap;      // consecutive sub-support path after which a positron escaped [mm]
};

// Survival with plain float arithmetic; __host__ __device__ so the analytic (--exact-range)
// device path and the host table use the same expression (prc.cu:65-72).
__host__ __device__ inline float survival(const Branch* br, int n, float r) {
    float s = 0.0f;
    for (int i = 0; i < n; ++i) {
        const float x = br[i].b * r, y = br[i].c * r;
        s += br[i].w * expf(-(powf(br[i].a * r, 1.0f + br[i].f) + x * x * sqrtf(x) + y * y * y * sqrtf(y)));
    }
    return s;
}

// A resolved isotope: weights fixed so the smallest branch absorbs the rounding (prc.cu:577-584)
// and the 99.95 % water-equivalent cutoff found by 64 bisection steps (prc.cu:83-91, 587).
struct RangeModel {
    int n = 0;
    Branch br[3] = {};
    float cutoff = 0.0f;

    bool resolve(const char* name) {
        for (const Isotope& iso : kIsotopeTable) {
            if (std::strcmp(iso.name, name) != 0) continue;
            n = iso.n;
            for (int b = 0; b < 3; ++b) br[b] = iso.br[b];
            float wsum = 0.0f;
            int smallest = 0;
            for (int b = 0; b < n; ++b) {
                wsum += br[b].w;
                if (br[b].w < br[smallest].w) smallest = b;
            }
            br[smallest].w += 1.0f - wsum;
            float lo = 0.0f, hi = 1.0f;
            while (1.0f - survival(br, n, hi) < 0.9995f && hi < 256.0f) hi *= 2.0f;
            for (int it = 0; it < 64; ++it) {
                const float mid = 0.5f * (lo + hi);
                if (1.0f - survival(br, n, mid) < 0.9995f) lo = mid;
                else hi = mid;
            }
            cutoff = hi;
            return true;
        }
        return false;
    }

    // Bins per mm and the 4097 samples S(j / scale), j = 0..4096 (prc.cu:626-628).
    float table_scale() const { return kRangeBins / cutoff; }
    std::vector<float> table() const {
        const float scale = table_scale();
        std::vector<float> t(kRangeBins + 1);
        for (int j = 0; j <= kRangeBins; ++j) t[j] = survival(br, n, j / scale);
        return t;
    }
};

}  // namespace prc
