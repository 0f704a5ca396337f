// prc_cli.cpp -- the `prc ISOTOPE NX NY NZ DX DY DZ [options]` command line, byte-compatible
// with jlherraiz/PRC_MLEM's executable (prc.cu:452-722): same options and defaults, same raw
// float32 I/O, same messages and exit codes.  All validation happens before the first CUDA call
// (the reference's CLI tests run with every GPU hidden); the device work goes through the
// C ABI of include/prc_b200.h.
#include "../../include/prc_b200.h"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace {

constexpr float kMinDensity = 1.0e-3f;
constexpr int kNearRays = 2048;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Everything the command line can set.  Defaults are the reference's (prc.cu:452-459); the
// last two fields are this engine's additions (--cache, --bf16-weights).
struct Settings {
    std::string isotope, mode = "correct", input = "ACTIVITY.raw", density = "DENSITY.raw", output;
    int dims[3] = {0, 0, 0};       // NX NY NZ
    float voxel[3] = {0, 0, 0};    // DX DY DZ [mm]
    int rays = 128, iterations = 20, save_every = 0;
    float beta = 0.2f, gamma = 20.0f, support_rho = 0.05f, air_cap_mm = 50.0f;
    bool reproject = false, trace_near_every_pass = false, exact_range = false, plain = false, bf16 = false;
    bool bf16_volumes = false, fp24 = false;
    int cache = PRC_CACHE_FULL;
    int tile = PRC_TILE_AUTO;
};

void print_usage(const char* prog, FILE* stream = stderr) {  // the usage text of prc.cu:461-484
    fprintf(stream,
            "Usage: %s ISOTOPE NX NY NZ DX DY DZ [options]\n"
            "  --mode correct|forward|adjoint   (default correct)\n"
            "  --input FILE      blurred (correct) or source (forward/adjoint) image, default ACTIVITY.raw\n"
            "  --density FILE    density map in g/cm3, default DENSITY.raw\n"
            "  --output FILE     default ACTIVITY_PRC_V2.raw (correct), ACTIVITY_FWD.raw, ACTIVITY_ADJ.raw\n"
            "  --rays N          even far-field rays per voxel (default 128)\n"
            "  --iterations N    accelerated MAP-EM iterations (default 20)\n"
            "  --beta B          relative-difference prior strength (default 0.2; 0 = no prior)\n"
            "                    Add --no-accel for plain Richardson-Lucy.\n"
            "  --gamma G         RDP edge preservation, larger keeps sharper edges (default 20)\n"
            "  --support-rho R   minimum density of voxels that can hold activity (default 0.05)\n"
            "  --air-cap-mm L    a positron that crossed L mm of air has escaped (default 50)\n"
            "  --save-every K    also write the estimate every K iterations\n"
            "  --reproject       also write A f of the result (_REPROJ.raw)\n"
            "  --exact-range     evaluate the survival function analytically, not from the table (validation)\n"
            "  --no-cache-near   trace the near block again in every pass (less GPU memory, slower)\n"
            "  --no-accel        plain MAP-EM without Biggs-Andrews extrapolation (validation)\n"
            "  --cache MODE      none|near|source|full: weights kept on the GPU between passes (default full)\n"
            "  --bf16-weights    store the projector weights in bfloat16 (mixed precision)\n"
            "  --bf16-volumes    bfloat16 weights, and bfloat16 volumes gathered inside MAP-EM\n"
            "  --fp24-weights    store the stored-field weights in 24 bits (fp32 rounded to 16 mantissa bits)\n"
            "  --tile SHAPE      auto|tune|8x2x2|16x2x1|32x1x1|4x4x2|16x1x2: source tile of the stored field\n"
            "                    (default auto; tune: time the candidates on a slab first)\n"
            "Isotopes:",
            prog);
    for (int i = 0; i < prc_isotope_count(); ++i) fprintf(stream, " %s", prc_isotope_name(i));
    fprintf(stream, "\n");
}

[[noreturn]] void die() { exit(EXIT_FAILURE); }

constexpr int kTune = 100;  // --tile tune: run the tile autotuner before building

// A whole-string decimal number.  The messages are the reference's, which its tests match.
template <class T>
T number(const char* text, const char* label) {
    char* end = nullptr;
    errno = 0;
    bool ok;
    T value;
    if constexpr (std::is_same_v<T, int>) {
        const long long v = strtoll(text, &end, 10);
        ok = v >= INT_MIN && v <= INT_MAX;
        value = (int)v;
    } else {
        value = strtof(text, &end);
        ok = std::isfinite(value);
    }
    if (errno != 0 || end == text || *end != '\0' || !ok) {
        fprintf(stderr, std::is_same_v<T, int> ? "Invalid integer for %s: %s\n" : "Invalid finite number for %s: %s\n",
                label, text);
        die();
    }
    return value;
}

// The option table: a name, whether it takes a value, and what it does with it.
using Apply = void (*)(Settings&, const char* value, const char* name);
struct Spec {
    const char* name;
    bool takes_value;
    Apply apply;
};
const Spec kSpecs[] = {
    {"--mode", true, [](Settings& s, const char* v, const char*) { s.mode = v; }},
    {"--input", true, [](Settings& s, const char* v, const char*) { s.input = v; }},
    {"--density", true, [](Settings& s, const char* v, const char*) { s.density = v; }},
    {"--output", true, [](Settings& s, const char* v, const char*) { s.output = v; }},
    {"--rays", true, [](Settings& s, const char* v, const char* n) { s.rays = number<int>(v, n); }},
    {"--iterations", true, [](Settings& s, const char* v, const char* n) { s.iterations = number<int>(v, n); }},
    {"--beta", true, [](Settings& s, const char* v, const char* n) { s.beta = number<float>(v, n); }},
    {"--gamma", true, [](Settings& s, const char* v, const char* n) { s.gamma = number<float>(v, n); }},
    {"--support-rho", true, [](Settings& s, const char* v, const char* n) { s.support_rho = number<float>(v, n); }},
    {"--air-cap-mm", true, [](Settings& s, const char* v, const char* n) { s.air_cap_mm = number<float>(v, n); }},
    {"--save-every", true, [](Settings& s, const char* v, const char* n) { s.save_every = number<int>(v, n); }},
    {"--reproject", false, [](Settings& s, const char*, const char*) { s.reproject = true; }},
    {"--no-cache-near", false, [](Settings& s, const char*, const char*) { s.trace_near_every_pass = true; }},
    {"--exact-range", false, [](Settings& s, const char*, const char*) { s.exact_range = true; }},
    {"--no-accel", false, [](Settings& s, const char*, const char*) { s.plain = true; }},
    {"--bf16-weights", false, [](Settings& s, const char*, const char*) { s.bf16 = true; }},
    {"--bf16-volumes", false, [](Settings& s, const char*, const char*) { s.bf16 = s.bf16_volumes = true; }},
    {"--fp24-weights", false, [](Settings& s, const char*, const char*) { s.fp24 = true; }},
    {"--cache", true,
     [](Settings& s, const char* v, const char*) {
         static const std::pair<const char*, int> modes[] = {{"none", PRC_CACHE_NONE},
                                                             {"near", PRC_CACHE_NEAR},
                                                             {"full", PRC_CACHE_FULL},
                                                             {"source", PRC_CACHE_SOURCE_MAJOR}};
         s.cache = -1;  // an unknown mode fails the parameter check below
         for (const auto& m : modes)
             if (!strcmp(v, m.first)) s.cache = m.second;
     }},
    {"--tile", true,
     [](Settings& s, const char* v, const char*) {
         static const std::pair<const char*, int> shapes[] = {{"auto", PRC_TILE_AUTO},     {"tune", kTune},
                                                              {"8x2x2", PRC_TILE_8x2x2},
                                                              {"16x2x1", PRC_TILE_16x2x1}, {"32x1x1", PRC_TILE_32x1x1},
                                                              {"4x4x2", PRC_TILE_4x4x2},   {"16x1x2", PRC_TILE_16x1x2}};
         s.tile = -1;  // an unknown shape fails the parameter check below
         for (const auto& t : shapes)
             if (!strcmp(v, t.first)) s.tile = t.second;
     }},
};

// Default output file of each mode (prc.cu:553-554).
const char* default_output(const std::string& mode) {
    return mode == "forward" ? "ACTIVITY_FWD.raw" : mode == "adjoint" ? "ACTIVITY_ADJ.raw" : "ACTIVITY_PRC_V2.raw";
}

Settings parse(int argc, char** argv) {
    Settings s;
    if (argc < 8) {  // the seven positional arguments are required
        print_usage(argv[0]);
        die();
    }
    s.isotope = argv[1];
    static const char* const dim_names[3] = {"NX", "NY", "NZ"}, *const voxel_names[3] = {"DX", "DY", "DZ"};
    for (int a = 0; a < 3; ++a) s.dims[a] = number<int>(argv[2 + a], dim_names[a]);
    for (int a = 0; a < 3; ++a) s.voxel[a] = number<float>(argv[5 + a], voxel_names[a]);
    for (int i = 8; i < argc; ++i) {
        const char* key = argv[i];
        const Spec* spec = nullptr;
        for (const Spec& candidate : kSpecs)
            if (!strcmp(key, candidate.name)) spec = &candidate;
        if (!spec) {
            fprintf(stderr, "Unknown option %s\n", key);
            print_usage(argv[0]);
            die();
        }
        const char* value = nullptr;
        if (spec->takes_value) {
            if (i + 1 == argc) {
                fprintf(stderr, "Missing value for %s\n", key);
                die();
            }
            value = argv[++i];
        }
        spec->apply(s, value, key);
    }
    // Every parameter in its range (the reference's conditions, prc.cu:540-546), then the
    // 32-bit voxel index limit on the exact 64-bit product (prc.cu:547-551).
    const bool in_range[] = {
        s.dims[0] > 0 && s.dims[1] > 0 && s.dims[2] > 0,
        s.voxel[0] > 0 && s.voxel[1] > 0 && s.voxel[2] > 0,
        s.rays >= 2 && s.rays % 2 == 0 && s.rays <= INT_MAX - 31,
        s.iterations >= 0 && s.iterations < INT_MAX,
        s.beta >= 0 && s.gamma >= 0 && s.support_rho >= 0 && s.air_cap_mm > 0,
        s.save_every >= 0 && s.cache >= 0 && s.tile >= 0,
        s.mode == "correct" || s.mode == "forward" || s.mode == "adjoint",
    };
    if (!std::all_of(std::begin(in_range), std::end(in_range), [](bool b) { return b; })) {
        fprintf(stderr, "Invalid geometry or solver parameters\n");
        die();
    }
    if ((long long)s.dims[0] * s.dims[1] * s.dims[2] > INT_MAX) {
        fprintf(stderr, "Volume exceeds the INT_MAX voxel index limit\n");
        die();
    }
    if (s.output.empty()) s.output = default_output(s.mode);
    return s;
}

// Checkpoint and reprojection names: the tag goes before the extension of the file name
// ("out.raw" -> "out_it003.raw"), or at the end when the file name has none or starts with its
// only dot; a dot in a directory name is never an extension (prc.cu:557-562).
std::string with_suffix(const std::string& path, const std::string& tag) {
    const size_t sep = path.find_last_of("/\\");
    const size_t name = sep == std::string::npos ? 0 : sep + 1;
    const size_t ext = path.find_last_of('.');
    if (ext == std::string::npos || ext <= name) return path + tag;
    std::string out = path;
    return out.insert(ext, tag);
}

// Reads exactly v->size() floats; false when the file is missing, short or too long.
bool read_raw_ok(const std::string& path, std::vector<float>* v) {  // prc.cu:339-347
    FILE* fp = fopen(path.c_str(), "rb");
    const bool ok = fp && fread(v->data(), sizeof(float), v->size(), fp) == v->size() && fgetc(fp) == EOF && !ferror(fp);
    if (fp) fclose(fp);
    return ok;
}

void read_failed(const std::string& path, size_t n) {
    fprintf(stderr, "Expected exactly %zu float32 values in %s\n", n, path.c_str());
    die();
}

// Writes an all-finite image; otherwise returns the reference's message and writes nothing.
std::string save_image_ok(const std::string& path, const float* host, size_t n) {  // prc.cu:349-360
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(host[i])) return "Non-finite output: " + path;
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp || fwrite(host, sizeof(float), n, fp) != n) {
        if (fp) fclose(fp);
        return "Cannot write " + path;
    }
    if (fclose(fp) != 0) return "Cannot write " + path;
    return "";
}

void save_image(const std::string& path, const float* host, size_t n) {
    const std::string err = save_image_ok(path, host, n);
    if (!err.empty()) {
        fprintf(stderr, "%s\n", err.c_str());
        die();
    }
}

// Checkpoints (--save-every) are written by a helper thread while the GPU runs the next
// iterations; a write error is reported, with the reference's message, before anything else is
// written.
// A host image buffer in pinned (page-locked) memory when the runtime can give it, so the
// device-to-host copies run at full speed; pageable memory otherwise.
struct HostImage {
    float* data = nullptr;
    size_t n = 0;
    bool pinned = false;
    std::vector<float> fallback;
    void resize(size_t count) {
        if (n == count) return;
        release();
        n = count;
        void* p = nullptr;
        if (prc_host_alloc(count * sizeof(float), &p) == PRC_OK) {
            data = static_cast<float*>(p), pinned = true;
        } else {
            fallback.resize(count), data = fallback.data(), pinned = false;
        }
    }
    void release() {
        if (pinned) prc_host_free(data);
        fallback.clear();
        data = nullptr, n = 0, pinned = false;
    }
    ~HostImage() { release(); }
};

struct CheckpointWriter {
    std::thread thread;
    HostImage image;
    std::string error;
    void finish() {
        if (thread.joinable()) thread.join();
        if (!error.empty()) {
            fprintf(stderr, "%s\n", error.c_str());
            die();
        }
    }
    void start(const std::string& path) {
        thread = std::thread([this, path] { error = save_image_ok(path, image.data, image.n); });
    }
};

void check(int rc) {
    if (rc != PRC_OK) {
        fprintf(stderr, "%s\n", prc_last_error());
        die();
    }
}

double host_sum(const float* v, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += v[i];
    return s;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc == 2 && (!strcmp(argv[1], "--help") || !strcmp(argv[1], "-h"))) {
        print_usage(argv[0], stdout);
        return EXIT_SUCCESS;
    }
    const Settings o = parse(argc, argv);
    float cutoff = 0.0f;
    if (prc_isotope_cutoff(o.isotope.c_str(), &cutoff) != PRC_OK) {
        print_usage(argv[0]);
        return EXIT_FAILURE;
    }
    const int nx = o.dims[0], ny = o.dims[1], nz = o.dims[2];
    const size_t n = (size_t)nx * ny * nz;

    // Host I/O (prc.cu:591-622, restructured): both files are read at once; as soon as the
    // density is complete and finite, a builder thread makes the first CUDA contact and builds
    // the projector (prc_create: clamp, support, source order, uploads, layout, normalisation)
    // while this thread finishes the input file and validates the activity.  The messages and
    // their precedence are the reference's: size errors density first, then the first voxel
    // where density or activity is non-finite, then "No activity".  Any of them stops the run
    // with nothing written, the builder's result discarded (a hidden GPU makes it fail quietly).
    const double t0 = now_s();
    std::vector<float> rho(n), img(n);
    bool img_ok = false;
    std::thread reader([&] { img_ok = read_raw_ok(o.input, &img); });
    const bool rho_ok = read_raw_ok(o.density, &rho);
    bool rho_finite = rho_ok;
    for (size_t i = 0; rho_finite && i < n; ++i) rho_finite = std::isfinite(rho[i]);

    prc_geometry geo{nx, ny, nz, o.voxel[0], o.voxel[1], o.voxel[2]};
    prc_options opts;
    prc_default_options(&opts);
    opts.rays = o.rays;
    opts.support_rho = o.support_rho;
    opts.air_cap_mm = o.air_cap_mm;
    opts.exact_range = o.exact_range;
    opts.cache = o.trace_near_every_pass ? PRC_CACHE_NONE : o.cache;
    opts.precision = o.bf16_volumes ? PRC_PRECISION_BF16_VOLUMES
                     : o.bf16       ? PRC_PRECISION_BF16
                     : o.fp24       ? PRC_PRECISION_FP24
                                    : PRC_PRECISION_FP32;
    opts.tile = o.tile;
    struct Build {
        prc_handle* h = nullptr;
        int rc = PRC_OK;
        std::string error;
        double seconds = 0.0;
    } build;
    std::thread builder;
    if (rho_finite) {
        builder = std::thread([&] {
            const double tb = now_s();
            if (opts.tile == kTune) {
                int tuned = PRC_TILE_AUTO;
                opts.tile = prc_tune_tile(&geo, o.isotope.c_str(), &opts, rho.data(), &tuned) == PRC_OK ? tuned
                                                                                                       : PRC_TILE_AUTO;
            }
            build.rc = prc_create(&geo, o.isotope.c_str(), &opts, rho.data(), &build.h);
            if (build.rc != PRC_OK) build.error = prc_last_error();
            build.seconds = now_s() - tb;
        });
    }
    auto stop = [&]() -> int {  // a validation failure: discard the build
        if (builder.joinable()) builder.join();
        if (build.h) prc_destroy(build.h);
        return EXIT_FAILURE;
    };
    reader.join();
    if (!rho_ok) read_failed(o.density, n);  // the reference's order: density first
    if (!img_ok) {
        stop();
        read_failed(o.input, n);
    }
    size_t n_active = 0;
    double input_sum = 0.0, support_sum = 0.0;
    for (size_t i = 0; i < n; ++i) {  // prc.cu:598-613
        if (!std::isfinite(rho[i]) || !std::isfinite(img[i])) {
            fprintf(stderr, "Non-finite density or activity at voxel %zu\n", i);
            return stop();
        }
        const float r = std::max(rho[i], kMinDensity);
        img[i] = std::max(img[i], 0.0f);
        input_sum += img[i];
        if (r >= o.support_rho) {
            ++n_active;
            support_sum += img[i];
        } else {
            img[i] = 0.0f;
        }
    }
    printf("isotope %s, grid %dx%dx%d, voxel %.3fx%.3fx%.3f mm, cutoff %.3f mm (water), air cap %.1f mm\n",
           o.isotope.c_str(), nx, ny, nz, o.voxel[0], o.voxel[1], o.voxel[2], cutoff, o.air_cap_mm);
    printf("tissue voxels %zu (%.1f%%), input counts in tissue %.6g of %.6g (%.2f%%)\n", n_active,
           100.0 * n_active / n, support_sum, input_sum, input_sum > 0 ? 100.0 * support_sum / input_sum : 0.0);
    if (support_sum == 0.0) {
        fprintf(stderr, "No activity in voxels with density >= %g: nothing to do\n", o.support_rho);
        return stop();
    }

    // The projector (its build overlapped the input's read and validation).
    double t = now_s();
    builder.join();
    if (build.rc != PRC_OK) {
        fprintf(stderr, "%s\n", build.error.c_str());
        return EXIT_FAILURE;
    }
    prc_handle* h = build.h;
    int64_t bytes = 0, far_entries = 0, far_t_entries = 0;
    int mode = 0;
    prc_device_bytes(h, &bytes);
    prc_cache_mode(h, &mode, &far_entries, &far_t_entries);
    printf("normalisation (%d near-block + %d far-field rays): %.2f s, cache %s, device memory %.0f MiB\n", kNearRays,
           o.rays, build.seconds,
           mode == PRC_CACHE_FULL ? "field (source+target major)" : mode == PRC_CACHE_SOURCE_MAJOR ? "field (source major)"
           : mode == PRC_CACHE_NEAR ? "near" : "none",
           bytes / 1048576.0);

    HostImage out;
    out.resize(n);
    if (o.mode == "forward" || o.mode == "adjoint") {  // prc.cu:648-657
        t = now_s();
        check(o.mode == "forward" ? prc_forward_host(h, img.data(), out.data) : prc_adjoint_host(h, img.data(), out.data));
        printf("%s: %.3f s\n", o.mode.c_str(), now_s() - t);
        save_image(o.output, out.data, n);
        printf("sum in %.6g, sum out %.6g, total %.2f s\n", support_sum, host_sum(out.data, n), now_s() - t0);
        out.release();
        prc_destroy(h);
        return EXIT_SUCCESS;
    }

    // MAP-EM (prc.cu:659-720)
    printf("MAP-EM: %d iterations, beta %.4g, gamma %.3g\n", o.iterations, o.beta, o.gamma);
    t = now_s();
    if (o.iterations == 0) {
        check(prc_em_run_host(h, img.data(), out.data, 0, o.beta, o.gamma, !o.plain));
    } else {
        check(prc_em_begin_host(h, img.data()));
        t = now_s();
        CheckpointWriter writer;
        for (int it = 1; it <= o.iterations; ++it) {
            check(prc_em_iterate(h, 1, o.beta, o.gamma, !o.plain, nullptr));
            if (it == 1 || it % 10 == 0 || it == o.iterations) {
                check(prc_synchronize(h));
                printf("iteration %d/%d: %.2f s\n", it, o.iterations, now_s() - t);
            }
            if (o.save_every > 0 && it % o.save_every == 0 && it < o.iterations) {
                char tag[32];
                snprintf(tag, sizeof(tag), "_it%03d", it);
                writer.finish();  // the previous checkpoint is on disk; its buffer is free
                writer.image.resize(n);
                check(prc_em_estimate_host(h, writer.image.data));
                writer.start(with_suffix(o.output, tag));
            }
        }
        writer.finish();
        check(prc_em_estimate_host(h, out.data));
    }
    const double t_iter = now_s() - t;
    save_image(o.output, out.data, n);
    if (o.reproject) {
        HostImage reproj;
        reproj.resize(n);
        check(prc_forward_host(h, out.data, reproj.data));
        save_image(with_suffix(o.output, "_REPROJ"), reproj.data, n);
    }
    printf("sum blurred (tissue) %.6g, sum corrected %.6g\n", support_sum, host_sum(out.data, n));
    printf("iterations %.2f s (%.2f s each), total %.2f s\n", t_iter, o.iterations ? t_iter / o.iterations : 0.0,
           now_s() - t0);
    out.release();
    prc_destroy(h);
    return EXIT_SUCCESS;
}
