// Command-line handling shared by the s1_compress / s1_decompress front ends. The flags, their
// parsing (std::stof / stoull / stoul / stoi) and the error convention ("error: <msg>" on stderr,
// exit status 1) follow c_codes/s1_compress.cpp:153-346 and c_codes/s1_decompress.cpp:5-154.
#pragma once
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "asz_b200.h"

namespace cli {

struct Args {
    std::string input, compressed, decompressed, plan;
    std::vector<uint64_t> dims;
    float rel_eb = 0;
    bool have_plan = false, t_min_set = false, t_max_set = false;
    asz_params p{};
};

inline const char *next(int argc, char **argv, int &i) {
    if (i + 1 >= argc) throw std::invalid_argument(std::string("missing value after ") + argv[i]);
    return argv[++i];
}

// Shared flags; returns false if `arg` is not one of them. `compress_side` enables the flags
// only s1_compress accepts.
inline bool parse_flag(const std::string &arg, int argc, char **argv, int &i, Args &a, bool compress_side) {
    asz_params &p = a.p;
    if (arg == "-f") return true;
    if (arg == "-i") {
        a.input = next(argc, argv, i);
        a.compressed = a.input + ".asz";
        a.decompressed = compress_side ? a.compressed + ".bin" : a.input + ".bin";
        return true;
    }
    if (arg == "-z") {
        a.compressed = next(argc, argv, i);
        a.decompressed = a.compressed + ".bin";
        return true;
    }
    if (arg == "-o") {
        a.decompressed = next(argc, argv, i);
        return true;
    }
    if (arg == "-3") {
        uint64_t d0 = std::stoul(next(argc, argv, i)), d1 = std::stoul(next(argc, argv, i)), d2 = std::stoul(next(argc, argv, i));
        a.dims = {d0, d1, d2};
        return true;
    }
    if (arg == "-M") {
        next(argc, argv, i);
        a.rel_eb = std::stof(next(argc, argv, i));
        return true;
    }
    if (arg == "--predictor-family") {
        std::string f = next(argc, argv, i);
        if (f == "cubic") p.predictor_family = ASZ_FAMILY_CUBIC;
        else if (f == "quintic") p.predictor_family = ASZ_FAMILY_QUINTIC;
        else throw std::invalid_argument("predictor_family must be cubic or quintic");
        return true;
    }
    if (arg == "--pivot-eb-ratio") return p.pivot_eb_ratio = std::stof(next(argc, argv, i)), true;
    if (arg == "--eb-ratio") return p.eb_ratio = std::stof(next(argc, argv, i)), true;
    if (arg == "--slope-ratio") return p.slope_ratio = std::stof(next(argc, argv, i)), true;
    if (arg == "--block-pivot-ratio") return p.block_pivot_ratio = std::stoull(next(argc, argv, i)), true;
    if (arg == "--max-layer-num") return p.max_layer_num = std::stoull(next(argc, argv, i)), true;
    if (arg == "--full-predictor-search-layer-num") return p.full_predictor_search_layer_num = std::stoull(next(argc, argv, i)), true;
    if (arg == "--t-precision") return p.t_precision = std::stoi(next(argc, argv, i)), true;
    if (!compress_side) return false;
    if (arg == "--predictor-plan") {
        a.plan = next(argc, argv, i);
        a.have_plan = true;
        return true;
    }
    if (arg == "--generate-config-sample-stride") return p.generate_config_sample_stride = std::stoull(next(argc, argv, i)), true;
    if (arg == "--h1-block-sampling-num") return p.h1_block_sampling_num = std::stoull(next(argc, argv, i)), true;
    if (arg == "--stat-eb-ratio") return p.stat_eb_ratio = std::stof(next(argc, argv, i)), true;
    if (arg == "--predictor-family-suffix-layers") return p.predictor_family_suffix_layers = std::stoull(next(argc, argv, i)), true;
    if (arg == "--predictor-family-sample-blocks") return p.predictor_family_sample_blocks = std::stoull(next(argc, argv, i)), true;
    if (arg == "--predictor-family-sample-point-limit")
        return p.predictor_family_sample_point_limit = std::stoull(next(argc, argv, i)), true;
    if (arg == "--predictor-family-sample-fraction-limit")
        return p.predictor_family_sample_fraction_limit = std::stof(next(argc, argv, i)), true;
    if (arg == "--predictor-family-coarse-probe-block-pivot-ratio")
        return p.predictor_family_coarse_probe_block_pivot_ratio = std::stoull(next(argc, argv, i)), true;
    if (arg == "--predictor-family-fine-probe-block-pivot-ratio")
        return p.predictor_family_fine_probe_block_pivot_ratio = std::stoull(next(argc, argv, i)), true;
    if (arg == "--predictor-family-fine-eb-threshold")
        return p.predictor_family_fine_eb_threshold = std::stof(next(argc, argv, i)), true;
    if (arg == "--default-slope-invalid-ratio-threshold")
        return p.default_slope_invalid_ratio_threshold = std::stof(next(argc, argv, i)), true;
    if (arg == "--default-slope-fallback") return p.default_slope_fallback = std::stof(next(argc, argv, i)), true;
    if (arg == "--default-slope-eb-span") return p.default_slope_eb_span = std::stof(next(argc, argv, i)), true;
    if (arg == "--t-min") return p.t_min = std::stof(next(argc, argv, i)), a.t_min_set = true, true;
    if (arg == "--t-max") return p.t_max = std::stof(next(argc, argv, i)), a.t_max_set = true, true;
    if (arg == "--report-t-histogram") return p.report_t_histogram = 1, true;
    return false;
}

inline std::vector<char> read_file(const std::string &path, const char *what) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error(std::string("cannot open ") + what + ": " + path);
    f.seekg(0, std::ios::end);
    std::streamoff n = f.tellg();
    f.seekg(0, std::ios::beg);
    std::vector<char> buf((size_t)std::max<std::streamoff>(n, 0));
    f.read(buf.data(), (std::streamsize)buf.size());
    if (!f) throw std::runtime_error(std::string("cannot read complete ") + what + ": " + path);
    return buf;
}

inline void write_file(const std::string &path, const void *data, size_t n, const char *what) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error(std::string("cannot open ") + what + ": " + path);
    f.write((const char *)data, (std::streamsize)n);
    if (!f) throw std::runtime_error(std::string("cannot write ") + what + ": " + path);
}

// The figures compress() prints after compressing (compress.tpp:306-319), in the float steps the
// reference's build executes. The error loop there is scalar: the squared errors go into one float
// through a fused multiply-add per value, in index order, and |d| into a running maximum. Then
// psnr = 10*log10f(((max-min)^2 / sum) * n), the division by n folded into the product, and
// dist = fma(-br, default_slope, psnr). The sum's order decides its last bits, so it is replayed on
// the host here (the library's asz_compress_stats sums in double on the device).
struct PrintedStats {
    float max_err, mse_sum;
};
__attribute__((target("fma"))) inline PrintedStats printed_stats(const float *x, const float *y, uint64_t n) {
    float sum = 0.0f, mx = 0.0f;
    for (uint64_t i = 0; i < n; i++) {
        const float d = x[i] - y[i];
        sum = __builtin_fmaf(d, d, sum);
        const float a = __builtin_fabsf(d);
        mx = mx > a ? mx : a;
    }
    return {mx, sum};
}

struct Ctx {
    asz_ctx *c = nullptr;
    Ctx() {
        c = asz_create(0);
        if (!c) throw std::runtime_error("cannot create a CUDA context on device 0");
    }
    ~Ctx() { asz_destroy(c); }
    void check(int rc) {
        if (rc != ASZ_OK) throw std::runtime_error(asz_last_error(c));
    }
};

}  // namespace cli
