// s2_many_prediction front end over the GPU sweep (asz_sweep): the reference tool's arguments,
// checks, stdout lines and per-predictor output files (c_codes/s2_many_prediction.cpp:442-566).
//
//   s2_many_prediction input dim0 dim1 dim2 output_prefix [family-or-stencil [eb0,eb1,...
//                      [legacy|augmented|transition [legacy|shared1d|common]]]]
//
// The reference writes its rows through the csv_tools library, which is not part of its tree;
// here each predictor's file <output_prefix>_<predictor>.csv is a plain CSV with a header row
// (rel_eb, the coefficient names, BR, H1, RMSE, MAE, PSNR, SAMPLES, ENCODE_SECONDS) and one row per
// (rel_eb, coefficient set), values printed with %.17g.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "asz_b200.h"

namespace {

struct Ctx {
    asz_ctx *c = nullptr;
    ~Ctx() {
        if (c) asz_destroy(c);
    }
};

void write_csv(const std::string &path, const std::string &predictor, const std::vector<asz_sweep_row> &rows) {
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) throw std::runtime_error("cannot open " + path);
    const bool six = predictor.rfind("1d6r", 0) == 0;
    std::fprintf(f, "rel_eb,%s,BR,H1,RMSE,MAE,PSNR,SAMPLES,ENCODE_SECONDS\n", six ? "a,b" : "t");
    for (const auto &r : rows) {
        std::fprintf(f, "%.17g,%.17g,", r.rel_eb, r.c0);
        if (six) std::fprintf(f, "%.17g,", r.c1);
        std::fprintf(f, "%.17g,%.17g,%.17g,%.17g,%.17g,%llu,%.17g\n", r.br, r.h1, r.rmse, r.mae, r.psnr,
                     (unsigned long long)r.samples, r.encode_seconds);
    }
    std::fclose(f);
}

}  // namespace

int main(int argc, char **argv) try {
    if (argc == 2 && std::string(argv[1]) == "--help") {
        std::printf("usage: s2_many_prediction input dim0 dim1 dim2 output_prefix [family-or-stencil [eb0,eb1,... [legacy|augmented|transition [legacy|shared1d|common]]]]\n");
        std::printf("family-or-stencil: 1d4r, 2d4r, 1d6r, all, or one exact stencil such as 1d4r2 or 1d6r0\n");
        return 0;
    }
    if (argc != 1 && (argc < 6 || argc > 10)) throw std::runtime_error("use --help for arguments");
    auto started = std::chrono::steady_clock::now();
    // The reference's defaults (its own dataset and output locations).
    std::string data_path = "/anvil/projects/x-cis240192/x-zjian1-in-cis240192/tensor-data/ISABEL/P/Pf01.bin";
    std::vector<uint64_t> shape = {100, 500, 500};
    std::vector<double> ebs = {1e-2, 1e-3, 1e-4, 1e-5, 1e-6};
    std::string prefix = "/home/x-zjian1/asz/csv/Pf01", family = "all";
    if (argc >= 6) {
        data_path = argv[1];
        for (int a = 0; a < 3; a++) shape[a] = std::stoull(argv[a + 2]);
        prefix = argv[5];
    }
    if (argc >= 7) family = argv[6];
    if (argc >= 8) {
        ebs.clear();
        std::stringstream ss(argv[7]);
        std::string b;
        while (std::getline(ss, b, ',')) ebs.push_back(std::stod(b));
    }
    const std::vector<std::string> stencils = {"1d4r0", "1d4r1", "1d4r2", "2d4r01", "2d4r02", "2d4r12", "1d6r0", "1d6r1", "1d6r2"};
    if (family != "all" && family != "1d4r" && family != "2d4r" && family != "1d6r" &&
        std::find(stencils.begin(), stencils.end(), family) == stencils.end())
        throw std::runtime_error("unknown predictor family or stencil");
    const std::string six = argc >= 9 ? argv[8] : "legacy";
    if (six != "legacy" && six != "augmented" && six != "transition")
        throw std::runtime_error("six-reference grid must be legacy, augmented or transition");
    const std::string targets = argc >= 10 ? argv[9] : "legacy";
    if (targets != "legacy" && targets != "shared1d" && targets != "common")
        throw std::runtime_error("target mode must be legacy, shared1d or common");
    uint64_t grid_size = 0;
    asz_sweep_coefs("1d6r0_xx0", six.c_str(), nullptr, nullptr, 0, &grid_size);
    std::printf("six_reference_grid=%s, candidates=%zu, targets=%s\n", six.c_str(), (size_t)grid_size, targets.c_str());
    if (ebs.empty()) throw std::runtime_error("error-bound grid is empty");
    for (double b : ebs)
        if (!std::isfinite(b) || b <= 0) throw std::runtime_error("error bounds must be positive and finite");
    std::vector<std::string> preds;
    for (const auto &s : stencils)
        if (family == "all" || s.rfind(family, 0) == 0)
            for (int o = 0; o < 3; o++) preds.push_back(s + "_xx" + std::to_string(o));
    for (const auto &p : preds)
        if (std::filesystem::exists(prefix + "_" + p + ".csv")) throw std::runtime_error("output already exists; use a fresh output prefix");
    auto parent = std::filesystem::path(prefix).parent_path();
    if (!parent.empty()) std::filesystem::create_directories(parent);
    uint64_t size = 1;
    for (uint64_t d : shape) {
        if (d < 12 || size > std::numeric_limits<uint64_t>::max() / d)
            throw std::runtime_error("invalid dimensions; each dimension must be at least 12");
        size *= d;
    }
    if (size > std::numeric_limits<uint64_t>::max() / sizeof(float) || std::filesystem::file_size(data_path) != size * sizeof(float))
        throw std::runtime_error("input size does not match float32 dimensions");
    std::vector<float> data(size);
    {
        std::ifstream in(data_path, std::ios::binary);
        in.read(reinterpret_cast<char *>(data.data()), (std::streamsize)(size * sizeof(float)));
        if (!in) throw std::runtime_error("input read failed");
    }
    Ctx ctx;
    ctx.c = asz_create(0);
    if (!ctx.c) throw std::runtime_error("no usable CUDA device");
    bool printed_range = false;
    for (const auto &p : preds) {
        auto t0 = std::chrono::steady_clock::now();
        uint64_t k = 0, n = 0;
        asz_sweep_coefs(p.c_str(), six.c_str(), nullptr, nullptr, 0, &k);
        std::vector<asz_sweep_row> rows(ebs.size() * k);
        float mm[2] = {0, 0};
        int rc = asz_sweep(ctx.c, data.data(), 0, shape.data(), p.c_str(), targets.c_str(), six.c_str(), ebs.data(), ebs.size(),
                           rows.data(), rows.size(), &n, mm);
        const std::string err = rc ? asz_last_error(ctx.c) : "";
        if (!printed_range && (rc == 0 || err == "constant input")) {  // s2_many_prediction.cpp:521-527
            std::printf("min_val=%f\n", (double)mm[0]);
            std::printf("max_val=%f\n", (double)mm[1]);
            printed_range = true;
        }
        if (rc) throw std::runtime_error(err);
        for (const auto &r : rows) {  // lossless_encode_and_write_csv (:431-438)
            if (p.rfind("1d6r", 0) == 0) std::printf("rel_eb=%f, a=%f, b=%f\n", r.rel_eb, r.c0, r.c1);
            else std::printf("rel_eb=%f, t=%f\n", r.rel_eb, r.c0);
            std::printf("BR=%f, CR=%f\n", r.br, r.cr);
            std::printf("H1=%f, H1_cr=%f\n", r.h1, r.h1_cr);
            std::printf("RMSE=%f, MAE=%f\n", r.rmse, r.mae);
            std::printf("PSNR=%f\n", r.psnr);
            std::printf("\n");
        }
        write_csv(prefix + "_" + p + ".csv", p, rows);
        std::printf("predictor=%s, elapsed_seconds=%.6f\n", p.c_str(),
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
    std::printf("total_seconds=%.6f\n", std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count());
    return 0;
} catch (const std::exception &e) {
    std::fflush(stdout);
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
}
