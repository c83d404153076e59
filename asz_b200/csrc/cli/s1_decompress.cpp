// Drop-in replacement for the reference's s1_decompress (c_codes/s1_decompress.cpp): same flags,
// the reconstruction file, and the stdout lines of decompress.tpp:198-207.
#include <cmath>

#include "cli_common.h"

int main(int argc, char *argv[]) try {
    if (argc == 2 && std::string(argv[1]) == "--help") {
        printf("usage: s1_decompress -i INPUT -z COMPRESSED -o RECONSTRUCTED -3 DIM0 DIM1 DIM2 -M REL REL_EB [options]\n");
        return 0;
    }
    cli::Args a;
    asz_default_params(&a.p);
    for (int i = 1; i < argc; i++) {
        std::string arg = argv[i];
        if (!cli::parse_flag(arg, argc, argv, i, a, false)) throw std::invalid_argument("unknown argument: " + arg);
    }
    if (a.compressed.empty() || a.decompressed.empty())
        throw std::invalid_argument("compressed-input and decompressed-output paths are required");
    if (a.dims.size() != 3 || a.dims[0] < 7 || a.dims[1] < 7 || a.dims[2] < 7)
        throw std::invalid_argument("all three dimensions must be at least 7");
    if (!(a.rel_eb > 0 && std::isfinite(a.rel_eb))) throw std::invalid_argument("relative error bound must be positive and finite");
    std::vector<char> z = cli::read_file(a.compressed, "compressed input");
    if (z.empty()) throw std::runtime_error("compressed input is empty: " + a.compressed);
    const uint64_t n = a.dims[0] * a.dims[1] * a.dims[2];
    std::vector<float> out(n);
    cli::Ctx ctx;
    asz_report r{};
    ctx.check(asz_decompress(ctx.c, (const uint8_t *)z.data(), z.size(), a.dims.data(), a.rel_eb, &a.p, out.data(), 0, &r));
    printf("Zstd decompression time: %f s\n", r.zstd_s);
    printf("Huffman decompression time: %f s\n", r.huffman_s);
    printf("Reconstruction setup time: %f s\n", 0.0);
    printf("Prediction reconstruction time: %f s\n", r.core_s);
    printf("Decompression time: %f s\n", r.total_s);
    float cr = (float)n * sizeof(float) / (float)z.size();
    printf("CR= %f\n", cr);
    printf("BR= %f\n", 8 * sizeof(float) / cr);
    cli::write_file(a.decompressed, out.data(), n * sizeof(float), "decompressed output");
    return 0;
} catch (const std::exception &e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
}
