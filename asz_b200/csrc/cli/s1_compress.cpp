// Drop-in replacement for the reference's s1_compress (c_codes/s1_compress.cpp): same flags,
// same .asz output, and the stdout report lines the reference prints (compress.tpp:149-319,
// get_default_slope.tpp:79-82, generate_config.tpp:6-49) that callers parse.
#include <cmath>
#include <cstring>
#include <map>

#include "cli_common.h"

int main(int argc, char *argv[]) try {
    if (argc == 2 && std::string(argv[1]) == "--help") {
        printf("usage: s1_compress -i INPUT -z COMPRESSED -o RECONSTRUCTED -3 DIM0 DIM1 DIM2 -M REL REL_EB [options]\n");
        return 0;
    }
    cli::Args a;
    asz_default_params(&a.p);
    for (int i = 1; i < argc; i++) {
        std::string arg = argv[i];
        if (!cli::parse_flag(arg, argc, argv, i, a, true)) throw std::invalid_argument("unknown argument: " + arg);
    }
    if (a.t_min_set != a.t_max_set) throw std::invalid_argument("t_min and t_max must be supplied together");
    a.p.t_range_set = a.t_min_set;
    if (a.input.empty() || a.compressed.empty()) throw std::invalid_argument("input and compressed-output paths are required");
    if (a.dims.size() != 3 || a.dims[0] < 7 || a.dims[1] < 7 || a.dims[2] < 7)
        throw std::invalid_argument("all three dimensions must be at least 7");
    if (!(a.rel_eb > 0 && std::isfinite(a.rel_eb))) throw std::invalid_argument("relative error bound must be positive and finite");
    const uint64_t n = a.dims[0] * a.dims[1] * a.dims[2];
    std::vector<char> raw = cli::read_file(a.input, "input");
    if (raw.size() != n * sizeof(float)) {
        if (raw.size() < n * sizeof(float)) throw std::runtime_error("cannot read complete input: " + a.input);
        throw std::runtime_error("input size does not match the dimensions: " + a.input);
    }
    cli::Ctx ctx;
    uint8_t *out = nullptr;
    size_t out_len = 0;
    asz_report r{};
    ctx.check(asz_compress(ctx.c, (const float *)raw.data(), 0, a.dims.data(), a.rel_eb, &a.p,
                           a.have_plan ? a.plan.c_str() : nullptr, &out, &out_len, &r));
    const asz_params &p = a.p;
    printf("Data range time: %f s\n", r.data_range_s);
    const char *reason[] = {"none", "invalid_ratio", "invalid_difference"};
    printf("Default slope statistics: max_invalid_ratio=%.6f, fallback=%s, reason=%s, slope=%.6f\n",
           r.slope_max_invalid_ratio, r.slope_fallback_reason ? "true" : "false", reason[r.slope_fallback_reason],
           r.default_slope);
    printf("Get default slope time: %f s\n", r.default_slope_s);
    printf("default_slope=%f\n", r.default_slope);
    if (!a.have_plan) {
        // generate_config's lines (generate_config.tpp:654, 672-673): layer i's winner is the plan's
        // i-th predictor from the end.
        std::vector<std::string> preds;
        {
            std::string pl = r.plan;
            size_t b = 0;
            while (b < pl.size()) {
                size_t e = pl.find(',', b);
                preds.push_back(pl.substr(b, e == std::string::npos ? std::string::npos : e - b));
                if (e == std::string::npos) break;
                b = e + 1;
            }
        }
        for (uint32_t i = 0; i < r.plan_search_layers && i < preds.size(); i++)
            printf("best_layer_predictor=%s, best_dist=%f\n", preds[preds.size() - 1 - i].c_str(), r.plan_best_dist[i]);
        // A layer with no candidate ends the search after printing its empty choice (-1e8 start score).
        if (r.plan_search_layers < p.max_layer_num) printf("best_layer_predictor=, best_dist=%f\n", -1e8f);
        printf("Generate config breakdown: statistics=%f s,sample prediction=%f s,lossless estimation=%f s\n", r.plan_stats_s,
               r.plan_sample_s, r.plan_lossless_s);
        printf("Generate config time: %f s\n", r.plan_s);
    }
    if (r.family_selected) {
        // select_predictor_family's lines (predictor_family.tpp:236-250).
        if (r.family_fallback)
            printf("Predictor family selection: selector=h1, suffix_layers=%lu, blocks=0, sampled_block_points=0, "
                   "sample_point_budget=%lu, probe_block_pivot_ratio=%lu, fallback=point_budget, family=cubic\n",
                   (unsigned long)r.fam_suffix_layers, (unsigned long)r.fam_budget, (unsigned long)r.fam_probe_bpr);
        else
            printf("Predictor family selection: selector=h1, suffix_layers=%lu, blocks=%lu, sampled_block_points=%lu, "
                   "sample_point_budget=%lu, probe_block_pivot_ratio=%lu, points=%lu, cubic_mse=%.12Le, quintic_mse=%.12Le, "
                   "cubic_psnr=%.12Le, quintic_psnr=%.12Le, cubic_h1=%.12Le, quintic_h1=%.12Le, six_score_gain=%.12Le, "
                   "family=%s\n",
                   (unsigned long)r.fam_suffix_layers, (unsigned long)r.fam_blocks, (unsigned long)r.fam_sampled_points,
                   (unsigned long)r.fam_budget, (unsigned long)r.fam_probe_bpr, (unsigned long)r.fam_points, r.fam_cubic_mse,
                   r.fam_quintic_mse, r.fam_cubic_psnr, r.fam_quintic_psnr, r.fam_cubic_h1, r.fam_quintic_h1, r.fam_score_gain,
                   r.quintic ? "quintic" : "cubic");
        printf("Predictor family selection time: %f s\n", r.family_s);
    }
    // print_config (generate_config.tpp:6-49).
    printf("predictor_vec={");
    {
        std::string pl = r.plan;
        size_t b = 0;
        bool first = true;
        while (b <= pl.size()) {
            size_t e = pl.find(',', b);
            printf("%s\"%s\"", first ? "" : ",", pl.substr(b, e == std::string::npos ? std::string::npos : e - b).c_str());
            first = false;
            if (e == std::string::npos) break;
            b = e + 1;
        }
    }
    printf("};\n");
    printf("pivot_eb_ratio=%.2f;\n", p.pivot_eb_ratio);
    printf("eb_ratio=%.2f;\n", p.eb_ratio);
    printf("slope_ratio=%.2f;\n", p.slope_ratio);
    printf("max_layer_num=%lu;\n", (unsigned long)p.max_layer_num);
    printf("full_predictor_search_layer_num=%lu;\n", (unsigned long)p.full_predictor_search_layer_num);
    printf("generate_config_sample_stride=%lu;\n", (unsigned long)p.generate_config_sample_stride);
    printf("h1_block_sampling_num=%lu;\n", (unsigned long)p.h1_block_sampling_num);
    printf("stat_eb_ratio=%.3f;\n", p.stat_eb_ratio);
    printf("predictor_family_suffix_layers=%lu;\n", (unsigned long)p.predictor_family_suffix_layers);
    printf("predictor_family_sample_blocks=%lu;\n", (unsigned long)p.predictor_family_sample_blocks);
    printf("predictor_family_sample_point_limit=%lu;\n", (unsigned long)p.predictor_family_sample_point_limit);
    printf("predictor_family_sample_fraction_limit=%.6f;\n", p.predictor_family_sample_fraction_limit);
    printf("predictor_family_coarse_probe_block_pivot_ratio=%lu;\n", (unsigned long)p.predictor_family_coarse_probe_block_pivot_ratio);
    printf("predictor_family_fine_probe_block_pivot_ratio=%lu;\n", (unsigned long)p.predictor_family_fine_probe_block_pivot_ratio);
    printf("predictor_family_fine_eb_threshold=%.12g;\n", p.predictor_family_fine_eb_threshold);
    printf("default_slope_invalid_ratio_threshold=%.3f;\n", p.default_slope_invalid_ratio_threshold);
    printf("default_slope_fallback=%.6f;\n", p.default_slope_fallback);
    printf("default_slope_eb_span=%.6f;\n", p.default_slope_eb_span);
    printf("t_precision=%d;\n", p.t_precision);
    printf("t_range=[%.6f,%.6f];\n", p.t_min, p.t_max);
    printf("t_candidates={");
    {
        int lo = (int)llroundf(p.t_min * (float)p.t_precision), hi = (int)llroundf(p.t_max * (float)p.t_precision);
        for (int t = lo; t <= hi; t++) printf("%s%.6f", t == lo ? "" : ",", (float)t / (float)p.t_precision);
    }
    printf("};\n");
    printf("block_t_candidates={%.6f,%.6f,%.6f,%.6f,%.6f};\n", 1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32);
    printf("block_pivot_ratio=%lu;\n", (unsigned long)p.block_pivot_ratio);
    printf("insufficient_sample_t=%.6f;\n", 4.0f / 16);
    printf("predictor_family=%s;\n", r.quintic ? "quintic" : "cubic");
    printf("pivot_stride={%u,%u,%u};\n", r.pivot_stride[0], r.pivot_stride[1], r.pivot_stride[2]);
    printf("block_shape={%u,%u,%u};\n", r.block_shape[0], r.block_shape[1], r.block_shape[2]);
    printf("block_num={%u,%u,%u};\n", r.block_num[0], r.block_num[1], r.block_num[2]);
    // compress() (compress.tpp:149-319).
    printf("min_val=%f max_val=%f\n", r.min_val, r.max_val);
    uint64_t nt = asz_debug_t(ctx.c, nullptr);
    printf("total_qb_num=%lu\n", (unsigned long)n);
    printf("t_int_vec.size()=%lu\n", (unsigned long)nt);
    if (p.report_t_histogram) {
        std::vector<int64_t> t(nt);
        asz_debug_t(ctx.c, t.data());
        std::map<int64_t, uint64_t> h;
        for (int64_t v : t) h[v]++;
        printf("T histogram:");
        bool first = true;
        for (auto &kv : h) {
            printf("%s%lld=%lu", first ? "" : ",", (long long)kv.first, (unsigned long)kv.second);
            first = false;
        }
        printf("\n");
        printf("T fallback count:%lu\n", (unsigned long)r.t_fallback_count);
    }
    printf("Huffman compression time: %f s\n", r.huffman_s);
    printf("Zstd compression time: %f s\n", r.zstd_s);
    printf("Core compression time: %f s\n", r.core_s + r.zstd_s);
    printf("Compression time: %f s\n", r.data_range_s + r.core_s + r.zstd_s);
    // The reconstruction comes back from the device for the reference's own error loop.
    std::vector<float> rec(n);
    if (asz_debug_recon(ctx.c, rec.data()) != n) throw std::runtime_error("reconstruction not available");
    const cli::PrintedStats st = cli::printed_stats((const float *)raw.data(), rec.data(), n);
    const float cr = (float)n * sizeof(float) / (float)out_len;
    const float br = 8 * sizeof(float) / cr;
    const float range = r.max_val - r.min_val;
    const float psnr = log10f(range * range / st.mse_sum * (float)n) * 10.0f;
    printf("max_err= %f (%f%%)\n", st.max_err, st.max_err * 100.0f / r.abs_eb);
    printf("CR: %f, BR: %f, PSNR: %f\n", cr, br, psnr);
    printf("dist=%f\n", std::fma(-br, r.default_slope, psnr));
    cli::write_file(a.compressed, out, out_len, "compressed output");
    asz_free(out);
    return 0;
} catch (const std::exception &e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
}
