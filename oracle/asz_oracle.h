/* C interface of the CPU oracle: a restatement of the ASZ reference compression path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load this library, and only as the checker. The product never links it.
 *
 * Every function follows the reference codec (the .tpp files and huffman.hpp under c_codes/asz_core) and the
 * floating-point form GCC 13.3 emits for it under the reference's flags
 * (-Ofast -march=native -mavx2 -mfma, c_codes/CMakeLists.txt:12). Each FMA, reciprocal and
 * rounding step is spelled out, so this file builds with -ffp-contract=off.
 */
#ifndef ASZ_ORACLE_H
#define ASZ_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Tunables of asz::param_c (c_codes/asz_core/asz_param.hpp:147-180). The defaults come from
 * aszo_default_params(). Fields the reference does not store in the .asz must be the same on
 * both sides. */
typedef struct aszo_params {
    float pivot_eb_ratio, eb_ratio, slope_ratio;
    uint64_t block_pivot_ratio;
    int32_t t_precision;
    float t_min, t_max;
    uint64_t h1_block_sampling_num;
    float stat_eb_ratio;
    float default_slope_invalid_ratio_threshold, default_slope_fallback, default_slope_eb_span;
    float insufficient_sample_t;
    uint64_t max_layer_num;                   /* plan search (generate_config.tpp:444-678) */
    uint64_t full_predictor_search_layer_num;
    uint64_t generate_config_sample_stride;
    uint64_t predictor_family_suffix_layers;  /* family selection (predictor_family.tpp:217-251) */
    uint64_t predictor_family_sample_blocks;
    uint64_t predictor_family_sample_point_limit;
    float predictor_family_sample_fraction_limit;
    uint64_t predictor_family_coarse_probe_block_pivot_ratio;
    uint64_t predictor_family_fine_probe_block_pivot_ratio;
    float predictor_family_fine_eb_threshold;
} aszo_params;

void aszo_default_params(aszo_params *p);

/* Result of aszo_compress. Buffers are malloc'd by the oracle; free them with aszo_free_result. */
typedef struct aszo_result {
    uint32_t layer_num;
    uint64_t *qb_len;        /* layer_num+1 stream lengths */
    int32_t **qb;            /* layer_num+1 QB streams (pivot stream first) */
    uint64_t t_len;
    int64_t *t_int;          /* per (block, round) t codes, block-major */
    float *recon;            /* in-place reconstruction (compressed_data) */
    uint8_t *pre_zstd;       /* header + t stream + QB streams, before zstd */
    uint64_t pre_zstd_len;
    uint8_t *asz;            /* final .asz bytes (zstd level 3) */
    uint64_t asz_len;
    float min_val, max_val, abs_eb, default_slope;
    uint64_t t_fallback_count;
    char plan[64 * 11 + 1];  /* plan used (searched when none was given) */
    uint32_t search_layers;  /* plan search: layers that chose a predictor */
    float best_dist[64];     /* plan search: the winning score of each of those layers */
    int32_t quintic;         /* family used */
    int32_t family_selected; /* 1: chosen by the selector (family -1) */
    int32_t family_fallback; /* selector: no block fit the point budget */
    uint64_t fam_suffix_layers, fam_blocks, fam_sampled_points, fam_budget, fam_probe_bpr, fam_points;
    long double fam_cubic_mse, fam_quintic_mse, fam_cubic_psnr, fam_quintic_psnr, fam_cubic_h1, fam_quintic_h1,
        fam_score_gain;
} aszo_result;

/* Compress with a given plan ("cubic2_012,cubic1_120,..."), quintic = force_quintic (0 or 1), or
 * -1 to run the reference's predictor-family selector. A NULL plan runs the reference's plan
 * search (param_c::generate_config).
 * Returns 0 or a negative error code; err (256 bytes) receives a message. */
int aszo_compress(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p,
                  const char *plan, int quintic, aszo_result *out, char *err);
void aszo_free_result(aszo_result *r);

/* As aszo_compress with a given plan and family, but the per-(block, round) t codes come from
 * t_int (block-major, block_num product x layer_num entries) instead of the coefficient selection.
 * The stream stores them; the reference's decompressor reads any code as t = code / t_precision. */
int aszo_compress_with_t(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p,
                         const char *plan, int quintic, const int64_t *t_int, uint64_t t_len, aszo_result *out,
                         char *err);

/* The gradient tuner's open-loop AB samples of every (block, round) group (block-major), read
 * from the original data on get_AB_map's lattice. Sizes come back in groups/samples; the arrays
 * are filled when they are non-NULL and cap >= samples (offsets: groups + 1 entries). */
int aszo_grad_samples(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p, const char *plan,
                      float *A, float *B, uint64_t *offsets, uint64_t cap, uint64_t *groups, uint64_t *samples,
                      char *err);

/* Decompress an .asz produced by the reference or by aszo_compress. */
int aszo_decompress(const uint8_t *asz, uint64_t asz_len, const uint64_t dims[3], float rel_eb,
                    const aszo_params *p, float *out, char *err);

/* Default rate-distortion slope (c_codes/asz_core/get_default_slope.tpp:6-83). */
float aszo_default_slope(const float *data, const uint64_t dims[3], float abs_eb, float min_val,
                         float max_val, const aszo_params *p);

/* Huffman-encode one stream exactly as huffman_encoder_class<T> does (save + encode), T=int32
 * (wide=0) or int64 (wide=1). Returns the byte count; out may be NULL to query the size. */
uint64_t aszo_huffman_encode(const void *symbols, uint64_t n, int wide, uint8_t *out);

/* Order probe for the hash-table emulation: builds std::unordered_map<tuple<int64,int64>,u64>
 * with the reference hash from keys (a[i], b[i]) in sequence and writes the iteration order
 * as indices of first occurrence into order (length = number of distinct keys, returned). */
uint64_t aszo_abmap_order(const int64_t *a, const int64_t *b, uint64_t n, uint64_t *order);
/* Same for std::unordered_map<int64_t,u64> (identity hash). */
uint64_t aszo_i64map_order(const int64_t *k, uint64_t n, uint64_t *order);

/* The reference's per-group proxy evaluation (c_codes/asz_core/get_h_psnr.tpp:6-31) on a map
 * built from the keys in sequence. Also returns the float fed to log10f (x) and the sum (mse). */
void aszo_h1_psnr(const int64_t *a, const int64_t *b, uint64_t n, float t, float abs_eb, float stat_eb,
                  float min_val, float max_val, float *h1, float *psnr, float *x, float *mse);

/* Prediction sweep (c_codes/s2_many_prediction.cpp), one row = one predictor, rel_eb and
 * coefficient set. Sums are before the divisions by the sample count. */
typedef struct aszo_sweep_row {
    double c0, c1;                 /* t (1d4r, 2d4r) or a, b (1d6r) */
    uint64_t samples, huffman_bytes, zstd_bytes;
    double mse_sum, rmse_sum, mae_sum;
    double br, cr, h1, h1_cr, rmse, mae, psnr;
} aszo_sweep_row;

/* Coefficients of a predictor ("1d4r0_xx2", "2d4r01_xx1", "1d6r2_xx0"): t = i/32 (1d4r), i/24
 * (2d4r), or the six-reference grid "legacy" | "augmented" | "transition" (1d6r). Returns the
 * count (arrays filled up to cap) or -1. */
int aszo_sweep_coefs(const char *predictor, const char *six_grid, double *c0, double *c1, uint64_t cap);
/* The targets in stream order as (i0, i1, i2) triples (up to cap); returns the count. targets:
 * "legacy" | "shared1d" | "common". */
uint64_t aszo_sweep_targets(const uint64_t dims[3], const char *predictor, const char *targets, uint64_t *coords,
                            uint64_t cap);
/* One row: QB stream (qb_out may be NULL), H1, Huffman + zstd sizes and the figures. */
int aszo_sweep_run(const float *data, const uint64_t dims[3], const char *predictor, const char *targets, double rel_eb,
                   float min_val, float max_val, double c0, double c1, int64_t *qb_out, uint64_t qb_cap,
                   aszo_sweep_row *row, char *err);
/* Fills br, cr, h1_cr, rmse, mae and psnr from the sizes and sums; range = max - min. */
void aszo_sweep_finish(aszo_sweep_row *row, double range);

#ifdef __cplusplus
}
#endif
#endif
