/* asz_b200: B200-native implementation of the ASZ compression hot path behind a C ABI.
 *
 * The reference (ASZ) has no library boundary of its own: callers drive the CLI binaries
 * s1_compress / s1_decompress and exchange raw float32 files and .asz streams. These entry points
 * replace that surface one for one:
 *
 *   asz_compress    replaces s1_compress's main (c_codes/s1_compress.cpp:153-341): parameter
 *                   validation (:49-99), data range (:101-140), plan preparation (:30-47) and
 *                   param_c<float>::compress() (c_codes/asz_core/compress.tpp:147-321).
 *   asz_decompress  replaces s1_decompress's main (c_codes/s1_decompress.cpp:5-149) and
 *                   param_c<float>::decompress() (c_codes/asz_core/decompress.tpp:79-208).
 *
 * The .asz bytes are the reference's bitstream: the same header, t stream, Huffman trees and
 * payloads, compressed by libzstd at level 3 on the host. For the same input, error bound, plan
 * and parameters the output equals s1_compress's byte for byte when both link the same libzstd.
 *
 * Errors: every call returns 0 on success or a negative ASZ_E* code; asz_last_error(ctx) holds
 * the message. The reference prints "error: <msg>" and exits 1 on the same conditions. Device
 * faults are never raised on purpose: kernels bound every loop and report through an error word.
 *
 * Threading: a context owns one CUDA stream and its device buffers. Calls on one context must
 * not overlap; separate contexts may be used from separate threads.
 */
#ifndef ASZ_B200_H
#define ASZ_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define ASZ_OK 0
#define ASZ_E_ARG -1      /* invalid argument (reference: std::invalid_argument) */
#define ASZ_E_DATA -2     /* invalid input data or stream (reference: std::runtime_error) */
#define ASZ_E_CUDA -3     /* CUDA runtime error */
#define ASZ_E_DEVICE -4   /* a kernel reported an inconsistency through its error word */
#define ASZ_E_UNSUPPORTED -5
#define ASZ_E_COMM -6     /* a caller's collective (asz_comm) failed */

/* Predictor family: ASZ_FAMILY_AUTO runs the reference's selector (predictor_family.tpp). */
#define ASZ_FAMILY_AUTO -1
#define ASZ_FAMILY_CUBIC 0
#define ASZ_FAMILY_QUINTIC 1

/* Every tunable of s1_compress / s1_decompress (c_codes/s1_compress.cpp:163-333), with the
 * defaults of asz::param_c (c_codes/asz_core/asz_param.hpp:147-180) from asz_default_params.
 * The reference does not store block_pivot_ratio, eb_ratio, pivot_eb_ratio or t_precision in the
 * .asz, so the decompressor must be given the values the compressor used. */
typedef struct asz_params {
    float pivot_eb_ratio;           /* --pivot-eb-ratio, default 0.05 */
    float eb_ratio;                 /* --eb-ratio, default 0.76 */
    float slope_ratio;              /* --slope-ratio, default 0.54 */
    uint64_t block_pivot_ratio;     /* --block-pivot-ratio, default 4 */
    uint64_t max_layer_num;         /* --max-layer-num, default 14 */
    uint64_t full_predictor_search_layer_num; /* default 4 */
    uint64_t generate_config_sample_stride;   /* default 5 */
    uint64_t h1_block_sampling_num; /* default 256 */
    float stat_eb_ratio;            /* default 0.2 */
    uint64_t predictor_family_suffix_layers;  /* default 6 */
    uint64_t predictor_family_sample_blocks;  /* default 8 */
    uint64_t predictor_family_sample_point_limit; /* default 32768 */
    float predictor_family_sample_fraction_limit; /* default 0.02 */
    uint64_t predictor_family_coarse_probe_block_pivot_ratio; /* default 3 */
    uint64_t predictor_family_fine_probe_block_pivot_ratio;   /* default 4 */
    float predictor_family_fine_eb_threshold; /* default 1e-4 */
    float default_slope_invalid_ratio_threshold; /* default 1 */
    float default_slope_fallback;   /* default 1000 */
    float default_slope_eb_span;    /* default 1.5 */
    int32_t t_precision;            /* --t-precision, default 32 */
    float t_min, t_max;             /* --t-min/--t-max, defaults 1/16 and 6/16 */
    int32_t t_range_set;            /* nonzero when t_min/t_max were given (they come together) */
    int32_t predictor_family;       /* ASZ_FAMILY_*, default AUTO */
    int32_t report_t_histogram;     /* --report-t-histogram */
} asz_params;

/* Timings (seconds) and figures of one call, matching the reference's stdout lines. */
typedef struct asz_report {
    double data_range_s;      /* "Data range time" */
    double default_slope_s;   /* "Get default slope time" */
    double plan_s;            /* "Generate config time" (auto plans) */
    double family_s;          /* "Predictor family selection time" */
    double core_s;            /* "Core compression time" without zstd (GPU rounds + Huffman) */
    double huffman_s;         /* "Huffman compression time" / "Huffman decompression time" */
    double zstd_s;            /* "Zstd compression time" / "Zstd decompression time" */
    double h2d_s, d2h_s;      /* host<->device copies inside the call */
    double total_s;           /* wall time of the whole call */
    float min_val, max_val, abs_eb, default_slope;
    float max_err, psnr, cr, br;
    uint64_t t_fallback_count;
    uint64_t pre_zstd_len, asz_len;
    uint64_t layer_num;
    float slope_max_invalid_ratio; /* "Default slope statistics" line */
    int32_t slope_fallback_reason; /* 0 none, 1 invalid_ratio, 2 invalid_difference */
    uint64_t ambiguous_decisions; /* per-block t decisions re-checked on the host */
    uint64_t reruns;              /* compressions repeated after a host re-check */
    uint64_t exact_groups;        /* (block, round) groups the certified fast path handed to the exact path */
    uint64_t serial_groups;       /* groups the exact kernels could not take (serial kernel) */
    uint64_t exact_window;        /* of exact_groups: errors spread wider than the fast path's histogram */
    uint64_t exact_undecided;     /* of exact_groups: a comparison the fast path's bounds could not settle */
    uint64_t wide_groups;         /* groups the fast path settled by counting their bins window by window */
    uint64_t kernel_launches;     /* this library's kernels launched by the call (CUB scans not counted) */
    /* Plan search (no plan given): "Generate config breakdown" phases (seconds), and per layer
     * from the finest the winning score ("best_layer_predictor=..., best_dist=..."); the winning
     * predictors are the plan read from its end. */
    double plan_stats_s, plan_sample_s, plan_lossless_s;
    uint32_t plan_search_layers;
    float plan_best_dist[64];
    /* Predictor-family selection (family ASZ_FAMILY_AUTO), the figures of its stdout line
     * (predictor_family.tpp:236-248): prediction MSE, PSNR and H1 per family, and the score. */
    int32_t family_selected, family_fallback;
    uint64_t fam_suffix_layers, fam_blocks, fam_sampled_points, fam_budget, fam_probe_bpr, fam_points;
    long double fam_cubic_mse, fam_quintic_mse, fam_cubic_psnr, fam_quintic_psnr, fam_cubic_h1, fam_quintic_h1,
        fam_score_gain;
    uint32_t pivot_stride[3], block_shape[3], block_num[3];
    int32_t quintic;
    char plan[64 * 11 + 1];       /* comma-separated predictor plan actually used */
} asz_report;

typedef struct asz_ctx asz_ctx;

void asz_default_params(asz_params *p);

/* Create a context bound to CUDA device `device`. Returns NULL on failure. */
asz_ctx *asz_create(int device);
void asz_destroy(asz_ctx *ctx);
const char *asz_last_error(const asz_ctx *ctx);

/* Run subsequent calls on the caller's stream (a cudaStream_t passed as a pointer); NULL
 * restores the context's own stream. */
int asz_set_stream(asz_ctx *ctx, void *cuda_stream);

/* Compress a C-order float32 field (dims[2] fastest). `in` is a host pointer, or a device
 * pointer when in_on_device is nonzero. `plan` is the reference's plan string
 * ("cubic2_012,cubic1_120,..."); NULL asks for the reference's automatic plan search.
 * On success *out receives a buffer of *out_len .asz bytes; release it with asz_free. */
int asz_compress(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                 const asz_params *p, const char *plan, uint8_t **out, size_t *out_len, asz_report *rep);

/* As asz_compress, with the per-(block, round) coefficients given instead of selected: t_int holds
 * block-major t codes (for block b = (b0 * block_num1 + b1) * block_num2 + b2 and round l, entry
 * b * layers + l), each within [t_min, t_max] * t_precision. The stream stores them and every
 * decoder, the reference's included (decompress.tpp:183-185 reads t as code / t_precision),
 * reconstructs with them. A plan and a fixed family are required. No counterpart in the reference:
 * it is the output stage of the gradient tuner (asz_b200/grad.py). */
int asz_compress_with_t(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                        const asz_params *p, const char *plan, const int64_t *t_int, uint64_t t_len, uint8_t **out,
                        size_t *out_len, asz_report *rep);

/* ---- Gradient tuner of the per-block coefficients (no counterpart in the reference) ----
 * A relaxed, differentiable form of the reference's H1-PSNR proxy (get_h_psnr.tpp:6-31) over
 * open-loop AB samples (get_AB_map.tpp:13-21 read from the original field), one group per
 * (block, round) indexed block * layers + round like the t stream. The relaxed proxy and its
 * derivative are defined in asz_b200/csrc/k_grad.cu. Flow: asz_grad_setup sizes the problem,
 * the caller allocates device buffers of those sizes, asz_grad_gather fills them, then
 * asz_grad_forward / asz_grad_backward evaluate J(t) and dJ/dt for a t per group (device pointers,
 * on cuda_stream), and asz_grad_tune runs the whole tuning (projected steps, snap to the t grid,
 * the reference's exact proxy as the judge against t = 1/4) and writes t codes for
 * asz_compress_with_t. Status 0 on success, 1 for a bad argument, 7 for a launch error. */
typedef struct asz_grad_problem {
    uint64_t groups;       /* blocks * layers */
    uint64_t samples;      /* AB samples over all groups (A, B buffer length) */
    uint64_t blocks, layers;
    float R2;              /* (max - min)^2 of the field */
    float abs_eb, default_slope;
    float t_min, t_max;
    int32_t t_precision;
} asz_grad_problem;

/* Range, error bound, default slope and plan geometry of a field (plan required); keeps a
 * reference to `in` (a copy for host input) until the next call. */
int asz_grad_setup(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                   const asz_params *p, const char *plan, asz_grad_problem *out);
/* Device buffers: A, B (samples floats), offsets (groups + 1 uint32), meta (groups * 4 floats:
 * layer eb, stat eb, 0.5 / stat eb, layer slope). Runs on the context's stream and waits. */
int asz_grad_gather(asz_ctx *ctx, float *A, float *B, uint32_t *offsets, float *meta);
/* J[g] for t[g] (relaxed proxy, lower is better). */
int asz_grad_forward(const float *A, const float *B, const uint32_t *offsets, const float *meta, float R2,
                     const float *t, uint64_t groups, float *J, void *cuda_stream);
/* grad_t[g] = grad_J[g] * dJ[g]/dt[g]. */
int asz_grad_backward(const float *A, const float *B, const uint32_t *offsets, const float *meta, float R2,
                      const float *t, const float *grad_J, uint64_t groups, float *grad_t, void *cuda_stream);
/* steps projected sign-gradient steps from t = 1/4 (step sizes step0 * 2^-k) inside [t_min, t_max],
 * snapped to codes on the t_precision grid; the reference's proxy (order-free sums, all samples)
 * keeps code 1/4 * t_precision unless the snapped code scores higher. The steps evaluate J on every
 * k-th sample of a group, k = ceil(n / step_cap) (step_cap 0 or above 1024: 1024). team: threads
 * per group (a multiple of 32 up to 512; 0 for the default 256). Writes t_codes[groups] (int64) and, if
 * non-NULL, t_relaxed[groups]; stats (3 uint32 on the device, zeroed by the caller) count tuned
 * groups, accepted codes, and groups whose quantised errors spread over more than 262144 bins
 * (the judge then keeps the default). */
int asz_grad_tune(const float *A, const float *B, const uint32_t *offsets, const float *meta, float R2, uint64_t groups,
                  float t_min, float t_max, int32_t t_precision, uint32_t steps, float step0, uint32_t step_cap,
                  uint32_t team, int64_t *t_codes, float *t_relaxed, uint32_t *stats, void *cuda_stream);

/* ---- Batches: many fields, one plan, one error bound (no counterpart in the reference, which
 * compresses one field per process). Each field gets the bytes asz_compress gives it: its own
 * range, default slope and geometry; the rounds of all fields run together, per round one
 * launch of each selection kernel and of the prediction kernel, each over a work queue of every
 * field's (block) groups or target lines, captured once per batch layout as a CUDA graph. The
 * persistent grids' CTAs per SM and the threads per target line come from an autotuner that times
 * the candidates on the first batch of a shape and reuses the choice. A field with a coefficient
 * decision that needs the host's log10f replay takes the single-field path (fields_fallback).
 * zstd runs on host threads as each field's stream is ready. */
typedef struct asz_batch_report {
    double total_s, h2d_s, prep_s, tune_s, rounds_s, encode_s, zstd_s; /* zstd_s: summed over threads */
    double rounds_ms;            /* device time of the captured round sequence */
    uint64_t input_bytes, output_bytes, kernel_launches;
    uint32_t tuned_now;          /* the autotuner ran in this call */
    uint32_t graph_reused;       /* the captured sequence of a previous call was replayed */
    uint32_t fields_fallback;    /* fields that took the single-field path */
    uint32_t fast_ctas_per_sm, round_ctas_per_sm, tpl_shift;  /* launch shapes in use */
} asz_batch_report;

/* in: count field pointers (host, or device when in_on_device); dims: 3 per field; plan required;
 * the family must be fixed. out[f] / out_len[f] receive each field's .asz (asz_free each);
 * reps (count entries) and brep are optional. */
int asz_compress_batch(asz_ctx *ctx, uint32_t count, const float *const *in, int in_on_device, const uint64_t *dims,
                       float rel_eb, const asz_params *p, const char *plan, uint8_t **out, size_t *out_len,
                       asz_report *reps, asz_batch_report *brep);

/* As asz_compress_batch, with each field's t codes given (t_tables[f], t_lens[f] entries,
 * block-major as for asz_compress_with_t) instead of selected: the time-series form, where the plan
 * of the first step is reused and each later step's coefficients come from the gradient tuner. */
int asz_compress_batch_with_t(asz_ctx *ctx, uint32_t count, const float *const *in, int in_on_device,
                              const uint64_t *dims, float rel_eb, const asz_params *p, const char *plan,
                              const int64_t *const *t_tables, const uint64_t *t_lens, uint8_t **out, size_t *out_len,
                              asz_report *reps, asz_batch_report *brep);

/* ---------------------------------------------------------------------------------------------
 * One field compressed by several ranks (one process per GPU), each holding a slab of axis-0
 * planes cut at block boundaries, for fields larger than one GPU's memory. The reference walks
 * the blocks of one field in raster order (compress.tpp:179-209); a slab is a run of axis-0
 * blocks, whose blocks are contiguous in every stream, so the ranks' stream pieces concatenated in
 * rank order are the single-field streams and rank 0's .asz is byte-identical to asz_compress's.
 * Exchanges: the data range (all ranks), the default slope's samples (all ranks), before each
 * axis-0 round the reconstructed planes just below each slab (from the rank below), the rerun
 * decision of the coefficient replay, the QB ranges and histograms (all ranks build the same
 * codes), and each rank's encoded pieces (to rank 0). The plan and the family must be given
 * (the plan search and the family selector sample the whole field). */

/* The caller's collectives over host buffers; each returns 0 on success. The library stages
 * device data through host memory and calls them in the same order on every rank. */
typedef struct asz_comm {
    int rank, size;
    void *user;
    /* In-place reduction over all ranks of count values: dtype 0 float32, 1 uint64, 2 int32;
     * op 0 sum, 1 min, 2 max. */
    int (*allreduce)(void *user, void *buf, uint64_t count, int dtype, int op);
    /* Each rank contributes `bytes` bytes; recv (size * bytes) receives them in rank order. */
    int (*allgather)(void *user, const void *send, uint64_t bytes, void *recv);
    int (*send)(void *user, const void *buf, uint64_t bytes, int dst);
    int (*recv)(void *user, void *buf, uint64_t bytes, int src);
} asz_comm;

/* The axis-0 planes a rank passes for its blocks [block_begin, block_end) of the plan's axis-0
 * blocks: planes [plane_begin, plane_begin + plane_count). Rank 0's slab starts at plane 0; any
 * other slab starts one plane past its first block's lower face, which belongs to the slab below.
 * blocks0 (optional) receives the field's number of axis-0 blocks. */
int asz_slab_planes(const uint64_t dims[3], const asz_params *p, const char *plan, uint64_t block_begin,
                    uint64_t block_end, uint64_t *plane_begin, uint64_t *plane_count, uint64_t *blocks0);

/* Compress this rank's slab: `planes` holds plane_count x dims[1] x dims[2] floats (host, or
 * device when on_device) as asz_slab_planes gives them; dims are the whole field's. Every rank
 * calls it with its own blocks; the blocks of all ranks, in rank order, cover the axis-0 blocks
 * exactly. Rank 0 receives the .asz in out/out_len (asz_free it); other ranks receive NULL/0.
 * rep (optional): the whole field's figures on every rank. A rank that fails returns nonzero;
 * the others then fail in their next exchange (the caller's collectives should time out). */
int asz_compress_slab(asz_ctx *ctx, const asz_comm *comm, const float *planes, int on_device, const uint64_t dims[3],
                      uint64_t block_begin, uint64_t block_end, float rel_eb, const asz_params *p, const char *plan,
                      uint8_t **out, size_t *out_len, asz_report *rep);

/* Decompress .asz bytes into `out` (prod(dims) floats; host pointer, or device pointer when
 * out_on_device is nonzero). */
int asz_decompress(asz_ctx *ctx, const uint8_t *in, size_t len, const uint64_t dims[3], float rel_eb,
                   const asz_params *p, float *out, int out_on_device, asz_report *rep);

void asz_free(void *ptr);
/* asz_free keeps released output buffers (at most 64 of them, 2 GiB in all) for later outputs of
 * the same or smaller size, whose memory is then already mapped. This frees them. No reference
 * counterpart. */
void asz_release_output_cache(void);

/* Error statistics of the last asz_compress call on this context, as the reference prints them
 * after compressing (compress.tpp:307-319): max |x - x'| and PSNR in dB. The input buffer given
 * to that call must still be valid (device input) or is the context's own copy (host input). */
int asz_compress_stats(asz_ctx *ctx, double *max_err, double *psnr);

/* Device-time profile by kernel family (CUDA events around each launch on the context's
 * stream). Off by default; enabling it adds one event pair per launch. */
typedef struct asz_profile_entry {
    char name[32];        /* kernel family, e.g. "tsel", "round_compress", "huff_encode" */
    uint64_t launches;
    double ms;            /* summed device time */
    uint64_t bytes;       /* algorithmic bytes moved by those launches (reads + writes) */
} asz_profile_entry;

int asz_profile_enable(asz_ctx *ctx, int on);

/* Per-block coefficient selection strategy. 0 (default): a certified order-free fast path settles
 * most (block, round) groups and the exact hash-order replay settles the rest, one launch per
 * round. 1: the exact replay for every group. 2: as 0, and plans with every round along axis 2
 * run all their rounds fused per column of lines held in shared memory (compression and
 * decompression). All give the reference's choices and bytes. */
int asz_set_tsel_mode(asz_ctx *ctx, int mode);
/* Copies up to max entries accumulated since the last reset; returns how many exist. */
int asz_profile_read(asz_ctx *ctx, asz_profile_entry *out, int max, int reset);

/* Error statistics of any reconstruction y of x (device pointers, n floats) that allocate nothing:
 * max |x - y| and PSNR = 10 log10(value_range^2 / mse), the figures asz_compress_stats gives for
 * the last compression. No reference counterpart: the reference computes these on the host inside
 * compress() (compress.tpp:307-319); this is the device form for callers without a context or
 * that must not allocate device memory. Scratch is a fixed 1 MiB device array in the library, so
 * n is limited to 65520 * 65536 values; larger n returns ASZ_E_ARG with a message. Squared
 * differences are summed in a fixed order, so repeated calls return identical bits.
 * Runs on the current device and on cuda_stream (NULL: the legacy default stream), and
 * synchronises that stream before it returns, so the figures are ready when the call ends. Each
 * call looks up the scratch array's device address in the current context (the lookup allocates
 * nothing). Calls on one device share the scratch: overlapping calls (from several threads or
 * streams) race and must be serialised by the caller. err (may be NULL) receives a message of at
 * most err_len bytes. */
int asz_error_stats_noalloc(const float *x, const float *y, uint64_t n, double value_range, void *cuda_stream,
                            double *max_err, double *psnr, char *err, size_t err_len);

/* ---------------------------------------------------------------------------------------------
 * Prediction sweep: the GPU form of the reference's study tool s2_many_prediction
 * (c_codes/s2_many_prediction.cpp:164-464, whose command line bin/s2_many_prediction keeps). One
 * call runs one predictor ("1d4r<axis>_xx<order>", "2d4r<axes>_xx<order>" with axes 01, 02 or 12,
 * "1d6r<axis>_xx<order>") over each relative error bound and each coefficient of the predictor's
 * grid: t = i/32, i = 0..12 (1d4r); t = i/24, i = -6..6 (2d4r); the six-reference grid "legacy",
 * "augmented" or "transition" (1d6r, six_reference_grid :89-124). Targets are "legacy",
 * "shared1d" (1d4r margin 5) or "common" (for_each_common_target :126-149). Each row carries the
 * tool's figures: BR and CR from the zstd-3 size of the Huffman-coded QB stream, H1, prediction
 * RMSE and MAE, PSNR, and the sample count. QB streams, H1, the Huffman and zstd sizes (so BR
 * and CR) are the reference's exactly; RMSE, MAE and PSNR come from sums taken in a different
 * order and agree to rounding (relative 1e-12 in the tests). */
typedef struct asz_sweep_row {
    double rel_eb, c0, c1;        /* c0 = t (1d4r, 2d4r) or a (1d6r); c1 = b (1d6r) */
    uint64_t samples, huffman_bytes, zstd_bytes;
    double mse_sum, rmse_sum, mae_sum;   /* sums over the targets, before the divisions */
    double br, cr, h1, h1_cr, rmse, mae, psnr;
    double encode_seconds;        /* this row's share of its batch's histogram, Huffman and zstd time */
} asz_sweep_row;

/* The coefficient grid of a predictor: fills c0/c1 up to cap, the count in *count. */
int asz_sweep_coefs(const char *predictor, const char *six_grid, double *c0, double *c1, uint64_t cap, uint64_t *count);
/* Host-side run of the kernel's target mapping (no GPU involved): the targets' (i0, i1, i2) in QB
 * stream order into coords[0, 3 x count) when coords is non-NULL (cap >= count). Returns
 * ASZ_E_DEVICE if the mapping misses or repeats a stream position. */
int asz_sweep_targets(const uint64_t dims[3], const char *predictor, const char *targets, uint64_t *coords, uint64_t cap,
                      uint64_t *count);
/* Rows for every rel_eb (outer) and coefficient (inner), the reference's order, into rows[0,
 * cap); *n_rows = n_eb x grid size (ASZ_E_ARG when cap is smaller). min_max (may be NULL)
 * receives the field's float minimum and maximum (std::min_element / std::max_element). The
 * field must have every dimension >= 12, finite values and max > min. */
int asz_sweep(asz_ctx *ctx, const float *data, int on_device, const uint64_t dims[3], const char *predictor,
              const char *targets, const char *six_grid, const double *rel_eb, uint64_t n_eb, asz_sweep_row *rows,
              uint64_t cap, uint64_t *n_rows, float *min_max);

/* Host-side self-check of the target geometry the round kernels use, for a field of the given
 * dims, plan and block ratio (no GPU involved): every stencil and sampling read is in bounds
 * and hits a value written in an earlier round, every point is written once, and the QB index
 * of every target equals its position in the reference's block-major loops
 * (compress.tpp:53-88). Returns the number of violations (0), or a negative error code. */
int64_t asz_check_geometry(const uint64_t dims[3], const char *plan, uint64_t block_pivot_ratio, int quintic);
/* The same for a frame whose blocks and pivot lattice start at `origin` (the predictor-family
 * probe's local contexts, predictor_family.tpp:40-60): positions below the origin, and the
 * origin's faces off the pivot lattice, keep their input values and are never written. */
int64_t asz_check_geometry_frame(const uint64_t dims[3], const uint64_t origin[3], const char *plan,
                                 uint64_t block_pivot_ratio, int quintic);

/* Host-side run of the device's std::unordered_map order emulation (no GPU involved), for
 * checking it against the real container: keys are (a[i], b[i]) pairs with the reference's
 * hash (asz_param.hpp:22-40) when pair is nonzero, else a[i] with the identity hash. Writes the
 * iteration order as indices of first occurrence; returns the number of distinct keys, or a
 * negative value if the emulated list is inconsistent. */
int64_t asz_check_hashorder(const int64_t *a, const int64_t *b, uint64_t n, int pair, uint64_t *order);

/* Internals of the last asz_compress call on this context, for parity checks: QB stream k
 * (0 = pivots, k = round k), per-(block, round) t codes, the in-place reconstruction and the
 * stream before zstd. Each copies into caller memory and returns the element count; pass NULL to
 * query the count. */
uint64_t asz_debug_qb(asz_ctx *ctx, uint32_t stream, int32_t *dst);
uint64_t asz_debug_t(asz_ctx *ctx, int64_t *dst);
uint64_t asz_debug_recon(asz_ctx *ctx, float *dst);
uint64_t asz_debug_pre_zstd(asz_ctx *ctx, uint8_t *dst);
/* Per (round, block): h1 of t = 1/16, 1/4, 9/32, 5/16, 11/32, then the five log10f arguments
 * (10 floats per group, round-major; all-ones bits where the block fell back). */
uint64_t asz_debug_proxies(asz_ctx *ctx, float *dst);

#ifdef __cplusplus
}
#endif
#endif
