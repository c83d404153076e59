// Host-callable launchers for the CUDA kernels, and the structs they share with the host.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "dev_common.cuh"
#include "tsel.cuh"

namespace asz {

// Kernels launched by this library on the calling thread (each launcher counts its own launches;
// library kernels such as CUB's scans are not counted).
uint64_t &launch_counter();
inline void count_launch() { ++launch_counter(); }


struct CodeEntry {
    uint32_t code;
    uint32_t len;
};

struct LutEntry {
    uint32_t sym;   // symbol index (value - offset), or tree node when len == 0
    uint32_t len;
};

// One stream of a batched decode (see k_huff.cu). Chunks of the stream are chunk0 .. chunk0 +
// nchunks - 1 in the global numbering; its tiles start at tile0.
struct DecStream {
    uint64_t bit_begin, bit_end;   // payload bits, absolute from the stream buffer base
    uint64_t chunk0, nchunks, tile0;
    uint64_t lut_off, child_off;   // entries into the batched table arenas
    uint64_t count;                // values the stream must produce
    int64_t offset;                // added to each symbol index
    void *out;                     // int64 values when wide, else int32
    uint32_t lut_bits, wide;
};

constexpr uint32_t kDecodeTile = 256;  // chunks per tile (threads per decode CTA)

// One candidate predictor of a plan-search layer (generate_config.tpp:526-604): its sample lattice
// (start, stride and count per axis; loop nest ax[0] outer .. ax[2] inner), stencil geometry along
// the prediction axis, t and error bound, and its offset in the layer's sample arrays.
struct PlanCand {
    uint64_t lo[3], st[3], cnt[3];
    uint64_t off;
    uint64_t hs, dist, right;
    float t, eb, neg_2_eb;
    int32_t dir;
    int32_t ax[3];
};

cudaError_t launch_range(const float *x, uint64_t n, int32_t *out, unsigned long long *nonfinite, cudaStream_t st);
cudaError_t launch_zero_first_last(const float *x, uint64_t n, unsigned long long *first, unsigned long long *last,
                                   cudaStream_t st);
// Batches (host/batch.cpp): one launch per round for every field of a batch. The fast selection and
// the round kernel take work items from a queue (a device counter, zero before the launch); items
// map to fields through an exclusive prefix of per-field item counts (nf + 1 entries). Groups the
// fast path hands off, and groups the exact path spills, are (field << 32 | group) entries.
cudaError_t launch_tsel_fast_batch(const BatchField *F, const uint64_t *goff, uint32_t nf, uint32_t l, const float *log2arena,
                                   float t_default, uint32_t *queue, unsigned long long *handoff_list, uint32_t *handoff_count,
                                   uint32_t grid, cudaStream_t st);
cudaError_t launch_tsel_exact_batch(const BatchField *F, uint32_t l, const float *log2arena, float t_default,
                                    const unsigned long long *list, const uint32_t *list_count, unsigned long long *spill,
                                    uint32_t *spill_count, uint32_t cap, unsigned grid, cudaStream_t st);
// Groups the batched exact kernel spilled (above its shared-memory capacity), a CTA each in a
// `stride`-byte slice of global scratch; what it cannot take goes to `spill`.
cudaError_t launch_tsel_exact_global_batch(const BatchField *F, uint32_t l, const float *log2arena, float t_default,
                                           const unsigned long long *list, const uint32_t *list_count,
                                           unsigned long long *spill, uint32_t *spill_count, uint8_t *scratch, uint64_t stride,
                                           uint32_t cap, unsigned grid, cudaStream_t st);
cudaError_t launch_tsel_v0_batch(const BatchField *F, uint32_t l, const float *log2arena, float t_default, uint8_t *scratch,
                                 uint64_t scratch_stride, uint32_t cap, uint32_t bcap, uint32_t tcap,
                                 const unsigned long long *list, const uint32_t *list_count, uint64_t slots, cudaStream_t st);
cudaError_t launch_pivot_compress_batch(const BatchField *F, const uint64_t *poff, uint32_t nf, uint64_t total_pivots,
                                        cudaStream_t st);
cudaError_t launch_tval_from_codes_batch(const BatchField *F, const uint64_t *goff, uint32_t nf, uint64_t total_blocks,
                                         uint32_t l, cudaStream_t st);
uint32_t round_tpl_log2(uint64_t t2);
uint64_t round_batch_items(const RoundGeom &rg, uint32_t tpl_log2);
cudaError_t launch_round_compress_batch(const BatchField *F, const uint64_t *ioff, uint32_t nf, uint32_t l, uint32_t *queue,
                                        uint32_t grid, cudaStream_t st);

// Open-loop AB samples of every (block, round) group for the gradient tuner (k_grad.cu).
cudaError_t launch_grad_gather(const FieldGeom &fg, const RoundGeom *rounds, const ClassInfo *classes, const float *x,
                               const uint32_t *off, uint64_t groups, float *A, float *B, uint32_t *err, cudaStream_t st);
cudaError_t launch_tval_from_codes(const int64_t *t_int, uint64_t nblocks, uint32_t L, uint32_t l, float tp, float *tval,
                                   cudaStream_t st);
cudaError_t launch_pivot_compress(const PivotGeom &pg, const float *in, float *rec, int32_t *qb, int32_t *qb_range,
                                  cudaStream_t st);
cudaError_t launch_pivot_decompress(const PivotGeom &pg, const int32_t *qb, float *rec, cudaStream_t st);
// One round over every target; `ent` holds the per-axis AxisEntry tables (RoundGeom::ent_off).
// Requires tcount[0] * tcount[1] < 2^32 and tcount[2] < 2^32 (checked by the host).
// hist (optional, kHistWin zeroed 64-bit bins): the QB histogram of the round's stream over
// [-kHistHalf, kHistHalf), added to hist; a QB outside the window sets *hist_over.
constexpr uint32_t kHistWin = 8192, kHistHalf = kHistWin / 2;
cudaError_t launch_round_compress(const FieldGeom &fg, const RoundGeom &rg, const AxisEntry *ent, const float *tval,
                                  const float *in, float *rec, int32_t *qb, int32_t *qb_range, uint32_t *err, int div_all,
                                  float *pred_out, cudaStream_t st, unsigned long long *hist = nullptr,
                                  uint32_t *hist_over = nullptr);
cudaError_t launch_round_decompress(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const AxisEntry *ent,
                                    const int64_t *t_int, const int32_t *qb, float *rec, uint32_t *err, cudaStream_t st);

// Fused rounds for plans whose every round runs along axis 2 (k_lines.cu). rounds and qoff (the
// stream offsets, pivots first) are device copies of the plan's round table; line_bytes is the
// size of one column's lines (at most lines_smem_limit()), and the field has at most 64 blocks
// along axis 2.
// set selects the columns of a launch (kColumnsAll, or kColumnsInterior: b0 >= 1 and b1 >= 1, at most
// block_shape[0] * block_shape[1] lines each; kColumnsEdge: the rest); a resumption lists column
// indices of the same set.
enum : uint32_t { kColumnsAll = 0, kColumnsInterior = 1, kColumnsEdge = 2 };
uint32_t lines_smem_limit();
cudaError_t launch_lines_decompress(const FieldGeom &fg, const RoundGeom *rounds, const AxisEntry *ent, const uint64_t *qoff,
                                    const int64_t *t_int, const int32_t *qb, float *rec, uint32_t *err, uint32_t set,
                                    uint32_t line_bytes, cudaStream_t st);
// A full pass (resume_in == nullptr) or the resumption of the listed (column, round) pairs. Blocks
// handed to the exact path are listed per round in bail_blocks + round * nblocks (bail_count[round])
// and their columns in resume_out (resume_count).
cudaError_t launch_lines_compress(const FieldGeom &fg, const RoundGeom *rounds, const AxisEntry *ent, const uint64_t *qoff,
                                  const ClassInfo *classes, const float *orig, float *rec, const float *log2arena, float R2,
                                  float t_default, float *tval, int64_t *t_int, uint32_t *fb_count, int32_t *qb,
                                  int32_t *qb_range, const uint32_t *overrides, uint32_t n_overrides, uint32_t *why,
                                  const uint32_t *resume_in, uint32_t n_resume, uint32_t *bail_blocks, uint32_t *bail_count,
                                  uint32_t *resume_out, uint32_t *resume_count, uint32_t *err, uint32_t set,
                                  uint32_t line_bytes, cudaStream_t st);

cudaError_t launch_error_stats(const float *x, const float *y, uint64_t n, unsigned int *max_bits, double *sse,
                               cudaStream_t st);

uint64_t tsel_scratch_bytes(uint32_t cap, uint32_t bcap, uint32_t tcap);
cudaError_t launch_tsel_v0(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                           const float *orig, const float *log2arena, float R2, float t_default, uint8_t *scratch,
                           uint64_t scratch_stride, uint32_t cap, uint32_t bcap, uint32_t tcap, float *tval, int64_t *t_int,
                           uint32_t *fb_count, AmbiguousRecord *amb, uint32_t amb_cap, uint32_t *amb_count,
                           const uint32_t *overrides, uint32_t n_overrides, float *proxies, const uint32_t *list,
                           const uint32_t *list_count, uint64_t slots, uint32_t *err, cudaStream_t st);
cudaError_t launch_tsel_fast(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                             const float *orig, const float *log2arena, float R2, float t_default, float *tval,
                             int64_t *t_int, uint32_t *fb_count, uint32_t *list_out, uint32_t *list_count,
                             const uint32_t *overrides, uint32_t n_overrides, uint32_t *why, cudaStream_t st,
                             uint32_t common_samples);
uint32_t exact_smem_bytes(uint32_t cap);
cudaError_t launch_tsel_exact(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                              const float *orig, const float *log2arena, float R2, float t_default, float *tval,
                              int64_t *t_int, uint32_t *fb_count, AmbiguousRecord *amb, uint32_t amb_cap,
                              uint32_t *amb_count, const uint32_t *overrides, uint32_t n_overrides, float *proxies,
                              const uint32_t *list, const uint32_t *list_count, uint32_t *spill, uint32_t *spill_count,
                              uint32_t cap, unsigned grid, cudaStream_t st);
// The exact replay with each CTA's working set in a slice of `scratch` (stride bytes, at least
// exact_smem_bytes(cap)) instead of shared memory, for groups of up to cap samples.
cudaError_t launch_tsel_exact_global(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes,
                                     const float *rec, const float *orig, const float *log2arena, float R2, float t_default,
                                     float *tval, int64_t *t_int, uint32_t *fb_count, AmbiguousRecord *amb, uint32_t amb_cap,
                                     uint32_t *amb_count, const uint32_t *overrides, uint32_t n_overrides, float *proxies,
                                     const uint32_t *list, const uint32_t *list_count, uint32_t *spill, uint32_t *spill_count,
                                     uint8_t *scratch, uint64_t stride, uint32_t cap, unsigned grid, cudaStream_t st);
cudaError_t launch_slope_exact_global(const SampleBox *boxes, const ProxyEval *evals, uint32_t n_evals, const float *orig,
                                      uint64_t n1n2, uint64_t n2, const float *log2arena, float R2, float *h1, float *x,
                                      uint32_t *m_out, uint32_t *err, uint8_t *scratch, uint64_t stride, uint32_t cap,
                                      uint32_t nboxes, cudaStream_t st);
cudaError_t launch_copy_box(const float *in, const uint64_t n[3], const uint64_t lo[3], const uint64_t m[3], float *out,
                            cudaStream_t st);
// out[k] = in[idx[k]] for k < n.
cudaError_t launch_gather(const float *in, const uint64_t *idx, uint64_t n, float *out, cudaStream_t st);
cudaError_t launch_plan_sample(const float *d, uint64_t n1, uint64_t n2, const PlanCand *cands, uint32_t ncands, uint64_t total,
                               int32_t *qb, float *e, int32_t *qb_range, cudaStream_t st);
cudaError_t launch_plan_mse(const PlanCand *cands, uint32_t ncands, const float *e, float *mse, cudaStream_t st);
cudaError_t launch_slope_exact(const SampleBox *boxes, const ProxyEval *evals, uint32_t n_evals, const float *orig,
                               uint64_t n1n2, uint64_t n2, const float *log2arena, float R2, float *h1, float *x,
                               uint32_t *m_out, uint32_t *err, uint32_t cap, uint32_t nboxes, cudaStream_t st);
cudaError_t launch_slope_v0(const FieldGeom &fg, const SampleBox *boxes, const ProxyEval *evals, uint32_t n_evals,
                            const float *orig, const float *log2arena, float R2, uint8_t *scratch, uint64_t scratch_stride,
                            uint32_t cap, uint32_t bcap, uint32_t tcap, float *h1, float *x, uint32_t *m_out, uint32_t *err,
                            uint32_t nboxes, cudaStream_t st);

template <class T>
cudaError_t launch_histogram(const T *s, uint64_t n, int64_t offset, uint64_t range, unsigned long long *hist,
                             cudaStream_t st);
template <class T>
cudaError_t launch_encode(const T *s, uint64_t n, int64_t offset, const CodeEntry *tab, uint64_t *bitoff, void *tmp,
                          size_t &tmp_bytes, uint32_t *out, cudaStream_t st);
// Tiled encoding of several streams of one symbol type in one launch (k_huff.cu). toff: exclusive
// prefix of the streams' tile counts (ns + 1 entries, tiles of enc_tile<T>() symbols);
// tile_state needs ntiles + 1 entries and err one, both cleared here; each stream's out is zeroed
// beforehand. After the launch *err is nonzero if a tile's wait for the bit counts before it ran
// out (the payload is then not valid). With tmp == nullptr, only sets tmp_bytes (no temporary
// space is used).
constexpr uint32_t kEncThreads = 256;
template <class T>
ASZ_HD constexpr uint32_t enc_tile() { return sizeof(T) == 4 ? 4096u : 2048u; }
struct EncStream {
    const void *s;          // int32 or int64 symbols
    uint64_t n;
    int64_t offset;         // the symbol of code table entry 0
    const CodeEntry *tab;
    uint32_t *out;          // payload words
};
template <class T>
cudaError_t launch_encode_tiles(const EncStream *streams, uint32_t ns, const uint64_t *toff, uint64_t ntiles, uint64_t *tile_state,
                                uint64_t *err, void *tmp, size_t &tmp_bytes, cudaStream_t st);
cudaError_t launch_scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, void *tmp, size_t &tmp_bytes, cudaStream_t st);
cudaError_t launch_decode_sync(const uint8_t *base, uint64_t chunk_bits, const DecStream *streams, const uint32_t *tile_stream,
                               uint64_t ntiles, uint32_t max_lut_bits, const LutEntry *luts, const uint32_t *childs,
                               int first_pass, uint64_t *start, uint64_t *end, uint64_t *count, const uint32_t *moved,
                               uint32_t *err, cudaStream_t st);
cudaError_t launch_decode_restart(const DecStream *streams, uint32_t nstreams, uint64_t nchunks, const uint64_t *end,
                                  uint64_t *start, uint32_t *moved, uint32_t *changed, cudaStream_t st);
cudaError_t launch_decode_check(const DecStream *streams, uint32_t nstreams, const uint64_t *off, const uint64_t *end,
                                uint32_t *err, cudaStream_t st);
cudaError_t launch_decode_write(const uint8_t *base, uint64_t chunk_bits, const DecStream *streams, const uint32_t *tile_stream,
                                uint64_t ntiles, uint32_t max_lut_bits, const LutEntry *luts, const uint32_t *childs,
                                const uint64_t *start, const uint64_t *off, uint32_t *err, cudaStream_t st);
template <class T>
cudaError_t launch_fill(T *out, uint64_t n, T v, cudaStream_t st);

// Prediction sweep (k_sweep.cu; c_codes/s2_many_prediction.cpp:126-397). Targets are visited as
// lines: loop levels 0 and 1 (axes axis[0], axis[1]) select a line, level 2 (axis[2], the QB
// order) runs along it. Legacy targets: start + index * step per level, per_line = count[2].
// Common targets (common = 1): every level covers [5, n - 5) and only points with an odd
// coordinate sum count, so a line whose outer coordinates have an even sum holds inner_odd
// targets (the odd inner coordinates) and the others inner_even; per_line is the larger.
struct SweepGeom {
    uint64_t n[3];
    uint64_t dist[2];          // linear neighbour distances (dist[1]: second 2D4R axis)
    uint64_t start[3], step[3], count[3];
    uint64_t inner_odd, inner_even;
    uint64_t lines, per_line, targets;
    uint32_t axis[3];
    uint32_t kind;             // 0: 1D4R, 1: 2D4R, 2: 1D6R
    uint32_t common;
    uint32_t line_per_thread;  // the QB-order axis is not the contiguous one: a thread walks a line
};
// Target `it` of the (line, position) space: false when the position is past its line's count
// (common targets); else its coordinates i[] and its index j in the QB stream. Lines before line
// (a, b) of the common targets, split by the parity of a + b, give j.
ASZ_HD bool sweep_target(const SweepGeom &g, uint64_t it, uint64_t i[3], uint64_t &j) {
    const uint64_t line = it / g.per_line, k = it - line * g.per_line;
    const uint64_t a = line / g.count[1], b = line - a * g.count[1];
    i[g.axis[0]] = g.start[0] + a * g.step[0];
    i[g.axis[1]] = g.start[1] + b * g.step[1];
    if (!g.common) {
        i[g.axis[2]] = g.start[2] + k * g.step[2];
        j = it;
        return true;
    }
    // (a + 5) + (b + 5) has the parity of a + b; the inner coordinate makes the sum odd.
    const bool odd_line = (a + b) & 1;
    if (k >= (odd_line ? g.inner_even : g.inner_odd)) return false;
    i[g.axis[2]] = (odd_line ? 6 : 5) + 2 * k;
    const uint64_t L1 = g.count[1];
    const uint64_t q0 = (a + 1) / 2 * ((L1 + 1) / 2) + a / 2 * (L1 / 2) + ((a & 1) ? b / 2 : (b + 1) / 2);
    const uint64_t q1 = a * L1 + b - q0;
    j = q0 * g.inner_odd + q1 * g.inner_even + k;
    return true;
}
// One coefficient set: 1D4R lo = 0.25 - t, hi = 0.25 + t; 2D4R hi weighs the first axis, lo the
// second; 1D6R c0 = a, c1 = b, w = 0.5 - (a + b).
struct SweepCoef {
    double c0, c1, w, lo, hi;
};
cudaError_t launch_sweep_predict(const float *d, const SweepGeom &g, const SweepCoef *coef, uint32_t ncoef, double abs_eb,
                                 double neg_2_eb, int64_t *qb, uint64_t qb_stride, double *part, long long *mm,
                                 cudaStream_t st);
uint32_t sweep_predict_grid(const SweepGeom &g);
cudaError_t launch_sweep_sums(const double *part, uint32_t nparts, uint32_t ncoef, double *sums, cudaStream_t st);
cudaError_t launch_sweep_stats(const int64_t *s, uint64_t n, int64_t offset, uint64_t range, unsigned long long *hist,
                               unsigned long long *first, cudaStream_t st);

}  // namespace asz
