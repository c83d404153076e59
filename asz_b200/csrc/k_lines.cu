// Fused rounds for plans whose every round runs along axis 2 (e.g. "cubic2_012" on every level).
//
// With all rounds on one axis, the pivot stride is 1 on the other two axes, so a block owns whole
// lines along axis 2 and every stencil read of a round stays on the target's own line. The lines of
// a "column" (the blocks sharing one (block0, block1) pair) can therefore be held in shared memory
// by one CTA for all rounds: the field is read and written once instead of once per round.
// Results are those of the per-round kernels (same stencils, same arithmetic, same QB indices);
// rounds run in the same order, and a round's coefficient selection sees the column after the
// previous round, as the per-round kernels do.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "geometry.cuh"
#include "launch.h"
#include "round_ops.cuh"
#include "tsel_fast.cuh"

namespace asz {
namespace {

constexpr uint32_t kMaxColumnBlocks = 64;  // blocks along axis 2 (the host checks the plan)

__host__ __device__ inline uint32_t column_count(uint32_t set, uint32_t nb0, uint32_t nb1) {
    if (set == kColumnsInterior) return (nb0 - 1) * (nb1 - 1);
    if (set == kColumnsEdge) return nb0 + nb1 - 1;
    return nb0 * nb1;
}

// The lines of column (b0, b1): coordinates [lo, lo + nl) on axes 0 and 1. A block's upper face is
// its own and its lower face the block below's, except at 0, so the columns' lines partition the
// (axis 0, axis 1) plane.
struct Column {
    uint32_t lo0, lo1, nl0, nl1;
};

__device__ __forceinline__ Column column_of(const FieldGeom &fg, uint32_t b0, uint32_t b1) {
    const uint32_t s0 = (uint32_t)fg.block_shape[0], s1 = (uint32_t)fg.block_shape[1];
    Column col;
    col.lo0 = b0 ? b0 * s0 + 1 : 0;
    col.lo1 = b1 ? b1 * s1 + 1 : 0;
    const uint32_t hi0 = (uint32_t)min((uint64_t)b0 * s0 + s0 + 1, fg.n[0]);
    const uint32_t hi1 = (uint32_t)min((uint64_t)b1 * s1 + s1 + 1, fg.n[1]);
    col.nl0 = hi0 > col.lo0 ? hi0 - col.lo0 : 0;
    col.nl1 = hi1 > col.lo1 ? hi1 - col.lo1 : 0;
    return col;
}

// Column sets of one launch: every column, the columns with b0 >= 1 and b1 >= 1 (at most
// block_shape[0] * block_shape[1] lines each), or the others (b0 == 0 or b1 == 0, one line more on
// each such axis). Splitting them lets the larger set run with less shared memory per CTA.
__device__ __forceinline__ void column_at(uint32_t set, uint32_t it, uint32_t nb1, uint32_t &b0, uint32_t &b1) {
    if (set == kColumnsInterior) {
        b0 = 1 + it / (nb1 - 1);
        b1 = 1 + it % (nb1 - 1);
    } else if (set == kColumnsEdge) {
        b0 = it < nb1 ? 0 : it - nb1 + 1;
        b1 = it < nb1 ? it : 0;
    } else {
        b0 = it / nb1;
        b1 = it % nb1;
    }
}

// Warp per line, coalesced along axis 2.
__device__ __forceinline__ void load_lines(const FieldGeom &fg, const Column &col, const float *__restrict__ g, float *s) {
    const uint32_t n2 = (uint32_t)fg.n[2], nl = col.nl0 * col.nl1;
    for (uint32_t line = threadIdx.x >> 5; line < nl; line += blockDim.x >> 5) {
        const uint32_t i0 = col.lo0 + line / col.nl1, i1 = col.lo1 + line % col.nl1;
        const float *src = g + ((uint64_t)i0 * fg.n[1] + i1) * n2;
        for (uint32_t x = threadIdx.x & 31; x < n2; x += 32) s[line * n2 + x] = src[x];
    }
}

__device__ __forceinline__ void store_lines(const FieldGeom &fg, const Column &col, const float *s, float *__restrict__ g) {
    const uint32_t n2 = (uint32_t)fg.n[2], nl = col.nl0 * col.nl1;
    for (uint32_t line = threadIdx.x >> 5; line < nl; line += blockDim.x >> 5) {
        const uint32_t i0 = col.lo0 + line / col.nl1, i1 = col.lo1 + line % col.nl1;
        float *dst = g + ((uint64_t)i0 * fg.n[1] + i1) * n2;
        for (uint32_t x = threadIdx.x & 31; x < n2; x += 32) dst[x] = s[line * n2 + x];
    }
}

__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

// ---------------------------------------------------------------------------------------------
// Decompression: every round of every column, from the pivots (already in rec) to the final
// values. decompress.tpp:34: value = fma(-qb, 2eb, pred) in double, t = t_int / t_precision.
struct DecShared {
    float t[kMaxColumnBlocks];
};

__global__ void __launch_bounds__(256)
    lines_decompress_kernel(FieldGeom fg, const RoundGeom *__restrict__ rounds, const AxisEntry *__restrict__ ent,
                            const uint64_t *__restrict__ qoff, const int64_t *__restrict__ t_int, const int32_t *__restrict__ qb,
                            float *__restrict__ rec, uint32_t set, uint32_t items, uint32_t *err_word) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DecShared &ds = *reinterpret_cast<DecShared *>(smem_raw);
    float *sl = reinterpret_cast<float *>(smem_raw + align16(sizeof(DecShared)));
    const uint32_t nb1 = (uint32_t)fg.block_num[1], nb2 = (uint32_t)fg.block_num[2];
    const uint32_t n2 = (uint32_t)fg.n[2], L = fg.layer_num;
    const float tp = (float)fg.t_precision;
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
        uint32_t b0, b1;
        column_at(set, it, nb1, b0, b1);
        const uint32_t c = b0 * nb1 + b1;
        const Column col = column_of(fg, b0, b1);
        const uint32_t nl = col.nl0 * col.nl1;
        __syncthreads();
        load_lines(fg, col, rec, sl);
        for (uint32_t l = 0; l < L; l++) {
            const RoundGeom &rg = rounds[l];
            if (threadIdx.x < nb2)
                ds.t[threadIdx.x] =
                    __fdiv_rn(__ll2float_rn(t_int[((uint64_t)c * nb2 + threadIdx.x) * L + l]), tp);
            __syncthreads();
            const double eb2 = __dadd_rn((double)rg.eb, (double)rg.eb);
            const uint32_t T2 = (uint32_t)rg.tcount[2], hs = (uint32_t)rg.hs;
            const AxisEntry *e0t = ent + rg.ent_off[0], *e1t = ent + rg.ent_off[1], *e2t = ent + rg.ent_off[2];
            const int32_t *qbl = qb + qoff[l + 1];
            const uint32_t work = nl * T2;
            for (uint32_t w = threadIdx.x; w < work; w += blockDim.x) {
                const uint32_t line = w / T2, k = w - line * T2;
                const uint32_t r0 = line / col.nl1;
                const AxisEntry e0 = load_entry(e0t + col.lo0 + r0), e1 = load_entry(e1t + col.lo1 + (line - r0 * col.nl1));
                const AxisEntry e2 = load_entry(e2t + k);
                const uint64_t qi = qb_index(rg, e0, e1, e2);
                if (qi >= rg.qb_total || e2.bb >= kMaxColumnBlocks) {
                    atomicOr(err_word, 4u);
                    continue;
                }
                float *ln = sl + line * n2;
                const float t = e2.stencil == kStencilCubic ? ds.t[e2.bb] : 0.0f;
                const float pred = predict_case(ln, e2.ii, hs, e2.stencil, t);
                ln[e2.ii] = __double2float_rn(__fma_rn(-(double)qbl[qi], eb2, (double)pred));
            }
            __syncthreads();
        }
        store_lines(fg, col, sl, rec);
    }
}

// ---------------------------------------------------------------------------------------------
// Compression.

// Samples of a block read from its column's lines in shared memory (the original values from
// global memory). The positions are those of the per-round fast kernel along axis 2.
struct LineSrc {
    fastsel::FastSampleGeo sg;
    const float *lines;
    const float *orig;
    uint64_t n1;
    uint32_t n2, lo0, lo1, nl1, hs;
    float neg;
    __device__ __forceinline__ void keys(uint32_t s, float &af, float &bf, bool &nz) const {
        using namespace fastsel;
        const uint32_t k0 = div_small(s, sg.c12);
        const uint32_t r = s - k0 * sg.c12.d;
        const uint32_t k1 = div_small(r, sg.c2);
        const uint32_t k2 = r - k1 * sg.cnt2;
        const uint32_t i0 = (uint32_t)(sg.lo[0] + k0 * sg.step[0]), i1 = (uint32_t)(sg.lo[1] + k1 * sg.step[1]);
        const uint32_t x = (uint32_t)(sg.lo[2] + k2 * sg.step[2]);
        const float *ln = lines + ((i0 - lo0) * nl1 + (i1 - lo1)) * n2;
        keys_of(ln[x - hs], ln[x - 3 * hs], ln[x + hs], ln[x + 3 * hs], orig[((uint64_t)i0 * n1 + i1) * n2 + x], neg, af, bf,
                nz);
    }
};

struct CompShared {
    fastsel::GroupShared gs;
    float t[kMaxColumnBlocks];  // this round's t per block of the column
};

// Per column, from its first round (or its resume entry) to the last round: coefficient selection
// of each block (certified fast path, fastsel::fast_group) and the round's targets, all on the
// lines in shared memory. A block whose choice needs the exact path stops its column at that round:
// the lines go back to rec, the block is listed for the exact path (bail_blocks + round * nblocks,
// bail_count[round]) and the column for resumption (resume_out: column, round). A resumed column
// starts with the t of its first round already chosen (tval) for each of its blocks.
__global__ void __launch_bounds__(fastsel::kThreads, 6)
    lines_compress_kernel(FieldGeom fg, const RoundGeom *__restrict__ rounds, const AxisEntry *__restrict__ ent,
                          const uint64_t *__restrict__ qoff, const ClassInfo *__restrict__ classes,
                          const float *__restrict__ orig, float *__restrict__ rec, const float *__restrict__ log2arena,
                          float R2, float t_default, float *__restrict__ tval, int64_t *__restrict__ t_int,
                          uint32_t *__restrict__ fb_count, int32_t *__restrict__ qb, int32_t *__restrict__ qb_range,
                          const uint32_t *__restrict__ overrides, uint32_t n_overrides, uint32_t *__restrict__ why,
                          const uint32_t *__restrict__ resume_in, uint32_t n_resume, uint32_t *__restrict__ bail_blocks,
                          uint32_t *__restrict__ bail_count, uint32_t *__restrict__ resume_out,
                          uint32_t *__restrict__ resume_count, uint32_t set, uint32_t *err_word) {
    using namespace fastsel;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CompShared &cs = *reinterpret_cast<CompShared *>(smem_raw);
    float *sl = reinterpret_cast<float *>(smem_raw + align16(sizeof(CompShared)));
    const uint32_t tid = threadIdx.x;
    const uint32_t nb0 = (uint32_t)fg.block_num[0], nb1 = (uint32_t)fg.block_num[1], nb2 = (uint32_t)fg.block_num[2];
    const uint64_t nblocks = (uint64_t)nb0 * nb1 * nb2;
    const uint32_t n2 = (uint32_t)fg.n[2], L = fg.layer_num;
    const uint32_t items = resume_in ? n_resume : column_count(set, nb0, nb1);
    for (int i = tid; i < 5 * kWinWords; i += kThreads) (&cs.gs.hist[0][0])[i] = 0;
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
        uint32_t b0, b1;
        if (resume_in) column_at(kColumnsAll, resume_in[2 * it], nb1, b0, b1);  // entries hold column indices
        else column_at(set, it, nb1, b0, b1);
        const uint32_t c = b0 * nb1 + b1;
        const uint32_t start = resume_in ? resume_in[2 * it + 1] : 0;
        const Column col = column_of(fg, b0, b1);
        const uint32_t nl = col.nl0 * col.nl1;
        __syncthreads();
        load_lines(fg, col, rec, sl);
        __syncthreads();
        bool bailed = false;
        for (uint32_t l = start; l < L; l++) {
            const RoundGeom &rg = rounds[l];
            const ClassInfo *cls = classes + 27 * l;
            // ---- Coefficient selection for each block of the column (compress.tpp:91-144).
            for (uint32_t b2 = 0; b2 < nb2; b2++) {
                const uint64_t g = ((uint64_t)b0 * nb1 + b1) * nb2 + b2;
                float t = 0.0f;
                if (resume_in && l == start) {
                    t = tval[g];  // settled before this launch
                } else {
                    const int ccls = (class_of(b0, nb0) * 3 + class_of(b1, nb1)) * 3 + class_of(b2, nb2);
                    const ClassInfo ci = cls[ccls];
                    bool forced = false;
                    float forced_t = 0.0f;
                    for (uint32_t i = 0; i < n_overrides; i++)
                        if (overrides[3 * i] == (uint32_t)g && overrides[3 * i + 1] == l) {
                            forced = true;
                            forced_t = __uint_as_float(overrides[3 * i + 2]);
                        }
                    uint32_t code = kFastDecided;
                    if (ci.fallback || ci.n == 0 || forced) {
                        t = forced ? forced_t : t_default;
                        if (!forced && tid == 0) atomicAdd(fb_count, 1u);
                    } else if (ci.n > 0xffffu) {  // a bin count could overflow its 16-bit half word
                        code = kFastHandoff;
                        if (tid == 0) atomicAdd(&why[0], 1u);
                    } else {
                        const uint64_t bb[3] = {b0, b1, b2};
                        FastSampleGeo sg;
                        uint32_t cnt[3];
                        for (int a = 0; a < 3; a++) {
                            uint64_t lo = bb[a] * fg.block_shape[a];
                            uint64_t hi = min((bb[a] + 1) * fg.block_shape[a] + 1, fg.n[a]);
                            if (a != 2 && lo != 0) lo += rg.stride[a];
                            if (a == 2) {
                                lo += 3 * rg.stride[a] / 2;
                                hi -= 3 * rg.stride[a] / 2;
                            }
                            sg.lo[a] = lo;
                            sg.step[a] = rg.stride[a] * ci.ss;
                            cnt[a] = (uint32_t)((hi - lo + sg.step[a] - 1) / sg.step[a]);
                        }
                        sg.cnt2 = cnt[2];
                        sg.c2 = small_div(cnt[2]);
                        sg.c12 = small_div(cnt[1] * cnt[2]);
                        const LineSrc src{sg, sl, orig, fg.n[1], n2, col.lo0, col.lo1, col.nl1, (uint32_t)rg.hs,
                                          rg.neg_2_stat_eb};
                        code = fast_group(cs.gs, src, ci.n, rg, log2arena + ci.log2_off, R2, why, t);
                    }
                    if (code == kFastHandoff) {
                        if (tid == 0) bail_blocks[(uint64_t)l * nblocks + atomicAdd(&bail_count[l], 1u)] = (uint32_t)g;
                        bailed = true;
                    } else if (tid == 0) {
                        tval[g] = t;
                        t_int[g * L + l] = lround_f(__fmul_rn(t, (float)fg.t_precision));
                    }
                }
                if (tid == 0) cs.t[b2] = t;
            }
            __syncthreads();
            if (bailed) {
                // The rest of the column waits for the exact path: its state goes back to memory.
                store_lines(fg, col, sl, rec);
                if (tid == 0) {
                    const uint32_t k = atomicAdd(resume_count, 1u);
                    resume_out[2 * k] = c;
                    resume_out[2 * k + 1] = l;
                }
                break;
            }
            // ---- The round's targets (compress.tpp:35-37 as emitted along axis 2: divide).
            const double ebd = (double)rg.eb, eb2 = __dadd_rn(ebd, ebd), rinv = __ddiv_rn(1.0, ebd);
            const uint32_t T2 = (uint32_t)rg.tcount[2], hs = (uint32_t)rg.hs;
            const AxisEntry *e0t = ent + rg.ent_off[0], *e1t = ent + rg.ent_off[1], *e2t = ent + rg.ent_off[2];
            int32_t *qbl = qb + qoff[l + 1];
            int32_t lo = INT32_MAX, hi = INT32_MIN;
            const uint32_t work = nl * T2;
#pragma unroll 4
            for (uint32_t w = tid; w < work; w += blockDim.x) {
                const uint32_t line = w / T2, k = w - line * T2;
                const uint32_t r0 = line / col.nl1, i0 = col.lo0 + r0, i1 = col.lo1 + (line - r0 * col.nl1);
                const AxisEntry e0 = load_entry(e0t + i0), e1 = load_entry(e1t + i1), e2 = load_entry(e2t + k);
                const uint64_t qi = qb_index(rg, e0, e1, e2);
                if (qi >= rg.qb_total || e2.bb >= kMaxColumnBlocks) {
                    atomicOr(err_word, 4u);
                    continue;
                }
                float *ln = sl + line * n2;
                const float t = e2.stencil == kStencilCubic ? cs.t[e2.bb] : 0.0f;
                const float pred = predict_case(ln, e2.ii, hs, e2.stencil, t);
                const double pd = (double)pred;
                const double diff = __dsub_rn(pd, (double)orig[((uint64_t)i0 * fg.n[1] + i1) * n2 + e2.ii]);
                const int32_t v = (int32_t)lround_d(quot_for_lround(__dmul_rn(diff, 0.5), ebd, rinv));
                qbl[qi] = v;
                ln[e2.ii] = __double2float_rn(__fma_rn(-(double)v, eb2, pd));
                lo = min(lo, v);
                hi = max(hi, v);
            }
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if ((tid & 31) == 0 && lo <= hi) {
                atomicMin(&qb_range[2 * (l + 1)], lo);
                atomicMax(&qb_range[2 * (l + 1) + 1], hi);
            }
            __syncthreads();
        }
        if (!bailed) store_lines(fg, col, sl, rec);
    }
}

}  // namespace

uint32_t lines_smem_limit() { return 96 * 1024; }

cudaError_t launch_lines_decompress(const FieldGeom &fg, const RoundGeom *rounds, const AxisEntry *ent, const uint64_t *qoff,
                                    const int64_t *t_int, const int32_t *qb, float *rec, uint32_t *err, uint32_t set,
                                    uint32_t line_bytes, cudaStream_t st) {
    const uint32_t items = column_count(set, (uint32_t)fg.block_num[0], (uint32_t)fg.block_num[1]);
    if (items == 0) return cudaSuccess;
    if (fg.block_num[2] > kMaxColumnBlocks) return cudaErrorInvalidValue;
    const uint32_t smem = (uint32_t)(align16(sizeof(DecShared)) + line_bytes);
    cudaError_t e = cudaFuncSetAttribute(lines_decompress_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lines_decompress_kernel, 256, smem);
    if (e != cudaSuccess) return e;
    const uint64_t cap = 148ull * (per_sm > 0 ? per_sm : 1);
    lines_decompress_kernel<<<(unsigned)(items < cap ? items : cap), 256, smem, st>>>(fg, rounds, ent, qoff, t_int, qb, rec, set,
                                                                                      items, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_lines_compress(const FieldGeom &fg, const RoundGeom *rounds, const AxisEntry *ent, const uint64_t *qoff,
                                  const ClassInfo *classes, const float *orig, float *rec, const float *log2arena, float R2,
                                  float t_default, float *tval, int64_t *t_int, uint32_t *fb_count, int32_t *qb,
                                  int32_t *qb_range, const uint32_t *overrides, uint32_t n_overrides, uint32_t *why,
                                  const uint32_t *resume_in, uint32_t n_resume, uint32_t *bail_blocks, uint32_t *bail_count,
                                  uint32_t *resume_out, uint32_t *resume_count, uint32_t *err, uint32_t set,
                                  uint32_t line_bytes, cudaStream_t st) {
    const uint32_t items =
        resume_in ? n_resume : column_count(set, (uint32_t)fg.block_num[0], (uint32_t)fg.block_num[1]);
    if (items == 0) return cudaSuccess;
    if (fg.block_num[2] > kMaxColumnBlocks) return cudaErrorInvalidValue;
    const uint32_t smem = (uint32_t)(align16(sizeof(CompShared)) + line_bytes);
    cudaError_t e = cudaFuncSetAttribute(lines_compress_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lines_compress_kernel, fastsel::kThreads, smem);
    if (e != cudaSuccess) return e;
    const uint64_t cap = 148ull * (per_sm > 0 ? per_sm : 1);
    lines_compress_kernel<<<(unsigned)(items < cap ? items : cap), fastsel::kThreads, smem, st>>>(
        fg, rounds, ent, qoff, classes, orig, rec, log2arena, R2, t_default, tval, t_int, fb_count, qb, qb_range, overrides,
        n_overrides, why, resume_in, n_resume, bail_blocks, bail_count, resume_out, resume_count, set, err);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz
