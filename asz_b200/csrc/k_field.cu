// Field-wide kernels: data range, pivot lattice, and the per-round prediction/quantisation.
//
// One launch per round covers every target of the round in every block (round-major). The
// reference walks block-major (compress.tpp:179-209), but the two orders give the same result.
// Every target is written once, by the block that owns it: lower faces on the non-prediction
// axes belong to the lower block (compress.tpp:59). Every stencil read hits a point finished in
// an earlier round or a pivot.
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "geometry.cuh"
#include "launch.h"
#include "round_ops.cuh"

namespace asz {

// ---------------------------------------------------------------------------------------------
// Data range (c_codes/s1_compress.cpp:128-138). std::minmax_element returns the first minimum and
// the last maximum, which matters only for the sign of a zero extremum; the host resolves that
// case with zero_first_last_kernel.

__device__ __forceinline__ int32_t ord_key(float v) {
    int32_t b = __float_as_int(v == 0.0f ? 0.0f : v);
    return b >= 0 ? b : (int32_t)(0x80000000u - (uint32_t)b) - 1;
}

// out[0] = min key, out[1] = max key (ordered-int encoding), out[2] = count of non-finite values.
__global__ void range_kernel(const float4 *__restrict__ x4, uint64_t n4, const float *__restrict__ tail, uint64_t ntail,
                             int32_t *out, unsigned long long *nonfinite) {
    int32_t mn = INT32_MAX, mx = INT32_MIN;
    unsigned long long bad = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    auto take = [&](float4 v) {
        const float a[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!isfinite(a[k])) {
                bad++;
                continue;
            }
            const int32_t o = ord_key(a[k]);
            mn = min(mn, o);
            mx = max(mx, o);
        }
    };
    // Four 16-byte loads per thread in flight per step, then the remainder one at a time.
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n4; i += 4 * stride) {
        const float4 v0 = __ldg(x4 + i), v1 = __ldg(x4 + i + stride), v2 = __ldg(x4 + i + 2 * stride),
                     v3 = __ldg(x4 + i + 3 * stride);
        take(v0);
        take(v1);
        take(v2);
        take(v3);
    }
    for (; i < n4; i += stride) take(__ldg(x4 + i));
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ntail; i += stride) {
        float v = tail[i];
        if (!isfinite(v)) bad++;
        else {
            mn = min(mn, ord_key(v));
            mx = max(mx, ord_key(v));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&out[0], mn);
        atomicMax(&out[1], mx);
        if (bad) atomicAdd(nonfinite, bad);
    }
}

// First and last index of a zero (either sign), for the sign of a zero minimum or maximum.
__global__ void zero_first_last_kernel(const float *__restrict__ x, uint64_t n, unsigned long long *first,
                                       unsigned long long *last) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
        if (x[i] == 0.0f) {
            atomicMin(first, (unsigned long long)i);
            atomicMax(last, (unsigned long long)i);
        }
}

// ---------------------------------------------------------------------------------------------
// Pivots (compress.tpp:162-175, decompress.tpp:160-171). Stream 0 is the pivot lattice in raster
// order. Compress: qb = llround(x * (0.5/pivot_eb)) (hoisted reciprocal, double), value
// qb*(2*pivot_eb) in double rounded to float.

__global__ void pivot_compress_kernel(PivotGeom pg, const float *__restrict__ in, float *__restrict__ rec,
                                      int32_t *__restrict__ qb, int32_t *qb_range) {
    const uint64_t total = pg.cnt[0] * pg.cnt[1] * pg.cnt[2];
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k2 = k % pg.cnt[2], k1 = (k / pg.cnt[2]) % pg.cnt[1], k0 = k / (pg.cnt[1] * pg.cnt[2]);
        uint64_t pos = (pg.origin[0] + k0 * pg.stride[0]) * pg.n1n2 + (pg.origin[1] + k1 * pg.stride[1]) * pg.n2 +
                       pg.origin[2] + k2 * pg.stride[2];
        int32_t q = (int32_t)lround_d(__dmul_rn((double)in[pos], pg.rp));
        qb[k] = q;
        rec[pos] = __double2float_rn(__dmul_rn((double)q, pg.peb2));
        lo = min(lo, q);
        hi = max(hi, q);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&qb_range[0], lo);
        atomicMax(&qb_range[1], hi);
    }
}

// Batched form: the pivots of every field of a batch, one item per pivot; a field's parameters
// come from its record, so a captured launch serves any data of the same shapes.
__global__ void pivot_compress_batch_kernel(const BatchField *__restrict__ F, const uint64_t *__restrict__ poff, uint32_t nf) {
    const uint64_t total = poff[nf];
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < total; gi += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f = field_of(poff, nf, gi);
        const BatchField &B = F[f];
        const PivotGeom &pg = B.pg;
        const uint64_t k = gi - poff[f];
        const uint64_t k2 = k % pg.cnt[2], k1 = (k / pg.cnt[2]) % pg.cnt[1], k0 = k / (pg.cnt[1] * pg.cnt[2]);
        const uint64_t pos = (pg.origin[0] + k0 * pg.stride[0]) * pg.n1n2 + (pg.origin[1] + k1 * pg.stride[1]) * pg.n2 +
                             pg.origin[2] + k2 * pg.stride[2];
        const int32_t q = (int32_t)lround_d(__dmul_rn((double)B.in[pos], pg.rp));
        B.qb[k] = q;
        B.rec[pos] = __double2float_rn(__dmul_rn((double)q, pg.peb2));
        // Range of stream 0: one atomic pair per warp when the warp's items share a field.
        const uint32_t act = __activemask();
        const uint32_t f0 = __shfl_sync(act, f, __ffs(act) - 1);
        if (__all_sync(act, f == f0)) {
            int32_t lo = q, hi = q;
            for (int o = 16; o > 0; o >>= 1) {
                const int32_t l2 = __shfl_xor_sync(act, lo, o), h2 = __shfl_xor_sync(act, hi, o);
                if ((act >> ((threadIdx.x ^ o) & 31)) & 1) {
                    lo = min(lo, l2);
                    hi = max(hi, h2);
                }
            }
            if ((threadIdx.x & 31) == (uint32_t)(__ffs(act) - 1)) {
                atomicMin(&B.qb_range[0], lo);
                atomicMax(&B.qb_range[1], hi);
            }
        } else {
            atomicMin(&B.qb_range[0], q);
            atomicMax(&B.qb_range[1], q);
        }
    }
}

__global__ void pivot_decompress_kernel(PivotGeom pg, const int32_t *__restrict__ qb, float *__restrict__ rec) {
    const uint64_t total = pg.cnt[0] * pg.cnt[1] * pg.cnt[2];
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k2 = k % pg.cnt[2], k1 = (k / pg.cnt[2]) % pg.cnt[1], k0 = k / (pg.cnt[1] * pg.cnt[2]);
        uint64_t pos = (pg.origin[0] + k0 * pg.stride[0]) * pg.n1n2 + (pg.origin[1] + k1 * pg.stride[1]) * pg.n2 +
                       pg.origin[2] + k2 * pg.stride[2];
        rec[pos] = __double2float_rn(__dmul_rn((double)qb[k], pg.peb2));
    }
}

// Thread layout of the round kernels: the targets form lines along axis 2 (tcount[2] long, one
// per (k0, k1)); a line is covered by tpl = 2^tpl_log2 threads and a CTA holds blockDim/tpl lines.
// All per-target geometry comes from the per-axis tables, so no division is done per target.
struct LineMap {
    uint32_t sub, row, lines_per_cta;
};

__device__ __forceinline__ LineMap line_map(uint32_t tpl_log2) {
    LineMap m;
    m.sub = threadIdx.x & ((1u << tpl_log2) - 1);
    m.row = threadIdx.x >> tpl_log2;
    m.lines_per_cta = blockDim.x >> tpl_log2;
    return m;
}

// Compress round: quantise the residual and write the reconstruction in place.
// compress.tpp:35-37 as emitted: axis 0 multiplies by the hoisted 0.5*(1/eb) (inlined loop),
// axes 1 and 2 divide (diff*0.5)/eb (out-of-line clone); value = fma(-qb, 2eb, pred) in double.
// kProbe: every axis divides, as the diagnostics instantiation that the predictor-family probe runs
// does (one out-of-line clone for all axes), and pred_out receives each target's prediction.
// Targets of line `line` (k0, k1) handled by the sub-th of the line's 2^tpl_log2 threads.
template <bool kProbe>
__device__ __forceinline__ void compress_line(const FieldGeom &fg, const RoundGeom &rg, const AxisEntry *__restrict__ ent,
                                              uint32_t tpl_log2, uint32_t sub, uint32_t line, const float *__restrict__ tval,
                                              const float *__restrict__ in, float *__restrict__ rec, int32_t *__restrict__ qb,
                                              uint32_t *err_word, float *__restrict__ pred_out, double ebd, double eb2,
                                              double rinv, double r0, int32_t &lo, int32_t &hi) {
    const AxisEntry *e0t = ent + rg.ent_off[0], *e1t = ent + rg.ent_off[1], *e2t = ent + rg.ent_off[2];
    const uint32_t T1 = (uint32_t)rg.tcount[1], T2 = (uint32_t)rg.tcount[2];
    const uint64_t n1n2 = fg.n[1] * fg.n[2], n2 = fg.n[2];
    const uint32_t nb1 = (uint32_t)fg.block_num[1], nb2 = (uint32_t)fg.block_num[2];
    const int dir = rg.dir;
    const uint32_t k0 = line / T1, k1 = line - k0 * T1;
    const AxisEntry e0 = load_entry(e0t + k0), e1 = load_entry(e1t + k1);
    const uint64_t line_pos = (uint64_t)e0.ii * n1n2 + (uint64_t)e1.ii * n2;
    const uint32_t line_blk = e0.bb * nb1 + e1.bb;
    const LineQB lq = line_qb(rg, e0, e1);
    for (uint32_t k2 = sub; k2 < T2; k2 += 1u << tpl_log2) {
        const AxisEntry e2 = load_entry(e2t + k2);
        const uint64_t pos = line_pos + e2.ii;
        const uint64_t qi = target_qb(rg, lq, e0, e1, e2);
        if (qi >= rg.qb_total) {
            atomicOr(err_word, 4u);
            continue;
        }
        const uint32_t sc = dir == 0 ? e0.stencil : dir == 1 ? e1.stencil : e2.stencil;
        const float t = sc == kStencilCubic ? tval[(uint64_t)line_blk * nb2 + e2.bb] : 0.0f;
        const float pred = predict_case(rec, pos, rg.dist, sc, t);
        const double pd = (double)pred;
        const double diff = __dsub_rn(pd, (double)in[pos]);
        const double q = dir == 0 && !kProbe ? __dmul_rn(diff, r0) : quot_for_lround(__dmul_rn(diff, 0.5), ebd, rinv);
        if (kProbe) pred_out[pos] = pred;
        const int32_t v = (int32_t)lround_d(q);
        qb[qi] = v;
        rec[pos] = __double2float_rn(__fma_rn(-(double)v, eb2, pd));
        lo = min(lo, v);
        hi = max(hi, v);
    }
}

// Two lines at once (lineB == UINT32_MAX: none). Both lines share the k2 sequence; each step loads
// both targets' inputs before it computes and stores either, so the loads overlap.
template <bool kProbe>
__device__ __forceinline__ void compress_lines2(const FieldGeom &fg, const RoundGeom &rg, const AxisEntry *__restrict__ ent,
                                                uint32_t tpl_log2, uint32_t sub, uint32_t lineA, uint32_t lineB,
                                                const float *__restrict__ tval, const float *__restrict__ in,
                                                float *__restrict__ rec, int32_t *__restrict__ qb, uint32_t *err_word,
                                                float *__restrict__ pred_out, double ebd, double eb2, double rinv, double r0,
                                                int32_t &lo, int32_t &hi, uint32_t *hsh, bool &hover) {
    const AxisEntry *e0t = ent + rg.ent_off[0], *e1t = ent + rg.ent_off[1], *e2t = ent + rg.ent_off[2];
    const uint32_t T1 = (uint32_t)rg.tcount[1], T2 = (uint32_t)rg.tcount[2];
    const uint64_t n1n2 = fg.n[1] * fg.n[2], n2 = fg.n[2];
    const uint32_t nb1 = (uint32_t)fg.block_num[1], nb2 = (uint32_t)fg.block_num[2];
    const int dir = rg.dir;
    const bool hasB = lineB != UINT32_MAX;
    // The stream's histogram window in shared memory (hsh == nullptr: not counted here).
    auto count = [&](int32_t v) {
        if (!hsh) return;
        const uint32_t b = (uint32_t)(v + kHistHalf);
        if (b < kHistWin) atomicAdd(&hsh[b], 1u);
        else hover = true;
    };
    const uint32_t a0 = lineA / T1, b0 = hasB ? lineB / T1 : a0;
    const AxisEntry e0A = load_entry(e0t + a0), e1A = load_entry(e1t + (lineA - a0 * T1));
    const AxisEntry e0B = load_entry(e0t + b0), e1B = load_entry(e1t + (hasB ? lineB - b0 * T1 : lineA - a0 * T1));
    const uint64_t posA0 = (uint64_t)e0A.ii * n1n2 + (uint64_t)e1A.ii * n2, posB0 = (uint64_t)e0B.ii * n1n2 + (uint64_t)e1B.ii * n2;
    const uint32_t blkA = e0A.bb * nb1 + e1A.bb, blkB = e0B.bb * nb1 + e1B.bb;
    const LineQB lqA = line_qb(rg, e0A, e1A), lqB = line_qb(rg, e0B, e1B);
    for (uint32_t k2 = sub; k2 < T2; k2 += 1u << tpl_log2) {
        const AxisEntry e2 = load_entry(e2t + k2);
        const uint64_t posA = posA0 + e2.ii, posB = posB0 + e2.ii;
        const uint64_t qiA = target_qb(rg, lqA, e0A, e1A, e2), qiB = target_qb(rg, lqB, e0B, e1B, e2);
        const uint32_t scA = dir == 0 ? e0A.stencil : dir == 1 ? e1A.stencil : e2.stencil;
        const uint32_t scB = dir == 0 ? e0B.stencil : dir == 1 ? e1B.stencil : e2.stencil;
        const bool okA = qiA < rg.qb_total, okB = hasB && qiB < rg.qb_total;
        if (!okA || (hasB && !okB)) atomicOr(err_word, 4u);
        StencilIn vA{}, vB{};
        float xA = 0.0f, xB = 0.0f, tA = 0.0f, tB = 0.0f;
        if (okA) {
            vA = load_stencil(rec, posA, rg.dist, scA);
            xA = __ldg(in + posA);
            if (scA == kStencilCubic) tA = __ldg(tval + (uint64_t)blkA * nb2 + e2.bb);
        }
        if (okB) {
            vB = load_stencil(rec, posB, rg.dist, scB);
            xB = __ldg(in + posB);
            if (scB == kStencilCubic) tB = __ldg(tval + (uint64_t)blkB * nb2 + e2.bb);
        }
        if (okA) {
            const float pred = predict_loaded(vA, scA, tA);
            const double pd = (double)pred;
            const double diff = __dsub_rn(pd, (double)xA);
            const double q = dir == 0 && !kProbe ? __dmul_rn(diff, r0) : quot_for_lround(__dmul_rn(diff, 0.5), ebd, rinv);
            if (kProbe) pred_out[posA] = pred;
            const int32_t v = (int32_t)lround_d(q);
            qb[qiA] = v;
            rec[posA] = __double2float_rn(__fma_rn(-(double)v, eb2, pd));
            lo = min(lo, v);
            hi = max(hi, v);
            count(v);
        }
        if (okB) {
            const float pred = predict_loaded(vB, scB, tB);
            const double pd = (double)pred;
            const double diff = __dsub_rn(pd, (double)xB);
            const double q = dir == 0 && !kProbe ? __dmul_rn(diff, r0) : quot_for_lround(__dmul_rn(diff, 0.5), ebd, rinv);
            if (kProbe) pred_out[posB] = pred;
            const int32_t v = (int32_t)lround_d(q);
            qb[qiB] = v;
            rec[posB] = __double2float_rn(__fma_rn(-(double)v, eb2, pd));
            lo = min(lo, v);
            hi = max(hi, v);
            count(v);
        }
    }
}

__device__ __forceinline__ void reduce_range(int32_t lo, int32_t hi, int32_t *qb_range) {
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0 && lo <= hi) {
        atomicMin(&qb_range[0], lo);
        atomicMax(&qb_range[1], hi);
    }
}

// Compress round: quantise the residual and write the reconstruction in place.
// compress.tpp:35-37 as emitted: axis 0 multiplies by the hoisted 0.5*(1/eb) (inlined loop),
// axes 1 and 2 divide (diff*0.5)/eb (out-of-line clone); value = fma(-qb, 2eb, pred) in double.
// kProbe: every axis divides, as the diagnostics instantiation that the predictor-family probe runs
// does (one out-of-line clone for all axes), and pred_out receives each target's prediction.
//
// hist (optional) receives the QB histogram of the round's stream over the window
// [-kHistHalf, kHistHalf): each CTA counts in shared memory and adds its nonzero bins at the end;
// a QB outside the window sets *hist_over, and the caller then counts that stream separately.
template <bool kProbe>
__global__ void __launch_bounds__(256, 3)
    round_compress_kernel(FieldGeom fg, RoundGeom rg, const AxisEntry *__restrict__ ent, uint32_t tpl_log2,
                          const float *__restrict__ tval, const float *__restrict__ in, float *__restrict__ rec,
                          int32_t *__restrict__ qb, int32_t *qb_range, uint32_t *err_word, float *__restrict__ pred_out,
                          unsigned long long *__restrict__ hist, uint32_t *hist_over) {
    extern __shared__ uint32_t hsh_raw[];
    uint32_t *hsh = hist ? hsh_raw : nullptr;
    if (hsh) {
        for (uint32_t i = threadIdx.x; i < kHistWin; i += blockDim.x) hsh[i] = 0;
        __syncthreads();
    }
    const double ebd = (double)rg.eb, eb2 = __dadd_rn(ebd, ebd), rinv = __ddiv_rn(1.0, ebd), r0 = __dmul_rn(rinv, 0.5);
    const uint32_t lines = (uint32_t)rg.tcount[0] * (uint32_t)rg.tcount[1];
    const LineMap m = line_map(tpl_log2);
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    bool hover = false;
    const uint32_t step = gridDim.x * m.lines_per_cta;
    for (uint32_t line = blockIdx.x * m.lines_per_cta + m.row; line < lines; line += 2 * step) {
        const uint32_t lineB = line + step < lines ? line + step : UINT32_MAX;
        compress_lines2<kProbe>(fg, rg, ent, tpl_log2, m.sub, line, lineB, tval, in, rec, qb, err_word, pred_out, ebd, eb2, rinv,
                                r0, lo, hi, hsh, hover);
    }
    reduce_range(lo, hi, qb_range);
    if (hsh) {
        if (hover) atomicOr(hist_over, 1u);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kHistWin; i += blockDim.x)
            if (hsh[i]) atomicAdd(&hist[i], (unsigned long long)hsh[i]);
    }
}

// The finest round along axis 2 (dir == 2, hs == 1): a warp per target line. The warp copies the
// whole line of the reconstruction and of the input (n2 floats each) into shared memory with
// 16-byte loads, then predicts its targets from there. The targets (odd points) and their stencil
// points (even points) cover the line, so the copy fetches no DRAM sector that per-target loads
// would not, with a quarter as many load instructions and no scattered ones. At hs >= 2 the
// per-target kernel measured as fast or faster (a line then holds fewer targets per staged byte),
// and so did a two-stage form with asynchronous copies and a form with two targets per lane step.
// Results are those of round_compress_kernel<false>: same entries, stencils, arithmetic and QB
// indices. A line's own targets are written to global memory only; the staged copy is read-only,
// and no target of the round reads a position that the round writes.
__device__ __forceinline__ void stencil_reach(uint32_t sc, uint32_t &neg, uint32_t &pos) {
    // Multiples of hs that the case reads below and above the target (predict_case).
    switch (sc) {
    case kStencilQuintic: neg = 5; pos = 5; break;
    case kStencilLeft1: neg = 1; pos = 0; break;
    case kStencilLeft2: neg = 1; pos = 1; break;
    case kStencilLeft3: neg = 1; pos = 3; break;
    case kStencilRight1: neg = 3; pos = 0; break;
    case kStencilRight2: neg = 3; pos = 1; break;
    default: neg = 3; pos = 3; break;
    }
}

__global__ void __launch_bounds__(256, 3)
    round_compress_line_kernel(FieldGeom fg, RoundGeom rg, const AxisEntry *__restrict__ ent, const float *__restrict__ tval,
                               const float *__restrict__ in, float *__restrict__ rec, int32_t *__restrict__ qb,
                               int32_t *qb_range, uint32_t *err_word, unsigned long long *__restrict__ hist,
                               uint32_t *hist_over) {
    extern __shared__ __align__(16) float line_smem[];
    const uint32_t n2 = (uint32_t)fg.n[2], n4 = n2 / 4;
    const uint32_t warps = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *hsh = hist ? reinterpret_cast<uint32_t *>(line_smem + (size_t)warps * 2 * n2) : nullptr;
    float *s_rec = line_smem + (size_t)warp * 2 * n2, *s_in = s_rec + n2;
    if (hsh) {
        for (uint32_t i = threadIdx.x; i < kHistWin; i += blockDim.x) hsh[i] = 0;
        __syncthreads();
    }
    bool hover = false;
    // Axis 2 divides (diff*0.5)/eb, as round_compress_kernel does off axis 0.
    const double ebd = (double)rg.eb, eb2 = __dadd_rn(ebd, ebd), rinv = __ddiv_rn(1.0, ebd);
    const AxisEntry *e0t = ent + rg.ent_off[0], *e1t = ent + rg.ent_off[1], *e2t = ent + rg.ent_off[2];
    const uint32_t T1 = (uint32_t)rg.tcount[1], T2 = (uint32_t)rg.tcount[2];
    const uint32_t lines = (uint32_t)rg.tcount[0] * T1;
    const uint64_t n1n2 = fg.n[1] * fg.n[2];
    const uint32_t nb1 = (uint32_t)fg.block_num[1], nb2 = (uint32_t)fg.block_num[2];
    const uint32_t hs = (uint32_t)rg.hs;
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    for (uint32_t line = blockIdx.x * warps + warp; line < lines; line += gridDim.x * warps) {
        const uint32_t k0 = line / T1, k1 = line - k0 * T1;
        const AxisEntry e0 = load_entry(e0t + k0), e1 = load_entry(e1t + k1);
        const uint64_t line_pos = (uint64_t)e0.ii * n1n2 + (uint64_t)e1.ii * n2;
        const uint32_t blk = e0.bb * nb1 + e1.bb;
        const LineQB lq = line_qb(rg, e0, e1);
        // Stage the line: four 16-byte loads per lane in flight before their stores.
        const float4 *g_rec4 = reinterpret_cast<const float4 *>(rec + line_pos);
        const float4 *g_in4 = reinterpret_cast<const float4 *>(in + line_pos);
        float4 *s_rec4 = reinterpret_cast<float4 *>(s_rec), *s_in4 = reinterpret_cast<float4 *>(s_in);
        for (uint32_t b = lane; b < n4; b += 64) {
            float4 a[2], c[2];
#pragma unroll
            for (uint32_t j = 0; j < 2; j++)
                if (b + 32 * j < n4) {
                    a[j] = g_rec4[b + 32 * j];
                    c[j] = __ldg(g_in4 + b + 32 * j);
                }
#pragma unroll
            for (uint32_t j = 0; j < 2; j++)
                if (b + 32 * j < n4) {
                    s_rec4[b + 32 * j] = a[j];
                    s_in4[b + 32 * j] = c[j];
                }
        }
        __syncwarp();
        for (uint32_t k2 = lane; k2 < T2; k2 += 32) {
            const AxisEntry e2 = load_entry(e2t + k2);
            const uint64_t qi = target_qb(rg, lq, e0, e1, e2);
            const uint32_t sc = e2.stencil, ii = e2.ii;
            uint32_t rn, rp;
            stencil_reach(sc, rn, rp);
            if (qi >= rg.qb_total || ii < rn * hs || ii + rp * hs >= n2) {
                atomicOr(err_word, 4u);
                continue;
            }
            const float t = sc == kStencilCubic ? __ldg(tval + (uint64_t)blk * nb2 + e2.bb) : 0.0f;
            const float pred = predict_case(s_rec, ii, hs, sc, t);
            const double pd = (double)pred;
            const double diff = __dsub_rn(pd, (double)s_in[ii]);
            const double q = quot_for_lround(__dmul_rn(diff, 0.5), ebd, rinv);
            const int32_t v = (int32_t)lround_d(q);
            qb[qi] = v;
            rec[line_pos + ii] = __double2float_rn(__fma_rn(-(double)v, eb2, pd));
            lo = min(lo, v);
            hi = max(hi, v);
            if (hsh) {
                const uint32_t bin = (uint32_t)(v + kHistHalf);
                if (bin < kHistWin) atomicAdd(&hsh[bin], 1u);
                else hover = true;
            }
        }
        __syncwarp();
    }
    reduce_range(lo, hi, qb_range);
    if (hsh) {
        if (hover) atomicOr(hist_over, 1u);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kHistWin; i += blockDim.x)
            if (hsh[i]) atomicAdd(&hist[i], (unsigned long long)hsh[i]);
    }
}

// Batched form: one work queue over the (field, item) pairs of a round, an item being
// kBatchChunks CTA-sized chunks of one field's target lines (256 >> tpl_log2 lines each).
constexpr uint32_t kBatchChunks = 8;

__global__ void __launch_bounds__(256, 5)
    round_compress_batch_kernel(const BatchField *__restrict__ F, const uint64_t *__restrict__ ioff, uint32_t nf, uint32_t l,
                                uint32_t *queue) {
    __shared__ uint64_t item;
    const uint64_t total = ioff[nf];
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(queue, 1u);
        __syncthreads();
        const uint64_t it = item;
        __syncthreads();
        if (it >= total) break;
        const uint32_t f = field_of(ioff, nf, it);
        const BatchField &B = F[f];
        const RoundGeom &rg = B.rounds[l];
        const uint32_t tpl = B.tpl_log2[l];
        const LineMap m = line_map(tpl);
        const double ebd = (double)rg.eb, eb2 = __dadd_rn(ebd, ebd), rinv = __ddiv_rn(1.0, ebd), r0 = __dmul_rn(rinv, 0.5);
        const uint32_t lines = (uint32_t)rg.tcount[0] * (uint32_t)rg.tcount[1];
        const uint64_t c0 = (it - ioff[f]) * kBatchChunks;
        int32_t lo = INT32_MAX, hi = INT32_MIN;
        for (uint32_t c = 0; c < kBatchChunks; c++) {
            const uint64_t line = (c0 + c) * m.lines_per_cta + m.row;
            if (line < lines)
                compress_line<false>(B.fg, rg, B.ent, tpl, m.sub, (uint32_t)line, B.tval, B.in, B.rec, B.qb + B.qoff[l + 1],
                                     &B.cnt->err, nullptr, ebd, eb2, rinv, r0, lo, hi);
        }
        reduce_range(lo, hi, B.qb_range + 2 * (l + 1));
    }
}

// Decompress round (decompress.tpp:34): value = fma(-qb, 2eb, pred) in double, t = t_int/t_precision.
// Two lines per step (lineB == UINT32_MAX: none): both targets' QB, t and stencil inputs are
// loaded before either is computed and stored. Within a round no target reads a position that the
// round writes, so the loads may run ahead of the stores.
__device__ __forceinline__ void decompress_lines2(const FieldGeom &fg, const RoundGeom &rg, uint32_t l,
                                                  const AxisEntry *__restrict__ ent, uint32_t tpl_log2, uint32_t sub,
                                                  uint32_t lineA, uint32_t lineB, const int64_t *__restrict__ t_int,
                                                  const int32_t *__restrict__ qb, float *__restrict__ rec, uint32_t *err_word,
                                                  double eb2, float tp) {
    const AxisEntry *e0t = ent + rg.ent_off[0], *e1t = ent + rg.ent_off[1], *e2t = ent + rg.ent_off[2];
    const uint32_t T1 = (uint32_t)rg.tcount[1], T2 = (uint32_t)rg.tcount[2];
    const uint64_t n1n2 = fg.n[1] * fg.n[2], n2 = fg.n[2];
    const uint32_t nb1 = (uint32_t)fg.block_num[1], nb2 = (uint32_t)fg.block_num[2];
    const int dir = rg.dir;
    const bool hasB = lineB != UINT32_MAX;
    const uint32_t a0 = lineA / T1, b0 = hasB ? lineB / T1 : a0;
    const AxisEntry e0A = load_entry(e0t + a0), e1A = load_entry(e1t + (lineA - a0 * T1));
    const AxisEntry e0B = load_entry(e0t + b0), e1B = load_entry(e1t + (hasB ? lineB - b0 * T1 : lineA - a0 * T1));
    const uint64_t posA0 = (uint64_t)e0A.ii * n1n2 + (uint64_t)e1A.ii * n2, posB0 = (uint64_t)e0B.ii * n1n2 + (uint64_t)e1B.ii * n2;
    const uint32_t blkA = e0A.bb * nb1 + e1A.bb, blkB = e0B.bb * nb1 + e1B.bb;
    const LineQB lqA = line_qb(rg, e0A, e1A), lqB = line_qb(rg, e0B, e1B);
    for (uint32_t k2 = sub; k2 < T2; k2 += 1u << tpl_log2) {
        const AxisEntry e2 = load_entry(e2t + k2);
        const uint64_t posA = posA0 + e2.ii, posB = posB0 + e2.ii;
        const uint64_t qiA = target_qb(rg, lqA, e0A, e1A, e2), qiB = target_qb(rg, lqB, e0B, e1B, e2);
        const uint32_t scA = dir == 0 ? e0A.stencil : dir == 1 ? e1A.stencil : e2.stencil;
        const uint32_t scB = dir == 0 ? e0B.stencil : dir == 1 ? e1B.stencil : e2.stencil;
        const bool okA = qiA < rg.qb_total, okB = hasB && qiB < rg.qb_total;
        if (!okA || (hasB && !okB)) atomicOr(err_word, 4u);
        StencilIn vA{}, vB{};
        int32_t qA = 0, qB = 0;
        int64_t tiA = 0, tiB = 0;
        if (okA) {
            vA = load_stencil(rec, posA, rg.dist, scA);
            qA = __ldg(qb + qiA);
            if (scA == kStencilCubic) tiA = __ldg(t_int + ((uint64_t)blkA * nb2 + e2.bb) * fg.layer_num + l);
        }
        if (okB) {
            vB = load_stencil(rec, posB, rg.dist, scB);
            qB = __ldg(qb + qiB);
            if (scB == kStencilCubic) tiB = __ldg(t_int + ((uint64_t)blkB * nb2 + e2.bb) * fg.layer_num + l);
        }
        if (okA) {
            const float t = scA == kStencilCubic ? __fdiv_rn(__ll2float_rn(tiA), tp) : 0.0f;
            const float pred = predict_loaded(vA, scA, t);
            rec[posA] = __double2float_rn(__fma_rn(-(double)qA, eb2, (double)pred));
        }
        if (okB) {
            const float t = scB == kStencilCubic ? __fdiv_rn(__ll2float_rn(tiB), tp) : 0.0f;
            const float pred = predict_loaded(vB, scB, t);
            rec[posB] = __double2float_rn(__fma_rn(-(double)qB, eb2, (double)pred));
        }
    }
}

__global__ void __launch_bounds__(256, 4)
    round_decompress_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const AxisEntry *__restrict__ ent, uint32_t tpl_log2,
                            const int64_t *__restrict__ t_int, const int32_t *__restrict__ qb, float *__restrict__ rec,
                            uint32_t *err_word) {
    const double ebd = (double)rg.eb, eb2 = __dadd_rn(ebd, ebd);
    const float tp = (float)fg.t_precision;
    const uint32_t lines = (uint32_t)rg.tcount[0] * (uint32_t)rg.tcount[1];
    const LineMap m = line_map(tpl_log2);
    const uint32_t step = gridDim.x * m.lines_per_cta;
    for (uint32_t line = blockIdx.x * m.lines_per_cta + m.row; line < lines; line += 2 * step) {
        const uint32_t lineB = line + step < lines ? line + step : UINT32_MAX;
        decompress_lines2(fg, rg, l, ent, tpl_log2, m.sub, line, lineB, t_int, qb, rec, err_word, eb2, tp);
    }
}

}  // namespace asz

// ---------------------------------------------------------------------------------------------
// Launchers (declared in launch.h).
namespace asz {

static unsigned grid_for(uint64_t n, unsigned threads, unsigned cap) {
    uint64_t b = (n + threads - 1) / threads;
    return (unsigned)(b < cap ? (b ? b : 1) : cap);
}

cudaError_t launch_range(const float *x, uint64_t n, int32_t *out, unsigned long long *nonfinite, cudaStream_t st) {
    // 128-bit loads when the pointer allows; otherwise (and for the tail) scalar loads.
    uint64_t n4 = ((uintptr_t)x % 16 == 0) ? n / 4 : 0;
    uint64_t ntail = n - 4 * n4;
    range_kernel<<<grid_for(n4 ? n4 : ntail, 256, 148 * 8), 256, 0, st>>>((const float4 *)x, n4, x + 4 * n4, ntail, out,
                                                                           nonfinite);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_zero_first_last(const float *x, uint64_t n, unsigned long long *first, unsigned long long *last,
                                   cudaStream_t st) {
    zero_first_last_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(x, n, first, last);
    count_launch();
    return cudaGetLastError();
}

// A caller's t codes for round l (block-major table, layer_num per block) as the floats the round
// kernels read: code / t_precision, exact on the t grid.
__global__ void tval_from_codes_kernel(const int64_t *__restrict__ t_int, uint64_t nblocks, uint32_t L, uint32_t l,
                                       float tp, float *__restrict__ tval) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < nblocks; g += (uint64_t)gridDim.x * blockDim.x)
        tval[g] = __fdiv_rn(__ll2float_rn(t_int[g * L + l]), tp);
}

// Batched form: every field's blocks of a batch (fields found by their block-offset prefix).
__global__ void tval_from_codes_batch_kernel(const BatchField *__restrict__ F, const uint64_t *__restrict__ goff, uint32_t nf,
                                             uint32_t l) {
    const uint64_t total = goff[nf];
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < total; gi += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f = field_of(goff, nf, gi);
        const BatchField &B = F[f];
        const uint64_t g = gi - goff[f];
        B.tval[g] = __fdiv_rn(__ll2float_rn(B.tint[g * B.fg.layer_num + l]), (float)B.fg.t_precision);
    }
}

cudaError_t launch_tval_from_codes_batch(const BatchField *F, const uint64_t *goff, uint32_t nf, uint64_t total_blocks,
                                         uint32_t l, cudaStream_t st) {
    if (total_blocks == 0) return cudaSuccess;
    tval_from_codes_batch_kernel<<<grid_for(total_blocks, 256, 148 * 8), 256, 0, st>>>(F, goff, nf, l);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_tval_from_codes(const int64_t *t_int, uint64_t nblocks, uint32_t L, uint32_t l, float tp, float *tval,
                                   cudaStream_t st) {
    if (nblocks == 0) return cudaSuccess;
    tval_from_codes_kernel<<<grid_for(nblocks, 256, 148 * 8), 256, 0, st>>>(t_int, nblocks, L, l, tp, tval);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pivot_compress(const PivotGeom &pg, const float *in, float *rec, int32_t *qb, int32_t *qb_range,
                                  cudaStream_t st) {
    uint64_t total = pg.cnt[0] * pg.cnt[1] * pg.cnt[2];
    pivot_compress_kernel<<<grid_for(total, 256, 148 * 16), 256, 0, st>>>(pg, in, rec, qb, qb_range);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pivot_compress_batch(const BatchField *F, const uint64_t *poff, uint32_t nf, uint64_t total_pivots,
                                        cudaStream_t st) {
    if (total_pivots == 0) return cudaSuccess;
    pivot_compress_batch_kernel<<<grid_for(total_pivots, 256, 148 * 16), 256, 0, st>>>(F, poff, nf);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pivot_decompress(const PivotGeom &pg, const int32_t *qb, float *rec, cudaStream_t st) {
    uint64_t total = pg.cnt[0] * pg.cnt[1] * pg.cnt[2];
    pivot_decompress_kernel<<<grid_for(total, 256, 148 * 16), 256, 0, st>>>(pg, qb, rec);
    count_launch();
    return cudaGetLastError();
}

static uint32_t tpl_log2_for(uint64_t t2) {
    uint32_t lg = 0;
    while ((1ull << lg) < t2 && lg < 8) lg++;
    return lg;
}

// The single-field round kernels give a line half as many threads as it has targets (each thread
// takes two targets of each of its two lines): measured faster than one thread per target.
static uint32_t round_lines_log2(uint64_t t2) {
    const uint32_t lg = tpl_log2_for(t2);
    return lg > 0 ? lg - 1 : 0;
}

static unsigned round_grid(const RoundGeom &rg, uint32_t tpl_log2) {
    const uint64_t lines = rg.tcount[0] * rg.tcount[1];
    const uint64_t per_cta = 256u >> tpl_log2;
    return grid_for(lines, (unsigned)(2 * per_cta), 148 * 32);
}

// round_compress_line_kernel takes the finest round along axis 2 when it can stage the lines with
// 16-byte loads: n2 a multiple of 4 (so every line starts on a 16-byte boundary) and both arrays
// 16-byte aligned; n2 <= 4096 bounds the staging buffers (32 KB a warp).
static bool line_kernel_fits(const FieldGeom &fg, const RoundGeom &rg, const float *in, const float *rec) {
    return rg.dir == 2 && rg.hs == 1 && fg.n[2] % 4 == 0 && fg.n[2] <= 4096 && (uintptr_t)in % 16 == 0 &&
           (uintptr_t)rec % 16 == 0 && rg.tcount[0] * rg.tcount[1] < (1ull << 32);
}

static cudaError_t launch_round_compress_lines(const FieldGeom &fg, const RoundGeom &rg, const AxisEntry *ent,
                                               const float *tval, const float *in, float *rec, int32_t *qb, int32_t *qb_range,
                                               uint32_t *err, cudaStream_t st, unsigned long long *hist, uint32_t *hist_over) {
    constexpr size_t kStageBudget = 96 * 1024;  // staging buffers of one CTA
    const size_t per_warp = 8 * fg.n[2];
    const unsigned warps = (unsigned)std::max<size_t>(1, std::min<size_t>(8, kStageBudget / per_warp));
    const size_t smem = warps * per_warp + (hist ? kHistWin * sizeof(uint32_t) : 0);
    cudaError_t e;
    if (smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(round_compress_line_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
        return e;
    int occ = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, round_compress_line_kernel, (int)(32 * warps), smem)) !=
        cudaSuccess)
        return e;
    const uint64_t lines = rg.tcount[0] * rg.tcount[1];
    const uint64_t ctas = std::min<uint64_t>((lines + warps - 1) / warps, 148ull * (uint64_t)std::max(occ, 1));
    round_compress_line_kernel<<<(unsigned)ctas, 32 * warps, smem, st>>>(fg, rg, ent, tval, in, rec, qb, qb_range, err, hist,
                                                                         hist_over);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_round_compress(const FieldGeom &fg, const RoundGeom &rg, const AxisEntry *ent, const float *tval,
                                  const float *in, float *rec, int32_t *qb, int32_t *qb_range, uint32_t *err, int div_all,
                                  float *pred_out, cudaStream_t st, unsigned long long *hist, uint32_t *hist_over) {
    if (rg.targets == 0) return cudaSuccess;
    if (!div_all && line_kernel_fits(fg, rg, in, rec))
        return launch_round_compress_lines(fg, rg, ent, tval, in, rec, qb, qb_range, err, st, hist, hist_over);
    const uint32_t lg = round_lines_log2(rg.tcount[2]);
    const size_t smem = hist ? kHistWin * sizeof(uint32_t) : 0;
    if (div_all)
        round_compress_kernel<true><<<round_grid(rg, lg), 256, smem, st>>>(fg, rg, ent, lg, tval, in, rec, qb, qb_range, err,
                                                                           pred_out, hist, hist_over);
    else
        round_compress_kernel<false><<<round_grid(rg, lg), 256, smem, st>>>(fg, rg, ent, lg, tval, in, rec, qb, qb_range, err,
                                                                            nullptr, hist, hist_over);
    count_launch();
    return cudaGetLastError();
}

uint32_t round_tpl_log2(uint64_t t2) { return tpl_log2_for(t2); }

uint64_t round_batch_items(const RoundGeom &rg, uint32_t tpl_log2) {
    const uint64_t lines = rg.tcount[0] * rg.tcount[1], per_cta = 256u >> tpl_log2;
    const uint64_t chunks = (lines + per_cta - 1) / per_cta;
    return rg.targets ? (chunks + kBatchChunks - 1) / kBatchChunks : 0;
}

cudaError_t launch_round_compress_batch(const BatchField *F, const uint64_t *ioff, uint32_t nf, uint32_t l, uint32_t *queue,
                                        uint32_t grid, cudaStream_t st) {
    round_compress_batch_kernel<<<grid ? grid : 148 * 5, 256, 0, st>>>(F, ioff, nf, l, queue);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_round_decompress(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const AxisEntry *ent,
                                    const int64_t *t_int, const int32_t *qb, float *rec, uint32_t *err, cudaStream_t st) {
    if (rg.targets == 0) return cudaSuccess;
    const uint32_t lg = round_lines_log2(rg.tcount[2]);
    round_decompress_kernel<<<round_grid(rg, lg), 256, 0, st>>>(fg, rg, l, ent, lg, t_int, qb, rec, err);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz

// ---------------------------------------------------------------------------------------------
// Error statistics of a reconstruction: max |x - y| (as float bits, non-negative) and the sum of
// squared differences in double.
namespace asz {
__global__ void error_stats_kernel(const float *__restrict__ x, const float *__restrict__ y, uint64_t n,
                                   unsigned int *max_bits, double *sse) {
    float mx = 0.0f;
    double s = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float d = fabsf(__fsub_rn(x[i], y[i]));
        mx = fmaxf(mx, d);
        double dd = (double)x[i] - (double)y[i];
        s = __fma_rn(dd, dd, s);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(max_bits, __float_as_uint(mx));
        atomicAdd(sse, s);
    }
}

cudaError_t launch_error_stats(const float *x, const float *y, uint64_t n, unsigned int *max_bits, double *sse,
                               cudaStream_t st) {
    error_stats_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(x, y, n, max_bits, sse);
    count_launch();
    return cudaGetLastError();
}
}  // namespace asz

namespace asz {
uint64_t &launch_counter() {
    thread_local uint64_t count = 0;
    return count;
}
}  // namespace asz

// Copy of the box [lo, lo + m) of a C-order field of shape n into a dense buffer of shape m (the
// predictor-family probe's local contexts).
namespace asz {
namespace {
__global__ void copy_box_kernel(const float *__restrict__ in, uint64_t n1, uint64_t n2, uint64_t lo0, uint64_t lo1, uint64_t lo2,
                                uint64_t m0, uint64_t m1, uint64_t m2, float *__restrict__ out) {
    const uint64_t total = m0 * m1 * m2;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i2 = k % m2, r = k / m2, i1 = r % m1, i0 = r / m1;
        out[k] = in[((lo0 + i0) * n1 + lo1 + i1) * n2 + lo2 + i2];
    }
}
}  // namespace

// out[k] = in[idx[k]]: the default slope's sample neighbourhoods of a slab (asz_compress_slab).
__global__ void gather_kernel(const float *__restrict__ in, const uint64_t *__restrict__ idx, uint64_t n,
                              float *__restrict__ out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = in[idx[k]];
}

cudaError_t launch_gather(const float *in, const uint64_t *idx, uint64_t n, float *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    gather_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(in, idx, n, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_copy_box(const float *in, const uint64_t n[3], const uint64_t lo[3], const uint64_t m[3], float *out,
                            cudaStream_t st) {
    const uint64_t total = m[0] * m[1] * m[2];
    if (total == 0) return cudaSuccess;
    copy_box_kernel<<<grid_for(total, 256, 148 * 8), 256, 0, st>>>(in, n[1], n[2], lo[0], lo[1], lo[2], m[0], m[1], m[2], out);
    count_launch();
    return cudaGetLastError();
}
}  // namespace asz
