// Certified order-free coefficient selection of one (block, round) group by one CTA: the shared
// algorithm of the per-round fast kernel (k_tsel_fast.cu) and the fused axis-2 rounds (k_lines.cu).
//
// The reference scores each candidate t with sums taken in std::unordered_map order
// (c_codes/asz_core/compress.tpp:91-144). This path computes the same per-sample terms with the
// reference's float operations, but sums them in any order: squared errors in double, and H1
// from a dense histogram of the quantised errors. It then bounds how far the reference's
// order-dependent float sums can be from these values:
// - mse:  n sequential roundings of non-negative partial sums, <= n * 2^-24 relative;
// - H1:   m_q sequential fused roundings, <= m_q * 2^-24 relative;
// - log10f: glibc's result is within 2.06 ulp of exact (measured over all floats); 3 ulp allowed.
// A candidate comparison whose sign holds over the whole interval is decided here. A group with
// any undecidable comparison goes to the exact path (k_tsel_exact.cu), which replays the maps'
// order. So does a group whose quantised errors span too many histogram windows (1024 bins per
// candidate, placed on the exact bin range or, when that is wider, counted window by window).
// Groups whose A keys are all zero give every candidate identical sums, and keep t = 1/4 exactly.
#pragma once
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "launch.h"
#include "tsel.cuh"

namespace asz {
namespace fastsel {

constexpr int kWin = 1024;         // histogram window (quantised-error values) per candidate
// Counts are 16-bit (a group has < 65536 samples), two per 32-bit word.
constexpr int kWinWords = kWin / 2;
// A group whose bins still overflow the window over the exact key ranges is counted in windows of
// 5 * kWin bins; beyond this many passes (all candidates together) it goes to the exact path.
constexpr uint32_t kMaxWidePasses = 40;

__device__ __forceinline__ int class_of(uint64_t b, uint64_t nb) { return b == 0 ? 0 : (b == nb - 1 ? 2 : 1); }

// AB keys of one sample from its four neighbours along the round axis and its original value
// (get_AB_map.tpp:18-21 as emitted), returned as the floats get_h1_psnr converts them to.
// The keys of a sample's A and B (the quantisation step of get_AB_map.tpp:20-21).
__device__ __forceinline__ void keys_of_ab(float A, float B, float neg, float &af, float &bf, bool &anz) {
    int64_t ak = lround_f(__fmul_rn(A, neg));
    int64_t bk = lround_f(__fmul_rn(B, neg));
    af = __ll2float_rn(ak);
    bf = __ll2float_rn(bk);
    anz = ak != 0;
}

__device__ __forceinline__ void keys_of(float m1, float m3, float p1, float p3, float x0, float neg, float &af, float &bf,
                                        bool &anz) {
    float A = __fsub_rn(__fadd_rn(m1, p1), __fadd_rn(m3, p3));
    float S4 = __fadd_rn(__fadd_rn(p1, p3), __fadd_rn(m1, m3));
    float B = __double2float_rn(__fma_rn((double)S4, 0.25, -(double)x0));
    keys_of_ab(A, B, neg, af, bf, anz);
}

__device__ __forceinline__ void sample_keys(const float *__restrict__ rec, const float *__restrict__ orig, uint64_t p,
                                            uint64_t d, float neg, float &af, float &bf, bool &anz) {
    keys_of(rec[p - d], rec[p - 3 * d], rec[p + d], rec[p + 3 * d], orig[p], neg, af, bf, anz);
}

// err and its quantisation bin for candidate t (get_h_psnr.tpp:14-17 as emitted).
__device__ __forceinline__ float cand_err(float af, float bf, float t2, float stat_eb) {
    return __fmul_rn(__fmaf_rn(bf, 2.0f, __fmul_rn(af, t2)), stat_eb);
}

__device__ __forceinline__ double ulp_f(double v) {
    v = fabs(v);
    if (!(v > 0) || isinf(v)) return 0x1p-149;
    int e = ilogb(v);
    return ldexp(1.0, max(e - 23, -149));
}

struct Interval {
    double lo, hi;
    bool exact_inf;  // psnr is +inf exactly (zero error)
};

// PSNR interval for the reference's float value given the order-free sum S of c*d^2 over n terms.
__device__ __forceinline__ Interval psnr_interval(double S, uint32_t n, float R2, float nf) {
    Interval iv;
    iv.exact_inf = false;
    if (S == 0.0) {
        iv.lo = iv.hi = INFINITY;
        iv.exact_inf = true;
        return iv;
    }
    const double g = (double)n * 0x1.0002p-24 + 0x1p-40;
    const double X = (double)R2 * (double)nf / S;
    const double xlo = X / (1.0 + g) * (1.0 - 0x1p-22), xhi = X / (1.0 - g) * (1.0 + 0x1p-22);
    const double llo = log10(xlo), lhi = log10(xhi);
    const double ul = ulp_f(fmax(fabs(llo), fabs(lhi)));
    const double up = ulp_f(10.0 * fmax(fabs(llo), fabs(lhi)));
    iv.lo = 10.0 * (llo - 3.0 * ul) - up - 1e-12 * fabs(llo);
    iv.hi = 10.0 * (lhi + 3.0 * ul) + up + 1e-12 * fabs(lhi);
    return iv;
}


// Quotient s / d for s * d < 2^32 with m = floor((2^32 - 1) / d) + 1 (d > 1): floor(s * m / 2^32)
// is exact because the error term s * (m * d - 2^32) / (d * 2^32) stays below 1/d.
struct SmallDiv {
    uint32_t d, m;
};

__device__ __forceinline__ SmallDiv small_div(uint32_t d) { return SmallDiv{d, d > 1 ? 0xffffffffu / d + 1u : 0u}; }
__device__ __forceinline__ uint32_t div_small(uint32_t s, SmallDiv q) { return q.d > 1 ? __umulhi(s, q.m) : s; }

struct FastSampleGeo {
    uint64_t lo[3], step[3];
    SmallDiv c2, c12;
    uint32_t cnt2;
};

__device__ __forceinline__ uint64_t fast_sample_pos(const FastSampleGeo &sg, uint32_t s, uint64_t n1, uint64_t n2) {
    const uint32_t k0 = div_small(s, sg.c12);
    const uint32_t r = s - k0 * sg.c12.d;
    const uint32_t k1 = div_small(r, sg.c2);
    const uint32_t k2 = r - k1 * sg.cnt2;
    const uint64_t i0 = sg.lo[0] + k0 * sg.step[0], i1 = sg.lo[1] + k1 * sg.step[1], i2 = sg.lo[2] + k2 * sg.step[2];
    return (i0 * n1 + i1) * n2 + i2;
}

// Threads per group: kThreads by default; the per-round kernel also has a 128-thread form for
// rounds with few groups, where the shorter per-group time of more threads wins.
constexpr int kThreads = 64;
constexpr int kMaxWarps = 4;

// Shared state of one group (one CTA).
struct GroupShared {
    uint32_t hist[5][kWinWords];
    Interval psnr[5];
    float fmin[kMaxWarps][2], fmax[kMaxWarps][2];
    double dsum[kMaxWarps][5];
    uint32_t cnt[kMaxWarps][5];
    uint32_t flag[kMaxWarps];
    uint32_t res_code;  // outcome of fast_group, broadcast to the CTA
    float res_t;
};

// Block-wide reductions over kT threads; every thread receives the result.
template <int kT>
__device__ __forceinline__ void block_minmax(GroupShared &sh, float &amin, float &amax, float &bmin, float &bmax) {
    for (int o = 16; o; o >>= 1) {
        amin = fminf(amin, __shfl_xor_sync(0xffffffffu, amin, o));
        amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        bmin = fminf(bmin, __shfl_xor_sync(0xffffffffu, bmin, o));
        bmax = fmaxf(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh.fmin[w][0] = amin;
        sh.fmin[w][1] = bmin;
        sh.fmax[w][0] = amax;
        sh.fmax[w][1] = bmax;
    }
    __syncthreads();
    amin = sh.fmin[0][0];
    bmin = sh.fmin[0][1];
    amax = sh.fmax[0][0];
    bmax = sh.fmax[0][1];
    for (int i = 1; i < kT / 32; i++) {
        amin = fminf(amin, sh.fmin[i][0]);
        bmin = fminf(bmin, sh.fmin[i][1]);
        amax = fmaxf(amax, sh.fmax[i][0]);
        bmax = fmaxf(bmax, sh.fmax[i][1]);
    }
}

// Sums of nv doubles and nv counts per thread, and the OR of a flag word. Fixed order (warp tree, then
// warps in index order), so every thread gets the same bits.
template <int kT, int NV>
__device__ __forceinline__ void block_sums(GroupShared &sh, double (&v)[NV], uint32_t (&c)[NV], uint32_t &flag) {
#pragma unroll
    for (int i = 0; i < NV; i++)
        for (int o = 16; o; o >>= 1) {
            v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
            c[i] += __shfl_xor_sync(0xffffffffu, c[i], o);
        }
    flag = __reduce_or_sync(0xffffffffu, flag);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int i = 0; i < NV; i++) {
            sh.dsum[w][i] = v[i];
            sh.cnt[w][i] = c[i];
        }
        sh.flag[w] = flag;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; i++) {
        v[i] = sh.dsum[0][i];
        c[i] = sh.cnt[0][i];
        for (int k = 1; k < kT / 32; k++) {
            v[i] += sh.dsum[k][i];
            c[i] += sh.cnt[k][i];
        }
    }
    flag = sh.flag[0];
    for (int k = 1; k < kT / 32; k++) flag |= sh.flag[k];
    __syncthreads();  // the staging arrays are reused by the next reduction
}

enum : uint32_t { kFastDecided = 0, kFastHandoff = 1 };

// Selects t for one group of n samples (n < 65536). Src::keys(s, af, bf, nz) gives the keys of
// sample s. Every thread of the CTA calls this and gets the same result: kFastDecided with t_out,
// or kFastHandoff when the exact path has to decide. The histograms are left zeroed.
template <class Src, int kT = kThreads>
__device__ uint32_t fast_group(GroupShared &sh, const Src &src, uint32_t n, const RoundGeom &rg, const float *l2, float R2,
                               uint32_t *why, float &t_out) {
    const uint32_t tid = threadIdx.x;
    const float cand[5] = {1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
    const float eb = rg.eb, neg_eb = __fdiv_rn(0.5f, eb), eb2 = __fadd_rn(eb, eb);
    // Window placement from the first kT samples (one per thread): their bin range per
    // candidate, centred in the window. A group whose samples overflow the window is redone
    // with the exact ranges of all samples.
    // Each thread's first two samples are loaded together and kept for the main pass.
    float af0 = 0.0f, bf0 = 0.0f, af1 = 0.0f, bf1 = 0.0f;
    bool nz0 = false, nz1 = false;
    float afmin = INFINITY, afmax = -INFINITY, bfmin = INFINITY, bfmax = -INFINITY;
    if (tid < n) {
        src.keys(tid, af0, bf0, nz0);
        if (tid + kT < n) src.keys(tid + kT, af1, bf1, nz1);
        afmin = afmax = af0;
        bfmin = bfmax = bf0;
    }
    block_minmax<kT>(sh, afmin, afmax, bfmin, bfmax);
    int64_t qlo[5];
    bool fits = true;
    for (int c = 0; c < 5; c++) {
        const float t2 = __fadd_rn(cand[c], cand[c]);
        const int64_t q0 = lround_f(__fmul_rn(cand_err(afmin, bfmin, t2, rg.stat_eb), neg_eb));
        const int64_t q1 = lround_f(__fmul_rn(cand_err(afmax, bfmax, t2, rg.stat_eb), neg_eb));
        if (q1 >= q0 && (uint64_t)q1 - (uint64_t)q0 < (uint64_t)kWin) qlo[c] = q0 - (kWin - 1 - (q1 - q0)) / 2;
        else fits = false;
    }
    double S[5];
    uint32_t anz = 0, out = 1;
    for (int attempt = 0; attempt < 2 && out; attempt++) {
        if (attempt == 1) {
            // Exact key ranges over all samples; the window is their bin range, or centred on
            // the bin of the mean keys when that range is wider than the window.
            afmin = bfmin = INFINITY;
            afmax = bfmax = -INFINITY;
            double ab[2] = {0.0, 0.0};
            for (uint32_t s = tid; s < n; s += kT) {
                float af, bf;
                bool nz;
                src.keys(s, af, bf, nz);
                afmin = fminf(afmin, af);
                afmax = fmaxf(afmax, af);
                bfmin = fminf(bfmin, bf);
                bfmax = fmaxf(bfmax, bf);
                ab[0] += (double)af;
                ab[1] += (double)bf;
            }
            block_minmax<kT>(sh, afmin, afmax, bfmin, bfmax);
            uint32_t dummy[2] = {0, 0}, none = 0;
            block_sums<kT, 2>(sh, ab, dummy, none);
            for (int c = 0; c < 5; c++) {
                const float t2 = __fadd_rn(cand[c], cand[c]);
                const int64_t q0 = lround_f(__fmul_rn(cand_err(afmin, bfmin, t2, rg.stat_eb), neg_eb));
                const int64_t q1 = lround_f(__fmul_rn(cand_err(afmax, bfmax, t2, rg.stat_eb), neg_eb));
                if (q1 >= q0 && (uint64_t)q1 - (uint64_t)q0 < (uint64_t)kWin) {
                    qlo[c] = q0;
                } else {
                    const float am = (float)(ab[0] / n), bm = (float)(ab[1] / n);
                    qlo[c] = lround_f(__fmul_rn(cand_err(am, bm, t2, rg.stat_eb), neg_eb)) - kWin / 2;
                }
            }
        } else if (!fits) {
            continue;
        }
        // Per-candidate sums and histograms over every sample.
        for (int c = 0; c < 5; c++) S[c] = 0.0;
        anz = 0;
        out = 0;
        for (uint32_t s = tid; s < n; s += kT) {
            float af, bf;
            bool nz;
            if (s == tid) {
                af = af0;
                bf = bf0;
                nz = nz0;
            } else if (s == tid + kT) {
                af = af1;
                bf = bf1;
                nz = nz1;
            } else {
                src.keys(s, af, bf, nz);
            }
            anz |= nz ? 1u : 0u;
#pragma unroll
            for (int c = 0; c < 5; c++) {
                const float t2 = __fadd_rn(cand[c], cand[c]);
                const float err = cand_err(af, bf, t2, rg.stat_eb);
                const int64_t q = lround_f(__fmul_rn(err, neg_eb));
                const float de = __fmaf_rn(-__ll2float_rn(q), eb2, err);
                const double dd = (double)de;
                S[c] = __fma_rn(dd, dd, S[c]);
                const uint64_t bin = (uint64_t)q - (uint64_t)qlo[c];
                if (bin < (uint64_t)kWin) atomicAdd(&sh.hist[c][bin >> 1], 1u << (16 * (bin & 1)));
                else out = 1;
            }
        }
        {
            // One reduction: S, and the OR of the flags (overflow in bit 0, a nonzero A key in bit 1).
            uint32_t flags = out | (anz << 1), dummy[5] = {0, 0, 0, 0, 0};
            block_sums<kT, 5>(sh, S, dummy, flags);
            out = flags & 1u;
            anz = (flags >> 1) & 1u;
        }
        if (out || !anz) {
            for (int i = tid; i < 5 * kWinWords; i += kT) (&sh.hist[0][0])[i] = 0;
            __syncthreads();
        }
        if (!anz) break;
    }
    if (!anz) {
        // Every candidate sees identical errors, so every comparison is fmaf(0, slope, 0 or NaN)
        // and nothing is accepted: t stays at 1/4.
        t_out = cand[1];
        return kFastDecided;
    }
    const float nf = __ull2float_rn((uint64_t)n), r = __fdiv_rn(1.0f, nf);
    double H[5];
    uint32_t mq[5];
    if (out) {
        // The bins of some candidate span more than the window even over the exact key ranges.
        // Count them window by window instead: per candidate, passes over the samples with all
        // five histogram regions used as one window of 5 * kWin bins.
        constexpr int kWide = 5 * kWin;
        int64_t q0c[5];
        uint32_t passes = 0;
        for (int c = 0; c < 5; c++) {
            const float t2 = __fadd_rn(cand[c], cand[c]);
            q0c[c] = lround_f(__fmul_rn(cand_err(afmin, bfmin, t2, rg.stat_eb), neg_eb));
            const int64_t q1 = lround_f(__fmul_rn(cand_err(afmax, bfmax, t2, rg.stat_eb), neg_eb));
            const uint64_t pc = ((uint64_t)q1 - (uint64_t)q0c[c]) / kWide + 1;
            passes += pc < (1u << 20) ? (uint32_t)pc : (1u << 20);
        }
        if (passes > kMaxWidePasses) {
            if (tid == 0) atomicAdd(&why[0], 1u);
            return kFastHandoff;
        }
        uint32_t *flat = &sh.hist[0][0];
        for (int c = 0; c < 5; c++) {
            const float t2 = __fadd_rn(cand[c], cand[c]);
            const int64_t q1 = lround_f(__fmul_rn(cand_err(afmax, bfmax, t2, rg.stat_eb), neg_eb));
            double h = 0.0;
            uint32_t k = 0;
            for (int64_t lo = q0c[c];; lo += kWide) {
                for (uint32_t s = tid; s < n; s += kT) {
                    float af, bf;
                    bool nz;
                    src.keys(s, af, bf, nz);
                    const int64_t q = lround_f(__fmul_rn(cand_err(af, bf, t2, rg.stat_eb), neg_eb));
                    const uint64_t bin = (uint64_t)q - (uint64_t)lo;
                    if (bin < (uint64_t)kWide) atomicAdd(&flat[bin >> 1], 1u << (16 * (bin & 1)));
                }
                __syncthreads();
                for (int i = tid; i < kWide / 2; i += kT) {
                    const uint32_t w = flat[i];
                    if (w) {
                        const uint32_t c0 = w & 0xffffu, c1 = w >> 16;
                        if (c0) {
                            const float p = __fmul_rn(__ull2float_rn((uint64_t)c0), r);
                            h = __fma_rn(-(double)p, (double)l2[c0], h);
                            k++;
                        }
                        if (c1) {
                            const float p = __fmul_rn(__ull2float_rn((uint64_t)c1), r);
                            h = __fma_rn(-(double)p, (double)l2[c1], h);
                            k++;
                        }
                        flat[i] = 0;
                    }
                }
                __syncthreads();
                if (q1 - lo < kWide) break;
            }
            H[c] = h;
            mq[c] = k;
        }
        if (tid == 0) atomicAdd(&why[2], 1u);
    } else if (n <= 2 * (uint32_t)kT) {
        // Every sample is held in registers: each one clears its bin with an atomic AND, and the
        // one that finds the count still there adds that bin's term. The window ends up zeroed
        // without a scan of all its bins, which dominates the cost of a small group.
#pragma unroll
        for (int c = 0; c < 5; c++) {
            H[c] = 0.0;
            mq[c] = 0;
        }
#pragma unroll
        for (uint32_t j = 0; j < 2; j++) {
            if (tid + j * kT >= n) break;
            const float af = j ? af1 : af0, bf = j ? bf1 : bf0;
#pragma unroll
            for (int c = 0; c < 5; c++) {
                const float t2 = __fadd_rn(cand[c], cand[c]);
                const int64_t q = lround_f(__fmul_rn(cand_err(af, bf, t2, rg.stat_eb), neg_eb));
                const uint64_t bin = (uint64_t)q - (uint64_t)qlo[c];  // < kWin: no sample left the window
                const uint32_t sh16 = 16u * (uint32_t)(bin & 1);
                const uint32_t cnt = (atomicAnd(&sh.hist[c][bin >> 1], ~(0xffffu << sh16)) >> sh16) & 0xffffu;
                if (cnt) {
                    const float p = __fmul_rn(__ull2float_rn((uint64_t)cnt), r);
                    H[c] = __fma_rn(-(double)p, (double)l2[cnt], H[c]);
                    mq[c]++;
                }
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < 5; c++) {
            double h = 0.0;
            uint32_t k = 0;
            for (int i = tid; i < kWinWords; i += kT) {
                uint32_t w = sh.hist[c][i];
                if (w) {
                    uint32_t c0 = w & 0xffffu, c1 = w >> 16;
                    if (c0) {
                        float p = __fmul_rn(__ull2float_rn((uint64_t)c0), r);
                        h = __fma_rn(-(double)p, (double)l2[c0], h);
                        k++;
                    }
                    if (c1) {
                        float p = __fmul_rn(__ull2float_rn((uint64_t)c1), r);
                        h = __fma_rn(-(double)p, (double)l2[c1], h);
                        k++;
                    }
                    sh.hist[c][i] = 0;
                }
            }
            H[c] = h;
            mq[c] = k;
        }
    }
    {
        uint32_t none = 0;
        block_sums<kT, 5>(sh, H, mq, none);
    }
    if (tid < 32) {
        // PSNR intervals of the five candidates in parallel, then the decision chain
        // (compress.tpp:127-142) on intervals by one lane.
        if (tid < 5) sh.psnr[tid] = psnr_interval(S[tid], n, R2, nf);
        __syncwarp();
        if (tid == 0) {
            const double slope = (double)rg.slope;
            bool sure = isfinite(slope) && slope > 0;
            int best = 1;
            for (int c = 0; c < 5 && sure; c++) {
                if (cand[c] == cand[best]) continue;
                const Interval Pc = sh.psnr[c], Pb = sh.psnr[best];
                const double gb = (double)mq[best] * 0x1.0002p-24 + 0x1p-40, gc = (double)mq[c] * 0x1.0002p-24 + 0x1p-40;
                bool accept;
                if (Pc.exact_inf || Pb.exact_inf) {
                    // inf - finite = inf (accept), finite - inf = -inf, inf - inf = NaN (reject).
                    accept = Pc.exact_inf && !Pb.exact_inf;
                } else {
                    double dlo = H[best] * (1.0 - gb) - H[c] * (1.0 + gc), dhi = H[best] * (1.0 + gb) - H[c] * (1.0 - gc);
                    dlo -= fabs(dlo) * 0x1p-23;
                    dhi += fabs(dhi) * 0x1p-23;
                    double plo = Pc.lo - Pb.hi, phi = Pc.hi - Pb.lo;
                    plo -= fabs(plo) * 0x1p-23;
                    phi += fabs(phi) * 0x1p-23;
                    double slo = dlo * slope + plo, shi = dhi * slope + phi;
                    slo -= 1e-9 * (fabs(dlo * slope) + fabs(plo));
                    shi += 1e-9 * (fabs(dhi * slope) + fabs(phi));
                    if (slo > 1e-30) accept = true;
                    else if (shi <= 0.0) accept = false;
                    else {
                        sure = false;
                        break;
                    }
                }
                if (accept) best = c;
            }
            if (!sure) atomicAdd(&why[1], 1u);
            sh.res_code = sure ? kFastDecided : kFastHandoff;
            sh.res_t = cand[best];
        }
    }
    __syncthreads();
    t_out = sh.res_t;
    return sh.res_code;
}

}  // namespace fastsel
}  // namespace asz
