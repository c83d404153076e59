// Per-(block, round) coefficient selection, fast path (c_codes/asz_core/compress.tpp:91-144).
//
// The reference scores each candidate t with sums taken in std::unordered_map order. This path
// computes the same per-sample terms with the reference's float operations, but sums them in
// any order: squared errors in double, and H1 from a dense histogram of the quantised errors.
// It then bounds how far the reference's order-dependent float sums can be from these values:
// - mse:  n sequential roundings of non-negative partial sums, <= n * 2^-24 relative;
// - H1:   m_q sequential fused roundings, <= m_q * 2^-24 relative;
// - log10f: glibc's result is within 2.06 ulp of exact (measured over all floats); 3 ulp allowed.
// A candidate comparison whose sign holds over the whole interval is decided here. A group with
// any undecidable comparison goes to the exact path (k_tsel.cu), which replays the maps' order.
// So does a group whose quantised errors do not fit the histogram window (1024 bins per candidate,
// placed on the exact bin range or, when that is wider, on the bin of the mean keys). Groups whose A
// keys are all zero give every candidate identical sums, and keep t = 1/4 exactly.
//
// One warp per group; the sample positions follow get_AB_map's loops (get_AB_map.tpp:13-15).
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "launch.h"
#include "tsel.cuh"

namespace asz {
namespace {

constexpr int kWin = 1024;         // histogram window (quantised-error values) per candidate
constexpr int kWarpsPerBlock = 8;
// Counts are 16-bit (a group has < 65536 samples), two per 32-bit word.
constexpr int kWinWords = kWin / 2;

__device__ __forceinline__ int class_of(uint64_t b, uint64_t nb) { return b == 0 ? 0 : (b == nb - 1 ? 2 : 1); }

struct SampleGeo {
    uint64_t lo[3], step[3];
    uint32_t cnt[3];
};

__device__ __forceinline__ uint64_t sample_pos(const SampleGeo &sg, uint32_t s, uint64_t n1, uint64_t n2) {
    uint32_t k2 = s % sg.cnt[2], k1 = (s / sg.cnt[2]) % sg.cnt[1], k0 = s / (sg.cnt[1] * sg.cnt[2]);
    uint64_t i0 = sg.lo[0] + k0 * sg.step[0], i1 = sg.lo[1] + k1 * sg.step[1], i2 = sg.lo[2] + k2 * sg.step[2];
    return (i0 * n1 + i1) * n2 + i2;
}

// AB keys of one sample (get_AB_map.tpp:18-21 as emitted), returned as the floats get_h1_psnr
// converts them to.
__device__ __forceinline__ void sample_keys(const float *__restrict__ rec, const float *__restrict__ orig, uint64_t p,
                                            uint64_t d, float neg, float &af, float &bf, bool &anz) {
    float m1 = rec[p - d], m3 = rec[p - 3 * d], p1 = rec[p + d], p3 = rec[p + 3 * d];
    float A = __fsub_rn(__fadd_rn(m1, p1), __fadd_rn(m3, p3));
    float S4 = __fadd_rn(__fadd_rn(p1, p3), __fadd_rn(m1, m3));
    float B = __double2float_rn(__fma_rn((double)S4, 0.25, -(double)orig[p]));
    int64_t ak = lround_f(__fmul_rn(A, neg));
    int64_t bk = lround_f(__fmul_rn(B, neg));
    af = __ll2float_rn(ak);
    bf = __ll2float_rn(bk);
    anz = ak != 0;
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
__device__ Interval psnr_interval(double S, uint32_t n, float R2, float nf) {
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

}  // namespace

// Groups are listed per round; list_out receives the groups this path could not settle.
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    tsel_fast_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const ClassInfo *__restrict__ classes,
                     const float *__restrict__ rec, const float *__restrict__ orig, const float *__restrict__ log2arena,
                     float R2, float t_default, float *__restrict__ tval, int64_t *__restrict__ t_int,
                     uint32_t *__restrict__ fb_count, uint32_t *__restrict__ list_out, uint32_t *__restrict__ list_count,
                     const uint32_t *__restrict__ overrides, uint32_t n_overrides, uint32_t *__restrict__ why) {
    extern __shared__ uint32_t hist_dyn[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t(*hist)[kWinWords] = (uint32_t(*)[kWinWords])(hist_dyn + warp * 5 * kWinWords);
    const uint64_t nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    const float cand[5] = {1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
    const int d = rg.dir;
    for (int c = 0; c < 5; c++)
        for (int i = lane; i < kWinWords; i += 32) hist[c][i] = 0;
    __syncwarp();
    for (uint64_t g = (uint64_t)blockIdx.x * kWarpsPerBlock + warp; g < nblocks; g += (uint64_t)gridDim.x * kWarpsPerBlock) {
        const uint64_t b2 = g % fg.block_num[2], b1 = (g / fg.block_num[2]) % fg.block_num[1],
                       b0 = g / (fg.block_num[1] * fg.block_num[2]);
        const uint64_t bb[3] = {b0, b1, b2};
        const int cls = (class_of(b0, fg.block_num[0]) * 3 + class_of(b1, fg.block_num[1])) * 3 + class_of(b2, fg.block_num[2]);
        const ClassInfo ci = classes[cls];
        bool forced = false;
        float forced_t = 0.0f;
        for (uint32_t i = 0; i < n_overrides; i++)
            if (overrides[3 * i] == (uint32_t)g && overrides[3 * i + 1] == l) {
                forced = true;
                forced_t = __uint_as_float(overrides[3 * i + 2]);
            }
        if (ci.fallback || ci.n == 0 || forced) {
            if (lane == 0) {
                float t = forced ? forced_t : t_default;
                if (!forced) atomicAdd(fb_count, 1u);
                tval[g] = t;
                t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(t, (float)fg.t_precision));
            }
            continue;
        }
        SampleGeo sg;
        for (int a = 0; a < 3; a++) {
            uint64_t lo = bb[a] * fg.block_shape[a];
            uint64_t hi = min((bb[a] + 1) * fg.block_shape[a] + 1, fg.n[a]);
            if (a != d && lo != 0) lo += rg.stride[a];
            if (a == d) {
                lo += 3 * rg.stride[a] / 2;
                hi -= 3 * rg.stride[a] / 2;
            }
            sg.lo[a] = lo;
            sg.step[a] = rg.stride[a] * ci.ss;
            sg.cnt[a] = (uint32_t)((hi - lo + sg.step[a] - 1) / sg.step[a]);
        }
        const uint32_t n = ci.n;
        const uint64_t n1 = fg.n[1], n2 = fg.n[2];
        if (n > 0xffffu) {  // a bin count could overflow its 16-bit half word
            if (lane == 0) {
                list_out[atomicAdd(list_count, 1u)] = (uint32_t)g;
                atomicAdd(&why[0], 1u);
            }
            continue;
        }
        // Pass 1: key ranges and sums, and whether any A key is nonzero.
        float afmin = INFINITY, afmax = -INFINITY, bfmin = INFINITY, bfmax = -INFINITY;
        double asum = 0.0, bsum = 0.0;
        bool anz = false;
        for (uint32_t s = lane; s < n; s += 32) {
            float af, bf;
            bool nz;
            sample_keys(rec, orig, sample_pos(sg, s, n1, n2), rg.dist, rg.neg_2_stat_eb, af, bf, nz);
            afmin = fminf(afmin, af);
            afmax = fmaxf(afmax, af);
            bfmin = fminf(bfmin, bf);
            bfmax = fmaxf(bfmax, bf);
            asum += (double)af;
            bsum += (double)bf;
            anz |= nz;
        }
        for (int o = 16; o; o >>= 1) {
            afmin = fminf(afmin, __shfl_xor_sync(0xffffffffu, afmin, o));
            afmax = fmaxf(afmax, __shfl_xor_sync(0xffffffffu, afmax, o));
            bfmin = fminf(bfmin, __shfl_xor_sync(0xffffffffu, bfmin, o));
            bfmax = fmaxf(bfmax, __shfl_xor_sync(0xffffffffu, bfmax, o));
            asum += __shfl_xor_sync(0xffffffffu, asum, o);
            bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
        }
        anz = __any_sync(0xffffffffu, anz);
        if (!anz) {
            // Every candidate sees identical errors, so every comparison is fmaf(0, slope, 0 or NaN)
            // and nothing is accepted: t stays at 1/4.
            if (lane == 0) {
                tval[g] = cand[1];
                t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(cand[1], (float)fg.t_precision));
            }
            continue;
        }
        const float eb = rg.eb, neg_eb = __fdiv_rn(0.5f, eb), eb2 = __fadd_rn(eb, eb);
        // Histogram window per candidate: the exact bin range when it fits, else centred on the
        // bin of the mean keys; samples outside it send the group to the exact path.
        int64_t qlo[5];
        for (int c = 0; c < 5; c++) {
            float t2 = __fadd_rn(cand[c], cand[c]);
            int64_t q0 = lround_f(__fmul_rn(cand_err(afmin, bfmin, t2, rg.stat_eb), neg_eb));
            int64_t q1 = lround_f(__fmul_rn(cand_err(afmax, bfmax, t2, rg.stat_eb), neg_eb));
            if (q1 >= q0 && (uint64_t)q1 - (uint64_t)q0 < (uint64_t)kWin) {
                qlo[c] = q0;
            } else {
                float am = (float)(asum / n), bm = (float)(bsum / n);
                qlo[c] = lround_f(__fmul_rn(cand_err(am, bm, t2, rg.stat_eb), neg_eb)) - kWin / 2;
            }
        }
        // Pass 2: per-candidate sums and histograms.
        double S[5] = {0, 0, 0, 0, 0};
        bool out = false;
        for (uint32_t s = lane; s < n; s += 32) {
            float af, bf;
            bool nz;
            sample_keys(rec, orig, sample_pos(sg, s, n1, n2), rg.dist, rg.neg_2_stat_eb, af, bf, nz);
#pragma unroll
            for (int c = 0; c < 5; c++) {
                float t2 = __fadd_rn(cand[c], cand[c]);
                float err = cand_err(af, bf, t2, rg.stat_eb);
                int64_t q = lround_f(__fmul_rn(err, neg_eb));
                float de = __fmaf_rn(-__ll2float_rn(q), eb2, err);
                double dd = (double)de;
                S[c] = __fma_rn(dd, dd, S[c]);
                const uint64_t bin = (uint64_t)q - (uint64_t)qlo[c];
                if (bin < (uint64_t)kWin) atomicAdd(&hist[c][bin >> 1], 1u << (16 * (bin & 1)));
                else out = true;
            }
        }
        out = __any_sync(0xffffffffu, out);
        if (out) {
            for (int c = 0; c < 5; c++)
                for (int i = lane; i < kWinWords; i += 32) hist[c][i] = 0;
            __syncwarp();
            if (lane == 0) {
                list_out[atomicAdd(list_count, 1u)] = (uint32_t)g;
                atomicAdd(&why[0], 1u);
            }
            continue;
        }
        __syncwarp();
        const float nf = __ull2float_rn((uint64_t)n), r = __fdiv_rn(1.0f, nf);
        const float *l2 = log2arena + ci.log2_off;
        double H[5];
        uint32_t mq[5];
#pragma unroll
        for (int c = 0; c < 5; c++) {
            double h = 0.0;
            uint32_t k = 0;
            for (int i = lane; i < kWinWords; i += 32) {
                uint32_t w = hist[c][i];
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
                    hist[c][i] = 0;
                }
            }
            for (int o = 16; o; o >>= 1) {
                h += __shfl_xor_sync(0xffffffffu, h, o);
                k += __shfl_xor_sync(0xffffffffu, k, o);
                S[c] += __shfl_xor_sync(0xffffffffu, S[c], o);
            }
            H[c] = h;
            mq[c] = k;
        }
        __syncwarp();
        if (lane == 0) {
            // Decision chain (compress.tpp:127-142) on intervals.
            Interval P[5];
            double hlo[5], hhi[5];
            for (int c = 0; c < 5; c++) {
                P[c] = psnr_interval(S[c], n, R2, nf);
                double gq = (double)mq[c] * 0x1.0002p-24 + 0x1p-40;
                hlo[c] = H[c] * (1.0 - gq);
                hhi[c] = H[c] * (1.0 + gq);
            }
            const double slope = (double)rg.slope;
            bool sure = isfinite(slope) && slope > 0;
            int best = 1;
            for (int c = 0; c < 5 && sure; c++) {
                if (cand[c] == cand[best]) continue;
                bool accept;
                if (P[c].exact_inf || P[best].exact_inf) {
                    // inf - finite = inf (accept), finite - inf = -inf, inf - inf = NaN (reject).
                    accept = P[c].exact_inf && !P[best].exact_inf;
                } else {
                    double dlo = hlo[best] - hhi[c], dhi = hhi[best] - hlo[c];
                    dlo -= fabs(dlo) * 0x1p-23;
                    dhi += fabs(dhi) * 0x1p-23;
                    double plo = P[c].lo - P[best].hi, phi = P[c].hi - P[best].lo;
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
            if (!sure) {
                list_out[atomicAdd(list_count, 1u)] = (uint32_t)g;
                atomicAdd(&why[1], 1u);
            } else {
                tval[g] = cand[best];
                t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(cand[best], (float)fg.t_precision));
            }
        }
        __syncwarp();
    }
}

cudaError_t launch_tsel_fast(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                             const float *orig, const float *log2arena, float R2, float t_default, float *tval,
                             int64_t *t_int, uint32_t *fb_count, uint32_t *list_out, uint32_t *list_count,
                             const uint32_t *overrides, uint32_t n_overrides, uint32_t *why, cudaStream_t st) {
    uint64_t nb = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    uint64_t blocks = (nb + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks > 148 * 64) blocks = 148 * 64;
    const int smem = kWarpsPerBlock * 5 * kWinWords * 4;
    cudaError_t e = cudaFuncSetAttribute(tsel_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    tsel_fast_kernel<<<(unsigned)blocks, kWarpsPerBlock * 32, smem, st>>>(fg, rg, l, classes, rec, orig, log2arena, R2,
                                                                          t_default, tval, t_int, fb_count, list_out,
                                                                          list_count, overrides, n_overrides, why);
    return cudaGetLastError();
}

}  // namespace asz
