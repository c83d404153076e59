// Differentiable per-block coefficient tuning: a relaxed form of the reference's H1-PSNR proxy
// (get_h_psnr.tpp:6-31) as a function of a continuous t, its derivative, and a tuner that replaces
// the 5-candidate scan (compress.tpp:91-144) by a few projected steps on it.
//
// Samples. Group (block b, round l), indexed b * layers + l like the t stream, has the AB-map
// sample lattice of get_AB_map (get_AB_map.tpp:13-15), but the samples are read OPEN LOOP, from
// the original field: A = (x-1 + x1) - (x-3 + x3) and B = (float)fma(x-3 + x3 + x-1 + x1, 0.25, -x)
// along the round axis, in the reference's float steps (get_AB_map.tpp:18-21). The interior 1D4R
// prediction error is then r(t) = A t + B. Open loop means every round's groups exist at once, so
// one launch covers all of them.
//
// Relaxed proxy of a group (n samples, layer error bound eb, slope from the layer's default slope,
// value range R), to be minimised:
//   q_s = clamp(r_s / (2 eb), -256, 256)                   bin coordinate of sample s
//   p_k = (1/n) sum_s w(q_s - k), w the unit triangle       soft histogram over integer bins
//   H   = -sum_k p_k log2(p_k + 1e-6)                       soft entropy (bits)
//   m   = (1/n) sum_s r_s^2                                 open-loop squared residual
//   mse = m c / (m + c), c = eb^2 / 3                      -> m for small residuals, -> the
//                                                            uniform quantisation noise eb^2/3
//   J   = slope * H - 10 log10(R^2 / mse)                   minus the relaxed score
// dJ/dt follows from dq_s/dt = A_s / (2 eb) (0 where clamped) and dm/dt = (2/n) sum r_s A_s; the
// triangle kernel gives dH/dq_s = (h'(p_{k0+1}) - h'(p_{k0})) / n with k0 = floor(q_s) and
// h'(p) = -(log2(p + 1e-6) + p / ((p + 1e-6) ln 2)).
//
// One CTA per group, its soft histogram (513 bins) in shared memory; sums in double.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "launch.h"
#include "tsel_fast.cuh"

namespace asz {
namespace grad {

constexpr int kHalfBins = 256;              // bins -256..256
constexpr int kBins = 2 * kHalfBins + 2;    // one spare
constexpr float kEps = 1e-6f;
constexpr double kTenOverLn10 = 4.3429448190325175;  // 10 / ln 10
constexpr float kInvLn2 = 1.4426950408889634f;

struct Meta {
    float eb, stat_eb, neg_2_stat_eb, slope;
};

// Bin coordinate, its clamp flag and the lower bin index (0-based in the window).
__device__ __forceinline__ void bin_of(float r, float inv2eb, float &f, int &k0, bool &clamped) {
    float q = r * inv2eb;
    clamped = !(q > -(float)kHalfBins && q < (float)kHalfBins);
    q = fminf(fmaxf(q, -(float)kHalfBins), (float)kHalfBins);
    float fl = floorf(q);
    if (fl >= (float)kHalfBins) fl = (float)kHalfBins - 1.0f;
    f = q - fl;
    k0 = (int)fl + kHalfBins;
}

struct Sums {
    double m, ra, H;  // mean r^2, sum r*A / n, soft entropy
    int klo, khi;     // lowest and highest bin with weight
};

// One CTA (the team: 32 to kMaxTeam threads, 256 by default) per group at a time. Its shared words
// (the soft histogram, h' values, or the judge's counts) are all zero between uses: every pass
// clears what it wrote, and only the bins a group touches are visited.
constexpr int kTeam = 256;
constexpr int kMaxTeam = 512;
constexpr int kTeamWarps = kMaxTeam / 32;
constexpr int kJudgeBins = 2048;              // judge window (quantised-error values)
constexpr uint32_t kMaxJudgeWindows = 128;    // beyond 128 * 2048 bins the judge keeps the default

struct TeamShared {
    float hist[kBins];   // soft histogram
    float hp[kBins];     // h'(p) per bin
    uint32_t counts[2][kJudgeBins];  // judge: one window of quantised-error counts per candidate
    double red[kTeamWarps][4];
    int imn[kTeamWarps], imx[kTeamWarps];
    long long lmn[kTeamWarps], lmx[kTeamWarps];
};

// Sums over the team in a fixed order (warp tree, then warps by index): every thread gets them.
__device__ void team_sum4(TeamShared &sh, double (&v)[4]) {
    for (int o = 16; o; o >>= 1)
        for (int i = 0; i < 4; i++) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int i = 0; i < 4; i++) sh.red[w][i] = v[i];
    __syncthreads();
    for (int i = 0; i < 4; i++) v[i] = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++)
        for (int i = 0; i < 4; i++) v[i] += sh.red[k][i];
    __syncthreads();
}

__device__ void team_sum3(TeamShared &sh, double &a, double &b, double &c) {
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh.red[w][0] = a;
        sh.red[w][1] = b;
        sh.red[w][2] = c;
    }
    __syncthreads();
    a = b = c = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
        a += sh.red[i][0];
        b += sh.red[i][1];
        c += sh.red[i][2];
    }
    __syncthreads();
}

template <class T>
__device__ void team_minmax(T (&mn)[kTeamWarps], T (&mx)[kTeamWarps], T &lo, T &hi) {
    for (int o = 16; o; o >>= 1) {
        const T l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        mn[w] = lo;
        mx[w] = hi;
    }
    __syncthreads();
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
        lo = mn[i] < lo ? mn[i] : lo;
        hi = mx[i] > hi ? mx[i] : hi;
    }
    __syncthreads();
}

// Soft histogram of the group's samples at t and the sums. keep: leave the histogram for
// group_grad (which clears it); otherwise it is cleared here.
__device__ Sums group_pass(TeamShared &sh, const float *__restrict__ A, const float *__restrict__ B, uint32_t n,
                           const Meta &mt, float t, bool keep) {
    const float inv2eb = 0.5f / mt.eb;
    double m = 0.0, ra = 0.0, H = 0.0;
    int klo = kBins, khi = -1;
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        const float a = A[s], r = fmaf(a, t, B[s]);
        float f;
        int k0;
        bool cl;
        bin_of(r, inv2eb, f, k0, cl);
        atomicAdd(&sh.hist[k0], 1.0f - f);
        atomicAdd(&sh.hist[k0 + 1], f);
        klo = min(klo, k0);
        khi = max(khi, k0 + 1);
        m += (double)r * r;
        ra += (double)r * a;
    }
    team_minmax(sh.imn, sh.imx, klo, khi);  // its barriers also complete the histogram
    const float inv_n = 1.0f / (float)n;
    for (int i = klo + (int)threadIdx.x; i <= khi; i += blockDim.x) {
        const float p = sh.hist[i] * inv_n;
        const float l2 = log2f(p + kEps);
        if (p > 0.0f) H -= (double)p * (double)l2;
        if (keep) sh.hp[i] = -(l2 + p / (p + kEps) * kInvLn2);  // h'(p) for group_grad
        sh.hist[i] = 0.0f;
    }
    team_sum3(sh, m, ra, H);
    return Sums{m / n, ra / n, H, klo, khi};
}

__device__ __forceinline__ double objective(const Sums &S, const Meta &mt, float R2) {
    const double c = (double)mt.eb * mt.eb / 3.0;
    const double mse = fmax(S.m * c / (S.m + c), 1e-300);
    return (double)mt.slope * S.H - 10.0 * log10((double)R2 / mse);
}

// dJ/dt after group_pass(keep) at the same t, from the h' values it left (the barriers of its
// final reduction made them visible).
__device__ double group_grad(TeamShared &sh, const float *__restrict__ A, const float *__restrict__ B, uint32_t n,
                             const Meta &mt, float t, const Sums &S) {
    const float inv2eb = 0.5f / mt.eb;
    double gh = 0.0, u0 = 0.0, u1 = 0.0;
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        const float a = A[s], r = fmaf(a, t, B[s]);
        float f;
        int k0;
        bool cl;
        bin_of(r, inv2eb, f, k0, cl);
        if (!cl) gh += (double)(sh.hp[k0 + 1] - sh.hp[k0]) * (double)(a * inv2eb);
    }
    team_sum3(sh, gh, u0, u1);  // its barriers end the reads of h'
    gh /= n;
    const double c = (double)mt.eb * mt.eb / 3.0;
    const double dlog = S.m > 0.0 ? c / (S.m * (S.m + c)) : 0.0;
    return (double)mt.slope * gh + kTenOverLn10 * dlog * 2.0 * S.ra;
}

__device__ __forceinline__ Meta load_meta(const float4 *meta, uint64_t g) {
    const float4 v = meta[g];
    Meta m{v.x, v.y, v.z, v.w};
    if (!isfinite(m.slope)) m.slope = 0.0f;
    return m;
}

__device__ __forceinline__ void team_clear(TeamShared &sh) {
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) sh.hist[i] = 0.0f;
    for (int i = threadIdx.x; i < 2 * kJudgeBins; i += blockDim.x) (&sh.counts[0][0])[i] = 0u;
    __syncthreads();
}

__global__ void __launch_bounds__(kMaxTeam)
    forward_kernel(const float *__restrict__ A, const float *__restrict__ B, const uint32_t *__restrict__ off,
                   const float4 *__restrict__ meta, float R2, const float *__restrict__ t, uint64_t groups,
                   float *__restrict__ J) {
    __shared__ TeamShared sh;
    team_clear(sh);
    for (uint64_t g = blockIdx.x; g < groups; g += gridDim.x) {
        const uint32_t o = off[g], n = off[g + 1] - o;
        if (n == 0) {
            if (threadIdx.x == 0) J[g] = 0.0f;
            continue;
        }
        const Meta mt = load_meta(meta, g);
        const Sums S = group_pass(sh, A + o, B + o, n, mt, t[g], false);
        if (threadIdx.x == 0) J[g] = (float)objective(S, mt, R2);
    }
}

__global__ void __launch_bounds__(kMaxTeam)
    backward_kernel(const float *__restrict__ A, const float *__restrict__ B, const uint32_t *__restrict__ off,
                    const float4 *__restrict__ meta, float R2, const float *__restrict__ t, const float *__restrict__ gJ,
                    uint64_t groups, float *__restrict__ gt) {
    __shared__ TeamShared sh;
    team_clear(sh);
    for (uint64_t g = blockIdx.x; g < groups; g += gridDim.x) {
        const uint32_t o = off[g], n = off[g + 1] - o;
        if (n == 0) {
            if (threadIdx.x == 0) gt[g] = 0.0f;
            continue;
        }
        const Meta mt = load_meta(meta, g);
        const Sums S = group_pass(sh, A + o, B + o, n, mt, t[g], true);
        const double d = group_grad(sh, A + o, B + o, n, mt, t[g], S);
        if (threadIdx.x == 0) gt[g] = (float)(d * (double)gJ[g]);
    }
}

// The reference's proxy scores -slope * h1 + psnr of candidates t[0] and t[1] (get_h_psnr.tpp:6-31
// on the keys of get_AB_map.tpp:18-21), with order-free double sums. One pass computes both
// candidates' errors and counts them in a window placed on sample 0's bin; a candidate whose
// errors spread beyond it is counted again window by window. Returns false when some candidate's
// errors span more than kMaxJudgeWindows windows.
__device__ bool exact_scores(TeamShared &sh, const float *__restrict__ A, const float *__restrict__ B, uint32_t n,
                             const Meta &mt, float R2, const float (&t)[2], double (&score)[2]) {
    const float neg_eb = __fdiv_rn(0.5f, mt.eb), eb2 = __fadd_rn(mt.eb, mt.eb);
    const float t2[2] = {__fadd_rn(t[0], t[0]), __fadd_rn(t[1], t[1])};
    long long w0[2], lo[2] = {LLONG_MAX, LLONG_MAX}, hi[2] = {LLONG_MIN, LLONG_MIN};
    {
        float af, bf;
        bool nz;
        fastsel::keys_of_ab(A[0], B[0], mt.neg_2_stat_eb, af, bf, nz);
        for (int c = 0; c < 2; c++)
            w0[c] = lround_f(__fmul_rn(fastsel::cand_err(af, bf, t2[c], mt.stat_eb), neg_eb)) - kJudgeBins / 2;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};  // mse[0], mse[1], h1[0], h1[1]
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        float af, bf;
        bool nz;
        fastsel::keys_of_ab(A[s], B[s], mt.neg_2_stat_eb, af, bf, nz);
        for (int c = 0; c < 2; c++) {
            const float err = fastsel::cand_err(af, bf, t2[c], mt.stat_eb);
            const long long q = lround_f(__fmul_rn(err, neg_eb));
            const float de = __fmaf_rn(-__ll2float_rn(q), eb2, err);
            acc[c] += (double)de * de;
            lo[c] = q < lo[c] ? q : lo[c];
            hi[c] = q > hi[c] ? q : hi[c];
            if (q >= w0[c] && q - w0[c] < kJudgeBins) atomicAdd(&sh.counts[c][q - w0[c]], 1u);
        }
    }
    for (int c = 0; c < 2; c++) team_minmax(sh.lmn, sh.lmx, lo[c], hi[c]);
    bool ok = true;
    for (int c = 0; c < 2; c++) {
        uint32_t *cnt = sh.counts[c];
        const bool fits = lo[c] >= w0[c] && hi[c] - w0[c] < kJudgeBins;
        if (fits) {
            for (int i = (int)(lo[c] - w0[c]) + threadIdx.x; i <= (int)(hi[c] - w0[c]); i += blockDim.x) {
                const uint32_t k = cnt[i];
                if (k) {
                    const double p = (double)k / n;
                    acc[2 + c] -= p * log2(p);
                    cnt[i] = 0u;
                }
            }
            continue;
        }
        for (int i = threadIdx.x; i < kJudgeBins; i += blockDim.x) cnt[i] = 0u;
        __syncthreads();
        if ((unsigned long long)(hi[c] - lo[c]) / kJudgeBins >= kMaxJudgeWindows) {
            ok = false;
            continue;
        }
        for (long long w = lo[c]; w <= hi[c]; w += kJudgeBins) {
            for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
                float af, bf;
                bool nz;
                fastsel::keys_of_ab(A[s], B[s], mt.neg_2_stat_eb, af, bf, nz);
                const long long q = lround_f(__fmul_rn(fastsel::cand_err(af, bf, t2[c], mt.stat_eb), neg_eb));
                if (q >= w && q - w < kJudgeBins) atomicAdd(&cnt[q - w], 1u);
            }
            __syncthreads();
            const int top = (int)min((long long)kJudgeBins - 1, hi[c] - w);
            for (int i = threadIdx.x; i <= top; i += blockDim.x) {
                const uint32_t k = cnt[i];
                if (k) {
                    const double p = (double)k / n;
                    acc[2 + c] -= p * log2(p);
                    cnt[i] = 0u;
                }
            }
            __syncthreads();
        }
    }
    team_sum4(sh, acc);
    for (int c = 0; c < 2; c++) {
        const double psnr = acc[c] > 0.0 ? 10.0 * log10((double)R2 * n / acc[c]) : INFINITY;
        score[c] = -(double)mt.slope * acc[2 + c] + psnr;
    }
    return ok;
}

// All of a group's tuning in one CTA: `steps` projected sign-gradient steps on J from t = 1/4 with
// step sizes step0 * 2^-k, inside [t_min, t_max]; the result snapped to the t grid; then the
// reference's proxy judges the snapped t against the default 1/4 and keeps the default unless
// the snapped t scores higher (the acceptance test of compress.tpp:136-140).
// stats: [0] groups tuned, [1] snapped t accepted, [2] quantised errors spread over more than
// kMaxJudgeWindows * kJudgeBins bins, so the judge kept the default.
// The steps see at most kStage samples of a group, staged in shared memory: every k-th sample,
// k = ceil(n / step_cap) (step_cap <= kStage; 0 means kStage). The judge sees all of them.
constexpr uint32_t kStage = 1024;

__global__ void __launch_bounds__(kMaxTeam)
    tune_kernel(const float *__restrict__ A, const float *__restrict__ B, const uint32_t *__restrict__ off,
                const float4 *__restrict__ meta, float R2, uint64_t groups, float t_min, float t_max, int32_t tp,
                uint32_t steps, float step0, uint32_t step_cap, int64_t *__restrict__ t_codes,
                float *__restrict__ t_relaxed, uint32_t *__restrict__ stats) {
    __shared__ TeamShared sh;
    __shared__ float sA[kStage], sB[kStage];
    if (step_cap == 0 || step_cap > kStage) step_cap = kStage;
    team_clear(sh);
    const int64_t code_lo = lround_f(__fmul_rn(t_min, (float)tp)), code_hi = lround_f(__fmul_rn(t_max, (float)tp));
    const int64_t code_def = lround_f(__fmul_rn(0.25f, (float)tp));
    for (uint64_t g = blockIdx.x; g < groups; g += gridDim.x) {
        const uint32_t o = off[g], n = off[g + 1] - o;
        if (n == 0) {
            if (threadIdx.x == 0) {
                t_codes[g] = code_def;
                if (t_relaxed) t_relaxed[g] = 0.25f;
            }
            continue;
        }
        const Meta mt = load_meta(meta, g);
        // The steps read their samples many times: stage them.
        const uint32_t stride = (n + step_cap - 1) / step_cap, ns = (n + stride - 1) / stride;
        __syncthreads();  // the previous group's passes are done with sA, sB
        for (uint32_t s = threadIdx.x; s < ns; s += blockDim.x) {
            sA[s] = A[o + s * stride];
            sB[s] = B[o + s * stride];
        }
        __syncthreads();
        float t = 0.25f, step = step0;
        for (uint32_t k = 0; k < steps; k++, step *= 0.5f) {
            const Sums S = group_pass(sh, sA, sB, ns, mt, t, true);
            const double d = group_grad(sh, sA, sB, ns, mt, t, S);
            if (d > 0.0) t -= step;
            else if (d < 0.0) t += step;
            t = fminf(fmaxf(t, t_min), t_max);
        }
        int64_t code = lround_f(__fmul_rn(t, (float)tp));
        code = code < code_lo ? code_lo : (code > code_hi ? code_hi : code);
        int64_t chosen = code_def;
        if (code != code_def) {
            const float cand[2] = {0.25f, (float)code / (float)tp};
            double sc[2];
            const bool ok = exact_scores(sh, A + o, B + o, n, mt, R2, cand, sc);
            if (!ok) {
                if (threadIdx.x == 0) atomicAdd(&stats[2], 1u);
            } else if (sc[1] - sc[0] > 0.0) {
                chosen = code;
                if (threadIdx.x == 0) atomicAdd(&stats[1], 1u);
            }
        }
        if (threadIdx.x == 0) {
            atomicAdd(&stats[0], 1u);
            t_codes[g] = chosen;
            if (t_relaxed) t_relaxed[g] = t;
        }
    }
}

// Open-loop AB samples of every group (see the file comment). One CTA per group; positions as in
// the fast selection (origin 0). err: bit 0 when a group's lattice does not hold off[] samples.
__global__ void __launch_bounds__(256)
    gather_kernel(FieldGeom fg, const RoundGeom *__restrict__ rounds, const ClassInfo *__restrict__ classes,
                  const float *__restrict__ x, const uint32_t *__restrict__ off, uint64_t groups, float *__restrict__ A,
                  float *__restrict__ B, uint32_t *err) {
    const uint32_t L = fg.layer_num;
    for (uint64_t gid = blockIdx.x; gid < groups; gid += gridDim.x) {
        const uint32_t o = off[gid], n = off[gid + 1] - o;
        if (n == 0) continue;
        const uint64_t g = gid / L, l = gid - g * L;
        const RoundGeom &rg = rounds[l];
        const uint64_t b2 = g % fg.block_num[2], b1 = (g / fg.block_num[2]) % fg.block_num[1],
                       b0 = g / (fg.block_num[1] * fg.block_num[2]);
        const uint64_t bb[3] = {b0, b1, b2};
        const int cls = (fastsel::class_of(b0, fg.block_num[0]) * 3 + fastsel::class_of(b1, fg.block_num[1])) * 3 +
                        fastsel::class_of(b2, fg.block_num[2]);
        const ClassInfo ci = classes[27 * l + cls];
        fastsel::FastSampleGeo sg;
        uint32_t cnt[3];
        const int d = rg.dir;
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
            cnt[a] = (uint32_t)((hi - lo + sg.step[a] - 1) / sg.step[a]);
        }
        if ((uint64_t)cnt[0] * cnt[1] * cnt[2] != n) {
            if (threadIdx.x == 0) atomicOr(err, 1u);
            continue;
        }
        sg.cnt2 = cnt[2];
        sg.c2 = fastsel::small_div(cnt[2]);
        sg.c12 = fastsel::small_div(cnt[1] * cnt[2]);
        for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
            const uint64_t p = fastsel::fast_sample_pos(sg, s, fg.n[1], fg.n[2]), dd = rg.dist;
            const float m1 = x[p - dd], m3 = x[p - 3 * dd], p1 = x[p + dd], p3 = x[p + 3 * dd];
            A[o + s] = __fsub_rn(__fadd_rn(m1, p1), __fadd_rn(m3, p3));
            const float S4 = __fadd_rn(__fadd_rn(p1, p3), __fadd_rn(m1, m3));
            B[o + s] = __double2float_rn(__fma_rn((double)S4, 0.25, -(double)x[p]));
        }
    }
}

unsigned grid_for(uint64_t items, unsigned per_cta) {
    uint64_t b = (items + per_cta - 1) / per_cta;
    const uint64_t cap = 148ull * 8;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

// Grid of the per-group kernels: one group per CTA at a time, up to 16 CTAs per SM.
unsigned group_grid(uint64_t groups) {
    const uint64_t cap = 148ull * 16;
    return (unsigned)(groups < 1 ? 1 : (groups > cap ? cap : groups));
}

}  // namespace grad

cudaError_t launch_grad_gather(const FieldGeom &fg, const RoundGeom *rounds, const ClassInfo *classes, const float *x,
                               const uint32_t *off, uint64_t groups, float *A, float *B, uint32_t *err, cudaStream_t st) {
    if (groups == 0) return cudaSuccess;
    grad::gather_kernel<<<grad::group_grid(groups), 256, 0, st>>>(fg, rounds, classes, x, off, groups, A, B, err);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz

using namespace asz;

extern "C" int asz_grad_forward(const float *A, const float *B, const uint32_t *offsets, const float *meta, float R2,
                                const float *t, uint64_t groups, float *J, void *cuda_stream) {
    if (groups == 0) return 0;
    if (!A || !B || !offsets || !meta || !t || !J) return 1;
    grad::forward_kernel<<<grad::group_grid(groups), grad::kTeam, 0, (cudaStream_t)cuda_stream>>>(A, B, offsets, (const float4 *)meta, R2, t, groups, J);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 7;
}

extern "C" int asz_grad_backward(const float *A, const float *B, const uint32_t *offsets, const float *meta, float R2,
                                 const float *t, const float *grad_J, uint64_t groups, float *grad_t, void *cuda_stream) {
    if (groups == 0) return 0;
    if (!A || !B || !offsets || !meta || !t || !grad_J || !grad_t) return 1;
    grad::backward_kernel<<<grad::group_grid(groups), grad::kTeam, 0, (cudaStream_t)cuda_stream>>>(A, B, offsets, (const float4 *)meta, R2, t, grad_J, groups, grad_t);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 7;
}

extern "C" int asz_grad_tune(const float *A, const float *B, const uint32_t *offsets, const float *meta, float R2,
                             uint64_t groups, float t_min, float t_max, int32_t t_precision, uint32_t steps, float step0,
                             uint32_t step_cap, uint32_t team, int64_t *t_codes, float *t_relaxed, uint32_t *stats,
                             void *cuda_stream) {
    if (groups == 0) return 0;
    if (team == 0) team = grad::kTeam;
    if (!A || !B || !offsets || !meta || !t_codes || !stats || t_precision <= 0 || !(t_min <= t_max) || team % 32 ||
        team > (uint32_t)grad::kMaxTeam)
        return 1;
    grad::tune_kernel<<<grad::group_grid(groups), team, 0, (cudaStream_t)cuda_stream>>>(
        A, B, offsets, (const float4 *)meta, R2, groups, t_min, t_max, t_precision, steps, step0, step_cap, t_codes, t_relaxed,
        stats);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? 0 : 7;
}
