// Per-(block, round) coefficient selection (c_codes/asz_core/compress.tpp:91-144) and the
// default-slope proxy evaluations (c_codes/asz_core/get_default_slope.tpp:6-83) on the GPU.
//
// The reference scores each candidate t with get_h1_psnr (c_codes/asz_core/get_h_psnr.tpp:6-31).
// That function sums floats while iterating two std::unordered_maps, so the sums depend on
// libstdc++'s iteration order. Each group therefore rebuilds both maps' exact linked-list order:
// nodes are inserted at the front of their bucket's run, or at the list head when the bucket is
// new, and the table is rehashed to the schedule in kSchedAt/kSchedBkt. All arithmetic follows
// the reference's emitted operations (see dev_common.cuh).
//
// log2f: the reference calls glibc log2f(p) with p = freq * (1/n). p depends only on the
// integer pair (freq, n), and n is fixed by the block geometry, so the host tabulates glibc's
// values per n and the kernel indexes the table.
// log10f: glibc's log10f is not correctly rounded (measured: at most 2.06 ulp from the exact
// value over all floats). The kernel computes log10 in double, rounds to float, and accepts a
// decision only if it holds for every result within 4 ulp of that. Otherwise it takes the
// decision the rounded value gives and records the group, so the host can replay it with
// glibc and request a corrected run.
//
// This is the first, serial form: one thread per group, with scratch in global memory.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "tsel.cuh"
#include "listsim.cuh"
#include "launch.h"

namespace asz {
namespace {


// Per-group scratch carved from one global arena. cap = max samples of the launch.
struct Scratch {
    int64_t *ka, *kb;      // AB keys per distinct entry (first-occurrence order)
    uint32_t *cnt;         // count per entry
    uint64_t *hash;        // reference hash per entry
    int32_t *nxt, *bkt;    // emulated linked list (cap+1 with sentinel) and bucket heads
    int32_t *tab;          // dedupe table (index into entries)
    int32_t *ord;          // AB map iteration order
    int64_t *qk;           // qb_map keys
    uint64_t *qc;          // qb_map counts
    int32_t *qnxt, *qbkt, *qtab;
    uint32_t cap, bcap, tcap;
};

// Lays out one group's arrays from `base` (8-byte aligned each) and returns the bytes used; with
// base == nullptr it only measures. The host sizes the per-group stride with the same function.
__host__ __device__ inline uint64_t carve_layout(uint8_t *base, uint32_t cap, uint32_t bcap, uint32_t tcap, Scratch *s) {
    uint64_t off = 0;
    auto take = [&](uint64_t bytes) {
        uint8_t *r = base ? base + off : nullptr;
        off += (bytes + 7) & ~7ull;
        return r;
    };
    Scratch t;
    t.ka = (int64_t *)take(8ull * cap);
    t.kb = (int64_t *)take(8ull * cap);
    t.hash = (uint64_t *)take(8ull * cap);
    t.qk = (int64_t *)take(8ull * cap);
    t.qc = (uint64_t *)take(8ull * cap);
    t.cnt = (uint32_t *)take(4ull * cap);
    t.nxt = (int32_t *)take(4ull * (cap + 1));
    t.bkt = (int32_t *)take(4ull * bcap);
    t.tab = (int32_t *)take(4ull * tcap);
    t.ord = (int32_t *)take(4ull * cap);
    t.qnxt = (int32_t *)take(4ull * (cap + 1));
    t.qbkt = (int32_t *)take(4ull * bcap);
    t.qtab = (int32_t *)take(4ull * tcap);
    t.cap = cap;
    t.bcap = bcap;
    t.tcap = tcap;
    if (s) *s = t;
    return (off + 255) & ~255ull;
}

__host__ __device__ inline uint64_t scratch_bytes(uint32_t cap, uint32_t bcap, uint32_t tcap) {
    return carve_layout(nullptr, cap, bcap, tcap, nullptr);
}

__device__ inline Scratch carve(uint8_t *base, uint32_t cap, uint32_t bcap, uint32_t tcap) {
    Scratch s;
    carve_layout(base, cap, bcap, tcap, &s);
    return s;
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

struct FieldRef {
    const float *ref;  // reference values (reconstruction, or the original field for the slope)
    const float *x0;   // the value at the sample point itself (original field)
    uint64_t n1n2, n2;
};

// get_AB_map over `box`, deduplicated in first-occurrence order into the scratch entries.
// Returns the number of distinct entries, or UINT32_MAX if the scratch is too small.
__device__ uint32_t build_abmap(const SampleBox &box, const FieldRef &f, Scratch &s) {
    for (uint32_t i = 0; i < s.tcap; i++) s.tab[i] = kNil;
    uint32_t m = 0;
    const uint64_t d = box.dist;
    for (uint64_t i0 = box.lo[0]; i0 < box.hi[0]; i0 += box.step[0])
        for (uint64_t i1 = box.lo[1]; i1 < box.hi[1]; i1 += box.step[1])
            for (uint64_t i2 = box.lo[2]; i2 < box.hi[2]; i2 += box.step[2]) {
                uint64_t p = i0 * f.n1n2 + i1 * f.n2 + i2;
                float m1 = f.ref[p - d], m3 = f.ref[p - 3 * d], p1 = f.ref[p + d], p3 = f.ref[p + 3 * d];
                // get_AB_map.tpp:18-21 as emitted: A=(x-1+x1)-(x-3+x3), S4=(x1+x3)+(x-1+x-3),
                // B=(float)fma(S4, 0.25, -x0) in double.
                float A = __fsub_rn(__fadd_rn(m1, p1), __fadd_rn(m3, p3));
                float S4 = __fadd_rn(__fadd_rn(p1, p3), __fadd_rn(m1, m3));
                float B = __double2float_rn(__fma_rn((double)S4, 0.25, -(double)f.x0[p]));
                int64_t ak = lround_f(__fmul_rn(A, box.neg_2_stat_eb));
                int64_t bk = lround_f(__fmul_rn(B, box.neg_2_stat_eb));
                uint64_t h = mix64((uint64_t)ak * 0x9e3779b97f4a7c15ull ^ (uint64_t)bk);
                uint32_t slot = (uint32_t)(h & (s.tcap - 1));
                // Linear probing over tcap > cap slots finds a free one within tcap probes; a
                // longer walk means the table is inconsistent, reported like an overflow.
                for (uint32_t probe = 0;; probe++) {
                    if (probe >= s.tcap) return UINT32_MAX;
                    int32_t e = s.tab[slot];
                    if (e == kNil) {
                        if (m >= s.cap) return UINT32_MAX;
                        s.tab[slot] = (int32_t)m;
                        s.ka[m] = ak;
                        s.kb[m] = bk;
                        s.cnt[m] = 1;
                        // asz_param.hpp:22-40: h = a*1145141919810 + b (wrapping).
                        s.hash[m] = (uint64_t)ak * 1145141919810ull + (uint64_t)bk;
                        m++;
                        break;
                    }
                    if (s.ka[e] == ak && s.kb[e] == bk) {
                        s.cnt[e]++;
                        break;
                    }
                    slot = (slot + 1) & (s.tcap - 1);
                }
            }
    // Reproduce the map's iteration order.
    ListSim L{s.nxt, s.bkt, s.hash, nullptr, s.cap, 0, 1, 0};
    L.init();
    for (uint32_t e = 0; e < m; e++) L.insert((int32_t)e);
    uint32_t k = 0;
    for (int32_t p = s.nxt[s.cap]; p != kNil && k < m; p = s.nxt[p]) s.ord[k++] = p;
    if (k != m || L.broken) return UINT32_MAX;
    return m;
}

// get_h1_psnr (get_h_psnr.tpp:6-31) as emitted. Writes h1 and the log10f argument x. Returns
// false if the bin table is inconsistent (no free slot within tcap probes).
__device__ bool eval_proxy(Scratch &s, uint32_t m, float t, float abs_eb, float stat_eb, float R2,
                           const float *log2tab, float &h1_out, float &x_out) {
    const float neg_2_eb = __fdiv_rn(0.5f, abs_eb);
    const float t2 = __fadd_rn(t, t), eb2 = __fadd_rn(abs_eb, abs_eb);
    for (uint32_t i = 0; i < s.tcap; i++) s.qtab[i] = kNil;
    ListSim Q{s.qnxt, s.qbkt, nullptr, s.qk, s.cap, 0, 1, 0};
    Q.init();
    float mse = 0.0f;
    uint64_t n = 0;
    uint32_t mq = 0;
    for (uint32_t k = 0; k < m; k++) {
        int32_t e = s.ord[k];
        float af = __ll2float_rn(s.ka[e]), bf = __ll2float_rn(s.kb[e]);
        float err = __fmul_rn(__fmaf_rn(bf, 2.0f, __fmul_rn(af, t2)), stat_eb);
        int64_t qb = lround_f(__fmul_rn(err, neg_2_eb));
        uint32_t slot = (uint32_t)(mix64((uint64_t)qb) & (s.tcap - 1));
        int32_t node = -1;
        for (uint32_t probe = 0; probe < s.tcap; probe++) {
            int32_t q = s.qtab[slot];
            if (q == kNil) {
                node = (int32_t)mq++;
                s.qtab[slot] = node;
                s.qk[node] = qb;
                s.qc[node] = 0;
                Q.insert(node);
                break;
            }
            if (s.qk[q] == qb) {
                node = q;
                break;
            }
            slot = (slot + 1) & (s.tcap - 1);
        }
        if (node < 0) return false;
        uint32_t c = s.cnt[e];
        s.qc[node] += c;
        float de = __fmaf_rn(-__ll2float_rn(qb), eb2, err);
        double de_d = (double)de;
        mse = __double2float_rn(__fma_rn((double)c, __dmul_rn(de_d, de_d), (double)mse));
        n += c;
    }
    float nf = __ull2float_rn(n);
    float h1 = 0.0f;
    float r = __fdiv_rn(1.0f, nf);
    uint32_t walked = 0;
    for (int32_t p = s.qnxt[s.cap]; p != kNil && walked < mq; p = s.qnxt[p], walked++) {
        uint64_t fq = s.qc[p];
        float pr = __fmul_rn(__ull2float_rn(fq), r);
        h1 = __fmaf_rn(-pr, log2tab[fq], h1);
    }
    h1_out = h1;
    x_out = __fmul_rn(__fdiv_rn(R2, mse), nf);
    return true;
}

// psnr = 10*log10f(x): the float value from a double-precision log10, and bounds that cover
// glibc's result (within 2.06 ulp of exact) with margin.
struct PsnrBand {
    float mid, lo, hi;
};
__device__ __forceinline__ float step_ulps(float v, int k) {
    int32_t b = __float_as_int(v);
    if (v == 0.0f) return k > 0 ? __int_as_float(k) : -__int_as_float(-k);
    if (b >= 0) return __int_as_float(b + k);
    return __int_as_float(b - k);
}
__device__ PsnrBand psnr_band(float x) {
    PsnrBand p;
    if (!(x > 0.0f) || isinf(x) || isnan(x)) {
        // log10f is exact at 0 (-inf), +inf (+inf) and NaN; negative x does not occur.
        float l = (x == 0.0f) ? -INFINITY : (isinf(x) ? INFINITY : __int_as_float(0x7fc00000));
        p.mid = p.lo = p.hi = __fmul_rn(10.0f, l);
        return p;
    }
    float l = __double2float_rn(log10((double)x));
    p.mid = __fmul_rn(10.0f, l);
    p.lo = __fmul_rn(10.0f, step_ulps(l, -4));
    p.hi = __fmul_rn(10.0f, step_ulps(l, 4));
    return p;
}

__device__ __forceinline__ int class_of(uint64_t b, uint64_t nb) { return b == 0 ? 0 : (b == nb - 1 ? 2 : 1); }

}  // namespace

// One thread per block for round `l`. Writes the chosen t (float) per block, its code into
// t_int[block * layer_num + l], and appends ambiguous decisions.
// Serial selection of group g of one field and round by one thread, with its scratch slot.
__device__ void v0_one(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *__restrict__ classes,
                       const float *__restrict__ rec, const float *__restrict__ orig, const float *__restrict__ log2arena,
                       float R2, float t_default, uint8_t *slot, uint32_t cap, uint32_t bcap, uint32_t tcap,
                       float *__restrict__ tval, int64_t *__restrict__ t_int, uint32_t *fb_count, AmbiguousRecord *amb,
                       uint32_t amb_cap, uint32_t *amb_count, const uint32_t *__restrict__ overrides, uint32_t n_overrides,
                       float *__restrict__ proxies, uint32_t *err_word, uint64_t g) {
    const uint64_t nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    if (g >= nblocks) return;
    const uint64_t b2 = g % fg.block_num[2], b1 = (g / fg.block_num[2]) % fg.block_num[1],
                   b0 = g / (fg.block_num[1] * fg.block_num[2]);
    const uint64_t bb[3] = {b0, b1, b2};
    const int cls = (class_of(b0, fg.block_num[0]) * 3 + class_of(b1, fg.block_num[1])) * 3 + class_of(b2, fg.block_num[2]);
    const ClassInfo ci = classes[cls];
    const int d = rg.dir;
    float best_t = t_default;
    bool fb = ci.fallback != 0;
    // Overrides: (block, round, float bits of t) settled by the host on a previous run.
    bool forced = false;
    float forced_t = 0.0f;
    for (uint32_t i = 0; i < n_overrides; i++)
        if (overrides[3 * i] == (uint32_t)g && overrides[3 * i + 1] == l) {
            forced = true;
            forced_t = __uint_as_float(overrides[3 * i + 2]);
        }
    if (!fb) {
        SampleBox box;
        for (int a = 0; a < 3; a++) {
            uint64_t lo = fg.origin[a] + bb[a] * fg.block_shape[a];
            uint64_t hi = min(fg.origin[a] + (bb[a] + 1) * fg.block_shape[a] + 1, fg.n[a]);
            if (a != d && lo != 0) lo += rg.stride[a];
            if (a == d) {
                lo += 3 * rg.stride[a] / 2;
                hi -= 3 * rg.stride[a] / 2;
            }
            box.lo[a] = lo;
            box.hi[a] = hi;
            box.step[a] = rg.stride[a] * ci.ss;
        }
        box.dist = rg.dist;
        box.neg_2_stat_eb = rg.neg_2_stat_eb;
        box.stat_eb = rg.stat_eb;
        box.n = ci.n;
        Scratch s = carve(slot, cap, bcap, tcap);
        FieldRef fr{rec, orig, fg.n[1] * fg.n[2], fg.n[2]};
        uint32_t m = ci.n == 0 ? 0 : build_abmap(box, fr, s);
        if (m == UINT32_MAX) {
            atomicOr(err_word, 1u);
            return;
        }
        if (m == 0) {
            fb = true;
        } else {
            const float *l2 = log2arena + ci.log2_off;
            // The five distinct t values of block_candidate_t (asz_param.hpp:203).
            const float cand[5] = {1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
            float h1v[5], xv[5];
            for (int c = 0; c < 5; c++)
                if (!eval_proxy(s, m, cand[c], rg.eb, rg.stat_eb, R2, l2, h1v[c], xv[c])) {
                    atomicOr(err_word, 1u);
                    return;
                }
            if (proxies) {
                for (int c = 0; c < 5; c++) {
                    proxies[(g * 10) + c] = h1v[c];
                    proxies[(g * 10) + 5 + c] = xv[c];
                }
            }
            // compress.tpp:127-142 with t starting at insufficient_sample_t (= 1/4).
            int best = 1;
            bool ambiguous = false;
            for (int c = 0; c < 5; c++) {
                if (cand[c] == cand[best]) continue;
                float d_h1 = __fsub_rn(h1v[best], h1v[c]);
                bool accept;
                if (__float_as_uint(xv[c]) == __float_as_uint(xv[best]) && isfinite(xv[c]) && xv[c] > 0.0f) {
                    // Same log10f argument: the PSNR difference is exactly 0. (For +inf, i.e. zero
                    // error, it is inf - inf = NaN instead, and the candidate is rejected below.)
                    accept = __fmaf_rn(d_h1, rg.slope, 0.0f) > 0.0f;
                } else {
                    PsnrBand pc = psnr_band(xv[c]), pb = psnr_band(xv[best]);
                    float s_mid = __fmaf_rn(d_h1, rg.slope, __fsub_rn(pc.mid, pb.mid));
                    float s_lo = __fmaf_rn(d_h1, rg.slope, __fsub_rn(pc.lo, pb.hi));
                    float s_hi = __fmaf_rn(d_h1, rg.slope, __fsub_rn(pc.hi, pb.lo));
                    bool sure = (s_lo > 0.0f) || !(s_hi > 0.0f);
                    if (!sure) ambiguous = true;
                    accept = s_mid > 0.0f;
                }
                if (accept) best = c;
            }
            best_t = cand[best];
            if (forced) {
                best_t = forced_t;
                ambiguous = false;
            }
            if (ambiguous) {
                uint32_t k = atomicAdd(amb_count, 1u);
                if (k < amb_cap) {
                    AmbiguousRecord &r = amb[k];
                    r.block = (uint32_t)g;
                    r.round = l;
                    r.provisional = (int32_t)lround_f(__fmul_rn(best_t, (float)fg.t_precision));
                    for (int c = 0; c < 5; c++) {
                        r.h1[c] = h1v[c];
                        r.x[c] = xv[c];
                    }
                }
            }
        }
    }
    if (fb) atomicAdd(fb_count, 1u);
    tval[g] = best_t;
    t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(best_t, (float)fg.t_precision));
}

__global__ void tsel_v0_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const ClassInfo *__restrict__ classes,
                               const float *__restrict__ rec, const float *__restrict__ orig,
                               const float *__restrict__ log2arena, float R2, float t_default,
                               uint8_t *scratch, uint64_t scratch_stride, uint32_t cap, uint32_t bcap, uint32_t tcap,
                               float *__restrict__ tval, int64_t *__restrict__ t_int, uint32_t *__restrict__ fb_count,
                               AmbiguousRecord *amb, uint32_t amb_cap, uint32_t *amb_count,
                               const uint32_t *__restrict__ overrides, uint32_t n_overrides,
                               float *__restrict__ proxies, const uint32_t *__restrict__ list,
                               const uint32_t *__restrict__ list_count, uint32_t *__restrict__ err_word) {
    const uint64_t nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    // With a list, each thread settles the listed groups tid, tid+nthreads, ... in its own scratch
    // slot; without one, thread g settles group g.
    const uint64_t items = list ? *list_count : nblocks;
    for (uint64_t it = tid; it < items; it += nthreads)
        v0_one(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, scratch + tid * scratch_stride, cap, bcap, tcap, tval,
               t_int, fb_count, amb, amb_cap, amb_count, overrides, n_overrides, proxies, err_word, list ? list[it] : it);
}

// Batched form over (field << 32 | group) entries of all fields of a batch.
__global__ void tsel_v0_batch_kernel(const BatchField *__restrict__ F, uint32_t l, const float *__restrict__ log2arena,
                                     float t_default, uint8_t *scratch, uint64_t scratch_stride, uint32_t cap, uint32_t bcap,
                                     uint32_t tcap, const unsigned long long *__restrict__ list,
                                     const uint32_t *__restrict__ list_count) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t items = *list_count;
    for (uint64_t it = tid; it < items; it += nthreads) {
        const unsigned long long e = list[it];
        const BatchField &B = F[e >> 32];
        const uint64_t nb = B.fg.block_num[0] * B.fg.block_num[1] * B.fg.block_num[2];
        v0_one(B.fg, B.rounds[l], l, B.classes + 27 * l, B.rec, B.in, log2arena, B.R2, t_default, scratch + tid * scratch_stride,
               cap, bcap, tcap, B.tval, B.tint, &B.cnt->fb, B.amb, B.amb_cap, &B.cnt->amb_count, nullptr, 0,
               B.proxies ? B.proxies + nb * l * 10 : nullptr, &B.cnt->err, e & 0xffffffffull);
    }
}

// Proxies of whole-field AB maps over the original data (the default slope's three axis maps, or
// the plan search's per-direction maps), each evaluated for every (t, eb) pair. One thread per map.
__global__ void slope_v0_kernel(FieldGeom fg, const SampleBox *__restrict__ boxes, const ProxyEval *__restrict__ evals,
                                uint32_t n_evals, const float *__restrict__ orig, const float *__restrict__ log2arena,
                                float R2, uint8_t *scratch, uint64_t scratch_stride, uint32_t cap, uint32_t bcap,
                                uint32_t tcap, float *__restrict__ h1_out, float *__restrict__ x_out,
                                uint32_t *__restrict__ m_out, uint32_t *__restrict__ err_word, uint32_t nboxes) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nboxes) return;
    SampleBox box = boxes[g];
    Scratch s = carve(scratch + g * scratch_stride, cap, bcap, tcap);
    FieldRef fr{orig, orig, fg.n[1] * fg.n[2], fg.n[2]};
    uint32_t m = build_abmap(box, fr, s);
    if (m == UINT32_MAX) {
        atomicOr(err_word, 2u);
        return;
    }
    m_out[g] = m;
    if (m == 0) return;
    for (uint32_t e = 0; e < n_evals; e++)
        if (!eval_proxy(s, m, evals[e].t, evals[e].abs_eb, box.stat_eb, R2, log2arena + box.log2_off,
                        h1_out[g * n_evals + e], x_out[g * n_evals + e])) {
            atomicOr(err_word, 2u);
            return;
        }
}

uint64_t tsel_scratch_bytes(uint32_t cap, uint32_t bcap, uint32_t tcap) { return scratch_bytes(cap, bcap, tcap); }

}  // namespace asz

namespace asz {
cudaError_t launch_tsel_v0(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                           const float *orig, const float *log2arena, float R2, float t_default, uint8_t *scratch,
                           uint64_t scratch_stride, uint32_t cap, uint32_t bcap, uint32_t tcap, float *tval, int64_t *t_int,
                           uint32_t *fb_count, AmbiguousRecord *amb, uint32_t amb_cap, uint32_t *amb_count,
                           const uint32_t *overrides, uint32_t n_overrides, float *proxies, const uint32_t *list,
                           const uint32_t *list_count, uint64_t slots, uint32_t *err, cudaStream_t st) {
    tsel_v0_kernel<<<(unsigned)((slots + 63) / 64), 64, 0, st>>>(fg, rg, l, classes, rec, orig, log2arena, R2, t_default,
                                                                  scratch, scratch_stride, cap, bcap, tcap, tval, t_int,
                                                                  fb_count, amb, amb_cap, amb_count, overrides, n_overrides,
                                                                  proxies, list, list_count, err);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_tsel_v0_batch(const BatchField *F, uint32_t l, const float *log2arena, float t_default, uint8_t *scratch,
                                 uint64_t scratch_stride, uint32_t cap, uint32_t bcap, uint32_t tcap,
                                 const unsigned long long *list, const uint32_t *list_count, uint64_t slots, cudaStream_t st) {
    tsel_v0_batch_kernel<<<(unsigned)((slots + 63) / 64), 64, 0, st>>>(F, l, log2arena, t_default, scratch, scratch_stride, cap,
                                                                        bcap, tcap, list, list_count);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_slope_v0(const FieldGeom &fg, const SampleBox *boxes, const ProxyEval *evals, uint32_t n_evals,
                            const float *orig, const float *log2arena, float R2, uint8_t *scratch, uint64_t scratch_stride,
                            uint32_t cap, uint32_t bcap, uint32_t tcap, float *h1, float *x, uint32_t *m_out, uint32_t *err,
                            uint32_t nboxes, cudaStream_t st) {
    slope_v0_kernel<<<1, 32, 0, st>>>(fg, boxes, evals, n_evals, orig, log2arena, R2, scratch, scratch_stride, cap, bcap, tcap,
                                      h1, x, m_out, err, nboxes);
    count_launch();
    return cudaGetLastError();
}
}  // namespace asz
