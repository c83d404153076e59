// Exact per-(block, round) coefficient selection for the groups the fast path could not settle,
// and the default-slope proxies (c_codes/asz_core/compress.tpp:91-144, get_AB_map.tpp:7-24,
// get_h_psnr.tpp:6-31, get_default_slope.tpp:15-39).
//
// One CTA per group, all state in shared memory:
//  1. sample keys in get_AB_map's scan order;
//  2. de-duplicate them (shared hash table) and compact the distinct keys in first-occurrence order;
//  3. rebuild std::unordered_map's iteration order without replaying insertions one by one. Within
//     one rehash stage the list is a sequence of bucket runs: runs ordered by the time their bucket
//     was first filled (newest first), nodes within a run newest first. A node's "time" in a stage
//     is its position in the previous stage's list if it was present at the rehash, else its
//     insertion index. So each stage is a parallel rank computation (atomics, one scan);
//  4. per evaluation: quantised errors in map order, the qb_map's own order (same method, identity
//     hash), then the two order-dependent float sums, one thread each, all evaluations at once.
// The result is the reference's float h1 and log10f argument bit for bit; the t decision then
// uses the same certified log10 step as the serial kernel.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "launch.h"
#include "listsim.cuh"
#include "tsel.cuh"

namespace asz {
namespace {

constexpr int kThreads = 512;  // 16 warps: 5 run the sum chains, 11 build the qb maps
constexpr int kMaxEvals = 22;  // default slope: 11 t values x 2 error bounds

__device__ __forceinline__ int class_of(uint64_t b, uint64_t nb) { return b == 0 ? 0 : (b == nb - 1 ? 2 : 1); }

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// A set of whole warps that synchronise on their own hardware barrier (bar 0 is the CTA's).
struct Team {
    int tid, size, bar;
    __device__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(size) : "memory"); }
};

// Exclusive scan of one value per team thread; total in *tot. warp_sums holds 32 ints.
__device__ int team_excl_scan(const Team &T, int v, int *warp_sums, int *tot) {
    const int lane = T.tid & 31, w = T.tid >> 5, nw = T.size >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    T.sync();
    if (w == 0) {
        int s = lane < nw ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;  // inclusive
    }
    T.sync();
    int base = w ? warp_sums[w - 1] : 0;
    int total = warp_sums[nw - 1];
    T.sync();
    if (tot) *tot = total;
    return base + x - v;
}

// Exclusive scan of a[0..n) in place; returns the total.
__device__ int team_scan_array(const Team &T, int *a, int n, int *warp_sums) {
    const int per = (n + T.size - 1) / T.size;
    const int beg = T.tid * per, end = min(beg + per, n);
    int local = 0;
    for (int i = beg; i < end; i++) local += a[i];
    int tot;
    int off = team_excl_scan(T, local, warp_sums, &tot);
    for (int i = beg; i < end; i++) {
        int v = a[i];
        a[i] = off;
        off += v;
    }
    T.sync();
    return tot;
}

// Iteration order of a std::unordered_map filled by inserting distinct elements 0..m-1 in order
// (stage method, see the file comment). code(e) is the element's hash. Writes ord[m].
// Scratch: tim, pos, ebk, nxt (m each), ctm, bsz, hed (buckets), arr (m+1).
template <class Code>
__device__ void map_order(const Team &T, int m, Code code, int *tim, int *pos, int *ebk, int *nxt, int *ctm, int *bsz,
                          int *hed, int *arr, int *ord, int *warp_sums) {
    int stage = 0;
    while (stage < kSchedLen && sched_at(stage) <= (uint64_t)m) {
        const int r = (int)sched_at(stage);
        const uint64_t beta = sched_bkt(stage);
        const int end = (stage + 1 < kSchedLen && sched_at(stage + 1) <= (uint64_t)m) ? (int)sched_at(stage + 1) - 1 : m;
        for (int e = T.tid; e < end; e += T.size) tim[e] = (stage == 0 || e >= r - 1) ? e : pos[e];
        for (uint64_t b = T.tid; b < beta; b += T.size) {
            ctm[b] = INT32_MAX;
            bsz[b] = 0;
            hed[b] = -1;
        }
        for (int t = T.tid; t < end; t += T.size) arr[t] = 0;
        T.sync();
        for (int e = T.tid; e < end; e += T.size) {
            int b = (int)(code(e) % beta);
            ebk[e] = b;
            atomicMin(&ctm[b], tim[e]);
            atomicAdd(&bsz[b], 1);
            nxt[e] = atomicExch(&hed[b], e);
        }
        T.sync();
        // arr[end-1-t] = size of the run whose bucket was created at time t.
        for (int e = T.tid; e < end; e += T.size) {
            int b = ebk[e];
            if (ctm[b] == tim[e]) arr[end - 1 - tim[e]] = bsz[b];
        }
        T.sync();
        team_scan_array(T, arr, end, warp_sums);  // arr[end-1-t] = nodes in runs created after t
        for (int e = T.tid; e < end; e += T.size) {
            int b = ebk[e], te = tim[e];
            int rank = 0, guard = 0;
            for (int x = hed[b]; x >= 0 && guard <= end; x = nxt[x], guard++)
                if (tim[x] > te) rank++;
            pos[e] = arr[end - 1 - ctm[b]] + rank;
        }
        T.sync();
        stage++;
    }
    for (int e = T.tid; e < m; e += T.size) ord[pos[e]] = e;
    T.sync();
}

struct ExactGroup {
    SampleBox box;
    uint32_t n;
};

// Shared-memory layout for groups of up to `cap` samples (offsets in bytes). The distinct
// entries and the AB map order persist; the sampling/de-duplication arrays and the later stage and
// qb_map arrays share one region.
struct Layout {
    uint32_t tcap, bmax;
    uint32_t ekey, ecnt, ord;                         // persistent
    uint32_t key, tkey, tfirst, tcnt, sslot;          // phase 1-3
    uint32_t tim, pos, ebk, nxt, ctm, bsz, hed, arr;  // phase 4-7 (stage scratch)
    uint32_t qtab, qfirst, qsum, qslot, qval, qc, qord;
    uint32_t total;
    __host__ __device__ Layout(uint32_t cap) {
        tcap = 16;
        while (tcap < 2 * cap) tcap <<= 1;
        bmax = (uint32_t)sched_buckets(cap);
        uint32_t off = 0;
        auto take = [&](uint32_t bytes) {
            uint32_t o = off;
            off += (bytes + 15) & ~15u;
            return o;
        };
        ekey = take(8 * cap);
        ecnt = take(4 * cap);
        ord = take(4 * cap);
        const uint32_t u = off;
        key = take(8 * cap);
        tkey = take(8 * tcap);
        tfirst = take(4 * tcap);
        tcnt = take(4 * tcap);
        sslot = take(4 * cap);
        const uint32_t end_a = off;
        off = u;
        tim = take(4 * cap);
        pos = take(4 * cap);
        ebk = take(4 * cap);
        nxt = take(4 * cap);
        ctm = take(4 * bmax);
        bsz = take(4 * bmax);
        hed = take(4 * bmax);
        arr = take(4 * (cap + 1));
        qtab = take(4 * tcap);
        qfirst = take(4 * tcap);
        qsum = take(4 * tcap);
        qslot = take(4 * cap);
        qval = take(4 * cap);
        qc = take(4 * cap);
        qord = take(4 * cap);
        total = off > end_a ? off : end_a;
    }
};

constexpr int kChainWarps = 5;  // warps 0..4: one mse chain each; the rest build qb maps

// Quantised error of an entry for one evaluation (get_h_psnr.tpp:14-19 as emitted).
__device__ __forceinline__ void entry_err(uint64_t kk, float t2, float stat_eb, float neg, float eb2, int &q, float &d) {
    float af = __ll2float_rn((int64_t)(int32_t)(uint32_t)(kk >> 32)), bf = __ll2float_rn((int64_t)(int32_t)(uint32_t)kk);
    float err = __fmul_rn(__fmaf_rn(bf, 2.0f, __fmul_rn(af, t2)), stat_eb);
    int64_t q64 = lround_f(__fmul_rn(err, neg));
    q = (int)q64;
    d = __fmaf_rn(-__ll2float_rn(q64), eb2, err);
}

// Evaluations of one group: h1 and the log10f argument for each (t, abs_eb).
// Returns false if the group does not fit `cap` or has keys outside int32.
__device__ bool exact_eval(const ExactGroup &eg, const float *__restrict__ ref, const float *__restrict__ x0, uint64_t n1n2,
                           uint64_t n2, const ProxyEval *evals, int n_evals, float R2, const float *__restrict__ log2tab,
                           uint8_t *smem, uint32_t cap, float *h1_out, float *x_out, uint32_t *m_out) {
    const uint32_t n = eg.n;
    if (n > cap || blockDim.x != (unsigned)kThreads) return false;
    const Layout Lo(cap);
    __shared__ int warp_sums[2][32];
    __shared__ int flag_wide, m_sh;
    __shared__ float h1_sh[5], mse_sh[5];
    __shared__ int mq_sh;
    const Team all{(int)threadIdx.x, (int)blockDim.x, 0};
    uint64_t *key = (uint64_t *)(smem + Lo.key), *tkey = (uint64_t *)(smem + Lo.tkey), *ekey = (uint64_t *)(smem + Lo.ekey);
    int *tfirst = (int *)(smem + Lo.tfirst), *tcnt = (int *)(smem + Lo.tcnt), *sslot = (int *)(smem + Lo.sslot);
    int *ecnt = (int *)(smem + Lo.ecnt), *ord = (int *)(smem + Lo.ord);
    int *tim = (int *)(smem + Lo.tim), *pos = (int *)(smem + Lo.pos), *ebk = (int *)(smem + Lo.ebk),
        *nxt = (int *)(smem + Lo.nxt), *ctm = (int *)(smem + Lo.ctm), *bsz = (int *)(smem + Lo.bsz),
        *hed = (int *)(smem + Lo.hed), *arr = (int *)(smem + Lo.arr);
    int *qtab = (int *)(smem + Lo.qtab), *qfirst = (int *)(smem + Lo.qfirst), *qsum = (int *)(smem + Lo.qsum),
        *qslot = (int *)(smem + Lo.qslot), *qval = (int *)(smem + Lo.qval), *qc = (int *)(smem + Lo.qc),
        *qord = (int *)(smem + Lo.qord);
    if (threadIdx.x == 0) flag_wide = 0;
    const uint64_t EMPTY = 0x8000000000000000ull;  // a = INT32_MIN: rejected below, so never a key
    for (uint32_t i = threadIdx.x; i < Lo.tcap; i += blockDim.x) {
        tkey[i] = EMPTY;
        tfirst[i] = INT32_MAX;
        tcnt[i] = 0;
    }
    all.sync();
    // 1. Sample keys in get_AB_map's scan order.
    const SampleBox &b = eg.box;
    uint32_t c[3];
    for (int a = 0; a < 3; a++) c[a] = b.hi[a] > b.lo[a] ? (uint32_t)((b.hi[a] - b.lo[a] + b.step[a] - 1) / b.step[a]) : 0;
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        uint32_t k2 = s % c[2], k1 = (s / c[2]) % c[1], k0 = s / (c[1] * c[2]);
        uint64_t p = (b.lo[0] + k0 * b.step[0]) * n1n2 + (b.lo[1] + k1 * b.step[1]) * n2 + (b.lo[2] + k2 * b.step[2]);
        const uint64_t d = b.dist;
        float m1 = ref[p - d], m3 = ref[p - 3 * d], p1 = ref[p + d], p3 = ref[p + 3 * d];
        float Af = __fsub_rn(__fadd_rn(m1, p1), __fadd_rn(m3, p3));
        float S4 = __fadd_rn(__fadd_rn(p1, p3), __fadd_rn(m1, m3));
        float Bf = __double2float_rn(__fma_rn((double)S4, 0.25, -(double)x0[p]));
        int64_t ak = lround_f(__fmul_rn(Af, b.neg_2_stat_eb)), bk = lround_f(__fmul_rn(Bf, b.neg_2_stat_eb));
        if (ak <= INT32_MIN || ak > INT32_MAX || bk < INT32_MIN || bk > INT32_MAX) flag_wide = 1;
        key[s] = ((uint64_t)(uint32_t)(int32_t)ak << 32) | (uint32_t)(int32_t)bk;
    }
    all.sync();
    if (flag_wide) return false;
    // 2. De-duplicate; first occurrence and count per distinct key.
    for (uint32_t s = threadIdx.x; s < n; s += blockDim.x) {
        uint64_t k = key[s];
        uint32_t slot = (uint32_t)(mix64(k) & (Lo.tcap - 1));
        for (uint32_t probe = 0; probe < Lo.tcap; probe++) {
            unsigned long long prev = atomicCAS((unsigned long long *)&tkey[slot], (unsigned long long)EMPTY, (unsigned long long)k);
            if (prev == EMPTY || prev == k) break;
            slot = (slot + 1) & (Lo.tcap - 1);
        }
        sslot[s] = (int)slot;
        atomicMin(&tfirst[slot], (int)s);
        atomicAdd(&tcnt[slot], 1);
    }
    all.sync();
    // 3. Distinct keys in first-occurrence order.
    {
        const uint32_t per = (n + blockDim.x - 1) / blockDim.x, beg = threadIdx.x * per, end = min(beg + per, n);
        int local = 0;
        for (uint32_t s = beg; s < end; s++) local += tfirst[sslot[s]] == (int)s;
        int tot;
        int off = team_excl_scan(all, local, warp_sums[0], &tot);
        for (uint32_t s = beg; s < end; s++)
            if (tfirst[sslot[s]] == (int)s) {
                ekey[off] = key[s];
                ecnt[off] = tcnt[sslot[s]];
                off++;
            }
        if (threadIdx.x == 0) m_sh = tot;
    }
    all.sync();
    const int m = m_sh;
    if (m_out && threadIdx.x == 0) *m_out = (uint32_t)m;
    if (m == 0) return true;
    // 4. AB map order; hash = a*1145141919810 + b (asz_param.hpp:22-40).
    auto abcode = [&](int e) {
        uint64_t k = ekey[e];
        int64_t a = (int32_t)(uint32_t)(k >> 32), bb = (int32_t)(uint32_t)k;
        return (uint64_t)a * 1145141919810ull + (uint64_t)bb;
    };
    map_order(all, m, abcode, tim, pos, ebk, nxt, ctm, bsz, hed, arr, ord, warp_sums[0]);
    // 5-7. Evaluations in batches of five: warps 0-4 run the mse chains while the other warps build
    // each evaluation's qb_map and run its h1 chain.
    const float nf = __ull2float_rn((uint64_t)n), rn = __fdiv_rn(1.0f, nf);
    for (int e0 = 0; e0 < n_evals; e0 += 5) {
        const int ne = min(5, n_evals - e0);
        const int warp = threadIdx.x >> 5;
        if (warp < kChainWarps) {
            // mse chain (get_h_psnr.tpp:12-22) in map order.
            if ((threadIdx.x & 31) == 0 && warp < ne) {
                const ProxyEval ev = evals[e0 + warp];
                const float neg = __fdiv_rn(0.5f, ev.abs_eb), t2 = __fadd_rn(ev.t, ev.t), eb2 = __fadd_rn(ev.abs_eb, ev.abs_eb);
                float mse = 0.0f;
                for (int k = 0; k < m; k++) {
                    const int e = ord[k];
                    int q;
                    float dv;
                    entry_err(ekey[e], t2, b.stat_eb, neg, eb2, q, dv);
                    double dd = (double)dv;
                    mse = __double2float_rn(__fma_rn((double)ecnt[e], __dmul_rn(dd, dd), (double)mse));
                }
                mse_sh[warp] = mse;
            }
        } else {
            const Team qt{(int)threadIdx.x - kChainWarps * 32, (int)blockDim.x - kChainWarps * 32, 1};
            for (int j = 0; j < ne; j++) {
                const ProxyEval ev = evals[e0 + j];
                const float neg = __fdiv_rn(0.5f, ev.abs_eb), t2 = __fadd_rn(ev.t, ev.t), eb2 = __fadd_rn(ev.abs_eb, ev.abs_eb);
                for (uint32_t i = qt.tid; i < Lo.tcap; i += qt.size) {
                    qtab[i] = INT32_MIN;
                    qfirst[i] = INT32_MAX;
                    qsum[i] = 0;
                }
                qt.sync();
                // Distinct q values, first occurrence in map order, summed counts.
                for (int k = qt.tid; k < m; k += qt.size) {
                    const int e = ord[k];
                    int q;
                    float dv;
                    entry_err(ekey[e], t2, b.stat_eb, neg, eb2, q, dv);
                    uint32_t slot = (uint32_t)(mix64((uint64_t)(uint32_t)q) & (Lo.tcap - 1));
                    for (uint32_t probe = 0; probe < Lo.tcap; probe++) {
                        int prev = atomicCAS(&qtab[slot], INT32_MIN, q);
                        if (prev == INT32_MIN || prev == q) break;
                        slot = (slot + 1) & (Lo.tcap - 1);
                    }
                    qslot[k] = (int)slot;
                    atomicMin(&qfirst[slot], k);
                    atomicAdd(&qsum[slot], ecnt[e]);
                }
                qt.sync();
                {
                    const int per = (m + qt.size - 1) / qt.size, beg = qt.tid * per, end = min(beg + per, m);
                    int local = 0;
                    for (int k = beg; k < end; k++) local += qfirst[qslot[k]] == k;
                    int tot;
                    int off = team_excl_scan(qt, local, warp_sums[1], &tot);
                    for (int k = beg; k < end; k++)
                        if (qfirst[qslot[k]] == k) {
                            qval[off] = qtab[qslot[k]];
                            qc[off] = qsum[qslot[k]];
                            off++;
                        }
                    if (qt.tid == 0) mq_sh = tot;
                }
                qt.sync();
                const int mq = mq_sh;
                auto qcode = [&](int e) { return (uint64_t)(int64_t)qval[e]; };
                map_order(qt, mq, qcode, tim, pos, ebk, nxt, ctm, bsz, hed, arr, qord, warp_sums[1]);
                // h1 chain (get_h_psnr.tpp:23-28).
                if (qt.tid == 0) {
                    float h1 = 0.0f;
                    for (int k = 0; k < mq; k++) {
                        int cnt = qc[qord[k]];
                        float pr = __fmul_rn(__ull2float_rn((uint64_t)cnt), rn);
                        h1 = __fmaf_rn(-pr, log2tab[cnt], h1);
                    }
                    h1_sh[j] = h1;
                }
                qt.sync();
            }
        }
        all.sync();
        if ((int)threadIdx.x < ne) {
            h1_out[e0 + threadIdx.x] = h1_sh[threadIdx.x];
            x_out[e0 + threadIdx.x] = __fmul_rn(__fdiv_rn(R2, mse_sh[threadIdx.x]), nf);
        }
        all.sync();
    }
    return true;
}

__device__ __forceinline__ float step_ulps(float v, int k) {
    int32_t b = __float_as_int(v);
    if (v == 0.0f) return k > 0 ? __int_as_float(k) : -__int_as_float(-k);
    if (b >= 0) return __int_as_float(b + k);
    return __int_as_float(b - k);
}

struct Band {
    float mid, lo, hi;
};
__device__ Band psnr_band(float x) {
    Band p;
    if (!(x > 0.0f) || isinf(x) || isnan(x)) {
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

}  // namespace

// Exact t selection for the listed groups of round l; groups that do not fit the arena go to
// `spill` for the serial kernel.
// Exact replay of group g of one field and round (compress.tpp:91-144 in the maps' order). The
// caller's spill(g) receives a group too large for shared memory (thread 0).
template <class Spill>
__device__ void exact_one(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *__restrict__ classes,
                          const float *__restrict__ rec, const float *__restrict__ orig, const float *__restrict__ log2arena,
                          float R2, float t_default, float *__restrict__ tval, int64_t *__restrict__ t_int, uint32_t *fb_count,
                          AmbiguousRecord *amb, uint32_t amb_cap, uint32_t *amb_count, const uint32_t *__restrict__ overrides,
                          uint32_t n_overrides, float *__restrict__ proxies, uint64_t g, uint8_t *smem, uint32_t cap,
                          float *h1v, float *xv, uint32_t &m_sh, const Spill &spill) {
    const uint64_t nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    const float cand[5] = {1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
    if (g >= nblocks) return;
    const uint64_t b2 = g % fg.block_num[2], b1 = (g / fg.block_num[2]) % fg.block_num[1],
                   b0 = g / (fg.block_num[1] * fg.block_num[2]);
    const uint64_t bb[3] = {b0, b1, b2};
    const int cls = (class_of(b0, fg.block_num[0]) * 3 + class_of(b1, fg.block_num[1])) * 3 + class_of(b2, fg.block_num[2]);
    const ClassInfo ci = classes[cls];
    const int d = rg.dir;
    ExactGroup eg;
    for (int a = 0; a < 3; a++) {
        uint64_t lo = fg.origin[a] + bb[a] * fg.block_shape[a];
        uint64_t hi = min(fg.origin[a] + (bb[a] + 1) * fg.block_shape[a] + 1, fg.n[a]);
        if (a != d && lo != 0) lo += rg.stride[a];
        if (a == d) {
            lo += 3 * rg.stride[a] / 2;
            hi -= 3 * rg.stride[a] / 2;
        }
        eg.box.lo[a] = lo;
        eg.box.hi[a] = hi;
        eg.box.step[a] = rg.stride[a] * ci.ss;
    }
    eg.box.dist = rg.dist;
    eg.box.neg_2_stat_eb = rg.neg_2_stat_eb;
    eg.box.stat_eb = rg.stat_eb;
    eg.n = ci.n;
    ProxyEval ev[5];
    for (int c = 0; c < 5; c++) ev[c] = ProxyEval{cand[c], rg.eb};
    if (threadIdx.x == 0) m_sh = 0;
    __syncthreads();
    bool ok = exact_eval(eg, rec, orig, fg.n[1] * fg.n[2], fg.n[2], ev, 5, R2, log2arena + ci.log2_off, smem, cap, h1v,
                         xv, &m_sh);
    __syncthreads();
    if (!ok) {
        if (threadIdx.x == 0) spill(g);
        __syncthreads();
        return;
    }
    if (threadIdx.x == 0) {
        float best_t = t_default;
        bool fb = m_sh == 0;
        bool forced = false;
        for (uint32_t i = 0; i < n_overrides; i++)
            if (overrides[3 * i] == (uint32_t)g && overrides[3 * i + 1] == l) {
                forced = true;
                best_t = __uint_as_float(overrides[3 * i + 2]);
            }
        if (!fb && !forced) {
            if (proxies)
                for (int c = 0; c < 5; c++) {
                    proxies[g * 10 + c] = h1v[c];
                    proxies[g * 10 + 5 + c] = xv[c];
                }
            int best = 1;
            bool ambiguous = false;
            for (int c = 0; c < 5; c++) {
                if (cand[c] == cand[best]) continue;
                float d_h1 = __fsub_rn(h1v[best], h1v[c]);
                bool accept;
                if (__float_as_uint(xv[c]) == __float_as_uint(xv[best]) && isfinite(xv[c]) && xv[c] > 0.0f) {
                    accept = __fmaf_rn(d_h1, rg.slope, 0.0f) > 0.0f;
                } else {
                    Band pc = psnr_band(xv[c]), pb = psnr_band(xv[best]);
                    float s_mid = __fmaf_rn(d_h1, rg.slope, __fsub_rn(pc.mid, pb.mid));
                    float s_lo = __fmaf_rn(d_h1, rg.slope, __fsub_rn(pc.lo, pb.hi));
                    float s_hi = __fmaf_rn(d_h1, rg.slope, __fsub_rn(pc.hi, pb.lo));
                    if (!((s_lo > 0.0f) || !(s_hi > 0.0f))) ambiguous = true;
                    accept = s_mid > 0.0f;
                }
                if (accept) best = c;
            }
            best_t = cand[best];
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
        if (fb) atomicAdd(fb_count, 1u);
        tval[g] = best_t;
        t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(best_t, (float)fg.t_precision));
    }
    __syncthreads();
}

struct ListSpill {
    uint32_t *list, *count;
    __device__ void operator()(uint64_t g) const { list[atomicAdd(count, 1u)] = (uint32_t)g; }
};

__global__ void __launch_bounds__(kThreads)
    tsel_exact_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const ClassInfo *__restrict__ classes,
                      const float *__restrict__ rec, const float *__restrict__ orig, const float *__restrict__ log2arena,
                      float R2, float t_default, float *__restrict__ tval, int64_t *__restrict__ t_int,
                      uint32_t *__restrict__ fb_count, AmbiguousRecord *amb, uint32_t amb_cap, uint32_t *amb_count,
                      const uint32_t *__restrict__ overrides, uint32_t n_overrides, float *__restrict__ proxies,
                      const uint32_t *__restrict__ list, const uint32_t *__restrict__ list_count, uint32_t *spill,
                      uint32_t *spill_count, uint32_t smem_bytes, uint32_t cap) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t items = *list_count;
    __shared__ float h1v[kMaxEvals], xv[kMaxEvals];
    __shared__ uint32_t m_sh;
    const ListSpill sp{spill, spill_count};
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x)
        exact_one(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int, fb_count, amb, amb_cap, amb_count,
                  overrides, n_overrides, proxies, list[it], smem, cap, h1v, xv, m_sh, sp);
}

// Batched form: the (field << 32 | group) entries that the batched fast path handed off, for all
// fields of a batch at once; spills go to one list of entries of the same form.
struct PairSpill {
    unsigned long long *list;
    uint32_t *count;
    uint32_t f;
    __device__ void operator()(uint64_t g) const { list[atomicAdd(count, 1u)] = ((unsigned long long)f << 32) | g; }
};

__global__ void __launch_bounds__(kThreads)
    tsel_exact_batch_kernel(const BatchField *__restrict__ F, uint32_t l, const float *__restrict__ log2arena,
                            float t_default, const unsigned long long *__restrict__ list, const uint32_t *__restrict__ list_count,
                            unsigned long long *spill, uint32_t *spill_count, uint32_t cap) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t items = *list_count;
    __shared__ float h1v[kMaxEvals], xv[kMaxEvals];
    __shared__ uint32_t m_sh;
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
        const unsigned long long e = list[it];
        const uint32_t f = (uint32_t)(e >> 32);
        const BatchField &B = F[f];
        const uint64_t nb = B.fg.block_num[0] * B.fg.block_num[1] * B.fg.block_num[2];
        const PairSpill sp{spill, spill_count, f};
        exact_one(B.fg, B.rounds[l], l, B.classes + 27 * l, B.rec, B.in, log2arena, B.R2, t_default, B.tval, B.tint, &B.cnt->fb,
                  B.amb, B.amb_cap, &B.cnt->amb_count, nullptr, 0, B.proxies ? B.proxies + nb * l * 10 : nullptr,
                  e & 0xffffffffull, smem, cap, h1v, xv, m_sh, sp);
    }
}

// Batched form of tsel_exact_global_kernel: the entries the batched exact kernel spilled (groups
// above its shared-memory capacity), a CTA per group in its slice of global scratch; what this
// cannot take (keys outside int32) goes on to `spill` for the serial kernel.
__global__ void __launch_bounds__(kThreads)
    tsel_exact_global_batch_kernel(const BatchField *__restrict__ F, uint32_t l, const float *__restrict__ log2arena,
                                   float t_default, const unsigned long long *__restrict__ list,
                                   const uint32_t *__restrict__ list_count, unsigned long long *spill, uint32_t *spill_count,
                                   uint8_t *scratch, uint64_t stride, uint32_t cap) {
    uint8_t *mine = scratch + blockIdx.x * stride;
    const uint32_t items = *list_count;
    __shared__ float h1v[kMaxEvals], xv[kMaxEvals];
    __shared__ uint32_t m_sh;
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
        const unsigned long long e = list[it];
        const uint32_t f = (uint32_t)(e >> 32);
        const BatchField &B = F[f];
        const uint64_t nb = B.fg.block_num[0] * B.fg.block_num[1] * B.fg.block_num[2];
        const PairSpill sp{spill, spill_count, f};
        exact_one(B.fg, B.rounds[l], l, B.classes + 27 * l, B.rec, B.in, log2arena, B.R2, t_default, B.tval, B.tint, &B.cnt->fb,
                  B.amb, B.amb_cap, &B.cnt->amb_count, nullptr, 0, B.proxies ? B.proxies + nb * l * 10 : nullptr,
                  e & 0xffffffffull, mine, cap, h1v, xv, m_sh, sp);
    }
}

__global__ void __launch_bounds__(kThreads)
    slope_exact_kernel(const SampleBox *__restrict__ boxes, const ProxyEval *__restrict__ evals, uint32_t n_evals,
                       const float *__restrict__ orig, uint64_t n1n2, uint64_t n2, const float *__restrict__ log2arena,
                       float R2, float *__restrict__ h1_out, float *__restrict__ x_out, uint32_t *__restrict__ m_out,
                       uint32_t *__restrict__ err_word, uint32_t smem_bytes, uint32_t cap) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ float h1v[kMaxEvals], xv[kMaxEvals];
    // Box blockIdx.x, evaluations [5 * blockIdx.y, 5 * blockIdx.y + 5): exact_eval runs five
    // evaluations side by side, so each CTA rebuilds the box's map and runs one batch of them.
    const uint32_t g = blockIdx.x, e0 = 5 * blockIdx.y;
    if (e0 >= n_evals) return;
    const uint32_t ne = min(5u, n_evals - e0);
    ExactGroup eg;
    eg.box = boxes[g];
    eg.n = eg.box.n;
    uint32_t m = 0;
    bool ok = exact_eval(eg, orig, orig, n1n2, n2, evals + e0, (int)ne, R2, log2arena + eg.box.log2_off, smem, cap, h1v, xv, &m);
    __syncthreads();
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(err_word, 2u);
        return;
    }
    if (threadIdx.x == 0 && blockIdx.y == 0) m_out[g] = m;
    for (uint32_t e = threadIdx.x; e < ne; e += blockDim.x) {
        h1_out[g * n_evals + e0 + e] = h1v[e];
        x_out[g * n_evals + e0 + e] = xv[e];
    }
}

// The same exact replay for groups larger than shared memory holds: each CTA works in its own
// slice of a global scratch arena (stride bytes, L2-resident) instead of shared memory, so a group
// of up to `cap` samples is still replayed by a whole CTA rather than by one thread. Groups it
// cannot take (more samples than cap, keys outside int32) go to `spill` for the serial kernel.
__global__ void __launch_bounds__(kThreads)
    tsel_exact_global_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const ClassInfo *__restrict__ classes,
                             const float *__restrict__ rec, const float *__restrict__ orig,
                             const float *__restrict__ log2arena, float R2, float t_default, float *__restrict__ tval,
                             int64_t *__restrict__ t_int, uint32_t *__restrict__ fb_count, AmbiguousRecord *amb,
                             uint32_t amb_cap, uint32_t *amb_count, const uint32_t *__restrict__ overrides,
                             uint32_t n_overrides, float *__restrict__ proxies, const uint32_t *__restrict__ list,
                             const uint32_t *__restrict__ list_count, uint32_t *spill, uint32_t *spill_count,
                             uint8_t *scratch, uint64_t stride, uint32_t cap) {
    uint8_t *mine = scratch + blockIdx.x * stride;
    const uint32_t items = *list_count;
    __shared__ float h1v[kMaxEvals], xv[kMaxEvals];
    __shared__ uint32_t m_sh;
    const ListSpill sp{spill, spill_count};
    for (uint32_t it = blockIdx.x; it < items; it += gridDim.x)
        exact_one(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int, fb_count, amb, amb_cap, amb_count,
                  overrides, n_overrides, proxies, list[it], mine, cap, h1v, xv, m_sh, sp);
}

__global__ void __launch_bounds__(kThreads)
    slope_exact_global_kernel(const SampleBox *__restrict__ boxes, const ProxyEval *__restrict__ evals, uint32_t n_evals,
                              const float *__restrict__ orig, uint64_t n1n2, uint64_t n2,
                              const float *__restrict__ log2arena, float R2, float *__restrict__ h1_out,
                              float *__restrict__ x_out, uint32_t *__restrict__ m_out, uint32_t *__restrict__ err_word,
                              uint8_t *scratch, uint64_t stride, uint32_t cap) {
    __shared__ float h1v[kMaxEvals], xv[kMaxEvals];
    const uint32_t g = blockIdx.x;
    ExactGroup eg;
    eg.box = boxes[g];
    eg.n = eg.box.n;
    bool ok = exact_eval(eg, orig, orig, n1n2, n2, evals, (int)n_evals, R2, log2arena + eg.box.log2_off,
                         scratch + g * stride, cap, h1v, xv, m_out + g);
    __syncthreads();
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(err_word, 2u);
        return;
    }
    for (uint32_t e = threadIdx.x; e < n_evals; e += blockDim.x) {
        h1_out[g * n_evals + e] = h1v[e];
        x_out[g * n_evals + e] = xv[e];
    }
}

// Shared-memory bytes the exact kernels need for groups of up to `cap` samples (also the size of
// a global-scratch slice).
uint32_t exact_smem_bytes(uint32_t cap) { return Layout(cap).total; }

cudaError_t launch_tsel_exact_global(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes,
                                     const float *rec, const float *orig, const float *log2arena, float R2, float t_default,
                                     float *tval, int64_t *t_int, uint32_t *fb_count, AmbiguousRecord *amb, uint32_t amb_cap,
                                     uint32_t *amb_count, const uint32_t *overrides, uint32_t n_overrides, float *proxies,
                                     const uint32_t *list, const uint32_t *list_count, uint32_t *spill, uint32_t *spill_count,
                                     uint8_t *scratch, uint64_t stride, uint32_t cap, unsigned grid, cudaStream_t st) {
    if (grid == 0) return cudaSuccess;
    tsel_exact_global_kernel<<<grid, kThreads, 0, st>>>(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int,
                                                        fb_count, amb, amb_cap, amb_count, overrides, n_overrides, proxies,
                                                        list, list_count, spill, spill_count, scratch, stride, cap);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_slope_exact_global(const SampleBox *boxes, const ProxyEval *evals, uint32_t n_evals, const float *orig,
                                      uint64_t n1n2, uint64_t n2, const float *log2arena, float R2, float *h1, float *x,
                                      uint32_t *m_out, uint32_t *err, uint8_t *scratch, uint64_t stride, uint32_t cap,
                                      uint32_t nboxes, cudaStream_t st) {
    if (nboxes == 0) return cudaSuccess;
    slope_exact_global_kernel<<<nboxes, kThreads, 0, st>>>(boxes, evals, n_evals, orig, n1n2, n2, log2arena, R2, h1, x, m_out,
                                                           err, scratch, stride, cap);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_tsel_exact(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                              const float *orig, const float *log2arena, float R2, float t_default, float *tval,
                              int64_t *t_int, uint32_t *fb_count, AmbiguousRecord *amb, uint32_t amb_cap,
                              uint32_t *amb_count, const uint32_t *overrides, uint32_t n_overrides, float *proxies,
                              const uint32_t *list, const uint32_t *list_count, uint32_t *spill, uint32_t *spill_count,
                              uint32_t cap, unsigned grid, cudaStream_t st) {
    uint32_t smem = exact_smem_bytes(cap);
    cudaError_t e = cudaFuncSetAttribute(tsel_exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    tsel_exact_kernel<<<grid, kThreads, smem, st>>>(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int,
                                                     fb_count, amb, amb_cap, amb_count, overrides, n_overrides, proxies, list,
                                                     list_count, spill, spill_count, smem, cap);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_tsel_exact_global_batch(const BatchField *F, uint32_t l, const float *log2arena, float t_default,
                                           const unsigned long long *list, const uint32_t *list_count,
                                           unsigned long long *spill, uint32_t *spill_count, uint8_t *scratch, uint64_t stride,
                                           uint32_t cap, unsigned grid, cudaStream_t st) {
    if (grid == 0) return cudaSuccess;
    tsel_exact_global_batch_kernel<<<grid, kThreads, 0, st>>>(F, l, log2arena, t_default, list, list_count, spill, spill_count,
                                                              scratch, stride, cap);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_tsel_exact_batch(const BatchField *F, uint32_t l, const float *log2arena, float t_default,
                                    const unsigned long long *list, const uint32_t *list_count, unsigned long long *spill,
                                    uint32_t *spill_count, uint32_t cap, unsigned grid, cudaStream_t st) {
    uint32_t smem = exact_smem_bytes(cap);
    cudaError_t e = cudaFuncSetAttribute(tsel_exact_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    tsel_exact_batch_kernel<<<grid, kThreads, smem, st>>>(F, l, log2arena, t_default, list, list_count, spill, spill_count, cap);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_slope_exact(const SampleBox *boxes, const ProxyEval *evals, uint32_t n_evals, const float *orig,
                               uint64_t n1n2, uint64_t n2, const float *log2arena, float R2, float *h1, float *x,
                               uint32_t *m_out, uint32_t *err, uint32_t cap, uint32_t nboxes, cudaStream_t st) {
    if (nboxes == 0) return cudaSuccess;
    uint32_t smem = exact_smem_bytes(cap);
    cudaError_t e = cudaFuncSetAttribute(slope_exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(nboxes, (n_evals + 4) / 5);
    slope_exact_kernel<<<grid, kThreads, smem, st>>>(boxes, evals, n_evals, orig, n1n2, n2, log2arena, R2, h1, x, m_out, err,
                                                  smem, cap);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz
