// CPU oracle: a restatement of the ASZ reference compression path, used only as a checker.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// load this library, and only to check or time against it. The product never links it.
//
// Scope: the plain path with a given plan and predictor family. That is the default-slope
// proxy, the per-(block, round) coefficient choice, the 1D4R/1D6R rounds with in-place
// reconstruction, the QB reorder, Huffman coding, stream assembly, zstd and decompression.
//
// Floating point. The reference is built with -Ofast -march=native -mavx2 -mfma
// (c_codes/CMakeLists.txt:12). The operation order and FMA contraction below were read from
// the code GCC 13.3 emits for the reference's sources, compiled here. Each fused step is an
// explicit fma()/fmaf() and every other step is a single IEEE operation. This file is built
// with -ffp-contract=off so the compiler adds nothing. Under -Ofast (-ffinite-math-only) GCC
// drops the reference's `psnr==INFINITY` tests (compress.tpp:131,136;
// get_default_slope.tpp:33), so they are absent here as well.
//
// Hash-table order. The proxies sum floats while iterating std::unordered_map, so their results
// depend on libstdc++'s iteration order. The restatement uses the same containers with the same
// hash (asz_param.hpp:22-40), key types and insertion sequence, so its order is the reference's.
#include "asz_oracle.h"
#include "zstd_decls.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <immintrin.h>
#include <limits>
#include <map>
#include <queue>
#include <stack>
#include <stdexcept>
#include <string>
#include <random>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace {

using std::vector;
using u64 = uint64_t;
using i64 = int64_t;
using qb_t = int32_t;

// asz_param.hpp:22-40: h = a*1145141919810 + b in wrapping 64-bit arithmetic.
struct ab_hash {
    size_t operator()(const std::tuple<i64, i64> &t) const {
        u64 h = (u64)std::get<0>(t);
        h = h * 1145141919810ull + (u64)std::get<1>(t);
        return (size_t)h;
    }
};
using ab_map = std::unordered_map<std::tuple<i64, i64>, u64, ab_hash>;

// llround of a float as GCC expands it under -Ofast: trunc(x + copysign(0.49999997f, x)).
static inline i64 lround_f(float x) {
    float h = std::copysign(0x1.fffffep-2f, x);
    float s = x + h;
    return (i64)s;
}
// Same for double: trunc(x + copysign(0.49999999999999994, x)).
static inline i64 lround_d(double x) {
    double h = std::copysign(0x1.fffffffffffffp-2, x);
    double s = x + h;
    return (i64)s;
}

// Quintic 1D6R weights (asz_param.hpp:72-74).
constexpr double QA = 3.0 / 256, QB = -25.0 / 256, QI = 0.5 - QA - QB;

struct field {
    u64 n[3];
    u64 size() const { return n[0] * n[1] * n[2]; }
    u64 pos(u64 i0, u64 i1, u64 i2) const { return i0 * n[1] * n[2] + i1 * n[2] + i2; }
};

// get_AB_map.tpp:7-24 (sample set and key quantisation).
template <class LOC, class STR>
void get_ab_map(ab_map &m, const float *d, const field &f, const LOC &loc, const STR &stride, u64 dist,
                float neg_2_stat_eb, u64 h1num) {
    u64 vol = (loc[0][1] - loc[0][0]) * (loc[1][1] - loc[1][0]) * (loc[2][1] - loc[2][0]);
    float q = (float)vol / (float)(stride[0] * stride[1] * stride[2] * h1num);
    u64 ss = (u64)std::cbrt((double)q);
    if (ss == 0) ss = 1;
    for (u64 i0 = loc[0][0]; i0 < loc[0][1]; i0 += stride[0] * ss)
        for (u64 i1 = loc[1][0]; i1 < loc[1][1]; i1 += stride[1] * ss)
            for (u64 i2 = loc[2][0]; i2 < loc[2][1]; i2 += stride[2] * ss) {
                u64 p = f.pos(i0, i1, i2);
                float m1 = d[p - dist], m3 = d[p - 3 * dist], p1 = d[p + dist], p3 = d[p + 3 * dist];
                float A = (m1 + p1) - (m3 + p3);
                float S4 = (p1 + p3) + (m1 + m3);
                float B = (float)std::fma((double)S4, 0.25, -(double)d[p]);
                i64 ak = lround_f(A * neg_2_stat_eb);
                i64 bk = lround_f(B * neg_2_stat_eb);
                m[{ak, bk}]++;
            }
}

// get_h_psnr.tpp:6-31. Returns also the log10f argument and the float sum for callers
// that need them.
void get_h1_psnr(float &h1, float &psnr, const ab_map &m, float t, float abs_eb, float stat_eb,
                 float min_val, float max_val, float *x_out = nullptr, float *mse_out = nullptr) {
    float neg_2_eb = 0.5f / abs_eb;
    float t2 = t + t, eb2 = abs_eb + abs_eb;
    std::unordered_map<i64, u64> qb_map;
    float mse = 0;
    u64 n = 0;
    for (const auto &[key, cnt] : m) {
        float af = (float)std::get<0>(key), bf = (float)std::get<1>(key);
        float err = std::fmaf(bf, 2.0f, af * t2) * stat_eb;
        i64 qb = lround_f(err * neg_2_eb);
        qb_map[qb] += cnt;
        float de = std::fmaf(-(float)qb, eb2, err);
        mse = (float)std::fma((double)cnt, (double)de * (double)de, (double)mse);
        n += cnt;
    }
    float nf = (float)n;
    h1 = 0;
    if (!qb_map.empty()) {
        float r = 1.0f / nf;
        for (const auto &[qb, freq] : qb_map) {
            float p = (float)freq * r;
            float L = log2f(p);
            h1 = std::fmaf(-p, L, h1);
        }
    }
    float R = max_val - min_val;
    float x = (R * R / mse) * nf;
    psnr = 10.0f * log10f(x);
    if (x_out) *x_out = x;
    if (mse_out) *mse_out = mse;
}

struct params_t {
    aszo_params p;
    vector<float> candidate_t, block_candidate_t;
    void init(const aszo_params &pp) {
        p = pp;
        candidate_t.clear();
        int lo = (int)llround(p.t_min * p.t_precision), hi = (int)llround(p.t_max * p.t_precision);
        for (int ti = lo; ti <= hi; ti++) candidate_t.push_back((float)ti / p.t_precision);
        block_candidate_t = {1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
    }
};

// get_default_slope.tpp:6-83.
float default_slope(const float *data, const field &f, float abs_eb, float min_val, float max_val,
                    const params_t &P) {
    const aszo_params &p = P.p;
    float ebs[2] = {abs_eb * p.default_slope_eb_span, abs_eb / p.default_slope_eb_span};
    float two_stat = abs_eb * p.stat_eb_ratio;
    float stat_eb = two_stat * 0.5f;
    float neg_2_stat_eb = 1.0f / two_stat;
    float avg_h1[2] = {0, 0}, avg_psnr[2] = {0, 0};
    u64 valid[2] = {0, 0};
    for (int dir = 0; dir < 3; dir++) {
        std::array<std::array<u64, 2>, 3> loc = {{{0, f.n[0]}, {0, f.n[1]}, {0, f.n[2]}}};
        loc[dir] = {3, f.n[dir] - 3};
        std::array<u64, 3> stride = {1, 1, 1};
        stride[dir] = 2;
        u64 dist = 1;
        for (int a = dir + 1; a < 3; a++) dist *= f.n[a];
        ab_map m;
        get_ab_map(m, data, f, loc, stride, dist, neg_2_stat_eb, p.h1_block_sampling_num);
        if (m.empty()) throw std::runtime_error("default slope: empty AB map");
        for (int i = 0; i < 2; i++)
            for (float t : P.candidate_t) {
                float h1, psnr;
                get_h1_psnr(h1, psnr, m, t, ebs[i], stat_eb, min_val, max_val);
                avg_h1[i] += h1;
                avg_psnr[i] += psnr;
                valid[i]++;
            }
    }
    u64 total = 3 * P.candidate_t.size();
    float recip = 1.0f / (float)total;
    float max_invalid = 0;
    for (int i = 0; i < 2; i++) {
        float inv = std::fmaf(-recip, (float)valid[i], 1.0f);
        max_invalid = std::max(inv, max_invalid);
    }
    if (max_invalid >= p.default_slope_invalid_ratio_threshold) return p.default_slope_fallback;
    // The tolerance scale uses the vectorised approximate reciprocal plus one Newton step that
    // GCC emits for average_h1[i]/=valid_case_num[i]; the differences use exact divisions.
    __m128 v = _mm_set_ps(1.0f, 1.0f, (float)valid[1], (float)valid[0]);
    __m128 r0 = _mm_rcp_ps(v);
    __m128 r1 = _mm_sub_ps(_mm_add_ps(r0, r0), _mm_mul_ps(r0, _mm_mul_ps(r0, v)));
    alignas(16) float rr[4];
    _mm_store_ps(rr, r1);
    float h1v0 = avg_h1[0] * rr[0], h1v1 = avg_h1[1] * rr[1];
    float h1_0 = avg_h1[0] / (float)valid[0], h1_1 = avg_h1[1] / (float)valid[1];
    float ps_0 = avg_psnr[0] / (float)valid[0], ps_1 = avg_psnr[1] / (float)valid[1];
    float h1_diff = h1_1 - h1_0, psnr_diff = ps_1 - ps_0;
    float scale = std::max(std::fabs(h1v1), std::fabs(h1v0));
    float tol = scale > 1.0f ? scale * 0x1p-17f : 0x1p-17f;
    // Ordered compares, as emitted: a NaN difference does not select the fallback.
    if (tol >= h1_diff || 0.0f >= psnr_diff) return p.default_slope_fallback;
    return psnr_diff / h1_diff;
}

struct codec {
    field f;
    params_t P;
    bool quintic = false;
    vector<std::string> plan;
    std::array<u64, 3> pivot_stride{}, block_shape{}, block_num{};
    float min_val = 0, max_val = 0, abs_eb = 0, default_slope_v = 0;
    const float *data = nullptr;
    vector<float> cd;  // compressed_data (in-place reconstruction)
    vector<vector<qb_t>> qbs;
    vector<i64> t_int;
    u64 t_fallback = 0;
    const int64_t *t_given = nullptr;  // block-major t codes to use instead of the selection

    void geometry() {  // generate_config.tpp:52-68
        pivot_stride = {1, 1, 1};
        for (auto &pr : plan) pivot_stride[pr[5] - '0'] *= 2;
        for (int a = 0; a < 3; a++) {
            block_shape[a] = pivot_stride[a] * P.p.block_pivot_ratio;
            block_num[a] = (f.n[a] + block_shape[a] - 1) / block_shape[a];
        }
    }

    // compress.tpp:91-144.
    float select_t(int dir, const std::array<std::array<u64, 2>, 3> &loc, const std::array<u64, 3> &stride,
                   float layer_eb, float slope, bool &fb) {
        fb = false;
        float best_t = P.p.insufficient_sample_t;
        if (loc[dir][1] <= loc[dir][0] + 3 * stride[dir]) {
            fb = true;
            return best_t;
        }
        std::array<std::array<u64, 2>, 3> sl;
        for (int a = 0; a < 3; a++) {
            sl[a] = {loc[a][0], loc[a][1]};
            if (a != dir && loc[a][0] != 0) sl[a][0] += stride[a];
        }
        sl[dir][0] += 3 * stride[dir] / 2;
        sl[dir][1] -= 3 * stride[dir] / 2;
        u64 sdist = stride[dir] / 2;
        for (int a = dir + 1; a < 3; a++) sdist *= f.n[a];
        float stat_eb = layer_eb * P.p.stat_eb_ratio;
        ab_map m;
        get_ab_map(m, cd.data(), f, sl, stride, sdist, 0.5f / stat_eb, P.p.h1_block_sampling_num);
        if (m.empty()) {
            fb = true;
            return best_t;
        }
        float best_h1, best_psnr;
        get_h1_psnr(best_h1, best_psnr, m, best_t, layer_eb, stat_eb, min_val, max_val);
        for (float c : P.block_candidate_t) {
            if (c == best_t) continue;
            float h1, psnr;
            get_h1_psnr(h1, psnr, m, c, layer_eb, stat_eb, min_val, max_val);
            float s = std::fmaf(best_h1 - h1, slope, psnr - best_psnr);
            if (s > 0) {
                best_t = c;
                best_h1 = h1;
                best_psnr = psnr;
            }
        }
        return best_t;
    }

    // compress.tpp:7-40 (prediction), and decompress.tpp:6-35 for the same stencils.
    inline float predict(u64 i, u64 hs, u64 right, u64 pos, u64 dist, float t) const {
        const float *c = cd.data();
        if (quintic && i >= 5 * hs && i + 5 * hs < right) {
            float s1 = c[pos - dist] + c[pos + dist];
            float s3 = c[pos - 3 * dist] + c[pos + 3 * dist];
            float s5 = c[pos - 5 * dist] + c[pos + 5 * dist];
            double acc = (double)s3 * QB;
            acc = std::fma((double)s1, QI, acc);
            acc = std::fma((double)s5, QA, acc);
            return (float)acc;
        }
        if (i <= hs) {
            if (i + hs >= right) return c[pos - dist];
            if (i + 3 * hs >= right) return (c[pos - dist] + c[pos + dist]) * 0.5f;
            return (std::fmaf(c[pos - dist], 3.0f, c[pos + dist] * 6.0f) - c[pos + 3 * dist]) * 0.125f;
        }
        if (i + hs >= right) return std::fmaf(c[pos - dist], 3.0f, -c[pos - 3 * dist]) * 0.5f;
        if (i + 3 * hs >= right)
            return std::fmaf(c[pos + dist], 3.0f, std::fmaf(c[pos - dist], 6.0f, -c[pos - 3 * dist])) * 0.125f;
        float s3 = c[pos - 3 * dist] + c[pos + 3 * dist];
        float s1 = c[pos - dist] + c[pos + dist];
        double td = t;
        float p1 = (float)((double)s3 * (0.25 - td));
        return (float)std::fma(0.25 + td, (double)s1, (double)p1);
    }

    // Target lattice and QB placement of one (block, round): compress.tpp:53-88.
    template <class FN>
    void for_targets(const std::array<std::array<u64, 2>, 3> &loc, const std::array<u64, 3> &stride, int dir,
                     int order, u64 &qb_base, FN fn) {
        std::array<u64, 3> left, shape;
        for (int a = 0; a < 3; a++) {
            left[a] = a == dir ? loc[a][0] + stride[a] / 2 : (loc[a][0] == 0 ? 0 : loc[a][0] + stride[a]);
            shape[a] = left[a] >= loc[a][1] ? 0 : (loc[a][1] - left[a] + stride[a] - 1) / stride[a];
        }
        u64 inner = order == 0 ? shape[0] : order == 1 ? shape[1] : 1;
        u64 dist = stride[dir] / 2;
        for (int a = dir + 1; a < 3; a++) dist *= f.n[a];
        u64 j0 = 0;
        for (u64 i0 = left[0]; i0 < loc[0][1]; i0 += stride[0], j0++) {
            u64 j1 = 0;
            for (u64 i1 = left[1]; i1 < loc[1][1]; i1 += stride[1], j1++) {
                u64 qi;
                if (order == 0) qi = (j1 * shape[2] + 0) * shape[0] + j0;
                else if (order == 1) qi = (j0 * shape[2] + 0) * shape[1] + j1;
                else qi = (j0 * shape[1] + j1) * shape[2] + 0;
                qi += qb_base;
                for (u64 i2 = left[2]; i2 < loc[2][1]; i2 += stride[2], qi += inner) {
                    u64 i = dir == 0 ? i0 : dir == 1 ? i1 : i2;
                    fn(i, stride[dir] / 2, loc[dir][1], f.pos(i0, i1, i2), dist, qi);
                }
            }
        }
        qb_base += shape[0] * shape[1] * shape[2];
    }

    u64 layer_qb_count(const std::array<std::array<u64, 2>, 3> &loc, const std::array<u64, 3> &stride, int dir) {
        u64 c = 1;
        for (int a = 0; a < 3; a++) {
            u64 left = a == dir ? loc[a][0] + stride[a] / 2 : (loc[a][0] == 0 ? 0 : loc[a][0] + stride[a]);
            c *= left >= loc[a][1] ? 0 : (loc[a][1] - left + stride[a] - 1) / stride[a];
        }
        return c;
    }

    std::array<std::array<u64, 2>, 3> block_loc(u64 b0, u64 b1, u64 b2) const {
        u64 b[3] = {b0, b1, b2};
        std::array<std::array<u64, 2>, 3> loc;
        for (int a = 0; a < 3; a++) loc[a] = {b[a] * block_shape[a], std::min((b[a] + 1) * block_shape[a] + 1, f.n[a])};
        return loc;
    }

    float layer_eb(u64 L, u64 l) const {
        return (float)((double)abs_eb * std::pow((double)P.p.eb_ratio, (double)(L - l - 1)));
    }

    // compress.tpp:147-231 (prediction part).
    void compress_core() {
        u64 N = f.size();
        cd.assign(data, data + N);
        u64 L = plan.size();
        qbs.assign(L + 1, {});
        t_int.clear();
        t_fallback = 0;
        // Pivots (compress.tpp:162-175): hoisted reciprocal 0.5/pivot_eb in double.
        float pivot_eb = abs_eb * P.p.pivot_eb_ratio;
        double peb = pivot_eb, rp = 0.5 / peb, peb2 = peb + peb;
        for (u64 i0 = 0; i0 < f.n[0]; i0 += pivot_stride[0])
            for (u64 i1 = 0; i1 < f.n[1]; i1 += pivot_stride[1])
                for (u64 i2 = 0; i2 < f.n[2]; i2 += pivot_stride[2]) {
                    u64 pos = f.pos(i0, i1, i2);
                    qb_t qb = (qb_t)lround_d((double)data[pos] * rp);
                    qbs[0].push_back(qb);
                    cd[pos] = (float)((double)qb * peb2);
                }
        for (u64 l = 0; l < L; l++) {
            u64 cnt = 0;
            for (u64 b0 = 0; b0 < block_num[0]; b0++)
                for (u64 b1 = 0; b1 < block_num[1]; b1++)
                    for (u64 b2 = 0; b2 < block_num[2]; b2++) {
                        std::array<u64, 3> stride = pivot_stride;
                        for (u64 k = 0; k < l; k++) stride[plan[k][5] - '0'] /= 2;
                        cnt += layer_qb_count(block_loc(b0, b1, b2), stride, plan[l][5] - '0');
                    }
            qbs[l + 1].assign(cnt, 0);
        }
        vector<u64> qb_base(L + 1, 0);
        for (u64 b0 = 0; b0 < block_num[0]; b0++)
            for (u64 b1 = 0; b1 < block_num[1]; b1++)
                for (u64 b2 = 0; b2 < block_num[2]; b2++) {
                    auto loc = block_loc(b0, b1, b2);
                    std::array<u64, 3> stride = pivot_stride;
                    for (u64 l = 0; l < L; l++) {
                        int dir = plan[l][5] - '0', order = plan[l][9] - '0';
                        float leb = layer_eb(L, l);
                        float slope =
                            (float)((double)default_slope_v * std::pow((double)P.p.slope_ratio, (double)((int)L - (int)l - 1)));
                        bool fb = false;
                        float t;
                        if (t_given) {
                            // A caller's t table (block-major codes): the stream stores and the
                            // decoder uses t_int / t_precision, which any code in range decodes.
                            t = (float)t_given[t_int.size()] / (float)P.p.t_precision;
                        } else {
                            t = select_t(dir, loc, stride, leb, slope, fb);
                        }
                        if (fb) t_fallback++;
                        t_int.push_back(lround_f(t * (float)P.p.t_precision));
                        // Quantisation: direction 0 multiplies by a hoisted 0.5*(1/eb); directions 1
                        // and 2 divide (compress.tpp:35 as emitted for block_compress_impl<false>).
                        double ebd = leb, eb2 = ebd + ebd, r0 = (1.0 / ebd) * 0.5;
                        vector<qb_t> &out = qbs[l + 1];
                        for_targets(loc, stride, dir, order, qb_base[l + 1],
                                    [&](u64 i, u64 hs, u64 right, u64 pos, u64 dist, u64 qi) {
                                        float pred = predict(i, hs, right, pos, dist, t);
                                        double pd = pred, diff = pd - (double)data[pos];
                                        double q = dir == 0 ? diff * r0 : (diff * 0.5) / ebd;
                                        qb_t qb = (qb_t)lround_d(q);
                                        out[qi] = qb;
                                        cd[pos] = (float)std::fma(-(double)qb, eb2, pd);
                                    });
                        stride[dir] /= 2;
                    }
                }
    }

    // The gradient tuner's open-loop samples: for every block (raster order) and round, the AB-map
    // lattice of select_t (compress.tpp:96-116 region, get_AB_map.tpp:9-17 loops) read from the
    // ORIGINAL data, recording A = (x-1 + x1) - (x-3 + x3) and B = (float)fma(S4, 0.25, -x) as
    // get_AB_map.tpp:18-19 computes them; a group that select_t would send to the fallback has none.
    void grad_samples(vector<float> &A, vector<float> &B, vector<uint64_t> &off) {
        const u64 L = plan.size();
        off.assign(1, 0);
        for (u64 b0 = 0; b0 < block_num[0]; b0++)
            for (u64 b1 = 0; b1 < block_num[1]; b1++)
                for (u64 b2 = 0; b2 < block_num[2]; b2++) {
                    auto loc = block_loc(b0, b1, b2);
                    std::array<u64, 3> stride = pivot_stride;
                    for (u64 l = 0; l < L; l++) {
                        const int dir = plan[l][5] - '0';
                        if (loc[dir][1] > loc[dir][0] + 3 * stride[dir]) {
                            std::array<std::array<u64, 2>, 3> sl;
                            for (int a = 0; a < 3; a++) {
                                sl[a] = {loc[a][0], loc[a][1]};
                                if (a != dir && loc[a][0] != 0) sl[a][0] += stride[a];
                            }
                            sl[dir][0] += 3 * stride[dir] / 2;
                            sl[dir][1] -= 3 * stride[dir] / 2;
                            u64 dist = stride[dir] / 2;
                            for (int a = dir + 1; a < 3; a++) dist *= f.n[a];
                            u64 vol = (sl[0][1] - sl[0][0]) * (sl[1][1] - sl[1][0]) * (sl[2][1] - sl[2][0]);
                            float q = (float)vol / (float)(stride[0] * stride[1] * stride[2] * P.p.h1_block_sampling_num);
                            u64 ss = (u64)std::cbrt((double)q);
                            if (ss == 0) ss = 1;
                            const float *d = data;
                            for (u64 i0 = sl[0][0]; i0 < sl[0][1]; i0 += stride[0] * ss)
                                for (u64 i1 = sl[1][0]; i1 < sl[1][1]; i1 += stride[1] * ss)
                                    for (u64 i2 = sl[2][0]; i2 < sl[2][1]; i2 += stride[2] * ss) {
                                        u64 p = f.pos(i0, i1, i2);
                                        float m1 = d[p - dist], m3 = d[p - 3 * dist], p1 = d[p + dist], p3 = d[p + 3 * dist];
                                        A.push_back((m1 + p1) - (m3 + p3));
                                        float S4 = (p1 + p3) + (m1 + m3);
                                        B.push_back((float)std::fma((double)S4, 0.25, -(double)d[p]));
                                    }
                        }
                        off.push_back(A.size());
                        stride[dir] /= 2;
                    }
                }
    }

    // decompress.tpp:79-196 (after the entropy stage).
    void decompress_core(float *out) {
        u64 N = f.size();
        cd.assign(N, 0.0f);
        u64 L = plan.size();
        float pivot_eb = abs_eb * P.p.pivot_eb_ratio;
        double peb2 = (double)pivot_eb + (double)pivot_eb;
        u64 k = 0;
        for (u64 i0 = 0; i0 < f.n[0]; i0 += pivot_stride[0])
            for (u64 i1 = 0; i1 < f.n[1]; i1 += pivot_stride[1])
                for (u64 i2 = 0; i2 < f.n[2]; i2 += pivot_stride[2]) {
                    if (k >= qbs[0].size()) throw std::runtime_error("compressed stream has too few QBs");
                    cd[f.pos(i0, i1, i2)] = (float)((double)qbs[0][k++] * peb2);
                }
        vector<float> lebs(L);
        for (u64 l = 0; l < L; l++) lebs[l] = layer_eb(L, l);
        vector<u64> qb_pos(L + 1, 0);
        u64 tp = 0;
        for (u64 b0 = 0; b0 < block_num[0]; b0++)
            for (u64 b1 = 0; b1 < block_num[1]; b1++)
                for (u64 b2 = 0; b2 < block_num[2]; b2++) {
                    auto loc = block_loc(b0, b1, b2);
                    std::array<u64, 3> stride = pivot_stride;
                    for (u64 l = 0; l < L; l++) {
                        if (tp >= t_int.size()) throw std::runtime_error("compressed stream contains too few t values");
                        float t = (float)t_int[tp++] / (float)P.p.t_precision;
                        int dir = plan[l][5] - '0', order = plan[l][9] - '0';
                        double ebd = lebs[l], eb2 = ebd + ebd;
                        const vector<qb_t> &in = qbs[l + 1];
                        u64 need = layer_qb_count(loc, stride, dir);
                        if (qb_pos[l + 1] > in.size() || need > in.size() - qb_pos[l + 1])
                            throw std::runtime_error("compressed stream has too few QBs");
                        for_targets(loc, stride, dir, order, qb_pos[l + 1],
                                    [&](u64 i, u64 hs, u64 right, u64 pos, u64 dist, u64 qi) {
                                        float pred = predict(i, hs, right, pos, dist, t);
                                        cd[pos] = (float)std::fma(-(double)in[qi], eb2, (double)pred);
                                    });
                        stride[dir] /= 2;
                    }
                }
        std::memcpy(out, cd.data(), N * sizeof(float));
    }
};

// ---------------------------------------------------------------------------------------------
// Huffman coder: huffman.hpp:17-784, restated with the same tree construction, tie-breaking,
// code assignment, DFS serialisation and LSB-first packing.
template <class T>
struct huff {
    struct node {
        u64 c = 0;
        int l = -1, r = -1;
    };
    vector<node> ht;
    bool usemp = false;
    T offset = 0;
    u64 maxval = 0, n = 0;
    unsigned mbft = 0;
    u64 root = 0;
    std::unordered_map<u64, std::pair<unsigned, u64>> code;  // symbol-offset -> (len, code)
    vector<u64> freq_of;                                     // per leaf index
    u64 bits = 0;

    static void put_be64(uint8_t *b, u64 v) {
        for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (56 - 8 * i));
    }

    void build(const T *s, u64 num) {
        T mn = s[0], mx = s[0];
        for (u64 i = 1; i < num; i++) {
            mn = std::min(mn, s[i]);
            mx = std::max(mx, s[i]);
        }
        offset = mn;
        maxval = (u64)(T)(mx - mn + 1);
        usemp = ((T)maxval >= (1 << 12) && num < 2 * (u64)mx) || (T)maxval >= (1 << 28);
        std::map<u64, u64> freq;
        for (u64 i = 0; i < num; i++) ++freq[(u64)(s[i] - offset)];
        ht.clear();
        freq_of.clear();
        for (auto &kv : freq) {
            node nd;
            nd.c = kv.first;
            ht.push_back(nd);
            freq_of.push_back(kv.second);
        }
        n = ht.size();
        code.clear();
        bits = 0;
        if (n == 1 || maxval == 1) {  // huffman.hpp:193-210
            mbft = 1;
            maxval = 1;
            offset = (T)(offset + (T)ht[0].c);
            ht[0].c = 0;
            code[0] = {1, 0};
            return;
        }
        mbft = 1;
        while ((1ull << mbft) < maxval) ++mbft;
        using pr = std::pair<u64, u64>;  // (node index, freq); min freq first, then min index
        auto cmp = [](const pr &u, const pr &v) { return u.second == v.second ? u.first > v.first : u.second > v.second; };
        std::priority_queue<pr, vector<pr>, decltype(cmp)> q(cmp);
        for (u64 i = 0; i < ht.size(); i++) q.push({i, freq_of[i]});
        while (q.size() > 1) {
            pr u = q.top();
            q.pop();
            pr v = q.top();
            q.pop();
            node nd;
            nd.l = (int)u.first;
            nd.r = (int)v.first;
            ht.push_back(nd);
            q.push({ht.size() - 1, u.second + v.second});
        }
        root = ht.size() - 1;
        dfs(root, 0, 0);
        for (u64 i = 0; i < n; i++) bits += freq_of[i] * code[ht[i].c].first;
    }
    void dfs(u64 u, unsigned len, u64 vec) {
        if (ht[u].l < 0) {
            if (len > 32) throw std::runtime_error("Huffman code longer than 32 bits");
            code[ht[u].c] = {len, vec};
            return;
        }
        dfs(ht[u].l, len + 1, vec);
        dfs(ht[u].r, len + 1, vec | (1ull << len));
    }
    u64 save_size() const {
        u64 s = 1 + 8 + 8 + 8;
        if (n > 1) s += (n * (mbft + 2) - 1 + 7) >> 3;
        return s;
    }
    u64 encode_size() const { return 8 + (maxval == 1 ? 0 : (bits + 7) >> 3); }

    struct bitw {
        uint8_t *p;
        unsigned mask = 0, idx = 0;
        void bit(unsigned v) {
            mask |= v << idx++;
            if (idx == 8) {
                *p++ = (uint8_t)mask;
                mask = idx = 0;
            }
        }
        void bits(u64 v, unsigned len) {
            for (unsigned k = 0; k < len; k++) bit((v >> k) & 1);
        }
        void flush() {
            if (idx > 0) *p++ = (uint8_t)mask;
        }
    };

    uint8_t *save(uint8_t *c) const {  // huffman.hpp:650-691
        *c++ = (uint8_t)((usemp << 7) | ((n == 1) << 6) | mbft);
        u64 ob = (u64)(i64)offset;
        for (int i = 0; i < 8; i++) *c++ = (uint8_t)(ob >> (8 * i));
        put_be64(c, n);
        c += 8;
        put_be64(c, maxval);
        c += 8;
        if (n <= 1) return c;
        bitw w{c};
        std::stack<u64> st;
        st.push(root);
        while (!st.empty()) {
            u64 u = st.top();
            st.pop();
            if (ht[u].l < 0) {
                w.bit(1);
                w.bits(ht[u].c, mbft);
            } else {
                w.bit(0);
                st.push((u64)ht[u].r);
                st.push((u64)ht[u].l);
            }
        }
        w.flush();
        return w.p;
    }
    uint8_t *encode(const T *s, u64 num, uint8_t *c) const {  // huffman.hpp:340-381
        if (maxval == 1) {
            put_be64(c, num ^ 0x1234abcd);
            return c + 8;
        }
        uint8_t *head = c;
        bitw w{c + 8};
        u64 len = 0;
        for (u64 i = 0; i < num; i++) {
            auto &e = code.at((u64)(s[i] - offset));
            len += e.first;
            w.bits(e.second, e.first);
        }
        w.flush();
        put_be64(head, len ^ 0x1234abcd);
        return w.p;
    }
};

// Huffman decoder: huffman.hpp:383-526 and 693-783. A plain tree walk (same output).
template <class T>
struct hdec {
    struct node {
        int l = -1, r = -1;
        u64 c = 0;
    };
    vector<node> ht;
    T offset = 0;
    u64 n = 0, maxval = 0;
    unsigned mbft = 0;
    static u64 be64(const uint8_t *b) {
        u64 v = 0;
        for (int i = 0; i < 8; i++) v = (v << 8) | b[i];
        return v;
    }
    const uint8_t *load(const uint8_t *b, const uint8_t *end) {
        if (end - b < 25) throw std::runtime_error("truncated Huffman header");
        mbft = b[0] & 0x3f;
        b++;
        u64 ob = 0;
        for (int i = 0; i < 8; i++) ob |= (u64)b[i] << (8 * i);
        b += 8;
        offset = (T)(i64)ob;
        n = be64(b);
        b += 8;
        maxval = be64(b);
        b += 8;
        ht.clear();
        if (n <= 1) return b;
        ht.push_back(node());
        vector<int> st{0};
        u64 i = 1;
        auto rd = [&](u64 k) -> unsigned {
            if ((k >> 3) >= (u64)(end - b)) throw std::runtime_error("truncated Huffman tree");
            return (b[k >> 3] >> (k & 7)) & 1;
        };
        while (!st.empty()) {
            int u = st.back();
            if (rd(i++) == 0) {
                ht.push_back(node());
                int id = (int)ht.size() - 1;
                if (ht[u].l < 0) ht[u].l = id;
                else ht[u].r = id;
                st.push_back(id);
            } else {
                u64 c = 0;
                for (unsigned j = 0; j < mbft; j++) c |= (u64)rd(i++) << j;
                node nd;
                nd.c = c;
                ht.push_back(nd);
                int id = (int)ht.size() - 1;
                if (ht[u].l < 0) ht[u].l = id;
                else ht[u].r = id;
                while (!st.empty() && ht[st.back()].r >= 0) st.pop_back();
            }
            if (ht.size() > 2 * n + 2) throw std::runtime_error("corrupt Huffman tree");
        }
        return b + ((i + 7) >> 3);
    }
    const uint8_t *decode(const uint8_t *b, const uint8_t *end, T *out, u64 count) {
        if (end - b < 8) throw std::runtime_error("truncated Huffman payload");
        if (maxval == 1 || n <= 1) {
            u64 c = be64(b) ^ 0x1234abcd;
            if (count && c != count) throw std::runtime_error("Huffman payload length does not match its value count");
            for (u64 i = 0; i < count; i++) out[i] = offset;
            return b + 8;
        }
        u64 len = be64(b) ^ 0x1234abcd;
        b += 8;
        if (((len + 7) >> 3) > (u64)(end - b)) throw std::runtime_error("truncated Huffman payload");
        u64 o = 0;
        int u = 0;
        for (u64 k = 0; k < len; k++) {
            unsigned bit = (b[k >> 3] >> (k & 7)) & 1;
            u = bit ? ht[u].r : ht[u].l;
            if (u < 0) throw std::runtime_error("corrupt Huffman payload");
            if (ht[u].l < 0) {
                if (o >= count) throw std::runtime_error("Huffman payload contains too many values");
                out[o++] = (T)(ht[u].c + offset);
                u = 0;
            }
        }
        if (u != 0) throw std::runtime_error("Huffman payload ends inside a code");
        if (o != count) throw std::runtime_error("Huffman payload contains too few values");
        return b + ((len + 7) >> 3);
    }
};

template <class T>
void append_stream(vector<uint8_t> &bs, const vector<T> &v) {
    u64 len = v.size();
    for (int i = 0; i < 8; i++) bs.push_back((uint8_t)(len >> (8 * i)));
    if (v.empty()) return;
    huff<T> h;
    h.build(v.data(), v.size());
    u64 sz = h.save_size() + h.encode_size();
    size_t off = bs.size();
    bs.resize(off + sz);
    uint8_t *p = h.save(bs.data() + off);
    p = h.encode(v.data(), v.size(), p);
    if (p != bs.data() + bs.size()) throw std::runtime_error("Huffman encoded size mismatch");
}

vector<std::string> parse_plan(const char *s) {
    vector<std::string> out;
    std::string t(s ? s : "");
    size_t b = 0;
    while (b <= t.size()) {
        size_t e = t.find(',', b);
        std::string pr = t.substr(b, e == std::string::npos ? std::string::npos : e - b);
        bool ok = pr.size() == 10 && pr.compare(0, 5, "cubic") == 0 && pr[5] >= '0' && pr[5] <= '2' && pr[6] == '_' &&
                  (pr.compare(7, 3, "120") == 0 || pr.compare(7, 3, "021") == 0 || pr.compare(7, 3, "012") == 0);
        if (!ok) throw std::invalid_argument("invalid predictor in plan: " + pr);
        out.push_back(pr);
        if (e == std::string::npos) break;
        b = e + 1;
    }
    return out;
}



// ---------------------------------------------------------------------------------------------
// Predictor-family selection: param_c::select_predictor_family and predictor_family_detail
// (predictor_family.tpp:1-252), with the long-double steps as the reference build emits them on
// x87: log2 and log10 through fyl2x, divisions by a count as a multiplication by its reciprocal,
// no infinity test in the score (finite-math), and floor through frndint.

static inline long double x87_fyl2x(long double x, long double y) {  // y * log2(x)
    long double r;
    __asm__("fyl2x" : "=t"(r) : "0"(x), "u"(y) : "st(1)");
    return r;
}
static inline long double x87_lg2() {
    long double r;
    __asm__("fldlg2" : "=t"(r));
    return r;
}

struct fam_result {
    u64 point_count = 0;
    long double prediction_mse = 0, reconstruction_mse = 0, reconstruction_psnr = 0, h1 = 0;
};

// entropy() (predictor_family.tpp:116-131).
static long double fam_entropy(const vector<qb_t> &qbs) {
    if (qbs.empty()) return 0;
    std::unordered_map<qb_t, u64> freq;
    for (qb_t q : qbs) freq[q]++;
    const long double r = 1.0L / (long double)qbs.size();
    long double h1 = 0;
    for (const auto &kv : freq) {
        const long double pr = (long double)kv.second * r;
        h1 = h1 - pr * x87_fyl2x(pr, 1.0L);
    }
    return h1;
}

// evaluate() (predictor_family.tpp:133-215) for one family on the target blocks.
static fam_result fam_evaluate(const codec &probe, const float *data, const vector<std::array<u64, 3>> &targets, bool quintic) {
    const u64 L = probe.plan.size();
    const float seed_eb = probe.abs_eb * probe.P.p.pivot_eb_ratio;
    vector<vector<qb_t>> layer_qbs(L);
    vector<long double> pred_sse(L, 0), rec_sse(L, 0);
    vector<u64> counts(L, 0);
    for (const auto &tb : targets) {
        std::array<u64, 3> cbb, tend, cb, ce, hb;
        for (int a = 0; a < 3; a++) {
            cbb[a] = tb[a] ? tb[a] - 1 : 0;
            tend[a] = tb[a] + 1;
            cb[a] = cbb[a] * probe.block_shape[a];
            ce[a] = std::min(tend[a] * probe.block_shape[a] + 1, probe.f.n[a]);
            const u64 left_halo = 5 * (probe.pivot_stride[a] / 2);
            hb[a] = cb[a] > left_halo ? cb[a] - left_halo : 0;
        }
        codec local;
        local.f = {{ce[0] - hb[0], ce[1] - hb[1], ce[2] - hb[2]}};
        vector<float> ldata(local.f.size());
        for (u64 i0 = hb[0]; i0 < ce[0]; i0++)
            for (u64 i1 = hb[1]; i1 < ce[1]; i1++)
                std::memcpy(&ldata[local.f.pos(i0 - hb[0], i1 - hb[1], 0)], &data[probe.f.pos(i0, i1, hb[2])],
                            local.f.n[2] * sizeof(float));
        local.data = ldata.data();
        local.cd = ldata;
        local.P = probe.P;
        local.quintic = quintic;
        local.plan = probe.plan;
        local.pivot_stride = probe.pivot_stride;
        local.block_shape = probe.block_shape;
        local.min_val = probe.min_val;
        local.max_val = probe.max_val;
        local.abs_eb = probe.abs_eb;
        local.default_slope_v = probe.default_slope_v;
        // Seed pivots on the context (global lattice), as in the whole-field compressor.
        const double peb = seed_eb, rp = 0.5 / peb, peb2 = peb + peb;
        for (u64 i0 = cb[0]; i0 < ce[0]; i0 += probe.pivot_stride[0])
            for (u64 i1 = cb[1]; i1 < ce[1]; i1 += probe.pivot_stride[1])
                for (u64 i2 = cb[2]; i2 < ce[2]; i2 += probe.pivot_stride[2]) {
                    const u64 pos = local.f.pos(i0 - hb[0], i1 - hb[1], i2 - hb[2]);
                    const qb_t qb = (qb_t)lround_d((double)ldata[pos] * rp);
                    local.cd[pos] = (float)((double)qb * peb2);
                }
        vector<long double> lp(L, 0), lr(L, 0);
        vector<u64> lc(L, 0);
        vector<qb_t> context_qbs;
        for (u64 b0 = cbb[0]; b0 < tend[0]; b0++)
            for (u64 b1 = cbb[1]; b1 < tend[1]; b1++)
                for (u64 b2 = cbb[2]; b2 < tend[2]; b2++) {
                    const bool target = b0 == tb[0] && b1 == tb[1] && b2 == tb[2];
                    const u64 bb[3] = {b0, b1, b2};
                    std::array<std::array<u64, 2>, 3> loc;
                    for (int a = 0; a < 3; a++)
                        loc[a] = {bb[a] * probe.block_shape[a] - hb[a],
                                  std::min((bb[a] + 1) * probe.block_shape[a] + 1, probe.f.n[a]) - hb[a]};
                    std::array<u64, 3> stride = probe.pivot_stride;
                    for (u64 l = 0; l < L; l++) {
                        const int dir = probe.plan[l][5] - '0', order = probe.plan[l][9] - '0';
                        const float leb = local.layer_eb(L, l);
                        const float slope =
                            (float)((double)probe.default_slope_v * std::pow((double)probe.P.p.slope_ratio, (double)((int64_t)L - (int64_t)l - 1)));
                        bool fb = false;
                        const float t = local.select_t(dir, loc, stride, leb, slope, fb);
                        vector<qb_t> &qv = target ? layer_qbs[l] : context_qbs;
                        if (!target) context_qbs.clear();
                        u64 base = qv.size();
                        qv.resize(base + local.layer_qb_count(loc, stride, dir));
                        // dot_compress<true>: the division form on every axis, and the diagnostics.
                        const double ebd = leb, eb2 = ebd + ebd;
                        local.for_targets(loc, stride, dir, order, base, [&](u64 i, u64 hs, u64 right, u64 pos, u64 dist, u64 qi) {
                            const float pred = local.predict(i, hs, right, pos, dist, t);
                            const double pd = pred, diff = pd - (double)ldata[pos];
                            const qb_t qb = (qb_t)lround_d((diff * 0.5) / ebd);
                            qv[qi] = qb;
                            local.cd[pos] = (float)std::fma(-(double)qb, eb2, pd);
                            if (target) {
                                const long double pe = (long double)pred - (long double)ldata[pos];
                                const long double re = (long double)local.cd[pos] - (long double)ldata[pos];
                                lp[l] = lp[l] + pe * pe;
                                lr[l] = lr[l] + re * re;
                                lc[l]++;
                            }
                        });
                        stride[dir] /= 2;
                    }
                }
        for (u64 l = 0; l < L; l++) {
            pred_sse[l] = pred_sse[l] + lp[l];
            rec_sse[l] = rec_sse[l] + lr[l];
            counts[l] += lc[l];
        }
    }
    fam_result r;
    long double wh1 = 0, ptot = 0, rtot = 0;
    for (u64 l = 0; l < L; l++) {
        if (counts[l] != layer_qbs[l].size()) throw std::runtime_error("predictor-family target count mismatch");
        r.point_count += counts[l];
        ptot = ptot + pred_sse[l];
        rtot = rtot + rec_sse[l];
        wh1 = wh1 + fam_entropy(layer_qbs[l]) * (long double)counts[l];
    }
    if (r.point_count == 0) throw std::runtime_error("predictor-family sample contains no target points");
    const long double rc = 1.0L / (long double)r.point_count;
    r.prediction_mse = ptot * rc;
    r.reconstruction_mse = rtot * rc;
    const long double range = (long double)probe.max_val - (long double)probe.min_val;
    r.reconstruction_psnr = r.reconstruction_mse == 0 ? (long double)INFINITY
                                                      : x87_fyl2x(range * range / r.reconstruction_mse, x87_lg2()) * 10.0L;
    r.h1 = wh1 * rc;
    return r;
}

// select_predictor_family (predictor_family.tpp:217-251). Fills the result's family fields.
static bool select_family(const codec &C, float rel_eb, aszo_result *out) {
    const aszo_params &p = C.P.p;
    codec probe;
    probe.f = C.f;
    probe.P = C.P;
    probe.P.p.h1_block_sampling_num = 256;  // not copied to the probe (copy_settings, :17-37)
    probe.min_val = C.min_val;
    probe.max_val = C.max_val;
    probe.abs_eb = C.abs_eb;
    probe.default_slope_v = C.default_slope_v;
    const u64 suffix = std::min<u64>(p.predictor_family_suffix_layers, C.plan.size());
    probe.plan.assign(C.plan.end() - suffix, C.plan.end());
    probe.P.p.block_pivot_ratio = rel_eb <= p.predictor_family_fine_eb_threshold ? p.predictor_family_fine_probe_block_pivot_ratio
                                                                                : p.predictor_family_coarse_probe_block_pivot_ratio;
    probe.geometry();
    // make_stratified_targets (:65-86).
    const u64 total = probe.block_num[0] * probe.block_num[1] * probe.block_num[2];
    const u64 sc = std::min<u64>(p.predictor_family_sample_blocks, total);
    std::mt19937_64 rng(0);
    vector<std::array<u64, 3>> cands;
    for (u64 s = 0; s < sc; s++) {
        const u64 sb = (u64)((unsigned __int128)s * total / sc), se = (u64)((unsigned __int128)(s + 1) * total / sc);
        u64 index = sb + rng() % (se - sb);
        std::array<u64, 3> t;
        t[2] = index % probe.block_num[2];
        index /= probe.block_num[2];
        t[1] = index % probe.block_num[1];
        t[0] = index / probe.block_num[1];
        cands.push_back(t);
    }
    // Point budget (:232-234): floor via frndint in round-down mode.
    const long double frac = (long double)C.f.size() * (long double)p.predictor_family_sample_fraction_limit;
    const u64 fraction_budget = (u64)floorl(frac);
    const u64 budget = std::min<u64>(p.predictor_family_sample_point_limit, fraction_budget);
    vector<std::array<u64, 3>> targets;
    u64 sampled = 0;
    for (const auto &c : cands) {  // apply_point_budget (:99-114)
        u64 pts = 1;
        for (int a = 0; a < 3; a++) {
            const u64 b = c[a] * probe.block_shape[a], e = std::min((c[a] + 1) * probe.block_shape[a] + 1, probe.f.n[a]);
            pts *= e - b;
        }
        if (sampled <= budget && pts <= budget - sampled) {
            targets.push_back(c);
            sampled += pts;
        }
    }
    out->family_selected = 1;
    out->fam_suffix_layers = suffix;
    out->fam_budget = budget;
    out->fam_probe_bpr = probe.P.p.block_pivot_ratio;
    out->fam_sampled_points = sampled;
    out->fam_blocks = targets.size();
    if (targets.empty()) {
        out->family_fallback = 1;
        return false;
    }
    const fam_result c = fam_evaluate(probe, C.data, targets, false);
    const fam_result q = fam_evaluate(probe, C.data, targets, true);
    const long double score = (c.h1 - q.h1) * (long double)C.default_slope_v + (q.reconstruction_psnr - c.reconstruction_psnr);
    out->fam_points = c.point_count;
    out->fam_cubic_mse = c.prediction_mse;
    out->fam_quintic_mse = q.prediction_mse;
    out->fam_cubic_psnr = c.reconstruction_psnr;
    out->fam_quintic_psnr = q.reconstruction_psnr;
    out->fam_cubic_h1 = c.h1;
    out->fam_quintic_h1 = q.h1;
    out->fam_score_gain = score;
    return score > 0;
}

// dot_sample_compress (generate_config.tpp:227-254) on the original data, in the form GCC emits:
// the edge stencils below, the interior as in dot_compress, the residual quantised in float
// (diff * neg_2_eb), and the squared error accumulated with one fmaf per sample.
static inline void dot_sample(vector<qb_t> &qv, float &mse, const float *d, u64 i, u64 hs, u64 right, u64 pos, u64 dist,
                              float t, float eb, float neg_2_eb) {
    float pred;
    const float xm1 = d[pos - dist];
    if (i <= hs) {
        if (i + hs >= right) pred = xm1;
        else if (i + 3 * hs >= right) pred = (d[pos + dist] + xm1) * 0.5f;
        else pred = std::fmaf(d[pos + dist], 6.0f, std::fmaf(xm1, 3.0f, -d[pos + 3 * dist])) * 0.125f;
    } else {
        const float xm3 = d[pos - 3 * dist];
        if (i + hs >= right) pred = std::fmaf(xm1, 3.0f, -xm3) * 0.5f;
        else if (i + 3 * hs >= right) pred = (std::fmaf(xm1, 6.0f, d[pos + dist] * 3.0f) - xm3) * 0.125f;
        else {
            float s1 = d[pos + dist] + xm1, s3 = xm3 + d[pos + 3 * dist];
            float p1 = (float)((double)s3 * (0.25 - (double)t));
            pred = (float)std::fma(0.25 + (double)t, (double)s1, (double)p1);
        }
    }
    const float diff = pred - d[pos];
    const qb_t qb = (qb_t)lround_f(diff * neg_2_eb);
    qv.push_back(qb);
    const float q2 = (float)(qb_t)((uint32_t)qb * 2u);
    const float e = std::fmaf(-eb, q2, diff);
    mse = std::fmaf(e, e, mse);
}

// block_sample_compress_cubicD_ORDER (generate_config.tpp:256-438) over the whole field: the
// innermost loop (axis = the order digit) runs at the lattice stride, the outer two at
// sample_stride times it; the prediction axis starts at its half stride.
static void sample_compress(vector<qb_t> &qv, float &mse, const float *d, const field &f, int dir, int order,
                            const u64 ps2[3], u64 S, float t, float eb, float neg_2_eb) {
    u64 st[3], lo[3];
    for (int a = 0; a < 3; a++) {
        st[a] = ps2[a] * (a == order ? 1 : S);
        lo[a] = a == dir ? ps2[dir] / 2 : 0;
    }
    const u64 hs = ps2[dir] / 2;
    u64 dist = hs;
    for (int a = dir + 1; a < 3; a++) dist *= f.n[a];
    static const int nest[3][3] = {{1, 2, 0}, {0, 2, 1}, {0, 1, 2}};  // loop axes, outer to inner
    const int *ax = nest[order];
    u64 ii[3];
    for (ii[ax[0]] = lo[ax[0]]; ii[ax[0]] < f.n[ax[0]]; ii[ax[0]] += st[ax[0]])
        for (ii[ax[1]] = lo[ax[1]]; ii[ax[1]] < f.n[ax[1]]; ii[ax[1]] += st[ax[1]])
            for (ii[ax[2]] = lo[ax[2]]; ii[ax[2]] < f.n[ax[2]]; ii[ax[2]] += st[ax[2]])
                dot_sample(qv, mse, d, ii[dir], hs, f.n[dir], f.pos(ii[0], ii[1], ii[2]), dist, t, eb, neg_2_eb);
}

template <class T> struct huff;

// generate_config (generate_config.tpp:444-678): reverse-greedy plan search from the finest layer.
static vector<std::string> generate_plan(const float *data, const field &f, float abs_eb, float min_val, float max_val,
                                         float slope, const params_t &P, vector<float> &dists) {
    const aszo_params &p = P.p;
    static const char *all9[9] = {"cubic0_120", "cubic0_021", "cubic0_012", "cubic1_120", "cubic1_021",
                                  "cubic1_012", "cubic2_120", "cubic2_021", "cubic2_012"};
    static const char *last3[3] = {"cubic0_012", "cubic1_012", "cubic2_012"};
    u64 ps[3] = {1, 1, 1};
    vector<std::string> plan;
    dists.clear();
    for (u64 layer = 0; layer < p.max_layer_num; layer++) {
        // As emitted: pow in double, products rounded to float, 0.5f/x for the 1/(2x) factors.
        const float layer_eb = (float)((double)abs_eb * std::pow((double)p.eb_ratio, (double)layer));
        const float neg_2_layer_eb = 0.5f / layer_eb;
        const float stat_eb = layer_eb * p.stat_eb_ratio;
        const float neg_2_stat_eb = 0.5f / stat_eb;
        const float lslope = (float)((double)slope * std::pow((double)p.slope_ratio, (double)layer));
        vector<std::string> cands;
        if (layer < p.full_predictor_search_layer_num) cands.assign(all9, all9 + 9);
        else cands.assign(last3, last3 + 3);
        ab_map maps[3];
        bool ready[3] = {false, false, false};
        vector<float> br(cands.size()), psnr(cands.size());
        vector<u64> num(cands.size(), 0);
        for (size_t c = 0; c < cands.size(); c++) {
            const int dir = cands[c][5] - '0', order = cands[c][9] - '0';
            ab_map &m = maps[dir];
            if (!ready[dir] && f.n[dir] > 3 * ps[dir]) {
                u64 ps2[3] = {ps[0], ps[1], ps[2]};
                ps2[dir] *= 2;
                std::array<std::array<u64, 2>, 3> loc = {{{0, f.n[0]}, {0, f.n[1]}, {0, f.n[2]}}};
                loc[dir] = {3 * ps2[dir] / 2, f.n[dir] - 3 * ps2[dir] / 2};
                u64 dist = ps2[dir];
                for (int a = dir + 1; a < 3; a++) dist *= f.n[a];
                dist /= 2;
                std::array<u64, 3> stride = {ps2[0], ps2[1], ps2[2]};
                get_ab_map(m, data, f, loc, stride, dist, neg_2_stat_eb, p.h1_block_sampling_num);
            }
            ready[dir] = true;
            // Best t on the map: score fmaf(-slope, h1, psnr), strictly better replaces.
            float best_t = 0.25f;
            if (!m.empty()) {
                float h1, ps_;
                get_h1_psnr(h1, ps_, m, 0.25f, layer_eb, stat_eb, min_val, max_val);
                float best = std::fmaf(-lslope, h1, ps_);
                for (float t : P.candidate_t) {
                    if (t == 0.25f) continue;
                    get_h1_psnr(h1, ps_, m, t, layer_eb, stat_eb, min_val, max_val);
                    float cur = std::fmaf(-lslope, h1, ps_);
                    if (cur > best) best_t = t;
                    best = cur > best ? cur : best;
                }
            }
            // Sampled compression with that t, then Huffman + zstd level 3 of its QBs.
            u64 ps2[3] = {ps[0], ps[1], ps[2]};
            ps2[dir] *= 2;
            vector<qb_t> qv;
            float mse = 0;
            sample_compress(qv, mse, data, f, dir, order, ps2, p.generate_config_sample_stride, best_t, layer_eb,
                            neg_2_layer_eb);
            if (!qv.empty()) {
                huff<qb_t> h;
                h.build(qv.data(), qv.size());
                vector<uint8_t> hb(h.save_size() + h.encode_size());
                uint8_t *w = h.save(hb.data());
                w = h.encode(qv.data(), qv.size(), w);
                if (w != hb.data() + hb.size()) throw std::runtime_error("Huffman encoded size mismatch");
                vector<uint8_t> z(ZSTD_compressBound(hb.size()));
                size_t zl = ZSTD_compress(z.data(), z.size(), hb.data(), hb.size(), 3);
                if (ZSTD_isError(zl)) throw std::runtime_error(ZSTD_getErrorName(zl));
                const float nf = (float)qv.size();
                br[c] = (float)zl * (8.0f / nf);
                const float mse_avg = mse / nf;
                const float R = max_val - min_val;
                psnr[c] = log10f(R * R / mse_avg) * 10.0f;
                num[c] = qv.size();
            }
        }
        // Best predictor: score psnr - slope*br (two roundings), strictly better replaces.
        int best = -1;
        float best_dist = 0;
        for (size_t c = 0; c < cands.size(); c++) {
            if (!num[c]) continue;
            const float dist = psnr[c] - lslope * br[c];
            if (best < 0 || dist > best_dist) {
                best = (int)c;
                best_dist = dist;
            }
        }
        if (best < 0) break;
        ps[cands[best][5] - '0'] *= 2;
        plan.insert(plan.begin(), cands[best]);
        dists.push_back(best_dist);
    }
    return plan;
}

void set_err(char *err, const char *m) {
    if (err) snprintf(err, 256, "%s", m);
}

}  // namespace

extern "C" {

void aszo_default_params(aszo_params *p) {
    p->pivot_eb_ratio = 0.05f;
    p->eb_ratio = 0.76f;
    p->slope_ratio = 0.54f;
    p->block_pivot_ratio = 4;
    p->t_precision = 32;
    p->t_min = 1.0f / 16;
    p->t_max = 6.0f / 16;
    p->h1_block_sampling_num = 256;
    p->stat_eb_ratio = 0.2f;
    p->default_slope_invalid_ratio_threshold = 1;
    p->default_slope_fallback = 1000;
    p->default_slope_eb_span = 1.5f;
    p->insufficient_sample_t = 4.0f / 16;
    p->max_layer_num = 14;
    p->full_predictor_search_layer_num = 4;
    p->generate_config_sample_stride = 5;
    p->predictor_family_suffix_layers = 6;
    p->predictor_family_sample_blocks = 8;
    p->predictor_family_sample_point_limit = 32768;
    p->predictor_family_sample_fraction_limit = 0.02f;
    p->predictor_family_coarse_probe_block_pivot_ratio = 3;
    p->predictor_family_fine_probe_block_pivot_ratio = 4;
    p->predictor_family_fine_eb_threshold = 1e-4f;
}

static int compress_impl(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p, const char *plan,
                         int quintic, const int64_t *t_given, uint64_t t_given_len, aszo_result *out, char *err) {
    try {
        std::memset(out, 0, sizeof(*out));
        codec C;
        C.t_given = t_given;
        C.f = {{dims[0], dims[1], dims[2]}};
        C.P.init(*p);
        C.quintic = quintic > 0;
        if (plan) C.plan = parse_plan(plan);
        C.data = data;
        u64 N = C.f.size();
        auto mm = std::minmax_element(data, data + N);
        C.min_val = *mm.first;
        C.max_val = *mm.second;
        if (C.min_val == C.max_val) throw std::runtime_error("max_val==min_val");
        C.abs_eb = rel_eb * (C.max_val - C.min_val);
        C.default_slope_v = default_slope(data, C.f, C.abs_eb, C.min_val, C.max_val, C.P);
        vector<float> dists;
        if (!plan) C.plan = generate_plan(data, C.f, C.abs_eb, C.min_val, C.max_val, C.default_slope_v, C.P, dists);
        if (C.plan.size() > 63) throw std::invalid_argument("predictor plan cannot contain more than 63 layers");
        if (C.plan.empty()) throw std::runtime_error("plan search found no layer");
        if (quintic < 0) C.quintic = select_family(C, rel_eb, out);
        out->quintic = C.quintic ? 1 : 0;
        {
            std::string pl;
            for (size_t i = 0; i < C.plan.size(); i++) pl += (i ? "," : "") + C.plan[i];
            snprintf(out->plan, sizeof(out->plan), "%s", pl.c_str());
            out->search_layers = (uint32_t)std::min<size_t>(dists.size(), 64);
            for (size_t i = 0; i < out->search_layers; i++) out->best_dist[i] = dists[i];
        }
        C.geometry();
        if (t_given && t_given_len != C.block_num[0] * C.block_num[1] * C.block_num[2] * C.plan.size())
            throw std::invalid_argument("t table length does not match the plan's blocks and rounds");
        C.compress_core();
        // Stream assembly: compress.tpp:233-291.
        vector<uint8_t> bs;
        uint8_t hdr[9];
        std::memcpy(hdr, &C.min_val, 4);
        std::memcpy(hdr + 4, &C.max_val, 4);
        hdr[8] = (uint8_t)(C.plan.size() | 0x40 | (C.quintic ? 0x80 : 0));
        bs.insert(bs.end(), hdr, hdr + 9);
        for (auto &pr : C.plan) {
            bs.push_back((uint8_t)pr[5]);
            bs.push_back((uint8_t)pr[9]);
        }
        append_stream<int64_t>(bs, C.t_int);
        for (auto &v : C.qbs) append_stream<int32_t>(bs, v);
        size_t bound = ZSTD_compressBound(bs.size());
        vector<uint8_t> z(bound);
        size_t zl = ZSTD_compress(z.data(), bound, bs.data(), bs.size(), 3);
        if (ZSTD_isError(zl)) throw std::runtime_error(ZSTD_getErrorName(zl));
        z.resize(zl);
        // Outputs.
        out->layer_num = (uint32_t)C.plan.size();
        out->qb_len = (uint64_t *)malloc(sizeof(uint64_t) * C.qbs.size());
        out->qb = (int32_t **)malloc(sizeof(int32_t *) * C.qbs.size());
        for (size_t i = 0; i < C.qbs.size(); i++) {
            out->qb_len[i] = C.qbs[i].size();
            out->qb[i] = (int32_t *)malloc(sizeof(int32_t) * std::max<size_t>(1, C.qbs[i].size()));
            std::memcpy(out->qb[i], C.qbs[i].data(), sizeof(int32_t) * C.qbs[i].size());
        }
        out->t_len = C.t_int.size();
        out->t_int = (int64_t *)malloc(sizeof(int64_t) * std::max<size_t>(1, C.t_int.size()));
        std::memcpy(out->t_int, C.t_int.data(), sizeof(int64_t) * C.t_int.size());
        out->recon = (float *)malloc(sizeof(float) * N);
        std::memcpy(out->recon, C.cd.data(), sizeof(float) * N);
        out->pre_zstd_len = bs.size();
        out->pre_zstd = (uint8_t *)malloc(bs.size());
        std::memcpy(out->pre_zstd, bs.data(), bs.size());
        out->asz_len = z.size();
        out->asz = (uint8_t *)malloc(z.size());
        std::memcpy(out->asz, z.data(), z.size());
        out->min_val = C.min_val;
        out->max_val = C.max_val;
        out->abs_eb = C.abs_eb;
        out->default_slope = C.default_slope_v;
        out->t_fallback_count = C.t_fallback;
        return 0;
    } catch (const std::exception &e) {
        set_err(err, e.what());
        return -1;
    }
}

int aszo_compress(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p, const char *plan,
                  int quintic, aszo_result *out, char *err) {
    return compress_impl(data, dims, rel_eb, p, plan, quintic, nullptr, 0, out, err);
}

int aszo_compress_with_t(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p, const char *plan,
                         int quintic, const int64_t *t_int, uint64_t t_len, aszo_result *out, char *err) {
    if (!plan || quintic < 0 || !t_int) {
        set_err(err, "a t table needs a plan and a family");
        return -1;
    }
    return compress_impl(data, dims, rel_eb, p, plan, quintic, t_int, t_len, out, err);
}

int aszo_grad_samples(const float *data, const uint64_t dims[3], float rel_eb, const aszo_params *p, const char *plan,
                      float *A, float *B, uint64_t *offsets, uint64_t cap, uint64_t *groups, uint64_t *samples, char *err) {
    try {
        codec C;
        C.f = {{dims[0], dims[1], dims[2]}};
        C.P.init(*p);
        C.plan = parse_plan(plan);
        C.data = data;
        u64 N = C.f.size();
        auto mm = std::minmax_element(data, data + N);
        C.min_val = *mm.first;
        C.max_val = *mm.second;
        if (C.min_val == C.max_val) throw std::runtime_error("max_val==min_val");
        C.abs_eb = rel_eb * (C.max_val - C.min_val);
        C.geometry();
        vector<float> a, b;
        vector<uint64_t> off;
        C.grad_samples(a, b, off);
        *groups = off.size() - 1;
        *samples = a.size();
        if (A && B && offsets && cap >= a.size()) {
            std::memcpy(A, a.data(), a.size() * 4);
            std::memcpy(B, b.data(), b.size() * 4);
            std::memcpy(offsets, off.data(), off.size() * 8);
        }
        return 0;
    } catch (const std::exception &e) {
        set_err(err, e.what());
        return -1;
    }
}

void aszo_free_result(aszo_result *r) {
    if (r->qb) {
        for (uint32_t i = 0; i <= r->layer_num; i++) free(r->qb[i]);
        free(r->qb);
    }
    free(r->qb_len);
    free(r->t_int);
    free(r->recon);
    free(r->pre_zstd);
    free(r->asz);
    std::memset(r, 0, sizeof(*r));
}

int aszo_decompress(const uint8_t *asz, uint64_t asz_len, const uint64_t dims[3], float rel_eb, const aszo_params *p,
                    float *out, char *err) {
    try {
        unsigned long long raw = ZSTD_getFrameContentSize(asz, asz_len);
        if (raw == 0ULL - 1 || raw == 0ULL - 2) throw std::runtime_error("not a zstd frame with a known size");
        vector<uint8_t> bs(raw);
        size_t got = ZSTD_decompress(bs.data(), raw, asz, asz_len);
        if (ZSTD_isError(got) || got != raw) throw std::runtime_error("ZSTD_decompress error in decompress()");
        const uint8_t *b = bs.data(), *end = bs.data() + bs.size();
        if (end - b < 9) throw std::runtime_error("truncated header");
        codec C;
        C.f = {{dims[0], dims[1], dims[2]}};
        C.P.init(*p);
        std::memcpy(&C.min_val, b, 4);
        std::memcpy(&C.max_val, b + 4, 4);
        uint8_t fl = b[8];
        u64 L = fl;
        if (fl & 0x40) {
            C.quintic = (fl & 0x80) != 0;
            L = fl & 0x3f;
        }
        b += 9;
        if ((u64)(end - b) < 2 * L) throw std::runtime_error("truncated header");
        for (u64 i = 0; i < L; i++) {
            if (b[0] < '0' || b[0] > '2' || b[1] < '0' || b[1] > '2')
                throw std::runtime_error("compressed stream contains an invalid predictor");
            std::string pr = "cubic";
            pr += (char)b[0];
            pr += "_";
            pr += b[1] == '0' ? "120" : b[1] == '1' ? "021" : "012";
            C.plan.push_back(pr);
            b += 2;
        }
        auto rd64 = [&](void) {
            if (end - b < 8) throw std::runtime_error("truncated stream length");
            u64 v = 0;
            for (int i = 0; i < 8; i++) v |= (u64)b[i] << (8 * i);
            b += 8;
            return v;
        };
        {
            u64 len = rd64();
            C.t_int.assign(len, 0);
            if (len) {
                hdec<int64_t> d;
                b = d.load(b, end);
                b = d.decode(b, end, C.t_int.data(), len);
            }
        }
        C.qbs.assign(L + 1, {});
        for (u64 i = 0; i <= L; i++) {
            u64 len = rd64();
            C.qbs[i].assign(len, 0);
            if (!len) continue;
            hdec<int32_t> d;
            b = d.load(b, end);
            b = d.decode(b, end, C.qbs[i].data(), len);
        }
        C.abs_eb = rel_eb * (C.max_val - C.min_val);
        C.geometry();
        C.decompress_core(out);
        return 0;
    } catch (const std::exception &e) {
        set_err(err, e.what());
        return -1;
    }
}

float aszo_default_slope(const float *data, const uint64_t dims[3], float abs_eb, float min_val, float max_val,
                         const aszo_params *p) {
    params_t P;
    P.init(*p);
    field f{{dims[0], dims[1], dims[2]}};
    return default_slope(data, f, abs_eb, min_val, max_val, P);
}

uint64_t aszo_huffman_encode(const void *symbols, uint64_t n, int wide, uint8_t *out) {
    vector<uint8_t> bs;
    if (wide) {
        const int64_t *s = (const int64_t *)symbols;
        append_stream<int64_t>(bs, vector<int64_t>(s, s + n));
    } else {
        const int32_t *s = (const int32_t *)symbols;
        append_stream<int32_t>(bs, vector<int32_t>(s, s + n));
    }
    if (out) std::memcpy(out, bs.data() + 8, bs.size() - 8);
    return bs.size() - 8;
}

uint64_t aszo_abmap_order(const int64_t *a, const int64_t *b, uint64_t n, uint64_t *order) {
    ab_map m;
    std::map<std::tuple<i64, i64>, u64> first;
    for (u64 i = 0; i < n; i++) {
        m[{a[i], b[i]}]++;
        first.emplace(std::tuple<i64, i64>{a[i], b[i]}, i);
    }
    u64 k = 0;
    for (auto &kv : m) order[k++] = first[kv.first];
    return k;
}

uint64_t aszo_i64map_order(const int64_t *keys, uint64_t n, uint64_t *order) {
    std::unordered_map<i64, u64> m;
    std::map<i64, u64> first;
    for (u64 i = 0; i < n; i++) {
        m[keys[i]]++;
        first.emplace(keys[i], i);
    }
    u64 k = 0;
    for (auto &kv : m) order[k++] = first[kv.first];
    return k;
}

void aszo_h1_psnr(const int64_t *a, const int64_t *b, uint64_t n, float t, float abs_eb, float stat_eb, float min_val,
                  float max_val, float *h1, float *psnr, float *x, float *mse) {
    ab_map m;
    for (u64 i = 0; i < n; i++) m[{a[i], b[i]}]++;
    get_h1_psnr(*h1, *psnr, m, t, abs_eb, stat_eb, min_val, max_val, x, mse);
}

}  // extern "C"
