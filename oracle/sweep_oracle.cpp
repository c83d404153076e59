// CPU oracle of the reference's prediction sweep tool (c_codes/s2_many_prediction.cpp).
//
// TEST INFRASTRUCTURE ONLY: part of libasz_oracle.so, loaded by tests/ as the checker of the
// CUDA sweep; never linked into the product.
//
// The floating-point forms follow what GCC 13.3 makes of the reference under its flags
// (-Ofast -march=native -mavx2 -mfma, c_codes/CMakeLists.txt:12), pinned target by target
// against the reference's own dot functions (oracle/s2_ref_dump.cpp) and, end to end, against
// the reference binary's outputs in tests/golden/s2_*.json:
//   - neighbour pairs are summed in float; 1D4R and 2D4R products of those sums with 0.25 -+ t
//     are exact in double, so their evaluation order does not matter;
//   - 1D6R: w = 0.5 - (a + b); pred = fma(w, s1, fma(a, s5, b * s3));
//   - e = pred - x; rmse_sum = fma(e, e, rmse_sum); mae_sum += |e|;
//   - qb = llround(e * neg_2_eb), which the compiler emits as trunc(v + copysign(0.5 - 2^-54, v));
//   - e2 = fma(-(2 qb), abs_eb, e); mse_sum = fma(e2, e2, mse_sum).
// This file builds with -ffp-contract=off, so every fused step above is an explicit std::fma.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "asz_oracle.h"
#include "zstd_decls.h"

namespace {

using u64 = uint64_t;

struct Pred {
    int kind = -1;     // 0: 1d4r, 1: 2d4r, 2: 1d6r
    int axis[2] = {-1, -1};
    int order = -1;    // QB order: the innermost loop axis
};

Pred parse_predictor(const std::string &p) {
    // "1d4r0_xx2", "2d4r01_xx1", "1d6r2_xx0" (s2_many_prediction.cpp:171-192, :548-552)
    Pred r;
    auto axis_at = [&](size_t i) { return (i < p.size() && p[i] >= '0' && p[i] <= '2') ? p[i] - '0' : -1; };
    if (p.rfind("1d4r", 0) == 0) r.kind = 0;
    else if (p.rfind("2d4r", 0) == 0) r.kind = 1;
    else if (p.rfind("1d6r", 0) == 0) r.kind = 2;
    else throw std::runtime_error("unknown predictor " + p);
    size_t i = 4;
    r.axis[0] = axis_at(i++);
    if (r.kind == 1) r.axis[1] = axis_at(i++);
    if (p.compare(i, 3, "_xx") != 0 || p.size() != i + 4) throw std::runtime_error("unknown predictor " + p);
    r.order = axis_at(i + 3);
    bool ok = r.axis[0] >= 0 && r.order >= 0;
    if (r.kind == 1) ok = ok && r.axis[1] >= 0 && ((r.axis[0] == 0 && r.axis[1] == 1) || (r.axis[0] == 0 && r.axis[1] == 2) ||
                                                    (r.axis[0] == 1 && r.axis[1] == 2));
    if (!ok) throw std::runtime_error("unknown predictor " + p);
    return r;
}

struct Range {
    u64 start, stop, step;
};

// The target loops of the reference's compress() (s2_many_prediction.cpp:204-397) for stride 1:
// the two axes other than the QB order run outside in increasing order, the order axis inside.
// 1D predictors: the prediction axis covers [m, n - m) every other point, the other axes all
// points (m = 3 for 1D4R, 5 for 1D4R "shared1d" and for 1D6R). 2D4R over axes (A, B): A and B
// cover [1, n - 1), the third axis [0, n), and every other point is taken along axis 0 for "01",
// axis 1 for "02" and axis 2 for "12".
void legacy_ranges(const Pred &p, const u64 n[3], bool shared1d, Range r[3]) {
    for (int x = 0; x < 3; x++) {
        bool pred_axis = x == p.axis[0] || (p.kind == 1 && x == p.axis[1]);
        u64 m = p.kind == 1 ? 1 : p.kind == 2 ? 5 : (shared1d ? 5 : 3);
        bool doubled = p.kind == 1 ? x == (p.axis[0] == 0 && p.axis[1] == 1 ? 0 : p.axis[0] == 0 ? 1 : 2) : x == p.axis[0];
        r[x].start = pred_axis ? m : 0;
        r[x].stop = pred_axis ? (n[x] > m ? n[x] - m : 0) : n[x];
        r[x].step = doubled ? 2 : 1;
    }
}

template <class F>
void for_each_target(const Pred &p, const u64 n[3], const std::string &targets, F f) {
    int outer[2], k = 0;
    for (int x = 0; x < 3; x++)
        if (x != p.order) outer[k++] = x;
    u64 i[3];
    if (targets == "common") {  // for_each_common_target (s2_many_prediction.cpp:126-149)
        const u64 m = 5;
        for (i[outer[0]] = m; i[outer[0]] + m < n[outer[0]]; i[outer[0]]++)
            for (i[outer[1]] = m; i[outer[1]] + m < n[outer[1]]; i[outer[1]]++)
                for (i[p.order] = m; i[p.order] + m < n[p.order]; i[p.order]++)
                    if ((i[0] + i[1] + i[2]) % 2 == 1) f(i[0], i[1], i[2]);
        return;
    }
    Range r[3];
    legacy_ranges(p, n, targets == "shared1d", r);
    for (i[outer[0]] = r[outer[0]].start; i[outer[0]] < r[outer[0]].stop; i[outer[0]] += r[outer[0]].step)
        for (i[outer[1]] = r[outer[1]].start; i[outer[1]] < r[outer[1]].stop; i[outer[1]] += r[outer[1]].step)
            for (i[p.order] = r[p.order].start; i[p.order] < r[p.order].stop; i[p.order] += r[p.order].step)
                f(i[0], i[1], i[2]);
}

void dists_of(const Pred &p, const u64 n[3], u64 d[2]) {  // s2_many_prediction.cpp:169-192
    auto dist = [&](int a) { return a == 0 ? n[1] * n[2] : a == 1 ? n[2] : (u64)1; };
    d[0] = dist(p.axis[0]);
    d[1] = p.kind == 1 ? dist(p.axis[1]) : 0;
}

int64_t llround_emitted(double v) { return (int64_t)(v + std::copysign(0x1.fffffffffffffp-2, v)); }

// six_reference_grid (s2_many_prediction.cpp:89-124).
std::vector<std::pair<double, double>> six_grid(const std::string &mode) {
    std::vector<std::pair<double, double>> g;
    if (mode == "transition") {
        g.push_back({1.0 / 6, 1.0 / 6});
        g.push_back({3.0 / 256, -25.0 / 256});
        for (int i = 0; i <= 12; i++) g.push_back({0.0, (8 - i) / 32.0});
        g.push_back({137.0 / 1536, 53.0 / 1536});
        for (int i = 0; i <= 12; i++) {
            // The division by 192 in the loop becomes a product with its rounded reciprocal.
            g.push_back({1.0 / 12, (40 - 3 * i) * (1.0 / 192.0)});
            g.push_back({3.0 / 512, (39 - 8 * i) / 512.0});
        }
        return g;
    }
    if (mode != "legacy" && mode != "augmented") throw std::runtime_error("six-reference grid must be legacy, augmented or transition");
    for (int i1 : {0, 11, 22, 31, 41})
        for (int i2 : {0, 113, 248, 341, 453, 567, 680, 793})
            g.push_back({1.0 / 6 - (double)((float)i1 / 186.0f), 1.0 / 6 - (double)((float)i2 / 1488.0f)});  // folded exactly
    if (mode == "augmented") {
        std::vector<std::pair<double, double>> exact = {{3.0 / 256, -25.0 / 256}};
        for (int i = 0; i <= 12; i++) exact.push_back({0.0, (8 - i) / 32.0});
        for (auto &c : exact) {
            bool found = false;
            for (auto &q : g)
                if (std::fabs(q.first - c.first) < 1e-7 && std::fabs(q.second - c.second) < 1e-7) {
                    q = c;
                    found = true;
                    break;
                }
            if (!found) g.push_back(c);
        }
    }
    return g;
}

}  // namespace

extern "C" {

int aszo_sweep_coefs(const char *predictor, const char *six_mode, double *c0, double *c1, uint64_t cap) {
    try {
        Pred p = parse_predictor(predictor);
        std::vector<std::pair<double, double>> g;
        if (p.kind == 0)  // t = i/32, i = 0..12 (:199-201)
            for (int i = 0; i <= 12; i++) g.push_back({(double)((float)i / 32.0f), 0.0});
        else if (p.kind == 1)  // t = i/24, i = -6..6 (:264-266), as i times the float reciprocal of 24
            for (int i = -6; i <= 6; i++) g.push_back({(double)((float)i * (1.0f / 24.0f)), 0.0});
        else
            g = six_grid(six_mode);
        for (u64 i = 0; i < g.size() && i < cap; i++) {
            c0[i] = g[i].first;
            c1[i] = g[i].second;
        }
        return (int)g.size();
    } catch (const std::exception &) {
        return -1;
    }
}

uint64_t aszo_sweep_targets(const uint64_t dims[3], const char *predictor, const char *targets, uint64_t *coords,
                            uint64_t cap) {
    Pred p = parse_predictor(predictor);
    u64 k = 0;
    for_each_target(p, dims, targets, [&](u64 i0, u64 i1, u64 i2) {
        if (k < cap) {
            coords[3 * k] = i0;
            coords[3 * k + 1] = i1;
            coords[3 * k + 2] = i2;
        }
        k++;
    });
    return k;
}

int aszo_sweep_run(const float *data, const uint64_t dims[3], const char *predictor, const char *targets, double rel_eb,
                   float min_val, float max_val, double c0, double c1, int64_t *qb_out, uint64_t qb_cap,
                   aszo_sweep_row *row, char *err) {
    try {
        Pred p = parse_predictor(predictor);
        std::string tg = targets;
        if (tg != "legacy" && tg != "shared1d" && tg != "common") throw std::runtime_error("target mode must be legacy, shared1d or common");
        u64 d[2];
        dists_of(p, dims, d);
        const u64 n1n2 = dims[1] * dims[2];
        // s2_many_prediction.cpp:195-196 (max_val and min_val are the float extremes as doubles)
        const double abs_eb = rel_eb * ((double)max_val - (double)min_val);
        const double neg_2_eb = 1 / (2 * abs_eb);
        const double w = 0.5 - (c0 + c1);
        std::vector<int64_t> qb;
        double mse = 0, rmse = 0, mae = 0;
        for_each_target(p, dims, tg, [&](u64 i0, u64 i1, u64 i2) {
            const u64 pos = i0 * n1n2 + i1 * dims[2] + i2;
            const float x = data[pos];
            double pred;
            if (p.kind == 0) {  // compress_1d4r_dot (:28-45)
                const float s3 = data[pos - 3 * d[0]] + data[pos + 3 * d[0]];
                const float s1 = data[pos - d[0]] + data[pos + d[0]];
                pred = (0.25 - c0) * (double)s3 + (0.25 + c0) * (double)s1;
            } else if (p.kind == 1) {  // compress_2d4r_dot (:47-65)
                const float sa = data[pos - d[0]] + data[pos + d[0]];
                const float sb = data[pos - d[1]] + data[pos + d[1]];
                pred = (0.25 + c0) * (double)sa + (0.25 - c0) * (double)sb;
            } else {  // compress_1d6r_dot (:67-87)
                const float s5 = data[pos - 5 * d[0]] + data[pos + 5 * d[0]];
                const float s3 = data[pos - 3 * d[0]] + data[pos + 3 * d[0]];
                const float s1 = data[pos - d[0]] + data[pos + d[0]];
                pred = std::fma(w, (double)s1, std::fma(c0, (double)s5, c1 * (double)s3));
            }
            const double e = pred - (double)x;
            rmse = std::fma(e, e, rmse);
            mae += std::fabs(e);
            const int64_t q = llround_emitted(e * neg_2_eb);
            qb.push_back(q);
            const double e2 = std::fma(-(double)(q * 2), abs_eb, e);
            mse = std::fma(e2, e2, mse);
        });
        if (qb.empty()) throw std::runtime_error("no prediction targets");
        if (qb_out) std::memcpy(qb_out, qb.data(), std::min<u64>(qb.size(), qb_cap) * sizeof(int64_t));
        const u64 S = qb.size();
        // get_H1 (c_codes/get_H.hpp): the map's iteration order, p = freq * (1 / size) with the
        // reciprocal taken once, and H1 -= p * log2(p) as one fused step.
        std::unordered_map<int64_t, u64> freq;
        for (int64_t v : qb) freq[v]++;
        double h1 = 0;
        const double inv = 1.0 / (double)S;
        for (auto &kv : freq) {
            const double pr = (double)kv.second * inv;
            h1 = std::fma(-pr, std::log2(pr), h1);
        }
        // lossless_encode_and_write_csv (:400-440): Huffman (save + encode) then zstd level 3.
        const u64 hb = aszo_huffman_encode(qb.data(), S, 1, nullptr);
        std::vector<uint8_t> hbuf(hb);
        aszo_huffman_encode(qb.data(), S, 1, hbuf.data());
        std::vector<uint8_t> zbuf(ZSTD_compressBound(hb));
        const size_t zb = ZSTD_compress(zbuf.data(), zbuf.size(), hbuf.data(), hb, 3);
        if (ZSTD_isError(zb)) throw std::runtime_error(ZSTD_getErrorName(zb));
        row->c0 = c0;
        row->c1 = c1;
        row->samples = S;
        row->huffman_bytes = hb;
        row->zstd_bytes = zb;
        row->mse_sum = mse;
        row->rmse_sum = rmse;
        row->mae_sum = mae;
        row->h1 = h1;
        aszo_sweep_finish(row, (double)max_val - (double)min_val);
        return 0;
    } catch (const std::exception &e) {
        if (err) {
            std::strncpy(err, e.what(), 255);
            err[255] = 0;
        }
        return -1;
    }
}

// The per-row figures (s2_many_prediction.cpp:423-430). The sums are divided by the size;
// psnr = 10 log10(range^2 / (mse_sum / size)) comes out as 10 log10((range^2 / mse_sum) * size).
void aszo_sweep_finish(aszo_sweep_row *r, double range) {
    const double S = (double)r->samples;
    r->cr = (double)(r->samples * sizeof(float)) / (double)r->zstd_bytes;
    r->br = (8 * sizeof(float)) / r->cr;
    r->h1_cr = (8 * sizeof(float)) / r->h1;
    r->rmse = std::sqrt(r->rmse_sum / S);
    r->mae = r->mae_sum / S;
    r->psnr = 10 * std::log10((range * range / r->mse_sum) * S);
}

}  // extern "C"
