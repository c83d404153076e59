// Host side of the prediction sweep (asz_sweep in include/asz_b200.h): the GPU form of the
// reference's study tool c_codes/s2_many_prediction.cpp.
//
// Per relative error bound, the predictor's coefficients go through in batches sized to the
// device memory: one launch predicts and quantises every target for every coefficient of the
// batch (k_sweep.cu); histograms and first positions of the QB symbols follow on the device; the
// host builds each stream's Huffman code and H1; one tiled launch encodes all streams; the host
// frames each stream as huffman_encoder_class<int64_t>::save + encode and compresses it with
// libzstd level 3 on its threads (lossless_encode_and_write_csv, :400-440).
//
// Host floating point restates the reference's forms under its -Ofast build and is compiled with
// -ffp-contract=off: the grid constants (a division in a loop becomes a product with the rounded
// reciprocal), H1 with p = freq * (1 / size) and H1 -= p log2 p fused, and the final figures with
// psnr = 10 log10((range^2 / mse_sum) * size).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../../include/asz_b200.h"
#include "../launch.h"
#include "buffers.h"
#include "huffman_host.h"
#include "internal.h"
#include "zstd_api.h"

using namespace asz;
using asz::host::DevBuf;
using asz::host::PinnedBuf;

namespace {

using u64 = uint64_t;
using clk = std::chrono::steady_clock;

// Per host worker: the framed stream, the zstd output and a zstd context, kept across rows and
// calls so that their pages are mapped once (first writes to fresh pages cost as much as zstd).
struct WorkerScratch {
    std::vector<uint8_t> buf, z;
    ZSTD_CCtx *cc = nullptr;
};

struct SweepState {
    DevBuf coef, qb, part, sums, mm, hist, first, tab, pay, enc, cub;
    PinnedBuf small, counts, payload;
    std::vector<WorkerScratch> ws;
};

struct Predictor {
    int kind = -1;  // 0: 1d4r, 1: 2d4r, 2: 1d6r
    int axis[2] = {-1, -1};
    int order = -1;
};

// Predictor names of s2_many_prediction.cpp:538-552: "<stencil>_xx<order>".
bool parse_predictor(const char *name, Predictor &p, std::string &err) {
    const std::string s = name ? name : "";
    err = "unknown predictor " + s;
    auto ax = [&](size_t i) { return i < s.size() && s[i] >= '0' && s[i] <= '2' ? s[i] - '0' : -1; };
    size_t i = 4;
    if (s.rfind("1d4r", 0) == 0) p.kind = 0;
    else if (s.rfind("2d4r", 0) == 0) p.kind = 1;
    else if (s.rfind("1d6r", 0) == 0) p.kind = 2;
    else return false;
    p.axis[0] = ax(i++);
    if (p.kind == 1) p.axis[1] = ax(i++);
    if (s.size() != i + 4 || s.compare(i, 3, "_xx") != 0) return false;
    p.order = ax(i + 3);
    if (p.axis[0] < 0 || p.order < 0) return false;
    if (p.kind == 1 && !(p.axis[1] > p.axis[0])) return false;
    return true;
}

// The target loops (stride 1). Legacy (s2_many_prediction.cpp:204-397): the two axes other than
// the QB order run outside in increasing order, the order axis inside; a 1D predictor's axis
// covers [m, n - m) every other point (m = 3 for 1D4R, 5 for 1D4R shared1d and for 1D6R), the
// other axes every point; 2D4R's two axes cover [1, n - 1), the third [0, n), every other point
// along axis 0 (pair 01), 1 (pair 02) or 2 (pair 12). Common (:126-149): [5, n - 5) on every
// axis, points with an odd coordinate sum.
bool sweep_geometry(const Predictor &p, const u64 n[3], const std::string &targets, SweepGeom &g) {
    std::memset(&g, 0, sizeof g);
    for (int a = 0; a < 3; a++) g.n[a] = n[a];
    auto dist = [&](int a) { return a == 0 ? n[1] * n[2] : a == 1 ? n[2] : (u64)1; };
    g.dist[0] = dist(p.axis[0]);
    g.dist[1] = p.kind == 1 ? dist(p.axis[1]) : 0;
    g.kind = (uint32_t)p.kind;
    int k = 0;
    for (int a = 0; a < 3; a++)
        if (a != p.order) g.axis[k++] = (uint32_t)a;
    g.axis[2] = (uint32_t)p.order;
    g.line_per_thread = p.order != 2;
    if (targets == "common") {
        g.common = 1;
        for (int l = 0; l < 3; l++) {
            const u64 m = n[g.axis[l]];
            g.start[l] = 5;
            g.step[l] = 1;
            g.count[l] = m > 10 ? m - 10 : 0;
        }
        const u64 c = g.count[2];
        g.inner_odd = (c + 1) / 2;  // 5, 7, ... below n - 5
        g.inner_even = c / 2;       // 6, 8, ...
        g.lines = g.count[0] * g.count[1];
        g.per_line = std::max(g.inner_odd, g.inner_even);
        const u64 L0 = g.count[0], L1 = g.count[1];
        const u64 q0 = (L0 + 1) / 2 * ((L1 + 1) / 2) + L0 / 2 * (L1 / 2);
        g.targets = q0 * g.inner_odd + (L0 * L1 - q0) * g.inner_even;
        return true;
    }
    const bool shared1d = targets == "shared1d";
    const int doubled = p.kind == 1 ? (p.axis[0] == 0 && p.axis[1] == 1 ? 0 : p.axis[0] == 0 ? 1 : 2) : p.axis[0];
    for (int l = 0; l < 3; l++) {
        const int a = (int)g.axis[l];
        const bool on = a == p.axis[0] || (p.kind == 1 && a == p.axis[1]);
        const u64 m = p.kind == 1 ? 1 : p.kind == 2 ? 5 : (shared1d ? 5 : 3);
        const u64 lo = on ? m : 0, hi = on ? (n[a] > m ? n[a] - m : 0) : n[a];
        g.start[l] = lo;
        g.step[l] = a == doubled ? 2 : 1;
        g.count[l] = hi > lo ? (hi - lo + g.step[l] - 1) / g.step[l] : 0;
    }
    g.lines = g.count[0] * g.count[1];
    g.per_line = g.count[2];
    g.targets = g.lines * g.per_line;
    return true;
}

// Coefficient grids (s2_many_prediction.cpp:89-124, :199-201, :264-266).
bool coef_grid(const Predictor &p, const std::string &six, std::vector<std::pair<double, double>> &g, std::string &err) {
    g.clear();
    if (p.kind == 0) {
        for (int i = 0; i <= 12; i++) g.push_back({(double)((float)i / 32.0f), 0.0});
        return true;
    }
    if (p.kind == 1) {  // i / 24 in float, as i times the float reciprocal of 24
        for (int i = -6; i <= 6; i++) g.push_back({(double)((float)i * (1.0f / 24.0f)), 0.0});
        return true;
    }
    if (six == "transition") {
        g.push_back({1.0 / 6, 1.0 / 6});
        g.push_back({3.0 / 256, -25.0 / 256});
        for (int i = 0; i <= 12; i++) g.push_back({0.0, (8 - i) / 32.0});
        g.push_back({137.0 / 1536, 53.0 / 1536});
        for (int i = 0; i <= 12; i++) {
            g.push_back({1.0 / 12, (40 - 3 * i) * (1.0 / 192.0)});
            g.push_back({3.0 / 512, (39 - 8 * i) / 512.0});
        }
        return true;
    }
    if (six != "legacy" && six != "augmented") {
        err = "six-reference grid must be legacy, augmented or transition";
        return false;
    }
    static const int k1[] = {0, 11, 22, 31, 41}, k2[] = {0, 113, 248, 341, 453, 567, 680, 793};
    for (int a : k1)
        for (int b : k2) g.push_back({1.0 / 6 - (double)((float)a / 186.0f), 1.0 / 6 - (double)((float)b / 1488.0f)});
    if (six == "augmented") {
        std::vector<std::pair<double, double>> exact = {{3.0 / 256, -25.0 / 256}};
        for (int i = 0; i <= 12; i++) exact.push_back({0.0, (8 - i) / 32.0});
        for (const auto &c : exact) {
            auto it = std::find_if(g.begin(), g.end(), [&](const std::pair<double, double> &q) {
                return std::fabs(q.first - c.first) < 1e-7 && std::fabs(q.second - c.second) < 1e-7;
            });
            if (it == g.end()) g.push_back(c);
            else *it = c;
        }
    }
    return true;
}

SweepCoef make_coef(const Predictor &p, double c0, double c1) {
    SweepCoef c{};
    c.c0 = c0;
    c.c1 = c1;
    c.w = 0.5 - (c0 + c1);
    if (p.kind == 0) {
        c.lo = 0.25 - c0;
        c.hi = 0.25 + c0;
    } else if (p.kind == 1) {
        c.hi = 0.25 + c0;
        c.lo = 0.25 - c0;
    }
    return c;
}

// get_H1 (c_codes/get_H.hpp): the symbols enter the map in order of first occurrence, which
// gives the reference's iteration order; p = freq * (1 / size); H1 -= p log2 p fused.
double h1_of(const u64 *hist, const u64 *first, u64 range, int64_t lo, u64 size) {
    std::vector<std::pair<u64, int64_t>> seen;
    for (u64 i = 0; i < range; i++)
        if (hist[i]) seen.push_back({first[i], lo + (int64_t)i});
    std::sort(seen.begin(), seen.end());
    std::unordered_map<int64_t, u64> m;
    for (const auto &s : seen) m.emplace(s.second, hist[(u64)(s.second - lo)]);
    const double inv = 1.0 / (double)size;
    double h1 = 0;
    for (const auto &kv : m) {
        const double pr = (double)kv.second * inv;
        h1 = std::fma(-pr, std::log2(pr), h1);
    }
    return h1;
}

void finish_row(asz_sweep_row &r, double range) {  // s2_many_prediction.cpp:423-430
    const double S = (double)r.samples;
    r.cr = (double)(r.samples * sizeof(float)) / (double)r.zstd_bytes;
    r.br = (8 * sizeof(float)) / r.cr;
    r.h1_cr = (8 * sizeof(float)) / r.h1;
    r.rmse = std::sqrt(r.rmse_sum / S);
    r.mae = r.mae_sum / S;
    r.psnr = 10 * std::log10((range * range / r.mse_sum) * S);
}

u64 host_workers() { return std::max(1u, std::thread::hardware_concurrency()); }

// f(i, w) for i in [0, n) on up to host_workers() threads; w is the calling worker's index.
template <class F>
void parallel_for(u64 n, F f) {
    const u64 nt = std::min<u64>(host_workers(), n);
    if (nt <= 1) {
        for (u64 i = 0; i < n; i++) f(i, 0);
        return;
    }
    std::atomic<u64> next{0};
    std::vector<std::thread> th;
    for (u64 t = 0; t < nt; t++)
        th.emplace_back([&, t] {
            for (u64 i; (i = next.fetch_add(1)) < n;) f(i, t);
        });
    for (auto &t : th) t.join();
}

constexpr u64 kMaxSymbolRange = 1ull << 27;

}  // namespace

#define CK(call)                                                                                         \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return host::ctx_fail(ctx, ASZ_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace asz::host {
void sweep_release(void *state) {
    SweepState *s = (SweepState *)state;
    if (!s) return;
    for (DevBuf *b : {&s->coef, &s->qb, &s->part, &s->sums, &s->mm, &s->hist, &s->first, &s->tab, &s->pay, &s->enc, &s->cub})
        b->release();
    s->small.release();
    s->counts.release();
    s->payload.release();
    for (WorkerScratch &w : s->ws)
        if (w.cc) ZSTD_freeCCtx(w.cc);
    delete s;
}
}  // namespace asz::host

extern "C" int asz_sweep_coefs(const char *predictor, const char *six_grid, double *c0, double *c1, uint64_t cap,
                               uint64_t *count) {
    Predictor p;
    std::string err;
    std::vector<std::pair<double, double>> g;
    if (!parse_predictor(predictor, p, err) || !coef_grid(p, six_grid ? six_grid : "legacy", g, err)) return ASZ_E_ARG;
    for (u64 i = 0; i < g.size() && i < cap; i++) {
        if (c0) c0[i] = g[i].first;
        if (c1) c1[i] = g[i].second;
    }
    if (count) *count = g.size();
    return ASZ_OK;
}

extern "C" int asz_sweep_targets(const uint64_t dims[3], const char *predictor, const char *targets, uint64_t *coords,
                                 uint64_t cap, uint64_t *count) {
    Predictor p;
    std::string err;
    const std::string tg = targets ? targets : "legacy";
    if (!dims || !count || !parse_predictor(predictor, p, err)) return ASZ_E_ARG;
    if (tg != "legacy" && tg != "shared1d" && tg != "common") return ASZ_E_ARG;
    SweepGeom g;
    sweep_geometry(p, dims, tg, g);
    *count = g.targets;
    if (!coords) return ASZ_OK;
    if (cap < g.targets) return ASZ_E_ARG;
    u64 visited = 0;
    for (u64 it = 0; it < g.lines * g.per_line; it++) {
        u64 i[3], j;
        if (!sweep_target(g, it, i, j)) continue;
        if (j >= g.targets) return ASZ_E_DEVICE;
        for (int a = 0; a < 3; a++) coords[3 * j + a] = i[a];
        visited++;
    }
    return visited == g.targets ? ASZ_OK : ASZ_E_DEVICE;
}

extern "C" int asz_sweep(asz_ctx *ctx, const float *data, int on_device, const uint64_t dims[3], const char *predictor,
                         const char *targets, const char *six_grid, const double *rel_eb, uint64_t n_eb, asz_sweep_row *rows,
                         uint64_t cap, uint64_t *n_rows, float *min_max) {
    if (!ctx) return ASZ_E_ARG;
    auto bad = [&](int code, const std::string &m) { return host::ctx_fail(ctx, code, m); };
    if (!data || !dims || !rel_eb || !n_rows) return bad(ASZ_E_ARG, "null argument");
    Predictor p;
    std::string err;
    if (!parse_predictor(predictor, p, err)) return bad(ASZ_E_ARG, err);
    const std::string tg = targets ? targets : "legacy", six = six_grid ? six_grid : "legacy";
    if (tg != "legacy" && tg != "shared1d" && tg != "common") return bad(ASZ_E_ARG, "target mode must be legacy, shared1d or common");
    std::vector<std::pair<double, double>> grid;
    if (!coef_grid(p, six, grid, err)) return bad(ASZ_E_ARG, err);
    if (n_eb == 0) return bad(ASZ_E_ARG, "error-bound grid is empty");
    for (u64 i = 0; i < n_eb; i++)
        if (!std::isfinite(rel_eb[i]) || rel_eb[i] <= 0) return bad(ASZ_E_ARG, "error bounds must be positive and finite");
    u64 N = 1;
    for (int a = 0; a < 3; a++) {  // s2_many_prediction.cpp:509-515
        if (dims[a] < 12 || N > ULLONG_MAX / dims[a]) return bad(ASZ_E_ARG, "invalid dimensions; each dimension must be at least 12");
        N *= dims[a];
    }
    SweepGeom g;
    sweep_geometry(p, dims, tg, g);
    const u64 K = grid.size(), S = g.targets;
    *n_rows = n_eb * K;
    if (cap < n_eb * K) return bad(ASZ_E_ARG, "row buffer too small");
    if (S == 0) return bad(ASZ_E_DATA, "no prediction targets");
    cudaStream_t st = host::ctx_stream(ctx);
    void *&sp = host::ctx_sweep_state(ctx);
    if (!sp) sp = new SweepState();
    SweepState &W = *(SweepState *)sp;

    const float *d_in = data;
    int rc;
    if (!on_device && (rc = host::ctx_upload(ctx, data, N, &d_in))) return rc;
    float mn, mx;  // s2_many_prediction.cpp:521-527
    if ((rc = host::ctx_range(ctx, d_in, N, true, mn, mx))) {
        if (rc == ASZ_E_DATA) return bad(ASZ_E_DATA, "input contains nonfinite values");
        return rc;
    }
    if (min_max) {
        min_max[0] = mn;
        min_max[1] = mx;
    }
    if (!(mx > mn)) return bad(ASZ_E_DATA, "constant input");
    const double range = (double)mx - (double)mn;

    // Coefficients per batch: their QB streams share the device with the field.
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const u64 budget = std::max<u64>(S * 8, std::min<u64>(free_b / 3, 24ull << 30));
    const u64 KB = std::max<u64>(1, std::min<u64>(K, budget / (S * 8)));
    const uint32_t nparts = sweep_predict_grid(g);
    CK(W.coef.reserve(KB * sizeof(SweepCoef)));
    CK(W.qb.reserve(KB * S * 8));
    CK(W.part.reserve(KB * nparts * 3 * sizeof(double)));
    CK(W.sums.reserve(KB * 3 * sizeof(double) + KB * 2 * sizeof(long long)));
    CK(W.small.reserve(KB * (sizeof(SweepCoef) + 3 * sizeof(double) + 2 * sizeof(long long))));
    SweepCoef *h_coef = (SweepCoef *)W.small.p;
    double *h_sums = (double *)(h_coef + KB);
    long long *h_mm = (long long *)(h_sums + 3 * KB);
    double *d_sums = W.sums.as<double>();
    long long *d_mm = (long long *)(d_sums + 3 * KB);
    int64_t *d_qb = W.qb.as<int64_t>();

    for (u64 e = 0; e < n_eb; e++) {
        const double abs_eb = rel_eb[e] * range;  // :195-196
        const double neg_2_eb = 1 / (2 * abs_eb);
        for (u64 k0 = 0; k0 < K; k0 += KB) {
            const u64 kc = std::min<u64>(KB, K - k0);
            for (u64 k = 0; k < kc; k++) {
                h_coef[k] = make_coef(p, grid[k0 + k].first, grid[k0 + k].second);
                h_mm[2 * k] = LLONG_MAX;
                h_mm[2 * k + 1] = LLONG_MIN;
            }
            CK(cudaMemcpyAsync(W.coef.p, h_coef, kc * sizeof(SweepCoef), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_mm, h_mm, kc * 2 * sizeof(long long), cudaMemcpyHostToDevice, st));
            CK(launch_sweep_predict(d_in, g, W.coef.as<SweepCoef>(), (uint32_t)kc, abs_eb, neg_2_eb, d_qb, S,
                                    W.part.as<double>(), d_mm, st));
            CK(launch_sweep_sums(W.part.as<double>(), nparts, (uint32_t)kc, d_sums, st));
            CK(cudaMemcpyAsync(h_sums, d_sums, kc * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(h_mm, d_mm, kc * 2 * sizeof(long long), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const auto t_enc = clk::now();
            // Histograms and first positions of every stream of the batch.
            std::vector<u64> hoff(kc + 1, 0);
            for (u64 k = 0; k < kc; k++) {
                const u64 r = (u64)(h_mm[2 * k + 1] - h_mm[2 * k]) + 1;
                if (h_mm[2 * k] > h_mm[2 * k + 1] || r > kMaxSymbolRange)
                    return bad(ASZ_E_UNSUPPORTED, "QB symbol range exceeds 2^27 values");
                hoff[k + 1] = hoff[k] + r;
            }
            const u64 htot = hoff[kc];
            CK(W.hist.reserve(htot * 8));
            CK(W.first.reserve(htot * 8));
            CK(W.counts.reserve(htot * 16));
            CK(cudaMemsetAsync(W.hist.p, 0, htot * 8, st));
            CK(cudaMemsetAsync(W.first.p, 0xff, htot * 8, st));
            for (u64 k = 0; k < kc; k++) {
                const int64_t *s = d_qb + k * S;
                CK(launch_sweep_stats(s, S, h_mm[2 * k], hoff[k + 1] - hoff[k], W.hist.as<unsigned long long>() + hoff[k],
                                      W.first.as<unsigned long long>() + hoff[k], st));
            }
            u64 *h_hist = (u64 *)W.counts.p, *h_first = h_hist + htot;
            CK(cudaMemcpyAsync(h_hist, W.hist.p, htot * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(h_first, W.first.p, htot * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            // Codes and H1 on the host threads.
            std::vector<HuffCode> code(kc);
            std::vector<double> h1(kc);
            std::vector<std::string> cerr(kc);
            std::vector<char> ok(kc, 1);
            parallel_for(kc, [&](u64 k, u64) {
                const u64 r = hoff[k + 1] - hoff[k];
                std::vector<u64> hv(h_hist + hoff[k], h_hist + hoff[k] + r);
                ok[k] = build_code(hv, h_mm[2 * k], h_mm[2 * k + 1], S, true, code[k], cerr[k]);
                h1[k] = h1_of(h_hist + hoff[k], h_first + hoff[k], r, h_mm[2 * k], S);
            });
            for (u64 k = 0; k < kc; k++)
                if (!ok[k]) return bad(ASZ_E_UNSUPPORTED, cerr[k]);
            // Encode every stream that has a payload in one tiled launch.
            std::vector<EncStream> es;
            std::vector<u64> toff{0}, tab_off(kc, 0), word_off(kc + 1, 0);
            u64 tab_tot = 0;
            for (u64 k = 0; k < kc; k++) {
                tab_off[k] = tab_tot;
                tab_tot += code[k].table.size();
                word_off[k + 1] = word_off[k] + (code[k].maxval == 1 ? 0 : (code[k].bits + 31) / 32);
            }
            CK(W.tab.reserve(std::max<u64>(tab_tot, 1) * sizeof(CodeEntry)));
            CK(W.pay.reserve(std::max<u64>(word_off[kc], 1) * 4));
            CK(W.payload.reserve(std::max<u64>(word_off[kc], 1) * 4 + tab_tot * sizeof(CodeEntry)));
            CodeEntry *h_tab = (CodeEntry *)(W.payload.p + word_off[kc] * 4);
            for (u64 k = 0; k < kc; k++) {
                std::memcpy(h_tab + tab_off[k], code[k].table.data(), code[k].table.size() * sizeof(CodeEntry));
                if (code[k].maxval == 1) continue;
                es.push_back(EncStream{d_qb + k * S, S, h_mm[2 * k], W.tab.as<CodeEntry>() + tab_off[k],
                                       W.pay.as<uint32_t>() + word_off[k]});
                toff.push_back(toff.back() + (S + enc_tile<int64_t>() - 1) / enc_tile<int64_t>());
            }
            const u64 nt = toff.back();
            if (nt) {
                CK(cudaMemcpyAsync(W.tab.p, h_tab, tab_tot * sizeof(CodeEntry), cudaMemcpyHostToDevice, st));
                CK(cudaMemsetAsync(W.pay.p, 0, word_off[kc] * 4, st));
                size_t tb = 0;
                CK(launch_encode_tiles<int64_t>(nullptr, 0, nullptr, nt, nullptr, nullptr, nullptr, tb, st));
                const u64 o_es = 0, o_toff = (es.size() * sizeof(EncStream) + 15) / 16 * 16,
                          o_bits = o_toff + (toff.size() * 8 + 15) / 16 * 16, o_scan = o_bits + (nt + 1) * 8 + 8;
                CK(W.enc.reserve(o_scan + (nt + 1) * 8 + 8));
                CK(W.cub.reserve(std::max<size_t>(tb, 16)));
                uint8_t *eb = W.enc.as<uint8_t>();
                CK(cudaMemcpyAsync(eb + o_es, es.data(), es.size() * sizeof(EncStream), cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(eb + o_toff, toff.data(), toff.size() * 8, cudaMemcpyHostToDevice, st));
                CK(cudaMemsetAsync(eb + o_bits + nt * 8, 0, 8, st));
                tb = W.cub.cap;
                CK(launch_encode_tiles<int64_t>((const EncStream *)(eb + o_es), (uint32_t)es.size(), (const u64 *)(eb + o_toff),
                                                nt, (u64 *)(eb + o_bits), (u64 *)(eb + o_scan), W.cub.p, tb, st));
                u64 enc_err = 0;
                CK(cudaMemcpyAsync(&enc_err, eb + o_scan, sizeof(u64), cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(W.payload.p, W.pay.p, word_off[kc] * 4, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                if (enc_err) return host::ctx_fail(ctx, ASZ_E_DEVICE, "Huffman encoder: a tile's wait for the tiles before it timed out");
            }
            // Frame each stream (save + encode, huffman.hpp) and compress it with zstd level 3.
            std::vector<u64> hb(kc), zb(kc);
            std::vector<char> zok(kc, 1);
            if (W.ws.size() < host_workers()) W.ws.resize(host_workers());
            parallel_for(kc, [&](u64 k, u64 w) {
                const HuffCode &c = code[k];
                WorkerScratch &sc = W.ws[w];
                const u64 pay = c.maxval == 1 ? 0 : (c.bits + 7) / 8, len = c.save_size() + 8 + pay;
                if (sc.buf.size() < len) sc.buf.resize(len);
                write_tree(c, sc.buf.data());
                write_len_word(c, sc.buf.data() + c.save_size());
                if (pay) std::memcpy(sc.buf.data() + c.save_size() + 8, W.payload.p + word_off[k] * 4, pay);
                if (sc.z.size() < ZSTD_compressBound(len)) sc.z.resize(ZSTD_compressBound(len));
                if (!sc.cc) sc.cc = ZSTD_createCCtx();
                const size_t n = sc.cc ? ZSTD_compressCCtx(sc.cc, sc.z.data(), sc.z.size(), sc.buf.data(), len, 3)
                                       : ZSTD_compress(sc.z.data(), sc.z.size(), sc.buf.data(), len, 3);
                zok[k] = !ZSTD_isError(n);
                hb[k] = len;
                zb[k] = n;
            });
            const double enc_s = std::chrono::duration<double>(clk::now() - t_enc).count();
            for (u64 k = 0; k < kc; k++) {
                if (!zok[k]) return bad(ASZ_E_DATA, "zstd compression failed");
                asz_sweep_row &r = rows[e * K + k0 + k];
                std::memset(&r, 0, sizeof r);
                r.rel_eb = rel_eb[e];
                r.c0 = grid[k0 + k].first;
                r.c1 = grid[k0 + k].second;
                r.samples = S;
                r.huffman_bytes = hb[k];
                r.zstd_bytes = zb[k];
                r.mse_sum = h_sums[3 * k];
                r.rmse_sum = h_sums[3 * k + 1];
                r.mae_sum = h_sums[3 * k + 2];
                r.h1 = h1[k];
                r.encode_seconds = enc_s / (double)kc;
                finish_row(r, range);
            }
        }
    }
    return ASZ_OK;
}
