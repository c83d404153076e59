// Host orchestration of the B200 compression path and the C ABI in include/asz_b200.h.
//
// Compress (c_codes/asz_core/compress.tpp:147-321 behind s1_compress.cpp:153-341):
//   data range on the GPU -> default slope (GPU proxies, glibc log10f on the host) -> pivots ->
//   per round: t selection and prediction kernels -> replay of ambiguous t decisions on the
//   host -> histograms -> Huffman codes built on the host -> GPU encoding -> stream assembly
//   -> libzstd level 3.
// Decompress (c_codes/asz_core/decompress.tpp:79-208): libzstd -> header and tree parsing ->
//   GPU Huffman decoding -> pivots -> per-round reconstruction kernels.
//
// Host floating point in this file restates the reference's scalar steps and is built with
// -ffp-contract=off; glibc's log10f, log2f, cbrt and pow are called where the reference calls
// them, so the host values are the reference's on the same machine.
#include <cuda_runtime.h>
#include <immintrin.h>

#include <algorithm>
#include <chrono>
#include <optional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <array>
#include <atomic>
#include <unordered_map>
#include <random>
#include <string>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../geometry.cuh"
#include "../launch.h"
#include "../listsim.cuh"
#include "../../../include/asz_b200.h"
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

double secs(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// llround of a float as the reference's -Ofast build computes it (see dev_common.cuh).
int64_t host_lround_f(float x) {
    volatile float h = std::copysign(0x1.fffffep-2f, x);
    volatile float s = x + h;
    return (int64_t)s;
}

struct Plan {
    std::vector<std::string> pred;  // "cubicD_OOO"
    std::vector<int> dir, order;
};

bool parse_plan(const char *text, Plan &plan, std::string &err) {
    // parse_predictor_plan (s1_compress.cpp:5-28).
    std::string t(text);
    size_t b = 0;
    while (b <= t.size()) {
        size_t e = t.find(',', b);
        std::string p = t.substr(b, e == std::string::npos ? std::string::npos : e - b);
        bool ok = false;
        for (int d = 0; d < 3; d++)
            for (const char *o : {"120", "021", "012"})
                if (p == std::string("cubic") + char('0' + d) + "_" + o) ok = true;
        if (!ok) {
            err = "invalid predictor in plan: " + p;
            return false;
        }
        plan.pred.push_back(p);
        plan.dir.push_back(p[5] - '0');
        plan.order.push_back(p[9] - '0');
        if (e == std::string::npos) break;
        b = e + 1;
    }
    if (plan.pred.empty()) {
        err = "predictor plan cannot be empty";
        return false;
    }
    return true;
}

struct Geometry {
    FieldGeom fg{};
    std::vector<RoundGeom> rounds;
    std::vector<u64> tab_count, tab_prefix;     // per round, per axis, per block
    std::vector<AxisEntry> ent;                 // per round, per axis, per lattice index
    std::vector<std::vector<ClassInfo>> classes;
    std::vector<uint32_t> cap;                  // max samples per round
    PivotGeom pg{};
    u64 pivots = 0, nblocks = 0;
};

}  // namespace

namespace {
// Worker threads kept for a context's host-side parallel loops: run(n, f) calls f(0..n-1) on the
// workers and the calling thread, and returns when all calls have returned.
class HostPool {
public:
    explicit HostPool(unsigned workers) {
        for (unsigned i = 0; i < workers; i++) th_.emplace_back([this] { loop(); });
    }
    ~HostPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void run(uint64_t n, const std::function<void(uint64_t)> &f) {
        {
            std::lock_guard<std::mutex> g(mu_);
            fn_ = &f;
            n_ = n;
            next_ = 0;
            active_ = th_.size();
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> l(mu_);
        done_.wait(l, [&] { return active_ == 0; });
        fn_ = nullptr;
    }

private:
    void work() {
        for (uint64_t j; (j = next_.fetch_add(1)) < n_;) (*fn_)(j);
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> g(mu_);
            if (--active_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(uint64_t)> *fn_ = nullptr;
    std::atomic<uint64_t> next_{0};
    uint64_t n_ = 0, gen_ = 0;
    size_t active_ = 0;
    bool stop_ = false;
};
}  // namespace

namespace {
// One host thread that runs submitted jobs in order: the Huffman code of a round's stream is built
// here while the device runs the later rounds. wait() returns when every submitted job is done.
class SerialWorker {
public:
    SerialWorker() : th_([this] { loop(); }) {}
    ~SerialWorker() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        th_.join();
    }
    void submit(std::function<void()> f) {
        {
            std::lock_guard<std::mutex> g(mu_);
            q_.push_back(std::move(f));
            pending_++;
        }
        cv_.notify_all();
    }
    void wait() {
        std::unique_lock<std::mutex> l(mu_);
        done_.wait(l, [&] { return pending_ == 0; });
    }

private:
    void loop() {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;
                f = std::move(q_.front());
                q_.erase(q_.begin());
            }
            f();
            std::lock_guard<std::mutex> g(mu_);
            if (--pending_ == 0) done_.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::vector<std::function<void()>> q_;
    size_t pending_ = 0;
    bool stop_ = false;
    std::thread th_;
};
}  // namespace

struct asz_ctx {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    // Copies of each round's histogram window run here, behind the round's kernel, while the main
    // stream goes on with the next round; their events (two per round) order the builder thread.
    cudaStream_t side = nullptr;
    std::vector<cudaEvent_t> round_ev;
    DevBuf hwin;          // per QB stream of the rounds: kHistWin 64-bit bins
    DevBuf slab_idx, slab_val, slab_cmp;  // slabs: slope-sample indices, gathered values, compact copy
    DevBuf gscratch, spill2;  // exact replay of groups larger than shared memory: working sets, what is left
    PinnedBuf hwin_host;  // their copies, with each stream's [min, max] and overflow word
    std::unique_ptr<SerialWorker> builder;
    std::string err;
    // Device buffers.
    DevBuf in, rec, qb, tval, tint, misc, scratch, log2arena, hist, codes, bitoff, cubtmp, payload, amb, overrides,
        classes, axis, pre, chunks, out, proxies, tlist, spill, iota, plan_qb, plan_e, plan_aux, plan_pay, probe_in, probe_pred,
        rounds_dev, lines_bail, lines_resume, enc;
    // Batches (asz_compress_batch): per-field slices of these arenas, the captured round sequence
    // of the last batch, and the launch shapes the autotuner chose per batch shape.
    DevBuf b_in, b_rec, b_qb, b_tval, b_tint, b_ent, b_cls, b_rounds, b_qoff, b_range, b_range0, b_prox, b_amb, b_cnt,
        b_fields, b_goff, b_poff, b_ioff, b_queue, b_hand, b_spill, b_spill2;
    std::vector<uint64_t> batch_graph_key;
    cudaGraphExec_t batch_graph = nullptr;
    std::map<std::vector<uint64_t>, std::array<uint32_t, 3>> batch_tuned;
    // 0: certified fast path + exact path for the rest; 1: exact path for all groups; 2: as 0, with
    // the rounds of all-axis-2 plans fused per column of lines.
    int tsel_mode = 0;
    // Cached glibc log2f tables, keyed by sample count.
    std::map<uint32_t, uint32_t> log2_off;
    std::vector<float> log2_host;
    u64 log2_dev_len = 0;
    // Last compress call, for the debug accessors.
    std::vector<u64> qb_off, qb_len;
    u64 t_len = 0, n_total = 0;
    const float *last_in = nullptr;   // device input of the last compress call
    // Gradient tuner problem (asz_grad_setup -> asz_grad_gather).
    Geometry grad_G;
    const float *grad_in = nullptr;
    std::vector<uint32_t> grad_off;
    std::vector<float> grad_meta;
    float last_min = 0, last_max = 0;
    PinnedBuf pre_zstd;   // the last compress call's stream before zstd
    PinnedBuf batch_pre[2];  // batches: two chunks of fields' streams, one encoding while one is compressed
    PinnedBuf raw_in;     // decompress: the stream after zstd
    bool have_last = false;
    // Profiling (asz_profile_*).
    bool prof = false;
    struct ProfSlot {
        std::string name;
        uint64_t launches = 0;
        double ms = 0;
        uint64_t bytes = 0;
    };
    std::vector<ProfSlot> prof_slots;
    struct Pending {
        cudaEvent_t a, b;
        size_t slot;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    // Prediction sweep (host/sweep.cpp): its buffers, owned there.
    void *sweep = nullptr;
    // zstd contexts kept across calls (one per concurrent user), and the decompression context.
    std::mutex zmu;
    std::vector<ZSTD_CCtx *> zfree;
    ZSTD_DCtx *zd = nullptr;
    // Host worker threads for the code builds (created on first use).
    std::unique_ptr<HostPool> pool;
};

namespace {
cudaEvent_t prof_event(asz_ctx *c) {
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
size_t prof_slot(asz_ctx *c, const char *name) {
    for (size_t i = 0; i < c->prof_slots.size(); i++)
        if (c->prof_slots[i].name == name) return i;
    c->prof_slots.push_back({name, 0, 0, 0});
    return c->prof_slots.size() - 1;
}
// Collects finished event pairs into the slots (called after a stream synchronisation).
void prof_collect(asz_ctx *c) {
    for (auto &p : c->pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        c->prof_slots[p.slot].ms += ms;
        c->prof_slots[p.slot].launches++;
        c->event_pool.push_back(p.a);
        c->event_pool.push_back(p.b);
    }
    c->pending.clear();
}
// RAII timer around one launch.
// Host wall time of one phase of a call, recorded as "host:<phase>" while profiling is on.
struct HostScope {
    asz_ctx *c;
    size_t slot = 0;
    clk::time_point t0;
    HostScope(asz_ctx *ctx, const char *name) : c(ctx) {
        if (!c->prof) return;
        slot = prof_slot(c, name);
        t0 = clk::now();
    }
    ~HostScope() {
        if (!c->prof) return;
        c->prof_slots[slot].ms += 1000.0 * secs(t0, clk::now());
        c->prof_slots[slot].launches++;
    }
};

struct ProfScope {
    asz_ctx *c;
    cudaEvent_t a = nullptr, b = nullptr;
    size_t slot = 0;
    ProfScope(asz_ctx *ctx, const char *name, uint64_t bytes) : c(ctx) {
        if (!c->prof) return;
        slot = prof_slot(c, name);
        c->prof_slots[slot].bytes += bytes;
        a = prof_event(c);
        b = prof_event(c);
        cudaEventRecord(a, c->stream);
    }
    ~ProfScope() {
        if (!a) return;
        cudaEventRecord(b, c->stream);
        c->pending.push_back({a, b, slot});
    }
};
}  // namespace

namespace {

int fail(asz_ctx *c, int code, const std::string &m) {
    c->err = m;
    return code;
}

// zstd level 3 through a context from the asz_ctx's pool (ZSTD_compressCCtx gives ZSTD_compress's
// bytes); safe from several threads at once.
size_t zstd3(asz_ctx *c, void *dst, size_t cap, const void *src, size_t n) {
    ZSTD_CCtx *z = nullptr;
    {
        std::lock_guard<std::mutex> g(c->zmu);
        if (!c->zfree.empty()) {
            z = c->zfree.back();
            c->zfree.pop_back();
        }
    }
    if (!z) z = ZSTD_createCCtx();
    if (!z) return ZSTD_compress(dst, cap, src, n, 3);
    const size_t r = ZSTD_compressCCtx(z, dst, cap, src, n, 3);
    std::lock_guard<std::mutex> g(c->zmu);
    c->zfree.push_back(z);
    return r;
}

// Output blocks (the .asz buffers that callers release with asz_free). Each carries a header with
// its capacity. asz_free returns a block to a small cache that later outputs take (best fit), so a
// caller compressing field after field reuses memory whose pages are already mapped: the first
// writes to fresh pages and their unmapping on release cost about as much as zstd itself. The
// cache holds at most kOutCacheBlocks blocks and kOutCacheBytes bytes; asz_release_output_cache
// empties it.
constexpr uint64_t kOutMagic = 0x415a534f55544255ull;
constexpr size_t kOutHeader = 64;
constexpr size_t kOutCacheBlocks = 64;
constexpr uint64_t kOutCacheBytes = 2ull << 30;
struct OutHeader {
    uint64_t magic, cap;
};
std::mutex g_out_mu;
std::vector<uint8_t *> g_out_cache;  // block starts (header), oldest first
uint64_t g_out_cached = 0;

uint8_t *out_alloc(size_t n) {
    {
        std::lock_guard<std::mutex> g(g_out_mu);
        size_t best = g_out_cache.size();
        for (size_t i = 0; i < g_out_cache.size(); i++) {
            const uint64_t cap = reinterpret_cast<OutHeader *>(g_out_cache[i])->cap;
            if (cap >= n && (best == g_out_cache.size() || cap < reinterpret_cast<OutHeader *>(g_out_cache[best])->cap)) best = i;
        }
        if (best < g_out_cache.size()) {
            uint8_t *b = g_out_cache[best];
            g_out_cache.erase(g_out_cache.begin() + (std::ptrdiff_t)best);
            g_out_cached -= reinterpret_cast<OutHeader *>(b)->cap;
            return b + kOutHeader;
        }
    }
    uint8_t *b = (uint8_t *)std::malloc(kOutHeader + (n ? n : 1));
    if (!b) return nullptr;
    *reinterpret_cast<OutHeader *>(b) = OutHeader{kOutMagic, (uint64_t)(n ? n : 1)};
    return b + kOutHeader;
}

void out_release(uint8_t *p) {
    uint8_t *b = p - kOutHeader;
    std::lock_guard<std::mutex> g(g_out_mu);
    g_out_cache.push_back(b);
    g_out_cached += reinterpret_cast<OutHeader *>(b)->cap;
    while (g_out_cache.size() > kOutCacheBlocks || g_out_cached > kOutCacheBytes) {
        g_out_cached -= reinterpret_cast<OutHeader *>(g_out_cache.front())->cap;
        std::free(g_out_cache.front());
        g_out_cache.erase(g_out_cache.begin());
    }
}

#define CK(call)                                                                    \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) return fail(ctx, ASZ_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int validate(asz_ctx *ctx, const asz_params &p, bool compress_side) {
    // validate_parameters (s1_compress.cpp:49-99) and s1_decompress.cpp:112-125.
    auto bad = [&](const char *m) { return fail(ctx, ASZ_E_ARG, m); };
    if (!(p.pivot_eb_ratio > 0 && p.pivot_eb_ratio <= 1)) return bad("pivot_eb_ratio must be in (0,1]");
    if (!(p.eb_ratio > 0 && p.eb_ratio <= 1)) return bad("eb_ratio must be in (0,1]");
    if (!(p.slope_ratio > 0 && p.slope_ratio <= 1)) return bad("slope_ratio must be in (0,1]");
    if (p.block_pivot_ratio == 0) return bad("block_pivot_ratio must be positive");
    if (p.max_layer_num == 0 || p.max_layer_num > 63) return bad("max_layer_num must be in [1,63]");
    if (p.full_predictor_search_layer_num == 0 || p.full_predictor_search_layer_num > 63)
        return bad("full_predictor_search_layer_num must be in [1,63]");
    if (p.t_precision < 16 || p.t_precision % 16 != 0) return bad("t_precision must be a positive multiple of 16");
    if (!compress_side) return ASZ_OK;
    if (p.generate_config_sample_stride == 0) return bad("generate_config_sample_stride must be positive");
    if (p.h1_block_sampling_num == 0) return bad("h1_block_sampling_num must be positive");
    if (!(p.stat_eb_ratio > 0 && p.stat_eb_ratio <= 1)) return bad("stat_eb_ratio must be in (0,1]");
    if (p.predictor_family_suffix_layers == 0) return bad("predictor_family_suffix_layers must be positive");
    if (p.predictor_family_sample_blocks == 0) return bad("predictor_family_sample_blocks must be positive");
    if (p.predictor_family_sample_point_limit == 0) return bad("predictor_family_sample_point_limit must be positive");
    if (!(p.predictor_family_sample_fraction_limit > 0 && p.predictor_family_sample_fraction_limit <= 1))
        return bad("predictor_family_sample_fraction_limit must be in (0,1]");
    if (p.predictor_family_coarse_probe_block_pivot_ratio == 0 || p.predictor_family_fine_probe_block_pivot_ratio == 0)
        return bad("predictor family probe block pivot ratios must be positive");
    if (!(p.predictor_family_fine_eb_threshold > 0 && std::isfinite(p.predictor_family_fine_eb_threshold)))
        return bad("predictor_family_fine_eb_threshold must be positive and finite");
    if (!(p.default_slope_invalid_ratio_threshold > 0 && p.default_slope_invalid_ratio_threshold <= 1))
        return bad("default_slope_invalid_ratio_threshold must be in (0,1]");
    if (!(p.default_slope_fallback > 0 && std::isfinite(p.default_slope_fallback)))
        return bad("default_slope_fallback must be positive and finite");
    if (!(p.default_slope_eb_span > 1 && std::isfinite(p.default_slope_eb_span)))
        return bad("default_slope_eb_span must be greater than 1 and finite");
    float tmin = p.t_min, tmax = p.t_max;
    if (!(tmin >= 0 && tmin <= tmax && tmax <= 0.5)) return bad("t range must satisfy 0 <= t_min <= t_max <= 0.5");
    float a = tmin * (float)p.t_precision, b = tmax * (float)p.t_precision;
    if (std::fabs(a - std::round(a)) > 1e-6 || std::fabs(b - std::round(b)) > 1e-6)
        return bad("t_min and t_max must be representable at t_precision");
    if (tmin > 4.0f / 16 || tmax < 5.0f / 16) return bad("t range must include 4/16 and 5/16");
    // set_t_candidates (asz_param.hpp:194-204).
    if (p.t_precision % 32 || tmin > 1.0f / 16 || tmax < 11.0f / 32)
        return bad("block t candidates require t_precision divisible by 32 and t range covering [1/16,11/32]");
    return ASZ_OK;
}

int validate_dims(asz_ctx *ctx, const uint64_t dims[3], float rel_eb) {
    if (!dims || dims[0] < 7 || dims[1] < 7 || dims[2] < 7) return fail(ctx, ASZ_E_ARG, "all three dimensions must be at least 7");
    if (!(rel_eb > 0 && std::isfinite(rel_eb))) return fail(ctx, ASZ_E_ARG, "relative error bound must be positive and finite");
    u64 n = 1;
    for (int a = 0; a < 3; a++) {
        if (n > std::numeric_limits<u64>::max() / dims[a]) return fail(ctx, ASZ_E_ARG, "data dimensions overflow the element count");
        n *= dims[a];
    }
    if (n > std::numeric_limits<size_t>::max() / sizeof(float))
        return fail(ctx, ASZ_E_ARG, "data dimensions exceed the addressable input size");
    return ASZ_OK;
}

// Plan geometry (generate_config.tpp:52-68) and per-round tables.
// The round kernels index lines (k0, k1) and positions along axis 2 in 32 bits, and the axis
// tables store coordinates and box extents in 32 bits.
bool kernel_limits_ok(const struct Geometry &G);

// Geometry of a compression of `dims` with `plan`; blocks and pivots start at `origin` (all zero
// for a whole field; the predictor-family probe's local contexts start past a halo).
// Slab of a field cut along axis 0 at block boundaries (asz_compress_slab): axis 0 has exactly
// `blocks0` blocks (the last one ends at the array's last plane, the slab's upper face), and with
// `skip_face` the plane at the origin belongs to the slab below, so the pivot lattice starts one
// pivot stride above it.
struct SlabGeom {
    u64 blocks0 = 0;
    bool skip_face = false;
};

void build_geometry(const uint64_t dims[3], const Plan &plan, const asz_params &p, float abs_eb, float default_slope,
                    bool quintic, Geometry &G, const uint64_t origin[3] = nullptr, const SlabGeom *slab = nullptr) {
    FieldGeom &fg = G.fg;
    const u64 L = plan.pred.size();
    for (int a = 0; a < 3; a++) {
        fg.n[a] = dims[a];
        fg.origin[a] = origin ? origin[a] : 0;
        fg.pivot_stride[a] = 1;
    }
    for (u64 l = 0; l < L; l++) fg.pivot_stride[plan.dir[l]] *= 2;
    for (int a = 0; a < 3; a++) {
        fg.block_shape[a] = fg.pivot_stride[a] * p.block_pivot_ratio;
        const u64 span = fg.n[a] > fg.origin[a] ? fg.n[a] - fg.origin[a] : 0;
        fg.block_num[a] = (span + fg.block_shape[a] - 1) / fg.block_shape[a];
    }
    if (slab && slab->blocks0) fg.block_num[0] = slab->blocks0;
    fg.layer_num = (uint32_t)L;
    fg.quintic = quintic ? 1 : 0;
    fg.t_precision = p.t_precision;
    G.nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    // Pivots (compress.tpp:162-175).
    G.pivots = 1;
    for (int a = 0; a < 3; a++) {
        const u64 o = fg.origin[a] + (a == 0 && slab && slab->skip_face ? fg.pivot_stride[0] : 0);
        const u64 span = fg.n[a] > o ? fg.n[a] - o : 0;
        G.pg.cnt[a] = (span + fg.pivot_stride[a] - 1) / fg.pivot_stride[a];
        G.pg.stride[a] = fg.pivot_stride[a];
        G.pg.origin[a] = o;
        G.pivots *= G.pg.cnt[a];
    }
    G.pg.n1n2 = fg.n[1] * fg.n[2];
    G.pg.n2 = fg.n[2];
    float pivot_eb = abs_eb * p.pivot_eb_ratio;
    G.pg.rp = 0.5 / (double)pivot_eb;
    G.pg.peb2 = (double)pivot_eb + (double)pivot_eb;

    u64 stride[3] = {fg.pivot_stride[0], fg.pivot_stride[1], fg.pivot_stride[2]};
    G.rounds.assign(L, RoundGeom{});
    G.classes.assign(L, std::vector<ClassInfo>(27));
    G.cap.assign(L, 0);
    G.tab_count.clear();
    G.tab_prefix.clear();
    G.ent.clear();
    for (u64 l = 0; l < L; l++) {
        RoundGeom &rg = G.rounds[l];
        const int d = plan.dir[l];
        rg.dir = d;
        rg.order = plan.order[l];
        for (int a = 0; a < 3; a++) rg.stride[a] = stride[a];
        rg.hs = stride[d] / 2;
        rg.dist = rg.hs;
        for (int a = d + 1; a < 3; a++) rg.dist *= fg.n[a];
        rg.targets = 1;
        for (int a = 0; a < 3; a++) {
            const u64 h = fg.origin[a];
            // First target: h + hs on the round axis; h (h == 0) or h + stride elsewhere.
            const u64 first = a == d ? h + rg.hs : (h == 0 ? 0 : h + stride[a]);
            const u64 step = a == d ? 2 * rg.hs : stride[a];
            rg.tcount[a] = fg.n[a] > first ? (fg.n[a] - first + step - 1) / step : 0;
            rg.targets *= rg.tcount[a];
        }
        // compress.tpp:194-195, decompress.tpp:156.
        rg.eb = (float)((double)abs_eb * std::pow((double)p.eb_ratio, (double)(L - l - 1)));
        rg.slope = (float)((double)default_slope * std::pow((double)p.slope_ratio, (double)((int)L - (int)l - 1)));
        rg.stat_eb = rg.eb * p.stat_eb_ratio;
        rg.neg_2_stat_eb = 0.5f / rg.stat_eb;
        // Per-axis box sizes (get_layer_qb_shape, asz_param.hpp:105-114).
        rg.qb_total = 1;
        for (int a = 0; a < 3; a++) {
            rg.axis_off[a] = (uint32_t)G.tab_count.size();
            u64 sum = 0;
            for (u64 b = 0; b < fg.block_num[a]; b++) {
                u64 lo = fg.origin[a] + b * fg.block_shape[a], hi = std::min(lo + fg.block_shape[a] + 1, fg.n[a]);
                u64 start = a == d ? lo + stride[a] / 2 : (lo == 0 ? 0 : lo + stride[a]);
                u64 c = start >= hi ? 0 : (hi - start + stride[a] - 1) / stride[a];
                G.tab_count.push_back(c);
                G.tab_prefix.push_back(sum);
                sum += c;
            }
            rg.total[a] = sum;
            rg.qb_total *= sum;
        }
        // Per-axis target tables for the round kernels.
        {
            AxisTables at{G.tab_count.data(), G.tab_prefix.data()};
            for (int a = 0; a < 3; a++) {
                rg.ent_off[a] = G.ent.size();
                for (u64 k = 0; k < rg.tcount[a]; k++) G.ent.push_back(axis_entry(fg, rg, at, a, k));
            }
        }
        // Block classes for coefficient selection (compress.tpp:96-116, get_AB_map.tpp:9-12).
        bool all_fb = true;
        for (int cls = 0; cls < 27; cls++) {
            int cc[3] = {cls / 9, (cls / 3) % 3, cls % 3};
            u64 rep[3];
            bool exists = true;
            for (int a = 0; a < 3; a++) {
                u64 nb = fg.block_num[a];
                if (cc[a] == 0) rep[a] = 0;
                else if (cc[a] == 2) {
                    if (nb < 2) exists = false;
                    rep[a] = nb - 1;
                } else {
                    if (nb < 3) exists = false;
                    rep[a] = 1;
                }
            }
            ClassInfo ci{1, 0, 0, 1, {0, 0, 0}, 0, 0};
            if (!exists) {
                G.classes[l][cls] = ci;
                continue;
            }
            u64 lo[3], hi[3];
            for (int a = 0; a < 3; a++) {
                lo[a] = fg.origin[a] + rep[a] * fg.block_shape[a];
                hi[a] = std::min(lo[a] + fg.block_shape[a] + 1, fg.n[a]);
            }
            if (hi[d] <= lo[d] + 3 * stride[d]) {
                G.classes[l][cls] = ci;
                continue;
            }
            for (int a = 0; a < 3; a++)
                if (a != d && lo[a] != 0) lo[a] += stride[a];
            lo[d] += 3 * stride[d] / 2;
            hi[d] -= 3 * stride[d] / 2;
            u64 vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
            float q = (float)vol / (float)(stride[0] * stride[1] * stride[2] * p.h1_block_sampling_num);
            u64 ss = (u64)std::cbrt((double)q);
            if (ss == 0) ss = 1;
            u64 n = 1;
            for (int a = 0; a < 3; a++) {
                u64 step = stride[a] * ss;
                const u64 c = hi[a] > lo[a] ? (hi[a] - lo[a] + step - 1) / step : 0;
                ci.cnt[a] = (uint32_t)c;
                n *= c;
            }
            auto magic = [](u64 dv) { return dv > 1 && dv <= 0xffffffffull ? (uint32_t)(0xffffffffull / dv + 1) : 0u; };
            ci.m2 = magic(ci.cnt[2]);
            ci.m12 = magic((u64)ci.cnt[1] * ci.cnt[2]);
            ci.ss = (uint32_t)ss;
            ci.n = (uint32_t)n;
            ci.fallback = n == 0 ? 1 : 0;
            if (n) all_fb = false;
            G.cap[l] = std::max<uint32_t>(G.cap[l], (uint32_t)n);
            G.classes[l][cls] = ci;
        }
        rg.fallback_all = all_fb ? 1 : 0;
        stride[d] /= 2;
    }
}

// Bytes of one column's lines for the fused axis-2 rounds (k_lines.cu), or 0 when the plan does not
// qualify: every round along axis 2, a whole field, at most 64 blocks along axis 2, and the lines of
// a column within the kernels' shared-memory budget.
uint32_t lines_smem_bytes(const Geometry &G) {
    const FieldGeom &fg = G.fg;
    if (G.rounds.empty() || G.rounds.size() > 63 || fg.origin[0] || fg.origin[1] || fg.origin[2] || fg.block_num[2] > 64)
        return 0;
    for (const RoundGeom &rg : G.rounds)
        if (rg.dir != 2 || rg.stride[0] != 1 || rg.stride[1] != 1 || rg.tcount[0] != fg.n[0] || rg.tcount[1] != fg.n[1])
            return 0;
    const u64 l0 = std::min<u64>(fg.block_shape[0] + 1, fg.n[0]), l1 = std::min<u64>(fg.block_shape[1] + 1, fg.n[1]);
    const u64 bytes = l0 * l1 * fg.n[2] * sizeof(float);
    return bytes <= lines_smem_limit() ? (uint32_t)bytes : 0;
}

// The fused launches of one pass: the interior columns with their smaller line buffer, then the
// edge columns (or every column in one launch when there is no interior).
struct LinesLaunch {
    uint32_t set, bytes;
};
std::vector<LinesLaunch> lines_launches(const Geometry &G, uint32_t edge_bytes) {
    const FieldGeom &fg = G.fg;
    if (fg.block_num[0] < 2 || fg.block_num[1] < 2) return {{kColumnsAll, edge_bytes}};
    const u64 inner = fg.block_shape[0] * fg.block_shape[1] * fg.n[2] * sizeof(float);
    return {{kColumnsInterior, (uint32_t)inner}, {kColumnsEdge, edge_bytes}};
}

bool kernel_limits_ok(const Geometry &G) {
    for (int a = 0; a < 3; a++)
        if (G.fg.n[a] >= (1ull << 32)) return false;
    for (const RoundGeom &rg : G.rounds) {
        if (rg.tcount[0] * rg.tcount[1] >= (1ull << 32) || rg.tcount[2] >= (1ull << 32)) return false;
        for (int a = 0; a < 3; a++)
            if (rg.total[a] >= (1ull << 32)) return false;
    }
    return true;
}

// glibc log2f(freq * (1/n)) for freq = 0..n (index 0 unused), cached per n.
uint32_t log2_table(asz_ctx *ctx, uint32_t n) {
    auto it = ctx->log2_off.find(n);
    if (it != ctx->log2_off.end()) return it->second;
    uint32_t off = (uint32_t)ctx->log2_host.size();
    float nf = (float)(u64)n;
    float r = 1.0f / nf;
    ctx->log2_host.push_back(0.0f);
    for (u64 f = 1; f <= n; f++) {
        float pr = (float)f * r;
        ctx->log2_host.push_back(log2f(pr));
    }
    ctx->log2_off[n] = off;
    return off;
}

int upload_log2(asz_ctx *ctx) {
    if (ctx->log2_dev_len == ctx->log2_host.size()) return ASZ_OK;
    CK(ctx->log2arena.reserve(ctx->log2_host.size() * sizeof(float)));
    if (ctx->log2arena.cap < ctx->log2_host.size() * sizeof(float)) return fail(ctx, ASZ_E_CUDA, "log2 arena");
    CK(cudaMemcpyAsync(ctx->log2arena.p, ctx->log2_host.data(), ctx->log2_host.size() * sizeof(float),
                       cudaMemcpyHostToDevice, ctx->stream));
    ctx->log2_dev_len = ctx->log2_host.size();
    return ASZ_OK;
}

// Scratch sizes for one AB map of up to `cap` samples.
void scratch_dims(uint32_t cap, uint32_t &bcap, uint32_t &tcap, u64 &stride) {
    cap = std::max<uint32_t>(cap, 1);
    bcap = (uint32_t)sched_buckets(cap);
    tcap = 16;
    while (tcap < 2 * cap) tcap <<= 1;
    stride = tsel_scratch_bytes(cap, bcap, tcap);
}

// Largest group (samples) the shared-memory exact kernel takes, within the per-CTA limit.
uint32_t exact_cap() {
    static uint32_t cap = 0;
    if (!cap) {
        int dev = 0, lim = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&lim, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        uint32_t c = 2048;
        while (c > 64 && exact_smem_bytes(c) + 2048 > (uint32_t)lim) c -= 64;
        cap = c;
    }
    return cap;
}

// Bytes of one CTA's slice of the global scratch for exact replays of up to cap samples.
u64 exact_global_stride(uint32_t cap) { return ((u64)exact_smem_bytes(cap) + 255) / 256 * 256; }

// AB maps larger than shared memory holds (dm->boxes, dm->evals uploaded): the exact kernel with
// each box's working set in global scratch, a CTA per box. done is false when a box needs the
// serial kernel (a key outside int32); the error word is then cleared for it.
int abmap_exact_global(asz_ctx *ctx, uint32_t ne, const float *field, u64 n1n2, u64 n2, float R2, uint32_t cap, uint32_t nb,
                       const char *prof_name, bool &done);

// Replays one ambiguous decision with glibc log10f (compress.tpp:127-142).
float replay_decision(const AmbiguousRecord &r, float slope) {
    const float cand[5] = {1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
    int best = 1;
    float best_h1 = r.h1[1], best_psnr = 10.0f * log10f(r.x[1]);
    for (int c = 0; c < 5; c++) {
        if (cand[c] == cand[best]) continue;
        float psnr = 10.0f * log10f(r.x[c]);
        float s = std::fma(best_h1 - r.h1[c], slope, psnr - best_psnr);
        if (s > 0) {
            best = c;
            best_h1 = r.h1[c];
            best_psnr = psnr;
        }
    }
    return cand[best];
}

}  // namespace

extern "C" {

void asz_default_params(asz_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->pivot_eb_ratio = 0.05f;
    p->eb_ratio = 0.76f;
    p->slope_ratio = 0.54f;
    p->block_pivot_ratio = 4;
    p->max_layer_num = 14;
    p->full_predictor_search_layer_num = 4;
    p->generate_config_sample_stride = 5;
    p->h1_block_sampling_num = 256;
    p->stat_eb_ratio = 0.2f;
    p->predictor_family_suffix_layers = 6;
    p->predictor_family_sample_blocks = 8;
    p->predictor_family_sample_point_limit = 32768;
    p->predictor_family_sample_fraction_limit = 0.02f;
    p->predictor_family_coarse_probe_block_pivot_ratio = 3;
    p->predictor_family_fine_probe_block_pivot_ratio = 4;
    p->predictor_family_fine_eb_threshold = 1e-4f;
    p->default_slope_invalid_ratio_threshold = 1;
    p->default_slope_fallback = 1000;
    p->default_slope_eb_span = 1.5f;
    p->t_precision = 32;
    p->t_min = 1.0f / 16;
    p->t_max = 6.0f / 16;
    p->predictor_family = ASZ_FAMILY_AUTO;
}

asz_ctx *asz_create(int device) {
    if (cudaSetDevice(device) != cudaSuccess) return nullptr;
    asz_ctx *c = new asz_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return nullptr;
    }
    c->stream = c->own;
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(c->own);
        delete c;
        return nullptr;
    }
    return c;
}

void asz_destroy(asz_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->batch_graph) cudaGraphExecDestroy(c->batch_graph);
    c->builder.reset();
    for (cudaEvent_t e : c->round_ev) cudaEventDestroy(e);
    if (c->side) cudaStreamDestroy(c->side);
    c->hwin.release();
    c->hwin_host.release();
    c->slab_idx.release();
    c->slab_val.release();
    c->slab_cmp.release();
    c->gscratch.release();
    c->spill2.release();
    for (DevBuf *b : {&c->in, &c->rec, &c->qb, &c->tval, &c->tint, &c->misc, &c->scratch, &c->log2arena, &c->hist, &c->codes,
                      &c->bitoff, &c->cubtmp, &c->payload, &c->amb, &c->overrides, &c->classes, &c->axis, &c->pre, &c->chunks,
                      &c->out, &c->proxies, &c->tlist, &c->spill, &c->iota, &c->plan_qb, &c->plan_e, &c->plan_aux,
                      &c->plan_pay, &c->probe_in, &c->probe_pred, &c->rounds_dev, &c->lines_bail,
                      &c->lines_resume, &c->enc, &c->b_in, &c->b_rec, &c->b_qb, &c->b_tval, &c->b_tint, &c->b_ent, &c->b_cls,
                      &c->b_rounds, &c->b_qoff, &c->b_range, &c->b_range0, &c->b_prox, &c->b_amb, &c->b_cnt, &c->b_fields,
                      &c->b_goff, &c->b_poff, &c->b_ioff, &c->b_queue, &c->b_hand, &c->b_spill, &c->b_spill2})
        b->release();
    c->pre_zstd.release();
    c->batch_pre[0].release();
    c->batch_pre[1].release();
    c->raw_in.release();
    for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
    asz::host::sweep_release(c->sweep);
    for (ZSTD_CCtx *z : c->zfree) ZSTD_freeCCtx(z);
    if (c->zd) ZSTD_freeDCtx(c->zd);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

const char *asz_last_error(const asz_ctx *c) { return c ? c->err.c_str() : "no context"; }

int asz_set_stream(asz_ctx *c, void *s) {
    if (!c) return ASZ_E_ARG;
    c->stream = s ? (cudaStream_t)s : c->own;
    return ASZ_OK;
}

void asz_free(void *p) {
    if (!p) return;
    // Every buffer this library hands out is an output block (out_alloc).
    out_release(static_cast<uint8_t *>(p));
}

void asz_release_output_cache(void) {
    std::lock_guard<std::mutex> g(g_out_mu);
    for (uint8_t *b : g_out_cache) std::free(b);
    g_out_cache.clear();
    g_out_cached = 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Compression.

namespace {

struct MiscLayout {  // small device words, one allocation
    int32_t range[2];
    unsigned long long nonfinite;
    unsigned long long zfirst, zlast;
    uint32_t err;
    uint32_t fb;
    uint32_t amb_count;
    uint32_t changed;
    uint32_t list_count[64];
    uint32_t spill_count[64];
    uint32_t spill2_count[64];  // groups the global-scratch exact kernel left to the serial one
    uint32_t all_count;
    uint32_t why[3];  // fast path: [0] handed off (bins too spread), [1] handed off (undecided), [2] settled window by window
    uint32_t dec_err;      // batched Huffman decoding: error bits
    uint32_t dec_changed;  // batched Huffman decoding: a chunk start moved in the last pass
    uint32_t resume_count;  // fused axis-2 compression: columns waiting for the exact path
    int32_t qb_range[2 * 64];
    uint32_t hist_over[64];  // round l: a QB of its stream fell outside the histogram window
    float h1[3 * 64];
    float x[3 * 64];
    uint32_t m[3];
    SampleBox boxes[3];
    ProxyEval evals[64];
};

int abmap_exact_global(asz_ctx *ctx, uint32_t ne, const float *field, u64 n1n2, u64 n2, float R2, uint32_t cap, uint32_t nb,
                       const char *prof_name, bool &done) {
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    cudaStream_t st = ctx->stream;
    const u64 stride = exact_global_stride(cap);
    CK(ctx->gscratch.reserve(nb * stride));
    CK(cudaMemsetAsync(&dm->err, 0, 4, st));
    {
        ProfScope ps(ctx, prof_name, 0);
        CK(launch_slope_exact_global(dm->boxes, dm->evals, ne, field, n1n2, n2, ctx->log2arena.as<float>(), R2, dm->h1, dm->x,
                                     dm->m, &dm->err, ctx->gscratch.as<uint8_t>(), stride, cap, nb, st));
    }
    uint32_t e1 = 0;
    CK(cudaMemcpyAsync(&e1, &dm->err, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    done = e1 == 0;
    if (!done) CK(cudaMemsetAsync(&dm->err, 0, 4, st));
    return ASZ_OK;
}

// first_max: a zero maximum takes the sign of the first largest element (std::max_element)
// instead of the last one (std::minmax_element).
int compute_range(asz_ctx *ctx, const float *d_in, u64 N, float &mn, float &mx, bool first_max = false) {
    MiscLayout init{};
    init.range[0] = INT32_MAX;
    init.range[1] = INT32_MIN;
    init.zfirst = ~0ull;
    init.zlast = 0;
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    CK(cudaMemcpyAsync(dm, &init, sizeof(MiscLayout), cudaMemcpyHostToDevice, ctx->stream));
    {
        ProfScope ps(ctx, "range", N * 4);
        CK(launch_range(d_in, N, dm->range, &dm->nonfinite, ctx->stream));
    }
    MiscLayout h;
    CK(cudaMemcpyAsync(&h, dm, offsetof(MiscLayout, err), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h.nonfinite) return fail(ctx, ASZ_E_DATA, "input contains a nonfinite value");
    auto tof = [](int32_t k) {
        uint32_t b = k >= 0 ? (uint32_t)k : ((uint32_t)k ^ 0x7fffffffu);
        float f;
        std::memcpy(&f, &b, 4);
        return f;
    };
    mn = tof(h.range[0]);
    mx = tof(h.range[1]);
    if (mn == 0.0f || mx == 0.0f) {
        // minmax_element keeps the first smallest and the last largest element; with zeros of
        // both signs present, that decides the stored sign.
        CK(launch_zero_first_last(d_in, N, &dm->zfirst, &dm->zlast, ctx->stream));
        unsigned long long fl[2];
        CK(cudaMemcpyAsync(fl, &dm->zfirst, 16, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (mn == 0.0f) CK(cudaMemcpy(&mn, d_in + fl[0], 4, cudaMemcpyDeviceToHost));
        if (mx == 0.0f) CK(cudaMemcpy(&mx, d_in + fl[first_max ? 0 : 1], 4, cudaMemcpyDeviceToHost));
    }
    return ASZ_OK;
}

// get_default_slope (c_codes/asz_core/get_default_slope.tpp:6-83).
// The three whole-field sample boxes of get_default_slope (get_default_slope.tpp:13-22): along
// direction d, [3, n_d - 3) with stride 2, the other axes whole, thinned by the sampling stride.
void slope_boxes(const uint64_t dims[3], const asz_params &p, float abs_eb, SampleBox boxes[3]) {
    const float two_stat = abs_eb * p.stat_eb_ratio;
    const float stat_eb = two_stat * 0.5f;
    const float neg = 1.0f / two_stat;
    for (int d = 0; d < 3; d++) {
        SampleBox &b = boxes[d];
        u64 lo[3] = {0, 0, 0}, hi[3] = {dims[0], dims[1], dims[2]}, st[3] = {1, 1, 1};
        lo[d] = 3;
        hi[d] = dims[d] - 3;
        st[d] = 2;
        u64 vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
        float q = (float)vol / (float)(st[0] * st[1] * st[2] * p.h1_block_sampling_num);
        u64 ss = (u64)std::cbrt((double)q);
        if (ss == 0) ss = 1;
        u64 n = 1;
        for (int a = 0; a < 3; a++) {
            b.lo[a] = lo[a];
            b.hi[a] = hi[a];
            b.step[a] = st[a] * ss;
            n *= hi[a] > lo[a] ? (hi[a] - lo[a] + b.step[a] - 1) / b.step[a] : 0;
        }
        b.dist = 1;
        for (int a = d + 1; a < 3; a++) b.dist *= dims[a];
        b.neg_2_stat_eb = neg;
        b.stat_eb = stat_eb;
        b.n = (uint32_t)n;
    }
}

// get_default_slope on given boxes over `field` (dims fdims): the whole field, or a compact copy of
// the boxes' samples whose boxes keep the samples' order.
int default_slope_on(asz_ctx *ctx, const float *field, const uint64_t fdims[3], SampleBox boxes[3], const asz_params &p,
                     float abs_eb, float mn, float mx, const std::vector<float> &cand_t, float &slope_out,
                     float &max_invalid_out, int &reason_out) {
    FieldGeom fg{};
    for (int a = 0; a < 3; a++) fg.n[a] = fdims[a];
    const uint64_t *dims = fdims;
    const float *d_in = field;
    const float ebs[2] = {abs_eb * p.default_slope_eb_span, abs_eb / p.default_slope_eb_span};
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    uint32_t cap = 1;
    for (int d = 0; d < 3; d++) {
        boxes[d].log2_off = boxes[d].n ? log2_table(ctx, boxes[d].n) : 0;
        cap = std::max<uint32_t>(cap, boxes[d].n);
    }
    const uint32_t ne = (uint32_t)(2 * cand_t.size());
    if (ne > 64) return fail(ctx, ASZ_E_UNSUPPORTED, "too many t candidates for the default slope");
    ProxyEval evals[64];
    for (int i = 0; i < 2; i++)
        for (size_t k = 0; k < cand_t.size(); k++) evals[i * cand_t.size() + k] = ProxyEval{cand_t[k], ebs[i]};
    int rc = upload_log2(ctx);
    if (rc) return rc;
    uint32_t bcap, tcap;
    u64 sstride;
    scratch_dims(cap, bcap, tcap, sstride);
    CK(ctx->scratch.reserve(3 * sstride));
    CK(cudaMemcpyAsync(dm->boxes, boxes, 3 * sizeof(SampleBox), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dm->evals, evals, sizeof(ProxyEval) * ne, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(&dm->err, 0, 4, ctx->stream));
    const float R = mx - mn;
    // The shared-memory exact kernel when the maps fit, else the same kernel with global scratch;
    // the serial kernel when a key exceeds int32 (the exact kernels then report error bit 2).
    bool serial = cap > exact_cap();
    if (!serial) {
        {
            ProfScope ps_slope(ctx, "slope", 0);
            CK(launch_slope_exact(dm->boxes, dm->evals, ne, d_in, dims[1] * dims[2], dims[2], ctx->log2arena.as<float>(),
                                  R * R, dm->h1, dm->x, dm->m, &dm->err, exact_cap(), 3, ctx->stream));
        }
        uint32_t e1 = 0;
        CK(cudaMemcpyAsync(&e1, &dm->err, 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (e1) {
            serial = true;
            CK(cudaMemsetAsync(&dm->err, 0, 4, ctx->stream));
        }
    }
    if (serial) {
        bool done = false;
        rc = abmap_exact_global(ctx, ne, d_in, dims[1] * dims[2], dims[2], R * R, cap, 3, "slope_global", done);
        if (rc) return rc;
        serial = !done;
    }
    if (serial) {
        ProfScope ps_slope(ctx, "slope_serial", 0);
        CK(launch_slope_v0(fg, dm->boxes, dm->evals, ne, d_in, ctx->log2arena.as<float>(), R * R, ctx->scratch.as<uint8_t>(),
                           sstride, cap, bcap, tcap, dm->h1, dm->x, dm->m, &dm->err, 3, ctx->stream));
    }
    std::vector<float> h1(3 * ne), x(3 * ne);
    uint32_t m[3], errw;
    CK(cudaMemcpyAsync(h1.data(), dm->h1, 4 * 3 * ne, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(x.data(), dm->x, 4 * 3 * ne, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(m, dm->m, 12, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&errw, &dm->err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (errw) return fail(ctx, ASZ_E_DEVICE, "default-slope kernel reported an internal error");
    float avg_h1[2] = {0, 0}, avg_psnr[2] = {0, 0};
    u64 valid[2] = {0, 0};
    for (int d = 0; d < 3; d++) {
        if (m[d] == 0)
            return fail(ctx, ASZ_E_DATA, "In get_default_slope, direction " + std::to_string(d) + " AB_map is empty");
        for (int i = 0; i < 2; i++)
            for (size_t k = 0; k < cand_t.size(); k++) {
                size_t e = (size_t)d * ne + i * cand_t.size() + k;
                float psnr = 10.0f * log10f(x[e]);
                avg_h1[i] += h1[e];
                avg_psnr[i] += psnr;
                valid[i]++;
            }
    }
    u64 total = 3 * cand_t.size();
    float recip = 1.0f / (float)total;
    float max_invalid = 0;
    for (int i = 0; i < 2; i++) {
        float inv = std::fma(-recip, (float)valid[i], 1.0f);
        max_invalid = std::max(inv, max_invalid);
    }
    max_invalid_out = max_invalid;
    reason_out = 0;
    if (max_invalid >= p.default_slope_invalid_ratio_threshold) {
        slope_out = p.default_slope_fallback;
        reason_out = 1;
        return ASZ_OK;
    }
    // Tolerance scale: the approximate reciprocal with one Newton step that the reference's
    // vectorised average_h1[i]/=valid_case_num[i] uses; the differences use exact divisions.
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
    if (tol >= h1_diff || 0.0f >= psnr_diff) {
        slope_out = p.default_slope_fallback;
        reason_out = 2;
    } else {
        slope_out = psnr_diff / h1_diff;
    }
    return ASZ_OK;
}

int default_slope(asz_ctx *ctx, const float *d_in, const uint64_t dims[3], const asz_params &p, float abs_eb, float mn,
                  float mx, const std::vector<float> &cand_t, float &slope_out, float &max_invalid_out, int &reason_out) {
    SampleBox boxes[3];
    slope_boxes(dims, p, abs_eb, boxes);
    return default_slope_on(ctx, d_in, dims, boxes, p, abs_eb, mn, mx, cand_t, slope_out, max_invalid_out, reason_out);
}

std::vector<float> candidate_t(const asz_params &p) {
    std::vector<float> c;
    int lo = (int)host_lround_f(p.t_min * (float)p.t_precision), hi = (int)host_lround_f(p.t_max * (float)p.t_precision);
    for (int ti = lo; ti <= hi; ti++) c.push_back((float)ti / (float)p.t_precision);
    return c;
}

struct StreamOut {
    HuffCode code;
    u64 count = 0;
    u64 payload_word_off = 0;  // in the payload arena (32-bit words)
    int64_t lo = 0, hi = -1;   // histogram range
    u64 hist_off = 0;
    bool prebuilt = false;     // code built during the rounds (no histogram pass here)
};

// ---------------------------------------------------------------------------------------------
// Plan search: param_c::generate_config (c_codes/asz_core/generate_config.tpp:444-678).
// Per layer, from the finest: for each candidate predictor, the best t on its direction's
// whole-field AB map (exact map order on the device, glibc log10f here), then a sampled open-loop
// compression of the original data (device), whose QBs are Huffman-coded (device) and compressed
// with libzstd level 3 (host threads); the candidate with the best psnr - slope * bit rate wins.
// The float steps follow the reference build's emitted code: pow in double with the products
// rounded to float, 0.5f/x for the 1/(2x) factors, fmaf(-slope, h1, psnr) for the t choice,
// bit rate = zstd_bytes * (8 / samples), psnr = log10f(range^2 / (mse / samples)) * 10, and a
// separately rounded slope * bit rate in the final score.

struct PlanSearchOut {
    std::vector<std::string> plan;
    std::vector<float> dists;  // winning score per layer, finest first
    double stats_s = 0, sample_s = 0, lossless_s = 0;
};

int plan_search(asz_ctx *ctx, const float *d_in, const uint64_t dims[3], const asz_params &p, float abs_eb, float mn, float mx,
                float slope, PlanSearchOut &out) {
    static const char *all9[9] = {"cubic0_120", "cubic0_021", "cubic0_012", "cubic1_120", "cubic1_021",
                                  "cubic1_012", "cubic2_120", "cubic2_021", "cubic2_012"};
    static const char *last3[3] = {"cubic0_012", "cubic1_012", "cubic2_012"};
    static const int nest[3][3] = {{1, 2, 0}, {0, 2, 1}, {0, 1, 2}};  // loop axes per order digit, outer to inner
    cudaStream_t st = ctx->stream;
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    const std::vector<float> cand_t = candidate_t(p);
    if (cand_t.size() > 21) return fail(ctx, ASZ_E_UNSUPPORTED, "too many t candidates for the plan search");
    const float R = mx - mn;
    FieldGeom fg{};
    for (int a = 0; a < 3; a++) fg.n[a] = dims[a];
    u64 ps[3] = {1, 1, 1};
    out = PlanSearchOut();
    for (u64 layer = 0; layer < p.max_layer_num; layer++) {
        const float layer_eb = (float)((double)abs_eb * std::pow((double)p.eb_ratio, (double)layer));
        const float neg_2_layer_eb = 0.5f / layer_eb;
        const float stat_eb = layer_eb * p.stat_eb_ratio;
        const float neg_2_stat_eb = 0.5f / stat_eb;
        const float lslope = (float)((double)slope * std::pow((double)p.slope_ratio, (double)layer));
        std::vector<std::string> cands;
        if (layer < p.full_predictor_search_layer_num) cands.assign(all9, all9 + 9);
        else cands.assign(last3, last3 + 3);
        // ---- Best t per direction on its AB map.
        auto t_stats = clk::now();
        float best_t[3] = {0.25f, 0.25f, 0.25f};
        {
            bool need[3] = {false, false, false};
            for (auto &c : cands) need[c[5] - '0'] = true;
            SampleBox boxes[3];
            int box_dir[3];
            uint32_t nb = 0, cap = 1;
            for (int d = 0; d < 3; d++) {
                if (!need[d] || !(dims[d] > 3 * ps[d])) continue;
                u64 ps2[3] = {ps[0], ps[1], ps[2]};
                ps2[d] *= 2;
                SampleBox &b = boxes[nb];
                u64 lo[3] = {0, 0, 0}, hi[3] = {dims[0], dims[1], dims[2]};
                lo[d] = 3 * ps2[d] / 2;
                hi[d] = dims[d] - 3 * ps2[d] / 2;
                u64 vol = (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]);
                float q = (float)vol / (float)(ps2[0] * ps2[1] * ps2[2] * p.h1_block_sampling_num);
                u64 ss = (u64)std::cbrt((double)q);
                if (ss == 0) ss = 1;
                u64 n = 1;
                for (int a = 0; a < 3; a++) {
                    b.lo[a] = lo[a];
                    b.hi[a] = hi[a];
                    b.step[a] = ps2[a] * ss;
                    n *= hi[a] > lo[a] ? (hi[a] - lo[a] + b.step[a] - 1) / b.step[a] : 0;
                }
                u64 dist = ps2[d];
                for (int a = d + 1; a < 3; a++) dist *= dims[a];
                b.dist = dist / 2;
                b.neg_2_stat_eb = neg_2_stat_eb;
                b.stat_eb = stat_eb;
                if (n > 0xffffffffull) return fail(ctx, ASZ_E_UNSUPPORTED, "plan-search AB map too large");
                b.n = (uint32_t)n;
                b.log2_off = n ? log2_table(ctx, (uint32_t)n) : 0;
                cap = std::max<uint32_t>(cap, (uint32_t)n);
                box_dir[nb++] = d;
            }
            if (nb) {
                const uint32_t ne = (uint32_t)cand_t.size();
                ProxyEval evals[64];
                for (uint32_t k = 0; k < ne; k++) evals[k] = ProxyEval{cand_t[k], layer_eb};
                int rc = upload_log2(ctx);
                if (rc) return rc;
                CK(cudaMemcpyAsync(dm->boxes, boxes, sizeof(SampleBox) * nb, cudaMemcpyHostToDevice, st));
                CK(cudaMemcpyAsync(dm->evals, evals, sizeof(ProxyEval) * ne, cudaMemcpyHostToDevice, st));
                CK(cudaMemsetAsync(&dm->err, 0, 4, st));
                CK(cudaMemsetAsync(dm->m, 0, sizeof(dm->m), st));
                bool serial = cap > exact_cap();
                if (!serial) {
                    {
                        ProfScope ps_(ctx, "plan_abmap", 0);
                        CK(launch_slope_exact(dm->boxes, dm->evals, ne, d_in, dims[1] * dims[2], dims[2], ctx->log2arena.as<float>(),
                                              R * R, dm->h1, dm->x, dm->m, &dm->err, exact_cap(), nb, st));
                    }
                    uint32_t e1 = 0;
                    CK(cudaMemcpyAsync(&e1, &dm->err, 4, cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    if (e1) {
                        serial = true;
                        CK(cudaMemsetAsync(&dm->err, 0, 4, st));
                    }
                }
                if (serial) {
                    bool done = false;
                    int rc2 = abmap_exact_global(ctx, ne, d_in, dims[1] * dims[2], dims[2], R * R, cap, nb,
                                                 "plan_abmap_global", done);
                    if (rc2) return rc2;
                    serial = !done;
                }
                if (serial) {
                    uint32_t bcap, tcap;
                    u64 sstride;
                    scratch_dims(cap, bcap, tcap, sstride);
                    CK(ctx->scratch.reserve(3 * sstride));
                    ProfScope ps_(ctx, "plan_abmap_serial", 0);
                    CK(launch_slope_v0(fg, dm->boxes, dm->evals, ne, d_in, ctx->log2arena.as<float>(), R * R,
                                       ctx->scratch.as<uint8_t>(), sstride, cap, bcap, tcap, dm->h1, dm->x, dm->m, &dm->err, nb,
                                       st));
                }
                std::vector<float> h1(nb * ne), x(nb * ne);
                uint32_t m[3], errw;
                CK(cudaMemcpyAsync(h1.data(), dm->h1, 4 * nb * ne, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(x.data(), dm->x, 4 * nb * ne, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(m, dm->m, 12, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(&errw, &dm->err, 4, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                if (errw) return fail(ctx, ASZ_E_DEVICE, "plan-search AB-map kernel reported an internal error");
                for (uint32_t bi = 0; bi < nb; bi++) {
                    if (m[bi] == 0) continue;  // empty map: t stays 1/4
                    auto score = [&](uint32_t k) {
                        const float psnr = 10.0f * log10f(x[bi * ne + k]);
                        return std::fma(-lslope, h1[bi * ne + k], psnr);
                    };
                    uint32_t k0 = ne;
                    for (uint32_t k = 0; k < ne; k++)
                        if (cand_t[k] == 0.25f) k0 = k;
                    float bt = 0.25f, best;
                    if (k0 < ne) {
                        best = score(k0);
                    } else {
                        // 1/4 outside the candidate range: evaluate it separately.
                        return fail(ctx, ASZ_E_UNSUPPORTED, "plan search needs t = 1/4 among the t candidates");
                    }
                    for (uint32_t k = 0; k < ne; k++) {
                        if (cand_t[k] == 0.25f) continue;
                        const float cur = score(k);
                        if (cur > best) bt = cand_t[k];
                        best = cur > best ? cur : best;
                    }
                    best_t[box_dir[bi]] = bt;
                }
            }
        }
        out.stats_s += secs(t_stats, clk::now());
        // ---- Sampled open-loop compression of every candidate (one launch), and its error sums.
        auto t_sample = clk::now();
        const uint32_t nc = (uint32_t)cands.size();
        std::vector<PlanCand> pc(nc);
        u64 total = 0;
        for (uint32_t c = 0; c < nc; c++) {
            const int dir = cands[c][5] - '0', order = cands[c][9] - '0';
            PlanCand &q = pc[c];
            u64 ps2[3] = {ps[0], ps[1], ps[2]};
            ps2[dir] *= 2;
            for (int a = 0; a < 3; a++) {
                q.st[a] = ps2[a] * (a == order ? 1 : p.generate_config_sample_stride);
                q.lo[a] = a == dir ? ps2[dir] / 2 : 0;
                q.cnt[a] = dims[a] > q.lo[a] ? (dims[a] - q.lo[a] + q.st[a] - 1) / q.st[a] : 0;
                q.ax[a] = nest[order][a];
            }
            q.off = total;
            q.hs = ps2[dir] / 2;
            u64 dist = q.hs;
            for (int a = dir + 1; a < 3; a++) dist *= dims[a];
            q.dist = dist;
            q.right = dims[dir];
            q.t = best_t[dir];
            q.eb = layer_eb;
            q.neg_2_eb = neg_2_layer_eb;
            q.dir = dir;
            total += q.cnt[0] * q.cnt[1] * q.cnt[2];
        }
        std::vector<u64> num(nc);
        for (uint32_t c = 0; c < nc; c++) num[c] = pc[c].cnt[0] * pc[c].cnt[1] * pc[c].cnt[2];
        CK(ctx->plan_qb.reserve(std::max<u64>(total, 1) * 4));
        CK(ctx->plan_e.reserve(std::max<u64>(total, 1) * 4));
        const u64 aux_cands = 0, aux_range = (nc * sizeof(PlanCand) + 255) & ~255ull, aux_mse = aux_range + 256;
        CK(ctx->plan_aux.reserve(aux_mse + 256));
        uint8_t *aux = ctx->plan_aux.as<uint8_t>();
        CK(cudaMemcpyAsync(aux + aux_cands, pc.data(), nc * sizeof(PlanCand), cudaMemcpyHostToDevice, st));
        std::vector<int32_t> rinit(2 * nc);
        for (uint32_t c = 0; c < nc; c++) {
            rinit[2 * c] = INT32_MAX;
            rinit[2 * c + 1] = INT32_MIN;
        }
        CK(cudaMemcpyAsync(aux + aux_range, rinit.data(), rinit.size() * 4, cudaMemcpyHostToDevice, st));
        const PlanCand *d_pc = (const PlanCand *)(aux + aux_cands);
        int32_t *d_qb = ctx->plan_qb.as<int32_t>();
        {
            ProfScope ps_(ctx, "plan_sample", total * 8);
            CK(launch_plan_sample(d_in, dims[1], dims[2], d_pc, nc, total, d_qb, ctx->plan_e.as<float>(), (int32_t *)(aux + aux_range),
                                  st));
        }
        {
            ProfScope ps_(ctx, "plan_mse", total * 4);
            CK(launch_plan_mse(d_pc, nc, ctx->plan_e.as<float>(), (float *)(aux + aux_mse), st));
        }
        std::vector<int32_t> ranges(2 * nc);
        std::vector<float> mse(nc);
        CK(cudaMemcpyAsync(ranges.data(), aux + aux_range, ranges.size() * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(mse.data(), aux + aux_mse, nc * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out.sample_s += secs(t_sample, clk::now());
        // ---- Huffman code of each candidate's QBs (device histogram and encoding), zstd on the host.
        auto t_lossless = clk::now();
        std::vector<u64> hist_off(nc, 0);
        u64 hist_total = 0;
        for (uint32_t c = 0; c < nc; c++) {
            if (!num[c]) continue;
            const u64 range = (u64)((int64_t)ranges[2 * c + 1] - (int64_t)ranges[2 * c]) + 1;
            if (range > (1ull << 27)) return fail(ctx, ASZ_E_UNSUPPORTED, "QB range too wide for the dense histogram");
            hist_off[c] = hist_total;
            hist_total += range;
        }
        CK(ctx->hist.reserve(std::max<u64>(hist_total, 1) * 8));
        CK(cudaMemsetAsync(ctx->hist.p, 0, std::max<u64>(hist_total, 1) * 8, st));
        unsigned long long *d_hist = ctx->hist.as<unsigned long long>();
        for (uint32_t c = 0; c < nc; c++) {
            if (!num[c]) continue;
            const u64 range = (u64)((int64_t)ranges[2 * c + 1] - (int64_t)ranges[2 * c]) + 1;
            ProfScope ps_(ctx, "plan_histogram", num[c] * 4);
            CK(launch_histogram<int32_t>(d_qb + pc[c].off, num[c], ranges[2 * c], range, d_hist + hist_off[c], st));
        }
        std::vector<u64> hist(hist_total);
        if (hist_total) CK(cudaMemcpyAsync(hist.data(), d_hist, hist_total * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::vector<HuffCode> codes(nc);
        std::vector<int64_t> sym_lo(nc, 0);
        std::vector<std::string> code_err(nc);
        std::vector<char> code_ok(nc, 1);
        {
            auto build_one = [&](uint32_t c) {
                if (!num[c]) return;
                const u64 range = (u64)((int64_t)ranges[2 * c + 1] - (int64_t)ranges[2 * c]) + 1;
                const u64 *h = hist.data() + hist_off[c];
                u64 a = 0, b = range;
                while (a < b && h[a] == 0) a++;
                while (b > a && h[b - 1] == 0) b--;
                std::vector<u64> hh(h + a, h + b);
                sym_lo[c] = (int64_t)ranges[2 * c] + (int64_t)a;
                code_ok[c] = build_code(hh, sym_lo[c], (int64_t)ranges[2 * c] + (int64_t)b - 1, num[c], false, codes[c], code_err[c]);
            };
            std::vector<std::thread> pool;
            for (uint32_t c = 1; c < nc; c++)
                if (num[c]) pool.emplace_back(build_one, c);
            build_one(0);
            for (auto &t : pool) t.join();
        }
        for (uint32_t c = 0; c < nc; c++)
            if (!code_ok[c]) return fail(ctx, ASZ_E_UNSUPPORTED, code_err[c]);
        // Encode all candidates into one payload arena.
        std::vector<u64> word_off(nc, 0), code_off(nc, 0);
        u64 words = 0, ncode = 0, max_count = 0;
        for (uint32_t c = 0; c < nc; c++) {
            if (!num[c]) continue;
            word_off[c] = words;
            words += (codes[c].bits + 31) / 32 + 2;
            code_off[c] = ncode;
            ncode += codes[c].table.size();
            max_count = std::max(max_count, num[c]);
        }
        std::vector<CodeEntry> ctab(std::max<u64>(ncode, 1));
        for (uint32_t c = 0; c < nc; c++)
            if (num[c]) std::copy(codes[c].table.begin(), codes[c].table.end(), ctab.begin() + code_off[c]);
        CK(ctx->codes.reserve(ctab.size() * sizeof(CodeEntry)));
        CK(cudaMemcpyAsync(ctx->codes.p, ctab.data(), ctab.size() * sizeof(CodeEntry), cudaMemcpyHostToDevice, st));
        CK(ctx->plan_pay.reserve(std::max<u64>(words, 1) * 4));
        CK(cudaMemsetAsync(ctx->plan_pay.p, 0, std::max<u64>(words, 1) * 4, st));
        CK(ctx->bitoff.reserve(std::max<u64>(max_count, 1) * 8));
        size_t tmp_bytes = 0;
        CK(launch_encode<int32_t>(nullptr, max_count, 0, nullptr, ctx->bitoff.as<u64>(), nullptr, tmp_bytes, nullptr, st));
        CK(ctx->cubtmp.reserve(tmp_bytes));
        for (uint32_t c = 0; c < nc; c++) {
            if (!num[c] || codes[c].maxval == 1) continue;
            size_t tb = ctx->cubtmp.cap;
            ProfScope ps_(ctx, "plan_encode", num[c] * 4);
            CK(launch_encode<int32_t>(d_qb + pc[c].off, num[c], sym_lo[c], ctx->codes.as<CodeEntry>() + code_off[c],
                                      ctx->bitoff.as<u64>(), ctx->cubtmp.p, tb, ctx->plan_pay.as<uint32_t>() + word_off[c], st));
        }
        std::vector<uint32_t> pay(std::max<u64>(words, 1));
        CK(cudaMemcpyAsync(pay.data(), ctx->plan_pay.p, std::max<u64>(words, 1) * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::vector<u64> zlen(nc, 0);
        std::vector<char> z_ok(nc, 1);
        {
            auto zstd_one = [&](uint32_t c) {
                if (!num[c]) return;
                const HuffCode &hc = codes[c];
                std::vector<uint8_t> bs(hc.save_size() + hc.encode_size());
                write_tree(hc, bs.data());
                write_len_word(hc, bs.data() + hc.save_size());
                if (hc.maxval != 1) std::memcpy(bs.data() + hc.save_size() + 8, pay.data() + word_off[c], (hc.bits + 7) >> 3);
                std::vector<uint8_t> z(ZSTD_compressBound(bs.size()));
                size_t zl = zstd3(ctx, z.data(), z.size(), bs.data(), bs.size());
                if (ZSTD_isError(zl)) z_ok[c] = 0;
                else zlen[c] = zl;
            };
            std::vector<std::thread> pool;
            for (uint32_t c = 1; c < nc; c++)
                if (num[c]) pool.emplace_back(zstd_one, c);
            zstd_one(0);
            for (auto &t : pool) t.join();
        }
        for (uint32_t c = 0; c < nc; c++)
            if (!z_ok[c]) return fail(ctx, ASZ_E_DATA, "ZSTD_compress failed in the plan search");
        out.lossless_s += secs(t_lossless, clk::now());
        // ---- Choose the layer's predictor.
        int best = -1;
        float best_dist = 0;
        for (uint32_t c = 0; c < nc; c++) {
            if (!num[c]) continue;
            const float nf = (float)num[c];
            const float br = (float)zlen[c] * (8.0f / nf);
            const float mse_avg = mse[c] / nf;
            const float psnr = log10f(R * R / mse_avg) * 10.0f;
            const float dist = psnr - lslope * br;
            if (best < 0 || dist > best_dist) {
                best = (int)c;
                best_dist = dist;
            }
        }
        if (best < 0) break;
        ps[cands[best][5] - '0'] *= 2;
        out.plan.insert(out.plan.begin(), cands[best]);
        out.dists.push_back(best_dist);
    }
    return ASZ_OK;
}

}  // namespace

// The compression core (compress.tpp:147-231): geometry, pivots, and every round with its per-block
// coefficient selection (fast path, exact replay, serial spill, host re-check of ambiguous
// decisions with reruns), leaving the reconstruction in ctx->rec, the QB streams in ctx->qb at
// o.qb_off and the t codes in ctx->tint.
struct CoreArgs {
    const float *d_in;
    const uint64_t *dims;
    const uint64_t *origin;  // frame origin, or nullptr for a whole field
    const Plan *plan;
    const asz_params *p;
    bool quintic;
    bool probe;              // predictor-family probe: divide on every axis, predictions to pred_out
    float *pred_out;
    float mn, mx, abs_eb, slope;
    const int64_t *t_given = nullptr;  // host table of block-major t codes replacing the selection
    u64 t_len = 0;
    // Count each round's QB histogram in its kernel and build the stream's Huffman code on the
    // context's builder thread while the later rounds run.
    bool prebuild = false;
    // Slabs (asz_compress_slab): the geometry options, a hook run before each round's selection
    // (the halo exchange before axis-0 rounds), and one that makes a rerun decision the same on
    // every rank (it receives this rank's and returns the agreed one).
    const SlabGeom *slab = nullptr;
    std::function<int(u64)> before_round = nullptr;
    std::function<int(bool &)> agree = nullptr;
};

// A QB stream's code built during the rounds (ok == false: the encoder counts and builds it).
struct PreCode {
    bool ok = false;
    int64_t lo = 0, hi = -1;
    HuffCode code;
};

struct CoreOut {
    Geometry G;
    std::vector<u64> qb_off, qb_len;
    std::vector<PreCode> pre;  // index s: QB stream s (0: pivots, 1..L: rounds)
};

int run_core(asz_ctx *ctx, const CoreArgs &a, CoreOut &o, asz_report &R) {
    const float *d_in = a.d_in;
    const uint64_t *dims = a.dims;
    const Plan &plan = *a.plan;
    const asz_params &p = *a.p;
    const bool quintic = a.quintic;
    const float mn = a.mn, mx = a.mx, abs_eb = a.abs_eb, slope = a.slope;
    const u64 N = dims[0] * dims[1] * dims[2];
    const u64 L = plan.pred.size();
    cudaStream_t st = ctx->stream;
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    int rc = 0;
    std::optional<HostScope> hs_prep(std::in_place, ctx, "host:prepare");
    Geometry &G = o.G;
    build_geometry(dims, plan, p, abs_eb, slope, quintic, G, a.origin, a.slab);
    if (!kernel_limits_ok(G)) return fail(ctx, ASZ_E_UNSUPPORTED, "field too large for the round kernels' 32-bit line indexing");
    u64 qb_sum = G.pivots;
    for (auto &rg : G.rounds) qb_sum += rg.qb_total;
    if (!a.origin && qb_sum != N) return fail(ctx, ASZ_E_DATA, "total_qb_num!=data.size()");
    // Buffers: reconstruction, QB streams (pivots first), per-block t.
    std::vector<u64> &qb_off = o.qb_off, &qb_len = o.qb_len;
    qb_off.assign(L + 1, 0);
    qb_len.assign(L + 1, 0);
    qb_len[0] = G.pivots;
    for (u64 l = 0; l < L; l++) qb_len[l + 1] = G.rounds[l].qb_total;
    u64 acc = 0;
    for (u64 s = 0; s <= L; s++) {
        qb_off[s] = acc;
        acc += qb_len[s];
    }
    CK(ctx->rec.reserve(N * sizeof(float)));
    // A frame's halo and unowned faces keep their input values (the reference starts from a copy).
    if (a.origin) CK(cudaMemcpyAsync(ctx->rec.p, d_in, N * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CK(ctx->qb.reserve(std::max<u64>(acc, 1) * sizeof(int32_t)));
    CK(ctx->tval.reserve(G.nblocks * sizeof(float)));
    CK(ctx->tint.reserve(G.nblocks * L * sizeof(int64_t)));
    CK(ctx->axis.reserve(std::max<size_t>(G.ent.size(), 1) * sizeof(AxisEntry)));
    CK(ctx->classes.reserve(27 * L * sizeof(ClassInfo)));
    const u64 amb_cap = 4096;
    CK(ctx->amb.reserve(amb_cap * sizeof(AmbiguousRecord)));
    CK(ctx->proxies.reserve(G.nblocks * L * 10 * sizeof(float)));
    CK(cudaMemsetAsync(ctx->proxies.p, 0xff, G.nblocks * L * 10 * sizeof(float), st));
    const AxisEntry *d_ent = ctx->axis.as<AxisEntry>();
    CK(cudaMemcpyAsync(ctx->axis.p, G.ent.data(), G.ent.size() * sizeof(AxisEntry), cudaMemcpyHostToDevice, st));
    for (u64 l = 0; l < L; l++)
        for (auto &ci : G.classes[l])
            if (ci.n) ci.log2_off = log2_table(ctx, ci.n);
    std::vector<ClassInfo> cls_flat;
    for (u64 l = 0; l < L; l++) cls_flat.insert(cls_flat.end(), G.classes[l].begin(), G.classes[l].end());
    CK(cudaMemcpyAsync(ctx->classes.p, cls_flat.data(), cls_flat.size() * sizeof(ClassInfo), cudaMemcpyHostToDevice, st));
    rc = upload_log2(ctx);
    if (rc) return rc;
    uint32_t capmax = 1;
    for (u64 l = 0; l < L; l++) capmax = std::max(capmax, G.cap[l]);
    uint32_t bcap, tcap;
    u64 sstride;
    scratch_dims(capmax, bcap, tcap, sstride);
    // Exact-path scratch: one slot per thread; every group in exact mode, otherwise a pool that
    // the listed groups share.
    const u64 slots = std::min<u64>(G.nblocks, 2048);
    CK(ctx->scratch.reserve(slots * sstride));
    CK(ctx->tlist.reserve(G.nblocks * sizeof(uint32_t)));
    CK(ctx->spill.reserve(G.nblocks * sizeof(uint32_t)));
    // Global scratch of the exact replay for groups above the shared-memory capacity: a slice per
    // CTA, at most 148 CTAs and 512 MiB.
    const u64 gstride = exact_global_stride(capmax);
    unsigned ggrid = 0;
    if (capmax > exact_cap()) {
        ggrid = (unsigned)std::max<u64>(1, std::min<u64>(148, (512ull << 20) / gstride));
        CK(ctx->gscratch.reserve(ggrid * gstride));
        CK(ctx->spill2.reserve(G.nblocks * sizeof(uint32_t)));
    }
    if (ctx->tsel_mode == 1) {
        std::vector<uint32_t> iota(G.nblocks);
        for (u64 i = 0; i < G.nblocks; i++) iota[i] = (uint32_t)i;
        CK(ctx->iota.reserve(G.nblocks * sizeof(uint32_t)));
        CK(cudaMemcpyAsync(ctx->iota.p, iota.data(), G.nblocks * 4, cudaMemcpyHostToDevice, st));
        uint32_t cnt = (uint32_t)G.nblocks;
        CK(cudaMemcpyAsync(&dm->all_count, &cnt, 4, cudaMemcpyHostToDevice, st));
    }
    const float Rg = mx - mn, R2 = Rg * Rg;
    const float t_default = 4.0f / 16;  // insufficient_sample_t (asz_param.hpp:206)
    int32_t init_range[2] = {INT32_MAX, INT32_MIN};
    std::vector<uint32_t> overrides;  // (block, round, t bits) settled by host replays
    std::vector<AmbiguousRecord> ambs;
    uint32_t fb_total = 0;
    int reruns = 0;
    float *d_rec = ctx->rec.as<float>();
    int32_t *d_qb = ctx->qb.as<int32_t>();
    float *d_tval = ctx->tval.as<float>();
    int64_t *d_tint = ctx->tint.as<int64_t>();
    // Every round along axis 2 on a whole field: all rounds fused per column of lines (k_lines.cu).
    if (a.t_given) {
        if (a.t_len != G.nblocks * L) return fail(ctx, ASZ_E_ARG, "t table length does not match the plan's blocks and rounds");
        CK(cudaMemcpyAsync(d_tint, a.t_given, a.t_len * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    }
    const uint32_t line_bytes = (!a.probe && !a.origin && !a.t_given && ctx->tsel_mode == 2) ? lines_smem_bytes(G) : 0;
    const int tsel_mode = ctx->tsel_mode == 2 ? 0 : ctx->tsel_mode;  // 2: the fast path with fused rounds
    const u64 ncols = G.fg.block_num[0] * G.fg.block_num[1];
    const RoundGeom *d_rounds = nullptr;
    const u64 *d_qoff = nullptr;
    u64 lines_alg_bytes = 0;
    if (line_bytes) {
        const u64 rbytes = L * sizeof(RoundGeom);
        CK(ctx->rounds_dev.reserve(rbytes + (L + 1) * sizeof(u64)));
        uint8_t *rd = ctx->rounds_dev.as<uint8_t>();
        CK(cudaMemcpyAsync(rd, G.rounds.data(), rbytes, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(rd + rbytes, qb_off.data(), (L + 1) * sizeof(u64), cudaMemcpyHostToDevice, st));
        d_rounds = (const RoundGeom *)rd;
        d_qoff = (const u64 *)(rd + rbytes);
        CK(ctx->lines_bail.reserve(std::max<u64>(G.nblocks * L, 1) * sizeof(uint32_t)));
        CK(ctx->lines_resume.reserve(std::max<u64>(4 * ncols, 1) * sizeof(uint32_t)));
        // Algorithmic bytes: the field loaded and stored once; per target its original value read
        // and its QB written; per coefficient sample its original value read.
        lines_alg_bytes = N * 8;
        for (u64 l = 0; l < L; l++) {
            lines_alg_bytes += G.rounds[l].targets * 8;
            for (int c = 0; c < 27; c++) {
                const ClassInfo &ci = G.classes[l][c];
                if (ci.fallback || !ci.n) continue;
                u64 m = 1;
                for (int ax = 0; ax < 3; ax++) {
                    const u64 nb = G.fg.block_num[ax], k = ax == 0 ? c / 9 : ax == 1 ? (c / 3) % 3 : c % 3;
                    m *= k == 0 ? 1 : k == 1 ? (nb > 2 ? nb - 2 : 0) : (nb >= 2 ? 1 : 0);
                }
                lines_alg_bytes += m * ci.n * 4;
            }
        }
    }
    u64 lines_exact = 0, lines_serial = 0;
    // Codes built during the rounds (CoreArgs::prebuild): each round's kernel counts its stream's
    // QB histogram window; a copy on the side stream behind the kernel and a code build on the
    // builder thread follow it, while the main stream runs the next rounds.
    const bool prebuild = a.prebuild && !line_bytes && !a.probe && !a.origin && L > 0;
    unsigned long long *d_hwin = nullptr;
    u64 *h_hist = nullptr;
    int32_t *h_rng = nullptr;
    uint32_t *h_over = nullptr;
    o.pre.assign(L + 1, PreCode{});
    if (prebuild) {
        CK(ctx->hwin.reserve(L * kHistWin * 8));
        CK(ctx->hwin_host.reserve(L * kHistWin * 8 + L * 8 + L * 4 + 8 + G.pivots * 4));
        d_hwin = ctx->hwin.as<unsigned long long>();
        h_hist = (u64 *)ctx->hwin_host.p;
        h_rng = (int32_t *)(h_hist + L * kHistWin);
        h_over = (uint32_t *)(h_rng + 2 * L);
        while (ctx->round_ev.size() < 2 * L) {
            cudaEvent_t e;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            ctx->round_ev.push_back(e);
        }
        if (!ctx->builder) ctx->builder = std::make_unique<SerialWorker>();
    }
    // Every return from here waits for the builder, which writes into o.pre.
    struct BuilderWait {
        SerialWorker *w;
        ~BuilderWait() {
            if (w) w->wait();
        }
    } builder_wait{prebuild ? ctx->builder.get() : nullptr};
    auto schedule_code = [&](u64 l) -> int {
        if (!prebuild) return ASZ_OK;
        cudaEvent_t ev_r = ctx->round_ev[2 * l], ev_c = ctx->round_ev[2 * l + 1];
        CK(cudaEventRecord(ev_r, st));
        CK(cudaStreamWaitEvent(ctx->side, ev_r, 0));
        CK(cudaMemcpyAsync(h_hist + l * kHistWin, d_hwin + l * kHistWin, kHistWin * 8, cudaMemcpyDeviceToHost, ctx->side));
        CK(cudaMemcpyAsync(h_rng + 2 * l, &dm->qb_range[2 * (l + 1)], 8, cudaMemcpyDeviceToHost, ctx->side));
        CK(cudaMemcpyAsync(h_over + l, &dm->hist_over[l], 4, cudaMemcpyDeviceToHost, ctx->side));
        CK(cudaEventRecord(ev_c, ctx->side));
        const u64 count = qb_len[l + 1];
        PreCode *pc = &o.pre[l + 1];
        const int dev = ctx->device;
        const u64 *hl = h_hist + l * kHistWin;
        const int32_t *rl = h_rng + 2 * l;
        const uint32_t *ol = h_over + l;
        ctx->builder->submit([=]() {
            cudaSetDevice(dev);
            if (cudaEventSynchronize(ev_c) != cudaSuccess) return;
            const int32_t lo = rl[0], hi = rl[1];
            if (*ol || count == 0 || lo > hi || lo < -(int32_t)kHistHalf || hi >= (int32_t)kHistHalf) return;
            const u64 *h = hl + (int64_t)lo + kHistHalf;
            u64 a0 = 0, b0 = (u64)(hi - lo) + 1;
            while (a0 < b0 && h[a0] == 0) a0++;
            while (b0 > a0 && h[b0 - 1] == 0) b0--;
            std::vector<u64> hh(h + a0, h + b0);
            std::string err;
            HuffCode code;
            if (!build_code(hh, (int64_t)lo + (int64_t)a0, (int64_t)lo + (int64_t)b0 - 1, count, false, code, err)) return;
            pc->code = std::move(code);
            pc->lo = (int64_t)lo + (int64_t)a0;
            pc->hi = (int64_t)lo + (int64_t)b0 - 1;
            pc->ok = true;
        });
        return ASZ_OK;
    };
    // The pivot stream's code, from a host copy of its QBs taken behind the pivot kernel (its
    // range is known only then, and it is small: one value per pivot).
    auto schedule_pivot_code = [&]() -> int {
        if (!prebuild || G.pivots == 0) return ASZ_OK;
        int32_t *h_prng = (int32_t *)(h_over + L);
        int32_t *h_piv = h_prng + 2;
        if (ctx->round_ev.size() < 2 * L + 2) {
            for (int k = 0; k < 2; k++) {
                cudaEvent_t e;
                CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                ctx->round_ev.push_back(e);
            }
        }
        cudaEvent_t ev_r = ctx->round_ev[2 * L], ev_c = ctx->round_ev[2 * L + 1];
        CK(cudaEventRecord(ev_r, st));
        CK(cudaStreamWaitEvent(ctx->side, ev_r, 0));
        CK(cudaMemcpyAsync(h_piv, d_qb + qb_off[0], G.pivots * 4, cudaMemcpyDeviceToHost, ctx->side));
        CK(cudaMemcpyAsync(h_prng, &dm->qb_range[0], 8, cudaMemcpyDeviceToHost, ctx->side));
        CK(cudaEventRecord(ev_c, ctx->side));
        const u64 count = G.pivots;
        PreCode *pc = &o.pre[0];
        const int dev = ctx->device;
        ctx->builder->submit([=]() {
            cudaSetDevice(dev);
            if (cudaEventSynchronize(ev_c) != cudaSuccess) return;
            const int32_t lo = h_prng[0], hi = h_prng[1];
            if (lo > hi || (u64)((int64_t)hi - lo) >= (1ull << 24)) return;
            std::vector<u64> h((u64)((int64_t)hi - lo) + 1, 0);
            for (u64 i = 0; i < count; i++) {
                const int64_t v = (int64_t)h_piv[i] - lo;
                if (v < 0 || v >= (int64_t)h.size()) return;
                h[(u64)v]++;
            }
            std::string err;
            HuffCode code;
            if (!build_code(h, lo, hi, count, false, code, err)) return;
            pc->code = std::move(code);
            pc->lo = lo;
            pc->hi = hi;
            pc->ok = true;
        });
        return ASZ_OK;
    };
    hs_prep.reset();
    std::optional<HostScope> hs_rounds(std::in_place, ctx, "host:rounds");
    while (true) {
        // Error word, fallback count, ambiguity count, QB ranges.
        if (prebuild) {
            ctx->builder->wait();  // builds of a previous attempt
            for (PreCode &pc : o.pre) pc = PreCode{};
            CK(cudaMemsetAsync(d_hwin, 0, L * kHistWin * 8, st));
            CK(cudaMemsetAsync(dm->hist_over, 0, sizeof(dm->hist_over), st));
        }
        CK(cudaMemsetAsync(&dm->err, 0, 3 * sizeof(uint32_t), st));
        CK(cudaMemsetAsync(dm->why, 0, sizeof(dm->why), st));
        for (u64 s = 0; s <= L; s++)
            CK(cudaMemcpyAsync(&dm->qb_range[2 * s], init_range, 8, cudaMemcpyHostToDevice, st));
        if (!overrides.empty()) {
            CK(ctx->overrides.reserve(overrides.size() * sizeof(uint32_t)));
            CK(cudaMemcpyAsync(ctx->overrides.p, overrides.data(), overrides.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, st));
        }
        // Pivots (compress.tpp:162-175).
        {
            ProfScope ps(ctx, "pivot_compress", G.pivots * 12);
            CK(launch_pivot_compress(G.pg, d_in, d_rec, d_qb + qb_off[0], &dm->qb_range[0], st));
        }
        rc = schedule_pivot_code();
        if (rc) return rc;
        if (line_bytes) {
            // Fused pass over all columns. Blocks the certified fast path cannot settle stop their
            // column at that round; the exact path then settles them round by round, and their
            // columns resume from there, until no column is left waiting (at most one pass per round).
            const uint32_t nov = (uint32_t)(overrides.size() / 3);
            uint32_t *d_bail = ctx->lines_bail.as<uint32_t>();
            uint32_t *d_res[2] = {ctx->lines_resume.as<uint32_t>(), ctx->lines_resume.as<uint32_t>() + 2 * ncols};
            uint32_t n_resume = 0;
            int cur = 0;
            lines_exact = lines_serial = 0;
            CK(cudaMemsetAsync(dm->spill_count, 0, sizeof(dm->spill_count), st));
            for (u64 pass = 0;; pass++) {
                if (pass > L) return fail(ctx, ASZ_E_DEVICE, "fused rounds did not finish");
                CK(cudaMemsetAsync(dm->list_count, 0, sizeof(dm->list_count), st));
                CK(cudaMemsetAsync(&dm->resume_count, 0, 4, st));
                {
                    ProfScope ps(ctx, "lines_compress", pass ? 0 : lines_alg_bytes);
                    std::vector<LinesLaunch> lls = lines_launches(G, line_bytes);
                    if (pass) lls = {{kColumnsAll, line_bytes}};  // resumptions list column indices
                    for (const LinesLaunch &ll : lls)
                        CK(launch_lines_compress(G.fg, d_rounds, d_ent, d_qoff, ctx->classes.as<ClassInfo>(), d_in, d_rec,
                                                 ctx->log2arena.as<float>(), R2, t_default, d_tval, d_tint, &dm->fb, d_qb,
                                                 dm->qb_range, ctx->overrides.as<uint32_t>(), nov, dm->why,
                                                 pass ? d_res[cur] : nullptr, n_resume, d_bail, dm->list_count,
                                                 d_res[cur ^ 1], &dm->resume_count, &dm->err, ll.set, ll.bytes, st));
                }
                uint32_t bails[64], spills[64], nres = 0;
                CK(cudaMemcpyAsync(bails, dm->list_count, sizeof(bails), cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(spills, dm->spill_count, sizeof(spills), cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(&nres, &dm->resume_count, 4, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                for (u64 l = 0; l < L; l++) lines_serial += spills[l];
                if (nres == 0) break;
                if (nres > ncols) return fail(ctx, ASZ_E_DEVICE, "fused rounds listed too many columns");
                CK(cudaMemsetAsync(dm->spill_count, 0, sizeof(dm->spill_count), st));
                for (u64 l = 0; l < L; l++) {
                    if (!bails[l]) continue;
                    if (bails[l] > G.nblocks) return fail(ctx, ASZ_E_DEVICE, "fused rounds listed too many blocks");
                    lines_exact += bails[l];
                    const RoundGeom &rg = G.rounds[l];
                    const ClassInfo *cls = ctx->classes.as<ClassInfo>() + 27 * l;
                    uint32_t *d_spill = ctx->spill.as<uint32_t>(), *d_scount = &dm->spill_count[l];
                    {
                        ProfScope ps(ctx, "tsel_exact", 0);
                        CK(launch_tsel_exact(G.fg, rg, (uint32_t)l, cls, d_rec, d_in, ctx->log2arena.as<float>(), R2, t_default,
                                             d_tval, d_tint, &dm->fb, ctx->amb.as<AmbiguousRecord>(), (uint32_t)amb_cap,
                                             &dm->amb_count, ctx->overrides.as<uint32_t>(), nov,
                                             ctx->proxies.as<float>() + G.nblocks * l * 10, d_bail + G.nblocks * l,
                                             &dm->list_count[l], d_spill, d_scount, exact_cap(), 148, st));
                    }
                    {
                        ProfScope ps(ctx, "tsel_serial", 0);
                        CK(launch_tsel_v0(G.fg, rg, (uint32_t)l, cls, d_rec, d_in, ctx->log2arena.as<float>(), R2, t_default,
                                          ctx->scratch.as<uint8_t>(), sstride, capmax, bcap, tcap, d_tval, d_tint, &dm->fb,
                                          ctx->amb.as<AmbiguousRecord>(), (uint32_t)amb_cap, &dm->amb_count,
                                          ctx->overrides.as<uint32_t>(), nov, ctx->proxies.as<float>() + G.nblocks * l * 10,
                                          d_spill, d_scount, slots, &dm->err, st));
                    }
                }
                n_resume = nres;
                cur ^= 1;
            }
        }
        for (u64 l = 0; l < L && !line_bytes; l++) {
            const RoundGeom &rg = G.rounds[l];
            const ClassInfo *cls = ctx->classes.as<ClassInfo>() + 27 * l;
            const uint32_t nov = (uint32_t)(overrides.size() / 3);
            if (a.before_round) {
                rc = a.before_round(l);
                if (rc) return rc;
            }
            if (a.t_given) {
                // The caller's t codes replace the coefficient selection.
                CK(launch_tval_from_codes(d_tint, G.nblocks, (uint32_t)L, (uint32_t)l, (float)p.t_precision, d_tval, st));
                ProfScope ps(ctx, "round_compress", rg.targets * 12);
                CK(launch_round_compress(G.fg, rg, d_ent, d_tval, d_in, d_rec, d_qb + qb_off[l + 1],
                                         &dm->qb_range[2 * (l + 1)], &dm->err, 0, nullptr, st,
                                         prebuild ? d_hwin + l * kHistWin : nullptr, prebuild ? &dm->hist_over[l] : nullptr));
                rc = schedule_code(l);
                if (rc) return rc;
                continue;
            }
            uint32_t *d_list = ctx->tlist.as<uint32_t>(), *d_lcount = &dm->list_count[l % 64];
            uint32_t *d_spill = ctx->spill.as<uint32_t>(), *d_scount = &dm->spill_count[l % 64];
            CK(cudaMemsetAsync(d_scount, 0, 4, st));
            if (tsel_mode == 0) {
                // Blocks per class (first, middle, last along each axis), for the algorithmic bytes
                // (one read of the 5 operands, 4 neighbours + original, per sample) and the group
                // size of the most populous class, which picks the kernel's CTA width.
                u64 per_axis[3][3];
                for (int a = 0; a < 3; a++) {
                    const u64 nb = G.fg.block_num[a];
                    per_axis[a][0] = 1;
                    per_axis[a][1] = nb > 2 ? nb - 2 : 0;
                    per_axis[a][2] = nb >= 2 ? 1 : 0;
                }
                u64 sample_bytes = 0, most = 0;
                uint32_t common_samples = 0;
                for (int c = 0; c < 27; c++) {
                    const ClassInfo &ci = G.classes[l][c];
                    if (ci.fallback || !ci.n) continue;
                    const u64 blocks = per_axis[0][c / 9] * per_axis[1][(c / 3) % 3] * per_axis[2][c % 3];
                    sample_bytes += blocks * ci.n * 20;
                    if (blocks > most || (blocks == most && ci.n > common_samples)) {
                        most = blocks;
                        common_samples = ci.n;
                    }
                }
                ProfScope ps(ctx, "tsel_fast", sample_bytes);
                CK(cudaMemsetAsync(d_lcount, 0, 4, st));
                CK(launch_tsel_fast(G.fg, rg, (uint32_t)l, cls, d_rec, d_in, ctx->log2arena.as<float>(), R2, t_default, d_tval,
                                    d_tint, &dm->fb, d_list, d_lcount, ctx->overrides.as<uint32_t>(), nov, dm->why, st,
                                    common_samples));
            } else {
                d_list = ctx->iota.as<uint32_t>();
                d_lcount = &dm->all_count;
            }
            {
                ProfScope ps(ctx, "tsel_exact", 0);
                CK(launch_tsel_exact(G.fg, rg, (uint32_t)l, cls, d_rec, d_in, ctx->log2arena.as<float>(), R2, t_default, d_tval,
                                     d_tint, &dm->fb, ctx->amb.as<AmbiguousRecord>(), (uint32_t)amb_cap, &dm->amb_count,
                                     ctx->overrides.as<uint32_t>(), nov, ctx->proxies.as<float>() + G.nblocks * l * 10,
                                     d_list, d_lcount, d_spill, d_scount, exact_cap(), 148, st));
            }
            // Groups larger than shared memory holds: the same replay with global scratch, a CTA
            // per group; only what that cannot take (keys outside int32) reaches the serial kernel.
            uint32_t *d_left = d_spill, *d_lcnt = d_scount;
            if (G.cap[l] > exact_cap()) {
                d_left = ctx->spill2.as<uint32_t>();
                d_lcnt = &dm->spill2_count[l % 64];
                CK(cudaMemsetAsync(d_lcnt, 0, 4, st));
                ProfScope ps(ctx, "tsel_exact_global", 0);
                CK(launch_tsel_exact_global(G.fg, rg, (uint32_t)l, cls, d_rec, d_in, ctx->log2arena.as<float>(), R2, t_default,
                                            d_tval, d_tint, &dm->fb, ctx->amb.as<AmbiguousRecord>(), (uint32_t)amb_cap,
                                            &dm->amb_count, ctx->overrides.as<uint32_t>(), nov,
                                            ctx->proxies.as<float>() + G.nblocks * l * 10, d_spill, d_scount, d_left, d_lcnt,
                                            ctx->gscratch.as<uint8_t>(), gstride, G.cap[l], ggrid, st));
            }
            {
                ProfScope ps(ctx, "tsel_serial", 0);
                CK(launch_tsel_v0(G.fg, rg, (uint32_t)l, cls, d_rec, d_in, ctx->log2arena.as<float>(), R2, t_default,
                                  ctx->scratch.as<uint8_t>(), sstride, capmax, bcap, tcap, d_tval, d_tint, &dm->fb,
                                  ctx->amb.as<AmbiguousRecord>(), (uint32_t)amb_cap, &dm->amb_count,
                                  ctx->overrides.as<uint32_t>(), nov, ctx->proxies.as<float>() + G.nblocks * l * 10, d_left,
                                  d_lcnt, slots, &dm->err, st));
            }
            ProfScope ps(ctx, "round_compress", rg.targets * 12);
            CK(launch_round_compress(G.fg, rg, d_ent, d_tval, d_in, d_rec, d_qb + qb_off[l + 1],
                                     &dm->qb_range[2 * (l + 1)], &dm->err, a.probe ? 1 : 0, a.pred_out, st,
                                     prebuild ? d_hwin + l * kHistWin : nullptr, prebuild ? &dm->hist_over[l] : nullptr));
            rc = schedule_code(l);
            if (rc) return rc;
        }
        uint32_t words[3];
        uint32_t lcounts[64], scounts[64];
        CK(cudaMemcpyAsync(words, &dm->err, sizeof(words), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(lcounts, dm->list_count, sizeof(lcounts), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(scounts, dm->spill_count, sizeof(scounts), cudaMemcpyDeviceToHost, st));
        uint32_t s2counts[64];
        CK(cudaMemcpyAsync(s2counts, dm->spill2_count, sizeof(s2counts), cudaMemcpyDeviceToHost, st));
        uint32_t why[3];
        CK(cudaMemcpyAsync(why, dm->why, sizeof(why), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        R.exact_window = why[0];
        R.exact_undecided = why[1];
        R.wide_groups = why[2];
        R.exact_groups = 0;
        R.serial_groups = 0;
        for (u64 l = 0; l < L && l < 64; l++) {
            if (tsel_mode == 0) R.exact_groups += lcounts[l];
            R.serial_groups += !line_bytes && G.cap[l] > exact_cap() ? s2counts[l] : scounts[l];
        }
        if (line_bytes) {
            R.exact_groups = lines_exact;
            R.serial_groups = lines_serial;
        }
        if (words[0]) return fail(ctx, ASZ_E_DEVICE, "round kernels reported an internal error " + std::to_string(words[0]));
        fb_total = words[1];
        uint32_t namb = words[2];
        if (namb > amb_cap) return fail(ctx, ASZ_E_UNSUPPORTED, "too many ambiguous coefficient decisions");
        ambs.resize(namb);
        if (namb) CK(cudaMemcpy(ambs.data(), ctx->amb.p, namb * sizeof(AmbiguousRecord), cudaMemcpyDeviceToHost));
        bool changed = false;
        for (const AmbiguousRecord &r : ambs) {
            float t = replay_decision(r, G.rounds[r.round].slope);
            int32_t code = (int32_t)host_lround_f(t * (float)p.t_precision);
            R.ambiguous_decisions++;
            if (code != r.provisional) {
                uint32_t bits;
                std::memcpy(&bits, &t, 4);
                overrides.push_back(r.block);
                overrides.push_back(r.round);
                overrides.push_back(bits);
                changed = true;
            }
        }
        if (a.agree) {
            rc = a.agree(changed);
            if (rc) return rc;
        }
        if (!changed) break;
        if (++reruns > 16) return fail(ctx, ASZ_E_DEVICE, "coefficient decisions did not settle");
    }
    R.reruns = (u64)reruns;
    R.t_fallback_count = fb_total;
    hs_rounds.reset();
    return ASZ_OK;
}


// ---------------------------------------------------------------------------------------------
// Predictor-family selection: param_c::select_predictor_family (predictor_family.tpp:217-251).
// Each sampled target block is compressed with its context (the blocks below it on each axis and
// a halo of input values) by the device core in a frame, once per family, with the probe's
// quantisation form; the target's predictions, reconstructions and QBs come back for the
// reference's long-double reductions. Those follow the reference build on x87: log2 and log10
// through fyl2x, divisions by a count as multiplications by its reciprocal, no infinity test
// in the score, and floor for the point budget.

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

struct FamilyEval {
    u64 points = 0;
    long double pred_mse = 0, rec_mse = 0, psnr = 0, h1 = 0;
};

long double family_entropy(const std::vector<int32_t> &qbs) {
    if (qbs.empty()) return 0;
    std::unordered_map<int32_t, u64> freq;
    for (int32_t q : qbs) freq[q]++;
    const long double r = 1.0L / (long double)qbs.size();
    long double h1 = 0;
    for (const auto &kv : freq) {
        const long double pr = (long double)kv.second * r;
        h1 = h1 - pr * x87_fyl2x(pr, 1.0L);
    }
    return h1;
}

struct FamilyProbe {
    const float *d_in;
    const uint64_t *dims;
    Plan plan;
    asz_params p;  // the probe's: block ratio, and h1_block_sampling_num at its default
    u64 ps[3], shape[3], bnum[3];
    float mn, mx, abs_eb, slope;
};

int family_evaluate(asz_ctx *ctx, const FamilyProbe &pr, const std::vector<std::array<u64, 3>> &targets, bool quintic,
                    FamilyEval &out) {
    cudaStream_t st = ctx->stream;
    const u64 L = pr.plan.pred.size();
    std::vector<std::vector<int32_t>> layer_qbs(L);
    std::vector<long double> pred_sse(L, 0), rec_sse(L, 0);
    std::vector<u64> counts(L, 0);
    for (const auto &tb : targets) {
        u64 cbb[3], cb[3], ce[3], hb[3], m[3], origin[3], tl[3];
        for (int a = 0; a < 3; a++) {
            cbb[a] = tb[a] ? tb[a] - 1 : 0;
            cb[a] = cbb[a] * pr.shape[a];
            ce[a] = std::min((tb[a] + 1) * pr.shape[a] + 1, pr.dims[a]);
            const u64 left_halo = 5 * (pr.ps[a] / 2);
            hb[a] = cb[a] > left_halo ? cb[a] - left_halo : 0;
            m[a] = ce[a] - hb[a];
            origin[a] = cb[a] - hb[a];
            tl[a] = tb[a] - cbb[a];  // target block in the frame
        }
        const u64 n = m[0] * m[1] * m[2];
        CK(ctx->probe_in.reserve(n * sizeof(float)));
        CK(ctx->probe_pred.reserve(n * sizeof(float)));
        CK(launch_copy_box(pr.d_in, pr.dims, hb, m, ctx->probe_in.as<float>(), st));
        CoreOut co;
        asz_report scratch{};
        CoreArgs ca{ctx->probe_in.as<float>(), m, origin, &pr.plan, &pr.p, quintic, true, ctx->probe_pred.as<float>(),
                    pr.mn, pr.mx, pr.abs_eb, pr.slope};
        int rc = run_core(ctx, ca, co, scratch);
        if (rc) return rc;
        std::vector<float> orig(n), rec(n), pred(n);
        u64 qtot = co.qb_off[L] + co.qb_len[L];
        std::vector<int32_t> qb(qtot);
        CK(cudaMemcpyAsync(orig.data(), ctx->probe_in.p, n * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rec.data(), ctx->rec.p, n * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(pred.data(), ctx->probe_pred.p, n * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(qb.data(), ctx->qb.p, qtot * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const Geometry &G = co.G;
        for (u64 l = 0; l < L; l++) {
            const RoundGeom &rg = G.rounds[l];
            // The target block's targets in block_compress_impl's loop order (compress.tpp:67-86).
            u64 lo[3], hi[3], left[3];
            for (int a = 0; a < 3; a++) {
                lo[a] = origin[a] + tl[a] * pr.shape[a];
                hi[a] = std::min(lo[a] + pr.shape[a] + 1, m[a]);
                left[a] = a == rg.dir ? lo[a] + rg.stride[a] / 2 : (lo[a] == 0 ? 0 : lo[a] + rg.stride[a]);
            }
            long double lp = 0, lr = 0;
            u64 lc = 0;
            for (u64 i0 = left[0]; i0 < hi[0]; i0 += rg.stride[0])
                for (u64 i1 = left[1]; i1 < hi[1]; i1 += rg.stride[1])
                    for (u64 i2 = left[2]; i2 < hi[2]; i2 += rg.stride[2]) {
                        const u64 pos = (i0 * m[1] + i1) * m[2] + i2;
                        const long double pe = (long double)pred[pos] - (long double)orig[pos];
                        const long double re = (long double)rec[pos] - (long double)orig[pos];
                        lp = lp + pe * pe;
                        lr = lr + re * re;
                        lc++;
                    }
            pred_sse[l] = pred_sse[l] + lp;
            rec_sse[l] = rec_sse[l] + lr;
            counts[l] += lc;
            // Its QB box, in stream order.
            u64 cc[3], pre[3];
            for (int a = 0; a < 3; a++) {
                cc[a] = G.tab_count[rg.axis_off[a] + tl[a]];
                pre[a] = G.tab_prefix[rg.axis_off[a] + tl[a]];
            }
            const u64 base = pre[0] * rg.total[1] * rg.total[2] + cc[0] * pre[1] * rg.total[2] + cc[0] * cc[1] * pre[2];
            const u64 size = cc[0] * cc[1] * cc[2];
            if (size != lc || base + size > co.qb_len[l + 1]) return fail(ctx, ASZ_E_DEVICE, "predictor-family target count mismatch");
            const int32_t *q = qb.data() + co.qb_off[l + 1] + base;
            layer_qbs[l].insert(layer_qbs[l].end(), q, q + size);
        }
    }
    out = FamilyEval();
    long double wh1 = 0, ptot = 0, rtot = 0;
    for (u64 l = 0; l < L; l++) {
        out.points += counts[l];
        ptot = ptot + pred_sse[l];
        rtot = rtot + rec_sse[l];
        wh1 = wh1 + family_entropy(layer_qbs[l]) * (long double)counts[l];
    }
    if (out.points == 0) return fail(ctx, ASZ_E_DATA, "predictor-family sample contains no target points");
    const long double rc = 1.0L / (long double)out.points;
    out.pred_mse = ptot * rc;
    out.rec_mse = rtot * rc;
    const long double range = (long double)pr.mx - (long double)pr.mn;
    out.psnr = out.rec_mse == 0 ? (long double)INFINITY : x87_fyl2x(range * range / out.rec_mse, x87_lg2()) * 10.0L;
    out.h1 = wh1 * rc;
    return ASZ_OK;
}

int select_family(asz_ctx *ctx, const float *d_in, const uint64_t dims[3], const asz_params &p, float rel_eb, float abs_eb,
                  float mn, float mx, float slope, const Plan &plan, bool &quintic, asz_report &R) {
    FamilyProbe pr;
    pr.d_in = d_in;
    pr.dims = dims;
    pr.p = p;
    pr.p.h1_block_sampling_num = 256;  // not copied to the probe (copy_settings, predictor_family.tpp:17-37)
    pr.mn = mn;
    pr.mx = mx;
    pr.abs_eb = abs_eb;
    pr.slope = slope;
    const u64 L = plan.pred.size();
    const u64 suffix = std::min<u64>(p.predictor_family_suffix_layers, L);
    std::string txt;
    for (u64 l = L - suffix; l < L; l++) txt += (l > L - suffix ? "," : "") + plan.pred[l];
    std::string perr;
    if (!parse_plan(txt.c_str(), pr.plan, perr)) return fail(ctx, ASZ_E_DEVICE, perr);
    pr.p.block_pivot_ratio = rel_eb <= p.predictor_family_fine_eb_threshold ? p.predictor_family_fine_probe_block_pivot_ratio
                                                                           : p.predictor_family_coarse_probe_block_pivot_ratio;
    for (int a = 0; a < 3; a++) pr.ps[a] = 1;
    for (u64 l = 0; l < suffix; l++) pr.ps[pr.plan.dir[l]] *= 2;
    for (int a = 0; a < 3; a++) {
        pr.shape[a] = pr.ps[a] * pr.p.block_pivot_ratio;
        pr.bnum[a] = (dims[a] + pr.shape[a] - 1) / pr.shape[a];
    }
    // make_stratified_targets (predictor_family.tpp:65-86).
    const u64 total = pr.bnum[0] * pr.bnum[1] * pr.bnum[2];
    const u64 sc = std::min<u64>(p.predictor_family_sample_blocks, total);
    std::mt19937_64 rng(0);
    std::vector<std::array<u64, 3>> cands;
    for (u64 s = 0; s < sc; s++) {
        const u64 sb = (u64)((unsigned __int128)s * total / sc), se = (u64)((unsigned __int128)(s + 1) * total / sc);
        u64 index = sb + rng() % (se - sb);
        std::array<u64, 3> t;
        t[2] = index % pr.bnum[2];
        index /= pr.bnum[2];
        t[1] = index % pr.bnum[1];
        t[0] = index / pr.bnum[1];
        cands.push_back(t);
    }
    const u64 N = dims[0] * dims[1] * dims[2];
    const u64 fraction_budget = (u64)floorl((long double)N * (long double)p.predictor_family_sample_fraction_limit);
    const u64 budget = std::min<u64>(p.predictor_family_sample_point_limit, fraction_budget);
    std::vector<std::array<u64, 3>> targets;
    u64 sampled = 0;
    for (const auto &c : cands) {  // apply_point_budget (predictor_family.tpp:99-114)
        u64 pts = 1;
        for (int a = 0; a < 3; a++) pts *= std::min((c[a] + 1) * pr.shape[a] + 1, dims[a]) - c[a] * pr.shape[a];
        if (sampled <= budget && pts <= budget - sampled) {
            targets.push_back(c);
            sampled += pts;
        }
    }
    R.family_selected = 1;
    R.fam_suffix_layers = suffix;
    R.fam_budget = budget;
    R.fam_probe_bpr = pr.p.block_pivot_ratio;
    R.fam_sampled_points = sampled;
    R.fam_blocks = targets.size();
    if (targets.empty()) {
        R.family_fallback = 1;
        quintic = false;
        return ASZ_OK;
    }
    FamilyEval c, q;
    int rc = family_evaluate(ctx, pr, targets, false, c);
    if (rc) return rc;
    rc = family_evaluate(ctx, pr, targets, true, q);
    if (rc) return rc;
    const long double score = (c.h1 - q.h1) * (long double)slope + (q.psnr - c.psnr);
    R.fam_points = c.points;
    R.fam_cubic_mse = c.pred_mse;
    R.fam_quintic_mse = q.pred_mse;
    R.fam_cubic_psnr = c.psnr;
    R.fam_quintic_psnr = q.psnr;
    R.fam_cubic_h1 = c.h1;
    R.fam_quintic_h1 = q.h1;
    R.fam_score_gain = score;
    quintic = score > 0;
    return ASZ_OK;
}

// ---- Entropy stage of one field: the t stream (int64) and L+1 QB streams (int32) Huffman-coded
// on the device and assembled with their headers into ctx->pre_zstd (compress.tpp:233-291).
struct EncodeArgs {
    const Geometry *G;
    const std::vector<u64> *qb_off, *qb_len;
    const int32_t *d_qb;       // streams at qb_off
    const int64_t *d_tint;     // t codes, block-major
    const int32_t *d_ranges;   // [min, max] per QB stream
    float mn, mx;
    bool quintic;
    const Plan *plan;
    const asz_params *p;
    const int64_t *t_given;    // a caller's t table, or nullptr
    u64 t_len, N;
    const std::vector<PreCode> *pre = nullptr;  // QB streams' codes built during the rounds
};

// Entropy stage of several fields at once: ranges, histograms, code builds (host threads over all
// streams of all fields), Huffman encoding, and the assembly of each field's pre-zstd stream into
// one pinned buffer (span[f] = offset, length). Each field's bytes are those of a single-field
// run; the fields only share the transfers and the synchronisations.
int encode_fields(asz_ctx *ctx, const std::vector<EncodeArgs> &A, std::vector<asz_report *> &Rs,
                  std::vector<std::pair<u64, u64>> &span, PinnedBuf &pb) {
    const u64 nf = A.size();
    cudaStream_t st = ctx->stream;
    const float t_default = 4.0f / 16;  // insufficient_sample_t (asz_param.hpp:206)
    std::optional<HostScope> hs_codes(std::in_place, ctx, "host:codes");
    auto t_huff = clk::now();
    std::vector<std::vector<StreamOut>> SO(nf);
    std::vector<std::vector<int32_t>> ranges(nf);
    for (u64 f = 0; f < nf; f++) {
        const u64 L = A[f].plan->pred.size();
        SO[f].resize(L + 2);  // index 0: t stream, 1..L+1: QB streams
        ranges[f].resize(2 * (L + 1));
        CK(cudaMemcpyAsync(ranges[f].data(), A[f].d_ranges, ranges[f].size() * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    u64 hist_total = 0;
    for (u64 f = 0; f < nf; f++) {
        const EncodeArgs &a = A[f];
        const u64 L = a.plan->pred.size();
        std::vector<StreamOut> &so = SO[f];
        so[0].count = a.G->nblocks * L;
        const float tv[6] = {t_default, 1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
        int64_t lo = INT64_MAX, hi = INT64_MIN;
        for (float t : tv) {
            int64_t c = host_lround_f(t * (float)a.p->t_precision);
            lo = std::min(lo, c);
            hi = std::max(hi, c);
        }
        for (u64 i = 0; a.t_given && i < a.t_len; i++) {
            lo = std::min(lo, a.t_given[i]);
            hi = std::max(hi, a.t_given[i]);
        }
        so[0].lo = lo;
        so[0].hi = hi;
        for (u64 s2 = 0; s2 <= L; s2++) {
            so[s2 + 1].count = (*a.qb_len)[s2];
            so[s2 + 1].lo = ranges[f][2 * s2];
            so[s2 + 1].hi = ranges[f][2 * s2 + 1];
            if (a.pre && s2 < a.pre->size() && (*a.pre)[s2].ok && so[s2 + 1].count) {
                const PreCode &pc = (*a.pre)[s2];
                so[s2 + 1].prebuilt = true;
                so[s2 + 1].lo = pc.lo;
                so[s2 + 1].hi = pc.hi;
                so[s2 + 1].code = pc.code;
            }
        }
        for (auto &o : so) {
            if (!o.count || o.prebuilt) continue;
            u64 range = (u64)(o.hi - o.lo) + 1;
            if (range > (1ull << 27)) return fail(ctx, ASZ_E_UNSUPPORTED, "QB range too wide for the dense histogram");
            o.hist_off = hist_total;
            hist_total += range;
        }
    }
    CK(ctx->hist.reserve(std::max<u64>(hist_total, 1) * 8));
    CK(cudaMemsetAsync(ctx->hist.p, 0, std::max<u64>(hist_total, 1) * 8, st));
    unsigned long long *d_hist = ctx->hist.as<unsigned long long>();
    for (u64 f = 0; f < nf; f++) {
        const EncodeArgs &a = A[f];
        const u64 L = a.plan->pred.size();
        std::vector<StreamOut> &so = SO[f];
        ProfScope ps_hist(ctx, "histogram", (a.G->nblocks * L) * 8 + a.N * 4);
        if (so[0].count)
            CK(launch_histogram<int64_t>(a.d_tint, so[0].count, so[0].lo, (u64)(so[0].hi - so[0].lo) + 1, d_hist + so[0].hist_off,
                                         st));
        for (u64 s2 = 0; s2 <= L; s2++)
            if (so[s2 + 1].count && !so[s2 + 1].prebuilt)
                CK(launch_histogram<int32_t>(a.d_qb + (*a.qb_off)[s2], (*a.qb_len)[s2], so[s2 + 1].lo,
                                             (u64)(so[s2 + 1].hi - so[s2 + 1].lo) + 1, d_hist + so[s2 + 1].hist_off, st));
    }
    std::optional<HostScope> hs_h(std::in_place, ctx, "host:codes_hist_d2h");
    std::vector<u64> hist(hist_total);
    if (hist_total) CK(cudaMemcpyAsync(hist.data(), d_hist, hist_total * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    hs_h.reset();
    std::optional<HostScope> hs_b(std::in_place, ctx, "host:codes_build");
    // Codes of all streams of all fields, on host threads.
    std::vector<std::pair<u64, u64>> jobs;
    for (u64 f = 0; f < nf; f++)
        for (u64 s2 = 0; s2 < SO[f].size(); s2++)
            if (SO[f][s2].count && !SO[f][s2].prebuilt) jobs.push_back({f, s2});
    std::vector<std::string> code_err(jobs.size());
    std::vector<char> code_ok(jobs.size(), 1);
    auto build_one = [&](u64 j) {
        StreamOut &o = SO[jobs[j].first][jobs[j].second];
        u64 range = (u64)(o.hi - o.lo) + 1;
        const u64 *h = hist.data() + o.hist_off;
        // Trim to the symbols present so the code's offset and range match the reference.
        u64 a0 = 0, b0 = range;
        while (a0 < b0 && h[a0] == 0) a0++;
        while (b0 > a0 && h[b0 - 1] == 0) b0--;
        std::vector<u64> hh(h + a0, h + b0);
        code_ok[j] = build_code(hh, o.lo + (int64_t)a0, o.lo + (int64_t)b0 - 1, o.count, jobs[j].second == 0, o.code,
                                code_err[j]);
        o.lo += (int64_t)a0;
    };
    // Waking the pool costs more than a few small builds (the t and pivot streams, when the
    // rounds' codes were built during the rounds), so those run here.
    u64 job_symbols = 0;
    for (auto &j : jobs) job_symbols += (u64)(SO[j.first][j.second].hi - SO[j.first][j.second].lo) + 1;
    if (jobs.size() > 2 && job_symbols > 4096) {
        if (!ctx->pool) ctx->pool = std::make_unique<HostPool>(std::min(15u, std::max(1u, std::thread::hardware_concurrency()) - 1));
        ctx->pool->run(jobs.size(), build_one);
    } else {
        for (u64 j = 0; j < jobs.size(); j++) build_one(j);
    }
    for (u64 j = 0; j < jobs.size(); j++)
        if (!code_ok[j]) return fail(ctx, ASZ_E_UNSUPPORTED, code_err[j]);
    u64 code_total = 0, words_total = 0, max_count = 0;
    std::vector<std::vector<u64>> code_off(nf);
    for (u64 f = 0; f < nf; f++) {
        code_off[f].assign(SO[f].size(), 0);
        for (u64 s2 = 0; s2 < SO[f].size(); s2++) {
            StreamOut &o = SO[f][s2];
            if (!o.count) continue;
            code_off[f][s2] = code_total;
            code_total += o.code.table.size();
            o.payload_word_off = words_total;
            words_total += (o.code.bits + 31) / 32 + 2;
            max_count = std::max(max_count, o.count);
        }
    }
    hs_b.reset();
    std::vector<CodeEntry> codes(std::max<u64>(code_total, 1));
    for (u64 f = 0; f < nf; f++)
        for (u64 s2 = 0; s2 < SO[f].size(); s2++)
            if (SO[f][s2].count)
                std::copy(SO[f][s2].code.table.begin(), SO[f][s2].code.table.end(), codes.begin() + code_off[f][s2]);
    CK(ctx->codes.reserve(codes.size() * sizeof(CodeEntry)));
    CK(cudaMemcpyAsync(ctx->codes.p, codes.data(), codes.size() * sizeof(CodeEntry), cudaMemcpyHostToDevice, st));
    CK(ctx->payload.reserve(std::max<u64>(words_total, 1) * 4));
    CK(cudaMemsetAsync(ctx->payload.p, 0, std::max<u64>(words_total, 1) * 4, st));
    uint32_t *d_pay = ctx->payload.as<uint32_t>();
    CodeEntry *d_codes = ctx->codes.as<CodeEntry>();
    hs_codes.reset();
    u64 enc_err[2] = {0, 0};  // the encoder's error words, read back with the sync below
    {
        // Every stream of every field in two launches, one per symbol type (the t streams are
        // int64, the QB streams int32).
        std::vector<EncStream> es[2];
        std::vector<u64> toff[2] = {{0}, {0}};
        u64 enc_bytes = 0;
        for (u64 f = 0; f < nf; f++) {
            const EncodeArgs &a = A[f];
            for (u64 s2 = 0; s2 < SO[f].size(); s2++) {
                StreamOut &o = SO[f][s2];
                if (!o.count || o.code.maxval == 1) continue;
                const int k = s2 == 0 ? 1 : 0;
                const void *sym = s2 == 0 ? (const void *)a.d_tint : (const void *)(a.d_qb + (*a.qb_off)[s2 - 1]);
                es[k].push_back(EncStream{sym, o.count, o.lo, d_codes + code_off[f][s2], d_pay + o.payload_word_off});
                const u64 tile = k ? enc_tile<int64_t>() : enc_tile<int32_t>();
                toff[k].push_back(toff[k].back() + (o.count + tile - 1) / tile);
                enc_bytes += o.count * (s2 == 0 ? 8 : 4) + (o.code.bits + 7) / 8;
            }
        }
        // Layout in ctx->enc: per type the stream records, the tile prefix, tile_bits, tile_scan.
        u64 off[2][4], bytes = 0;
        auto place = [&](u64 n) {
            const u64 o = bytes;
            bytes += (n + 15) / 16 * 16;
            return o;
        };
        size_t tmp_bytes = 0;
        for (int k = 0; k < 2; k++) {
            const u64 nt = toff[k].back();
            off[k][0] = place(es[k].size() * sizeof(EncStream));
            off[k][1] = place(toff[k].size() * sizeof(u64));
            off[k][2] = place((nt + 1) * sizeof(u64));
            off[k][3] = place((nt + 1) * sizeof(u64));
            size_t tb = 0;
            if (k == 0) CK(launch_encode_tiles<int32_t>(nullptr, 0, nullptr, nt, nullptr, nullptr, nullptr, tb, st));
            else CK(launch_encode_tiles<int64_t>(nullptr, 0, nullptr, nt, nullptr, nullptr, nullptr, tb, st));
            tmp_bytes = std::max(tmp_bytes, tb);
        }
        CK(ctx->enc.reserve(std::max<u64>(bytes, 16)));
        CK(ctx->cubtmp.reserve(std::max<size_t>(tmp_bytes, 16)));
        uint8_t *eb = ctx->enc.as<uint8_t>();
        ProfScope ps(ctx, "huff_encode", enc_bytes);
        for (int k = 0; k < 2; k++) {
            const u64 nt = toff[k].back();
            if (!nt) continue;
            CK(cudaMemcpyAsync(eb + off[k][0], es[k].data(), es[k].size() * sizeof(EncStream), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(eb + off[k][1], toff[k].data(), toff[k].size() * sizeof(u64), cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(eb + off[k][2] + nt * sizeof(u64), 0, sizeof(u64), st));  // the scan's total
            size_t tb = ctx->cubtmp.cap;
            const EncStream *E = (const EncStream *)(eb + off[k][0]);
            const u64 *T = (const u64 *)(eb + off[k][1]);
            u64 *tbits = (u64 *)(eb + off[k][2]), *tscan = (u64 *)(eb + off[k][3]);
            if (k == 0) CK(launch_encode_tiles<int32_t>(E, (uint32_t)es[k].size(), T, nt, tbits, tscan, ctx->cubtmp.p, tb, st));
            else CK(launch_encode_tiles<int64_t>(E, (uint32_t)es[k].size(), T, nt, tbits, tscan, ctx->cubtmp.p, tb, st));
            CK(cudaMemcpyAsync(&enc_err[k], tscan, sizeof(u64), cudaMemcpyDeviceToHost, st));
        }
    }
    // Stream assembly (compress.tpp:233-291) in pinned memory: the host writes the headers and
    // code trees while each payload is copied from the device straight into its place.
    span.assign(nf, {0, 0});
    u64 all_len = 0;
    for (u64 f = 0; f < nf; f++) {
        const u64 L = A[f].plan->pred.size();
        u64 total_len = 9 + 2 * L;
        for (auto &o : SO[f]) total_len += 8 + (o.count ? o.code.save_size() + o.code.encode_size() : 0);
        span[f] = {all_len, total_len};
        all_len += total_len;
    }
    CK(pb.reserve(all_len));
    pb.len = all_len;
    // The encoding launches finish before the copy timer starts, so that d2h_s holds the copies
    // (and the host's header writing between them) and none of the kernels' time.
    CK(cudaStreamSynchronize(st));
    if (enc_err[0] | enc_err[1]) return fail(ctx, ASZ_E_DEVICE, "Huffman encoder: a tile's wait for the tiles before it timed out");
    auto t_d2h = clk::now();
    {
        HostScope hs(ctx, "host:assembly");
        for (u64 f = 0; f < nf; f++) {
            const EncodeArgs &a = A[f];
            const Plan &plan = *a.plan;
            const u64 L = plan.pred.size();
            uint8_t *const bs0 = pb.p + span[f].first;
            uint8_t *w = bs0;
            std::memcpy(w, &a.mn, 4);
            std::memcpy(w + 4, &a.mx, 4);
            w[8] = (uint8_t)(L | 0x40 | (a.quintic ? 0x80 : 0));
            w += 9;
            for (u64 l = 0; l < L; l++) {
                w[0] = (uint8_t)plan.pred[l][5];
                w[1] = (uint8_t)plan.pred[l][9];
                w += 2;
            }
            for (const StreamOut &o : SO[f]) {
                for (int i = 0; i < 8; i++) w[i] = (uint8_t)(o.count >> (8 * i));
                w += 8;
                if (!o.count) continue;
                write_tree(o.code, w);
                w += o.code.save_size();
                write_len_word(o.code, w);
                w += 8;
                if (o.code.maxval != 1) {
                    u64 nb = (o.code.bits + 7) >> 3;
                    if (nb) CK(cudaMemcpyAsync(w, d_pay + o.payload_word_off, nb, cudaMemcpyDeviceToHost, st));
                    w += nb;
                }
            }
            if ((u64)(w - bs0) != span[f].second) return fail(ctx, ASZ_E_DEVICE, "Huffman encoded size mismatch");
        }
        CK(cudaStreamSynchronize(st));
    }
    const double d2h = secs(t_d2h, clk::now()), huff = secs(t_huff, clk::now());
    for (asz_report *r : Rs)
        if (r) {
            r->d2h_s = d2h;
            r->huffman_s = huff;
        }
    return ASZ_OK;
}

static int compress_entry(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                          const asz_params *pp, const char *plan_text, const int64_t *t_given, uint64_t t_len, uint8_t **out,
                          size_t *out_len, asz_report *rep) {
    if (!ctx) return ASZ_E_ARG;
    auto t_start = clk::now();
    const uint64_t launches0 = launch_counter();
    ctx->err.clear();
    ctx->have_last = false;
    if (!in || !out || !out_len) return fail(ctx, ASZ_E_ARG, "null argument");
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    int rc = validate(ctx, p, true);
    if (rc) return rc;
    rc = validate_dims(ctx, dims, rel_eb);
    if (rc) return rc;
    Plan plan;
    std::string perr;
    if (plan_text) {
        if (!parse_plan(plan_text, plan, perr)) return fail(ctx, ASZ_E_ARG, perr);
        if (plan.pred.size() > 63) return fail(ctx, ASZ_E_ARG, "predictor plan cannot contain more than 63 layers");
    }
    bool quintic = p.predictor_family == ASZ_FAMILY_QUINTIC;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, ASZ_E_CUDA, "cudaSetDevice");
    const u64 N = dims[0] * dims[1] * dims[2];
    
    cudaStream_t st = ctx->stream;
    asz_report R{};

    CK(ctx->misc.reserve(sizeof(MiscLayout)));
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    // Input.
    const float *d_in = in;
    auto t0 = clk::now();
    if (!in_on_device) {
        CK(ctx->in.reserve(N * sizeof(float)));
        CK(cudaMemcpyAsync(ctx->in.p, in, N * sizeof(float), cudaMemcpyHostToDevice, st));
        d_in = ctx->in.as<float>();
    }
    CK(cudaStreamSynchronize(st));
    R.h2d_s = secs(t0, clk::now());
    // Data range (s1_compress.cpp:131-138).
    auto t_range = clk::now();
    float mn, mx;
    {
        HostScope hs(ctx, "host:range");
        rc = compute_range(ctx, d_in, N, mn, mx);
    }
    if (rc) return rc;
    R.data_range_s = secs(t_range, clk::now());
    if (mn == mx) return fail(ctx, ASZ_E_DATA, "max_val==min_val");
    const float abs_eb = rel_eb * (mx - mn);
    // Default slope.
    auto t_slope = clk::now();
    const std::vector<float> cand = candidate_t(p);
    float slope, max_invalid = 0;
    int reason = 0;
    {
        HostScope hs(ctx, "host:slope");
        rc = default_slope(ctx, d_in, dims, p, abs_eb, mn, mx, cand, slope, max_invalid, reason);
    }
    if (rc) return rc;
    R.default_slope_s = secs(t_slope, clk::now());
    if (!plan_text) {
        // Plan search (s1_compress.cpp:30-47 with no --predictor-plan).
        auto t_plan = clk::now();
        PlanSearchOut ps;
        {
            HostScope hs(ctx, "host:plan_search");
            rc = plan_search(ctx, d_in, dims, p, abs_eb, mn, mx, slope, ps);
        }
        if (rc) return rc;
        R.plan_s = secs(t_plan, clk::now());
        R.plan_stats_s = ps.stats_s;
        R.plan_sample_s = ps.sample_s;
        R.plan_lossless_s = ps.lossless_s;
        R.plan_search_layers = (uint32_t)std::min<size_t>(ps.dists.size(), 64);
        for (uint32_t i = 0; i < R.plan_search_layers; i++) R.plan_best_dist[i] = ps.dists[i];
        if (ps.plan.empty()) return fail(ctx, ASZ_E_DATA, "plan search found no layer");
        std::string txt;
        for (size_t i = 0; i < ps.plan.size(); i++) txt += (i ? "," : "") + ps.plan[i];
        if (!parse_plan(txt.c_str(), plan, perr)) return fail(ctx, ASZ_E_DEVICE, perr);
        if (plan.pred.size() > 63) return fail(ctx, ASZ_E_ARG, "predictor plan cannot contain more than 63 layers");
    }
    const u64 L = plan.pred.size();
    if (p.predictor_family == ASZ_FAMILY_AUTO) {
        // prepare_compression_plan (s1_compress.cpp:41-42): the family selector runs after the plan.
        auto t_fam = clk::now();
        {
            HostScope hs(ctx, "host:family_selection");
            rc = select_family(ctx, d_in, dims, p, rel_eb, abs_eb, mn, mx, slope, plan, quintic, R);
        }
        if (rc) return rc;
        R.family_s = secs(t_fam, clk::now());
    }

    auto t_core = clk::now();
    CoreOut co;
    {
        CoreArgs ca{d_in, dims, nullptr, &plan, &p, quintic, false, nullptr, mn, mx, abs_eb, slope, t_given, t_len};
        ca.prebuild = true;
        rc = run_core(ctx, ca, co, R);
        if (rc) return rc;
    }
    Geometry &G = co.G;
    std::vector<u64> &qb_off = co.qb_off, &qb_len = co.qb_len;
    {
        const std::vector<EncodeArgs> ea{EncodeArgs{&G, &qb_off, &qb_len, ctx->qb.as<int32_t>(), ctx->tint.as<int64_t>(),
                                                    dm->qb_range, mn, mx, quintic, &plan, &p, t_given, t_len, N, &co.pre}};
        std::vector<asz_report *> rs{&R};
        std::vector<std::pair<u64, u64>> span;
        rc = encode_fields(ctx, ea, rs, span, ctx->pre_zstd);
        if (rc) return rc;
    }
    PinnedBuf &pb = ctx->pre_zstd;
    R.core_s = secs(t_core, clk::now());
    // zstd level 3 (compress.tpp:294-299).
    auto t_z = clk::now();
    HostScope hs_z(ctx, "host:zstd");
    size_t bound = ZSTD_compressBound(pb.len);
    uint8_t *z = out_alloc(bound);
    if (!z) return fail(ctx, ASZ_E_DATA, "out of host memory");
    size_t zl = zstd3(ctx, z, bound, pb.p, pb.len);
    if (ZSTD_isError(zl)) {
        out_release(z);
        return fail(ctx, ASZ_E_DATA, std::string("ZSTD_compress: ") + ZSTD_getErrorName(zl));
    }
    R.zstd_s = secs(t_z, clk::now());
    *out = z;
    *out_len = zl;
    // Report.
    ctx->qb_off = qb_off;
    ctx->qb_len = qb_len;
    ctx->t_len = G.nblocks * L;
    ctx->n_total = N;
    ctx->last_in = d_in;
    ctx->last_min = mn;
    ctx->last_max = mx;
    ctx->have_last = true;
    if (rep) {
        R.min_val = mn;
        R.max_val = mx;
        R.abs_eb = abs_eb;
        R.default_slope = slope;
        R.slope_max_invalid_ratio = max_invalid;
        R.slope_fallback_reason = reason;
        R.pre_zstd_len = pb.len;
        R.asz_len = zl;
        R.layer_num = L;
        R.quintic = quintic ? 1 : 0;
        for (int a = 0; a < 3; a++) {
            R.pivot_stride[a] = (uint32_t)G.fg.pivot_stride[a];
            R.block_shape[a] = (uint32_t)G.fg.block_shape[a];
            R.block_num[a] = (uint32_t)G.fg.block_num[a];
        }
        std::string pl;
        for (u64 l = 0; l < L; l++) pl += (l ? "," : "") + plan.pred[l];
        std::snprintf(R.plan, sizeof(R.plan), "%s", pl.c_str());
        R.cr = (float)N * sizeof(float) / (float)zl;
        R.br = 8 * sizeof(float) / R.cr;
        R.kernel_launches = launch_counter() - launches0;
        R.total_s = secs(t_start, clk::now());
        *rep = R;
    }
    return ASZ_OK;
}

extern "C" int asz_compress(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                            const asz_params *pp, const char *plan_text, uint8_t **out, size_t *out_len, asz_report *rep) {
    return compress_entry(ctx, in, in_on_device, dims, rel_eb, pp, plan_text, nullptr, 0, out, out_len, rep);
}

extern "C" int asz_compress_with_t(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                                   const asz_params *pp, const char *plan_text, const int64_t *t_int, uint64_t t_len,
                                   uint8_t **out, size_t *out_len, asz_report *rep) {
    if (!ctx) return ASZ_E_ARG;
    ctx->err.clear();
    if (!plan_text || !t_int) return fail(ctx, ASZ_E_ARG, "a t table needs a plan and the table");
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    if (p.predictor_family == ASZ_FAMILY_AUTO) return fail(ctx, ASZ_E_ARG, "a t table needs a fixed predictor family");
    // Codes on the t grid within [t_min, t_max] (s1_compress.cpp:92-98 bound the range).
    const int64_t lo = (int64_t)std::llround((double)p.t_min * p.t_precision);
    const int64_t hi = (int64_t)std::llround((double)p.t_max * p.t_precision);
    for (uint64_t i = 0; i < t_len; i++)
        if (t_int[i] < lo || t_int[i] > hi) return fail(ctx, ASZ_E_ARG, "t code outside [t_min, t_max] at index " + std::to_string(i));
    return compress_entry(ctx, in, in_on_device, dims, rel_eb, &p, plan_text, t_int, t_len, out, out_len, rep);
}

// ---------------------------------------------------------------------------------------------
// Gradient tuner problem: the open-loop AB samples of every (block, round) group (k_grad.cu).

extern "C" int asz_grad_setup(asz_ctx *ctx, const float *in, int in_on_device, const uint64_t dims[3], float rel_eb,
                              const asz_params *pp, const char *plan_text, asz_grad_problem *out) {
    if (!ctx) return ASZ_E_ARG;
    ctx->err.clear();
    if (!in || !plan_text || !out) return fail(ctx, ASZ_E_ARG, "null argument");
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    int rc = validate(ctx, p, true);
    if (rc) return rc;
    rc = validate_dims(ctx, dims, rel_eb);
    if (rc) return rc;
    Plan plan;
    std::string perr;
    if (!parse_plan(plan_text, plan, perr)) return fail(ctx, ASZ_E_ARG, perr);
    if (plan.pred.size() > 63) return fail(ctx, ASZ_E_ARG, "predictor plan cannot contain more than 63 layers");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, ASZ_E_CUDA, "cudaSetDevice");
    const u64 N = dims[0] * dims[1] * dims[2];
    cudaStream_t st = ctx->stream;
    CK(ctx->misc.reserve(sizeof(MiscLayout)));
    const float *d_in = in;
    if (!in_on_device) {
        CK(ctx->in.reserve(N * sizeof(float)));
        CK(cudaMemcpyAsync(ctx->in.p, in, N * sizeof(float), cudaMemcpyHostToDevice, st));
        d_in = ctx->in.as<float>();
    }
    float mn, mx;
    rc = compute_range(ctx, d_in, N, mn, mx);
    if (rc) return rc;
    if (mn == mx) return fail(ctx, ASZ_E_DATA, "max_val==min_val");
    const float abs_eb = rel_eb * (mx - mn);
    const std::vector<float> cand = candidate_t(p);
    float slope, max_invalid = 0;
    int reason = 0;
    rc = default_slope(ctx, d_in, dims, p, abs_eb, mn, mx, cand, slope, max_invalid, reason);
    if (rc) return rc;
    Geometry &G = ctx->grad_G;
    build_geometry(dims, plan, p, abs_eb, slope, p.predictor_family == ASZ_FAMILY_QUINTIC, G);
    if (!kernel_limits_ok(G)) return fail(ctx, ASZ_E_UNSUPPORTED, "field too large for 32-bit line indexing");
    const u64 L = plan.pred.size(), groups = G.nblocks * L;
    ctx->grad_off.assign(groups + 1, 0);
    ctx->grad_meta.assign(groups * 4, 0.0f);
    u64 acc = 0;
    const FieldGeom &fg = G.fg;
    auto cls_of = [](u64 b, u64 nb) { return b == 0 ? 0 : (b == nb - 1 ? 2 : 1); };
    for (u64 g = 0; g < G.nblocks; g++) {
        const u64 b2 = g % fg.block_num[2], b1 = (g / fg.block_num[2]) % fg.block_num[1], b0 = g / (fg.block_num[1] * fg.block_num[2]);
        const int c = (cls_of(b0, fg.block_num[0]) * 3 + cls_of(b1, fg.block_num[1])) * 3 + cls_of(b2, fg.block_num[2]);
        for (u64 l = 0; l < L; l++) {
            const u64 gid = g * L + l;
            const ClassInfo &ci = G.classes[l][c];
            ctx->grad_off[gid] = (uint32_t)acc;
            acc += ci.fallback ? 0 : ci.n;
            if (acc > 0xffffffffull) return fail(ctx, ASZ_E_UNSUPPORTED, "more than 2^32 - 1 tuner samples");
            const RoundGeom &rg = G.rounds[l];
            float *m = &ctx->grad_meta[gid * 4];
            m[0] = rg.eb;
            m[1] = rg.stat_eb;
            m[2] = rg.neg_2_stat_eb;
            m[3] = rg.slope;
        }
    }
    ctx->grad_off[groups] = (uint32_t)acc;
    ctx->grad_in = d_in;
    asz_grad_problem P{};
    P.groups = groups;
    P.samples = acc;
    P.blocks = G.nblocks;
    P.layers = L;
    P.R2 = (mx - mn) * (mx - mn);
    P.abs_eb = abs_eb;
    P.default_slope = slope;
    P.t_min = p.t_min;
    P.t_max = p.t_max;
    P.t_precision = p.t_precision;
    *out = P;
    return ASZ_OK;
}

extern "C" int asz_grad_gather(asz_ctx *ctx, float *A, float *B, uint32_t *offsets, float *meta) {
    if (!ctx) return ASZ_E_ARG;
    ctx->err.clear();
    if (!ctx->grad_in || ctx->grad_off.empty()) return fail(ctx, ASZ_E_ARG, "asz_grad_setup has not run");
    if (!A || !B || !offsets || !meta) return fail(ctx, ASZ_E_ARG, "null argument");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, ASZ_E_CUDA, "cudaSetDevice");
    const Geometry &G = ctx->grad_G;
    const u64 L = G.rounds.size(), groups = G.nblocks * L;
    cudaStream_t st = ctx->stream;
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    CK(cudaMemcpyAsync(offsets, ctx->grad_off.data(), (groups + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(meta, ctx->grad_meta.data(), groups * 4 * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(ctx->rounds_dev.reserve(L * sizeof(RoundGeom)));
    CK(cudaMemcpyAsync(ctx->rounds_dev.p, G.rounds.data(), L * sizeof(RoundGeom), cudaMemcpyHostToDevice, st));
    std::vector<ClassInfo> cls_flat;
    for (u64 l = 0; l < L; l++) cls_flat.insert(cls_flat.end(), G.classes[l].begin(), G.classes[l].end());
    CK(ctx->classes.reserve(cls_flat.size() * sizeof(ClassInfo)));
    CK(cudaMemcpyAsync(ctx->classes.p, cls_flat.data(), cls_flat.size() * sizeof(ClassInfo), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(&dm->err, 0, 4, st));
    {
        ProfScope ps(ctx, "grad_gather", (u64)ctx->grad_off[groups] * 28);
        CK(launch_grad_gather(G.fg, ctx->rounds_dev.as<RoundGeom>(), ctx->classes.as<ClassInfo>(), ctx->grad_in, offsets, groups,
                              A, B, &dm->err, st));
    }
    uint32_t errw = 0;
    CK(cudaMemcpyAsync(&errw, &dm->err, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (errw) return fail(ctx, ASZ_E_DEVICE, "tuner sample lattice does not match the class sample counts");
    return ASZ_OK;
}

// ---------------------------------------------------------------------------------------------
// Decompression.

namespace {

// Zero bytes after the stream for the decoder's read-ahead.
constexpr u64 kDecodePad = 64;

// One stream to decode: its parsed code, the values it must produce and where they go.
struct DecodeJob {
    const HuffParsed *hp;
    u64 count;
    void *out;
    bool wide;
};

// Decode every stream of a .asz in one batched launch per pass (k_huff.cu). The stream bytes are
// on the device at d_base (256-byte aligned, padded by kDecodePad). Errors of the payloads are
// left in dm->dec_err for the caller to read with its final synchronisation.
int gpu_decode_all(asz_ctx *ctx, const std::vector<DecodeJob> &jobs, const uint8_t *d_base, MiscLayout *dm, cudaStream_t st) {
    const u64 C = 1024;  // chunk bits
    std::vector<DecStream> ds;
    std::vector<uint32_t> tile_stream;
    std::vector<LutEntry> luts;
    std::vector<uint32_t> childs;
    u64 nchunks = 0;
    uint32_t max_lut_bits = 1;
    for (const DecodeJob &j : jobs) {
        const HuffParsed &hp = *j.hp;
        if (!j.count) continue;
        if (hp.single) {
            if (hp.single_count != j.count) return fail(ctx, ASZ_E_DATA, "Huffman payload length does not match its value count");
            if (j.wide) CK(launch_fill<int64_t>((int64_t *)j.out, j.count, (int64_t)hp.offset, st));
            else CK(launch_fill<int32_t>((int32_t *)j.out, j.count, (int32_t)hp.offset, st));
            continue;
        }
        DecStream d{};
        d.bit_begin = hp.payload_off * 8;
        d.bit_end = d.bit_begin + hp.payload_bits;
        d.chunk0 = nchunks;
        d.nchunks = std::max<u64>(1, (hp.payload_bits + C - 1) / C);
        d.tile0 = tile_stream.size();
        d.lut_off = luts.size();
        d.child_off = childs.size();
        d.count = j.count;
        d.offset = hp.offset;
        d.out = j.out;
        d.lut_bits = hp.lut_bits;
        d.wide = j.wide ? 1 : 0;
        luts.insert(luts.end(), hp.lut.begin(), hp.lut.end());
        childs.insert(childs.end(), hp.child.begin(), hp.child.end());
        const u64 tiles = (d.nchunks + kDecodeTile - 1) / kDecodeTile;
        tile_stream.insert(tile_stream.end(), tiles, (uint32_t)ds.size());
        nchunks += d.nchunks;
        max_lut_bits = std::max(max_lut_bits, hp.lut_bits);
        ds.push_back(d);
    }
    CK(cudaMemsetAsync(&dm->dec_err, 0, 4, st));
    if (ds.empty()) return ASZ_OK;
    if (childs.empty()) childs.push_back(0);
    // Tables and descriptors in one upload.
    const u64 ds_bytes = ds.size() * sizeof(DecStream), ts_bytes = tile_stream.size() * 4, lut_bytes = luts.size() * sizeof(LutEntry),
              ch_bytes = childs.size() * 4;
    auto al = [](u64 x) { return (x + 255) & ~255ull; };
    const u64 o_ts = al(ds_bytes), o_lut = o_ts + al(ts_bytes), o_ch = o_lut + al(lut_bytes), total = o_ch + al(ch_bytes);
    std::vector<uint8_t> blob(total);
    std::memcpy(blob.data(), ds.data(), ds_bytes);
    std::memcpy(blob.data() + o_ts, tile_stream.data(), ts_bytes);
    std::memcpy(blob.data() + o_lut, luts.data(), lut_bytes);
    std::memcpy(blob.data() + o_ch, childs.data(), ch_bytes);
    CK(ctx->codes.reserve(total));
    uint8_t *dc = ctx->codes.as<uint8_t>();
    CK(cudaMemcpyAsync(dc, blob.data(), total, cudaMemcpyHostToDevice, st));
    const DecStream *d_ds = (const DecStream *)dc;
    const uint32_t *d_ts = (const uint32_t *)(dc + o_ts);
    const LutEntry *d_lut = (const LutEntry *)(dc + o_lut);
    const uint32_t *d_ch = (const uint32_t *)(dc + o_ch);
    // Per-chunk arrays: start, end, count, off (count + 1 entries for the scan), moved (u32).
    CK(ctx->chunks.reserve(4 * (nchunks + 1) * 8 + (nchunks + 1) * 4 + 64));
    u64 *d_start = ctx->chunks.as<u64>(), *d_end = d_start + nchunks + 1, *d_cnt = d_end + nchunks + 1, *d_off = d_cnt + nchunks + 1;
    uint32_t *d_moved = reinterpret_cast<uint32_t *>(d_off + nchunks + 1);
    CK(cudaMemsetAsync(d_cnt + nchunks, 0, 8, st));
    const uint32_t nst = (uint32_t)ds.size();
    const u64 ntiles = tile_stream.size();
    for (u64 it = 0;; it++) {
        {
            ProfScope ps(ctx, "huff_decode_sync", 0);
            CK(launch_decode_sync(d_base, C, d_ds, d_ts, ntiles, max_lut_bits, d_lut, d_ch, it == 0 ? 1 : 0, d_start, d_end, d_cnt,
                                  d_moved, &dm->dec_err, st));
        }
        CK(cudaMemsetAsync(&dm->dec_changed, 0, 4, st));
        CK(launch_decode_restart(d_ds, nst, nchunks, d_end, d_start, d_moved, &dm->dec_changed, st));
        uint32_t changed;
        CK(cudaMemcpyAsync(&changed, &dm->dec_changed, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (!changed) break;
        // Every pass that moves a start fixes at least one more chunk, so this ends.
        if (it > nchunks + 2) return fail(ctx, ASZ_E_DATA, "Huffman payload does not synchronise");
    }
    size_t tb = 0;
    CK(launch_scan_u64(d_cnt, d_off, nchunks + 1, nullptr, tb, st));
    CK(ctx->cubtmp.reserve(tb));
    tb = ctx->cubtmp.cap;
    CK(launch_scan_u64(d_cnt, d_off, nchunks + 1, ctx->cubtmp.p, tb, st));
    CK(launch_decode_check(d_ds, nst, d_off, d_end, &dm->dec_err, st));
    ProfScope ps_w(ctx, "huff_decode_write", 0);
    CK(launch_decode_write(d_base, C, d_ds, d_ts, ntiles, max_lut_bits, d_lut, d_ch, d_start, d_off, &dm->dec_err, st));
    return ASZ_OK;
}

}  // namespace

extern "C" int asz_decompress(asz_ctx *ctx, const uint8_t *in, size_t len, const uint64_t dims[3], float rel_eb,
                              const asz_params *pp, float *out, int out_on_device, asz_report *rep) {
    if (!ctx) return ASZ_E_ARG;
    auto t_start = clk::now();
    const uint64_t launches0 = launch_counter();
    ctx->err.clear();
    if (!in || !out) return fail(ctx, ASZ_E_ARG, "null argument");
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    int rc = validate(ctx, p, false);
    if (rc) return rc;
    rc = validate_dims(ctx, dims, rel_eb);
    if (rc) return rc;
    if (len == 0) return fail(ctx, ASZ_E_DATA, "compressed input is empty");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, ASZ_E_CUDA, "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    asz_report R{};
    // zstd (decompress.tpp:83-86).
    auto t_z = clk::now();
    unsigned long long raw = ZSTD_getFrameContentSize(in, len);
    if (raw == ZSTD_CONTENTSIZE_ERROR || raw == ZSTD_CONTENTSIZE_UNKNOWN || raw > (1ull << 40))
        return fail(ctx, ASZ_E_DATA, "ZSTD_decompress error in decompress()");
    CK(ctx->raw_in.reserve(raw + kDecodePad));
    uint8_t *const bsp = ctx->raw_in.p;
    std::memset(bsp + raw, 0, kDecodePad);
    size_t got;
    {
        HostScope hs(ctx, "host:zstd");
        if (!ctx->zd) ctx->zd = ZSTD_createDCtx();
        got = ctx->zd ? ZSTD_decompressDCtx(ctx->zd, bsp, raw, in, len) : ZSTD_decompress(bsp, raw, in, len);
    }
    if (ZSTD_isError(got) || got != raw) return fail(ctx, ASZ_E_DATA, "ZSTD_decompress error in decompress()");
    R.zstd_s = secs(t_z, clk::now());
    auto t_h = clk::now();
    // Header (decompress.tpp:89-119).
    if (raw < 9) return fail(ctx, ASZ_E_DATA, "truncated header");
    float mn, mx;
    std::memcpy(&mn, bsp, 4);
    std::memcpy(&mx, bsp + 4, 4);
    uint8_t flags = bsp[8];
    u64 L = flags;
    bool quintic = p.predictor_family == ASZ_FAMILY_QUINTIC;
    if (flags & 0x40) {
        quintic = (flags & 0x80) != 0;
        L = flags & 0x3f;
    }
    u64 pos = 9;
    if (raw - pos < 2 * L) return fail(ctx, ASZ_E_DATA, "truncated header");
    std::string ptxt;
    for (u64 l = 0; l < L; l++) {
        uint8_t a = bsp[pos], o = bsp[pos + 1];
        if (a < '0' || a > '2' || o < '0' || o > '2') return fail(ctx, ASZ_E_DATA, "compressed stream contains an invalid predictor");
        ptxt += (l ? "," : "") + std::string("cubic") + (char)a + "_" + (o == '0' ? "120" : o == '1' ? "021" : "012");
        pos += 2;
    }
    Plan plan;
    std::string perr;
    if (L == 0 || !parse_plan(ptxt.c_str(), plan, perr)) return fail(ctx, ASZ_E_DATA, "compressed stream contains no rounds");
    auto rd64 = [&](u64 &v) {
        if (raw - pos < 8) return false;
        v = 0;
        for (int i = 0; i < 8; i++) v |= (u64)bsp[pos + i] << (8 * i);
        pos += 8;
        return true;
    };
    std::vector<HuffParsed> hp(L + 2);
    std::vector<u64> counts(L + 2), sbeg(L + 2, 0), send(L + 2, 0);
    // Stream boundaries from the headers alone: a tree takes n (mbft + 2) - 1 bits and a payload
    // the bits its length word gives (none for a single symbol), so every stream's start is known
    // before any tree is read (huffman.hpp:322-338).
    auto be64 = [&](u64 at) {
        u64 v = 0;
        for (int i = 0; i < 8; i++) v = (v << 8) | bsp[at + i];
        return v;
    };
    for (u64 s = 0; s < L + 2; s++) {
        if (!rd64(counts[s])) return fail(ctx, ASZ_E_DATA, "truncated stream length");
        if (!counts[s]) continue;
        if (pos > raw || raw - pos < 25) return fail(ctx, ASZ_E_DATA, "truncated Huffman header");
        const unsigned mbft = bsp[pos] & 0x3f;
        const u64 n = be64(pos + 9), maxval = be64(pos + 17);
        if (n == 0) return fail(ctx, ASZ_E_DATA, "Huffman stream with no symbols");
        if (n > 1 && (mbft == 0 || mbft > 63 || n > (1ull << 31))) return fail(ctx, ASZ_E_DATA, "corrupt Huffman tree header");
        const u64 tree = n > 1 ? (n * (mbft + 2) - 1 + 7) / 8 : 0;
        sbeg[s] = pos;
        if (raw - pos - 25 < tree + 8) return fail(ctx, ASZ_E_DATA, "truncated Huffman payload");
        u64 q = pos + 25 + tree;
        const u64 w = be64(q) ^ 0x1234abcdull;
        q += 8;
        if (n > 1 && maxval != 1) {
            if (w > (raw - q) * 8) return fail(ctx, ASZ_E_DATA, "truncated Huffman payload");
            q += (w + 7) / 8;
        }
        send[s] = pos = q;
    }
    // Trees and lookup tables on the context's worker threads; each stream must end where the
    // next one starts.
    {
        std::vector<std::string> perr(L + 2);
        std::vector<char> pok(L + 2, 1);
        auto parse_one = [&](uint64_t s) {
            if (!counts[s]) return;
            u64 at = sbeg[s];
            pok[s] = parse_stream(bsp, raw, at, hp[s], perr[s]) && at == send[s];
            if (!pok[s] && perr[s].empty()) perr[s] = "corrupt Huffman stream";
        };
        if (!ctx->pool) ctx->pool = std::make_unique<HostPool>(std::min(15u, std::max(1u, std::thread::hardware_concurrency()) - 1));
        ctx->pool->run(L + 2, parse_one);
        for (u64 s = 0; s < L + 2; s++) {
            if (!pok[s]) return fail(ctx, ASZ_E_DATA, perr[s]);
            // Every code is at least one bit, and a single-symbol stream still has to fit the
            // field's bookkeeping: larger counts are corrupt (and would overflow the output sizing).
            if (counts[s] && (hp[s].single ? counts[s] > (1ull << 40) : counts[s] > hp[s].payload_bits))
                return fail(ctx, ASZ_E_DATA, "compressed stream has an impossible value count");
        }
    }
    const float abs_eb = rel_eb * (mx - mn);
    Geometry G;
    build_geometry(dims, plan, p, abs_eb, 0.0f, quintic, G);
    if (!kernel_limits_ok(G)) return fail(ctx, ASZ_E_UNSUPPORTED, "field too large for the round kernels' 32-bit line indexing");
    const u64 N = dims[0] * dims[1] * dims[2];
    if (counts[0] < G.nblocks * L) return fail(ctx, ASZ_E_DATA, "compressed stream contains too few t values");
    if (counts[1] < G.pivots) return fail(ctx, ASZ_E_DATA, "compressed stream has too few QBs");
    for (u64 l = 0; l < L; l++)
        if (counts[l + 2] < G.rounds[l].qb_total) return fail(ctx, ASZ_E_DATA, "compressed stream has too few QBs");
    // Device: stream bytes, t codes, QB streams.
    CK(ctx->misc.reserve(sizeof(MiscLayout)));
    CK(ctx->pre.reserve(raw + kDecodePad));
    // The copy is waited for inside its timer, so h2d_s holds the transfer itself.
    auto t0 = clk::now();
    CK(cudaMemcpyAsync(ctx->pre.p, bsp, raw + kDecodePad, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    R.h2d_s += secs(t0, clk::now());
    std::vector<u64> qoff(L + 1);
    u64 qtot = 0;
    for (u64 s = 0; s <= L; s++) {
        qoff[s] = qtot;
        qtot += counts[s + 1];
    }
    CK(ctx->tint.reserve(std::max<u64>(counts[0], 1) * 8));
    CK(ctx->qb.reserve(std::max<u64>(qtot, 1) * 4));
    std::optional<HostScope> hs_dec(std::in_place, ctx, "host:huffman_decode");
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    {
        std::vector<DecodeJob> jobs;
        jobs.push_back({&hp[0], counts[0], ctx->tint.p, true});
        for (u64 s = 0; s <= L; s++) jobs.push_back({&hp[s + 1], counts[s + 1], ctx->qb.as<int32_t>() + qoff[s], false});
        rc = gpu_decode_all(ctx, jobs, ctx->pre.as<uint8_t>(), dm, st);
        if (rc) return rc;
    }
    hs_dec.reset();
    R.huffman_s = secs(t_h, clk::now());
    // Reconstruction.
    auto t_core = clk::now();
    std::optional<HostScope> hs_rec(std::in_place, ctx, "host:reconstruct");
    float *d_out = out;
    if (!out_on_device) {
        CK(ctx->rec.reserve(N * sizeof(float)));
        d_out = ctx->rec.as<float>();
    }
    CK(ctx->axis.reserve(std::max<size_t>(G.ent.size(), 1) * sizeof(AxisEntry)));
    const AxisEntry *d_ent = ctx->axis.as<AxisEntry>();
    CK(cudaMemcpyAsync(ctx->axis.p, G.ent.data(), G.ent.size() * sizeof(AxisEntry), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(&dm->err, 0, 4, st));
    {
        ProfScope ps(ctx, "pivot_decompress", G.pivots * 8);
        CK(launch_pivot_decompress(G.pg, ctx->qb.as<int32_t>() + qoff[0], d_out, st));
    }
    if (const uint32_t line_bytes = ctx->tsel_mode == 2 ? lines_smem_bytes(G) : 0) {
        // Every round along axis 2: all rounds fused per column of lines (k_lines.cu).
        const u64 rbytes = L * sizeof(RoundGeom);
        CK(ctx->rounds_dev.reserve(rbytes + (L + 1) * sizeof(u64)));
        uint8_t *rd = ctx->rounds_dev.as<uint8_t>();
        CK(cudaMemcpyAsync(rd, G.rounds.data(), rbytes, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(rd + rbytes, qoff.data(), (L + 1) * sizeof(u64), cudaMemcpyHostToDevice, st));
        u64 tgt = 0;
        for (u64 l = 0; l < L; l++) tgt += G.rounds[l].targets;
        // Algorithmic bytes: the field loaded and stored once, one QB read per target.
        ProfScope ps(ctx, "lines_decompress", N * 8 + tgt * 4);
        for (const LinesLaunch &ll : lines_launches(G, line_bytes))
            CK(launch_lines_decompress(G.fg, (const RoundGeom *)rd, d_ent, (const u64 *)(rd + rbytes),
                                       ctx->tint.as<int64_t>(), ctx->qb.as<int32_t>(), d_out, &dm->err, ll.set, ll.bytes, st));
    } else {
        for (u64 l = 0; l < L; l++) {
            ProfScope ps(ctx, "round_decompress", G.rounds[l].targets * 8);
            CK(launch_round_decompress(G.fg, G.rounds[l], (uint32_t)l, d_ent, ctx->tint.as<int64_t>(),
                                       ctx->qb.as<int32_t>() + qoff[l + 1], d_out, &dm->err, st));
        }
    }
    uint32_t errw, decw;
    CK(cudaMemcpyAsync(&errw, &dm->err, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&decw, &dm->dec_err, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    hs_rec.reset();
    // Payload errors first: the reconstruction ran on whatever was decoded (bounded, no faults).
    if (decw & (8u | 16u)) return fail(ctx, ASZ_E_DATA, "corrupt Huffman payload");
    if (decw & 128u) return fail(ctx, ASZ_E_DATA, "Huffman payload ends inside a code");
    if (decw & 32u) return fail(ctx, ASZ_E_DATA, "Huffman payload contains too few values");
    if (decw & 64u) return fail(ctx, ASZ_E_DATA, "Huffman payload contains too many values");
    if (errw) return fail(ctx, ASZ_E_DEVICE, "reconstruction kernels reported an internal error");
    R.core_s = secs(t_core, clk::now());
    if (!out_on_device) {
        auto t1 = clk::now();
        CK(cudaMemcpyAsync(out, d_out, N * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        R.d2h_s = secs(t1, clk::now());
    }
    if (rep) {
        R.min_val = mn;
        R.max_val = mx;
        R.abs_eb = abs_eb;
        R.layer_num = L;
        R.quintic = quintic;
        R.asz_len = len;
        R.pre_zstd_len = raw;
        R.cr = (float)N * sizeof(float) / (float)len;
        R.br = 8 * sizeof(float) / R.cr;
        std::snprintf(R.plan, sizeof(R.plan), "%s", ptxt.c_str());
        for (int a = 0; a < 3; a++) {
            R.pivot_stride[a] = (uint32_t)G.fg.pivot_stride[a];
            R.block_shape[a] = (uint32_t)G.fg.block_shape[a];
            R.block_num[a] = (uint32_t)G.fg.block_num[a];
        }
        R.kernel_launches = launch_counter() - launches0;
        R.total_s = secs(t_start, clk::now());
        *rep = R;
    }
    return ASZ_OK;
}

// ---------------------------------------------------------------------------------------------
// Debug accessors for the last asz_compress call.

extern "C" uint64_t asz_debug_qb(asz_ctx *ctx, uint32_t stream, int32_t *dst) {
    if (!ctx || !ctx->have_last || stream >= ctx->qb_len.size()) return 0;
    if (dst) cudaMemcpy(dst, ctx->qb.as<int32_t>() + ctx->qb_off[stream], ctx->qb_len[stream] * 4, cudaMemcpyDeviceToHost);
    return ctx->qb_len[stream];
}

extern "C" uint64_t asz_debug_t(asz_ctx *ctx, int64_t *dst) {
    if (!ctx || !ctx->have_last) return 0;
    if (dst) cudaMemcpy(dst, ctx->tint.p, ctx->t_len * 8, cudaMemcpyDeviceToHost);
    return ctx->t_len;
}

extern "C" uint64_t asz_debug_recon(asz_ctx *ctx, float *dst) {
    if (!ctx || !ctx->have_last) return 0;
    if (dst) cudaMemcpy(dst, ctx->rec.p, ctx->n_total * 4, cudaMemcpyDeviceToHost);
    return ctx->n_total;
}

extern "C" uint64_t asz_debug_proxies(asz_ctx *ctx, float *dst) {
    if (!ctx || !ctx->have_last) return 0;
    uint64_t n = ctx->t_len * 10;
    if (dst) cudaMemcpy(dst, ctx->proxies.p, n * 4, cudaMemcpyDeviceToHost);
    return n;
}

extern "C" uint64_t asz_debug_pre_zstd(asz_ctx *ctx, uint8_t *dst) {
    if (!ctx || !ctx->have_last) return 0;
    if (dst && ctx->pre_zstd.len) std::memcpy(dst, ctx->pre_zstd.p, ctx->pre_zstd.len);
    return ctx->pre_zstd.len;
}

extern "C" int asz_compress_stats(asz_ctx *ctx, double *max_err, double *psnr) {
    if (!ctx) return ASZ_E_ARG;
    if (!ctx->have_last) return fail(ctx, ASZ_E_ARG, "no compression on this context");
    cudaStream_t st = ctx->stream;
    struct {
        unsigned int mx;
        unsigned int pad;
        double sse;
    } h{}, *d = (decltype(&h))ctx->misc.as<uint8_t>();
    CK(cudaMemsetAsync(d, 0, sizeof(h), st));
    CK(launch_error_stats(ctx->last_in, ctx->rec.as<float>(), ctx->n_total, &d->mx, &d->sse, st));
    CK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float m;
    std::memcpy(&m, &h.mx, 4);
    double mse = h.sse / (double)ctx->n_total;
    double range = (double)ctx->last_max - (double)ctx->last_min;
    if (max_err) *max_err = m;
    if (psnr) *psnr = 10.0 * std::log10(range * range / mse);
    return ASZ_OK;
}

extern "C" int asz_profile_enable(asz_ctx *ctx, int on) {
    if (!ctx) return ASZ_E_ARG;
    ctx->prof = on != 0;
    return ASZ_OK;
}

extern "C" int asz_profile_read(asz_ctx *ctx, asz_profile_entry *out, int max, int reset) {
    if (!ctx) return ASZ_E_ARG;
    cudaStreamSynchronize(ctx->stream);
    prof_collect(ctx);
    int n = (int)ctx->prof_slots.size();
    for (int i = 0; i < n && i < max && out; i++) {
        std::snprintf(out[i].name, sizeof(out[i].name), "%s", ctx->prof_slots[i].name.c_str());
        out[i].launches = ctx->prof_slots[i].launches;
        out[i].ms = ctx->prof_slots[i].ms;
        out[i].bytes = ctx->prof_slots[i].bytes;
    }
    if (reset) ctx->prof_slots.clear();
    return n;
}

// ---------------------------------------------------------------------------------------------
// Geometry self-check (see include/asz_b200.h).

extern "C" int64_t asz_check_geometry(const uint64_t dims[3], const char *plan_text, uint64_t bpr, int quintic) {
    const uint64_t zero[3] = {0, 0, 0};
    return asz_check_geometry_frame(dims, zero, plan_text, bpr, quintic);
}

extern "C" int64_t asz_check_geometry_frame(const uint64_t dims[3], const uint64_t origin[3], const char *plan_text,
                                            uint64_t bpr, int quintic) {
    if (!dims || !origin || !plan_text || bpr == 0) return ASZ_E_ARG;
    Plan plan;
    std::string err;
    if (!parse_plan(plan_text, plan, err)) return ASZ_E_ARG;
    const u64 N = dims[0] * dims[1] * dims[2];
    if (N > (1ull << 26)) return ASZ_E_UNSUPPORTED;
    for (int a = 0; a < 3; a++)
        if (origin[a] >= dims[a]) return ASZ_E_ARG;
    const bool whole = origin[0] == 0 && origin[1] == 0 && origin[2] == 0;
    asz_params p;
    asz_default_params(&p);
    p.block_pivot_ratio = bpr;
    Geometry G;
    build_geometry(dims, plan, p, 1.0f, 1.0f, quintic != 0, G, origin);
    const FieldGeom &fg = G.fg;
    const u64 L = plan.pred.size();
    int64_t bad = 0;
    // Stamps: 0 = input value or pivot, l+1 = written by round l, -1 = a target not yet written.
    // Every point starts as an input value; the targets of all rounds are marked first.
    std::vector<int32_t> stamp(N, 0);
    {
        u64 str[3] = {fg.pivot_stride[0], fg.pivot_stride[1], fg.pivot_stride[2]};
        for (u64 l = 0; l < L; l++) {
            const RoundGeom &rg = G.rounds[l];
            for (u64 b0 = 0; b0 < fg.block_num[0]; b0++)
                for (u64 b1 = 0; b1 < fg.block_num[1]; b1++)
                    for (u64 b2 = 0; b2 < fg.block_num[2]; b2++) {
                        u64 bb[3] = {b0, b1, b2}, lo[3], hi[3];
                        for (int a = 0; a < 3; a++) {
                            u64 l0 = fg.origin[a] + bb[a] * fg.block_shape[a];
                            hi[a] = std::min(l0 + fg.block_shape[a] + 1, fg.n[a]);
                            lo[a] = a == rg.dir ? l0 + str[a] / 2 : (l0 == 0 ? 0 : l0 + str[a]);
                        }
                        for (u64 i0 = lo[0]; i0 < hi[0]; i0 += str[0])
                            for (u64 i1 = lo[1]; i1 < hi[1]; i1 += str[1])
                                for (u64 i2 = lo[2]; i2 < hi[2]; i2 += str[2]) {
                                    int32_t &s0 = stamp[(i0 * fg.n[1] + i1) * fg.n[2] + i2];
                                    if (s0 == -1) bad++;  // a point targeted twice
                                    s0 = -1;
                                }
                    }
            str[rg.dir] /= 2;
        }
    }
    // Pivots: never targets.
    for (u64 i0 = fg.origin[0]; i0 < fg.n[0]; i0 += fg.pivot_stride[0])
        for (u64 i1 = fg.origin[1]; i1 < fg.n[1]; i1 += fg.pivot_stride[1])
            for (u64 i2 = fg.origin[2]; i2 < fg.n[2]; i2 += fg.pivot_stride[2])
                if (stamp[(i0 * fg.n[1] + i1) * fg.n[2] + i2] != 0) bad++;
    AxisTables at{G.tab_count.data(), G.tab_prefix.data()};
    u64 written = G.pivots;
    for (u64 l = 0; l < L; l++) {
        const RoundGeom &rg = G.rounds[l];
        const int32_t cur = (int32_t)l + 1;
        auto readable = [&](int64_t q) { return q >= 0 && (u64)q < N && stamp[q] >= 0 && stamp[q] < cur; };
        // Reference order of QB indices: blocks in raster order, targets in compress.tpp:67-86 order.
        std::vector<u64> ref_pos(rg.qb_total, ~0ull);
        u64 base = 0;
        for (u64 b0 = 0; b0 < fg.block_num[0]; b0++)
            for (u64 b1 = 0; b1 < fg.block_num[1]; b1++)
                for (u64 b2 = 0; b2 < fg.block_num[2]; b2++) {
                    u64 bb[3] = {b0, b1, b2}, lo[3], hi[3], sh[3];
                    for (int a = 0; a < 3; a++) {
                        u64 l0 = fg.origin[a] + bb[a] * fg.block_shape[a];
                        hi[a] = std::min(l0 + fg.block_shape[a] + 1, fg.n[a]);
                        lo[a] = a == rg.dir ? l0 + rg.stride[a] / 2 : (l0 == 0 ? 0 : l0 + rg.stride[a]);
                        sh[a] = lo[a] >= hi[a] ? 0 : (hi[a] - lo[a] + rg.stride[a] - 1) / rg.stride[a];
                    }
                    for (u64 i0 = lo[0], j0 = 0; i0 < hi[0]; i0 += rg.stride[0], j0++)
                        for (u64 i1 = lo[1], j1 = 0; i1 < hi[1]; i1 += rg.stride[1], j1++)
                            for (u64 i2 = lo[2], j2 = 0; i2 < hi[2]; i2 += rg.stride[2], j2++) {
                                u64 li = rg.order == 0 ? (j1 * sh[2] + j2) * sh[0] + j0
                                        : rg.order == 1 ? (j0 * sh[2] + j2) * sh[1] + j1
                                                        : (j0 * sh[1] + j1) * sh[2] + j2;
                                if (base + li >= rg.qb_total) bad++;
                                else ref_pos[base + li] = (i0 * fg.n[1] + i1) * fg.n[2] + i2;
                            }
                    base += sh[0] * sh[1] * sh[2];
                }
        if (base != rg.qb_total) bad++;
        std::vector<uint8_t> used(rg.qb_total, 0);
        std::vector<u64> targets;
        for (u64 k = 0; k < rg.targets; k++) {
            Target t = locate(fg, rg, at, k);
            if (t.pos >= N || t.qi >= rg.qb_total || used[t.qi] || t.block >= G.nblocks) {
                bad++;
                continue;
            }
            {
                // The round kernels' table form of the same target.
                const u64 T1 = rg.tcount[1], T2 = rg.tcount[2];
                const u64 k2 = k % T2, line = k / T2, k0 = line / T1, k1 = line % T1;
                const AxisEntry &e0 = G.ent[rg.ent_off[0] + k0], &e1 = G.ent[rg.ent_off[1] + k1], &e2 = G.ent[rg.ent_off[2] + k2];
                const u64 pos = ((u64)e0.ii * fg.n[1] + e1.ii) * fg.n[2] + e2.ii;
                const u64 blk = ((u64)e0.bb * fg.block_num[1] + e1.bb) * fg.block_num[2] + e2.bb;
                const uint32_t sc = rg.dir == 0 ? e0.stencil : rg.dir == 1 ? e1.stencil : e2.stencil;
                if (pos != t.pos || qb_index(rg, e0, e1, e2) != t.qi || blk != t.block ||
                    sc != stencil_case(t.i, rg.hs, t.right, quintic != 0))
                    bad++;
            }
            used[t.qi] = 1;
            if (ref_pos[t.qi] != t.pos) bad++;
            if (stamp[t.pos] != -1) bad++;
            // The stencil branch exactly as predict() selects it.
            const int64_t pos = (int64_t)t.pos, d = (int64_t)rg.dist;
            const u64 i = t.i, hs = rg.hs, right = t.right;
            std::vector<int64_t> rd;
            if (quintic && i >= 5 * hs && i + 5 * hs < right) rd = {-1, 1, -3, 3, -5, 5};
            else if (i <= hs) {
                if (i + hs >= right) rd = {-1};
                else if (i + 3 * hs >= right) rd = {-1, 1};
                else rd = {-1, 1, 3};
            } else if (i + hs >= right) rd = {-1, -3};
            else if (i + 3 * hs >= right) rd = {-1, 1, -3};
            else rd = {-3, 3, -1, 1};
            for (int64_t o : rd)
                if (!readable(pos + o * d)) bad++;
            targets.push_back(t.pos);
        }
        for (u64 q = 0; q < rg.qb_total; q++)
            if (!used[q]) bad++;
        // Coefficient-selection samples: x0 is an unwritten target of this round, the four
        // references are earlier values (compress.tpp:102-120, get_AB_map.tpp:13-19).
        for (u64 g = 0; g < G.nblocks; g++) {
            u64 bb[3] = {g / (fg.block_num[1] * fg.block_num[2]), (g / fg.block_num[2]) % fg.block_num[1], g % fg.block_num[2]};
            int cls = 0;
            for (int a = 0; a < 3; a++) cls = cls * 3 + (bb[a] == 0 ? 0 : (bb[a] == fg.block_num[a] - 1 ? 2 : 1));
            const ClassInfo &ci = G.classes[l][cls];
            if (ci.fallback) continue;
            u64 lo[3], hi[3], step[3], cnt = 1;
            for (int a = 0; a < 3; a++) {
                lo[a] = fg.origin[a] + bb[a] * fg.block_shape[a];
                hi[a] = std::min(lo[a] + fg.block_shape[a] + 1, fg.n[a]);
                if (a != rg.dir && lo[a] != 0) lo[a] += rg.stride[a];
                if (a == rg.dir) {
                    lo[a] += 3 * rg.stride[a] / 2;
                    hi[a] -= 3 * rg.stride[a] / 2;
                }
                step[a] = rg.stride[a] * ci.ss;
                cnt *= hi[a] > lo[a] ? (hi[a] - lo[a] + step[a] - 1) / step[a] : 0;
            }
            if (cnt != ci.n) bad++;
            for (u64 i0 = lo[0]; i0 < hi[0]; i0 += step[0])
                for (u64 i1 = lo[1]; i1 < hi[1]; i1 += step[1])
                    for (u64 i2 = lo[2]; i2 < hi[2]; i2 += step[2]) {
                        int64_t pos = (int64_t)((i0 * fg.n[1] + i1) * fg.n[2] + i2), d = (int64_t)rg.dist;
                        if (pos < 0 || (u64)pos >= N || stamp[pos] != -1) bad++;
                        for (int64_t o : {-1, 1, -3, 3})
                            if (!readable(pos + o * d)) bad++;
                    }
        }
        for (u64 q : targets) stamp[q] = cur;
        written += targets.size();
    }
    if (whole && written != N) bad++;
    for (u64 q = 0; q < N; q++)
        if (stamp[q] < 0) {
            bad++;
            break;
        }
    return bad;
}

extern "C" int64_t asz_check_hashorder(const int64_t *a, const int64_t *b, uint64_t n, int pair, uint64_t *order) {
    if (!a || (pair && !b) || !order) return ASZ_E_ARG;
    std::map<std::pair<int64_t, int64_t>, uint64_t> first;
    std::vector<uint64_t> firsts;
    std::vector<uint64_t> hash;
    std::vector<int64_t> keys;
    for (uint64_t i = 0; i < n; i++) {
        std::pair<int64_t, int64_t> k{a[i], pair ? b[i] : 0};
        if (first.emplace(k, i).second) {
            firsts.push_back(i);
            hash.push_back(pair ? (uint64_t)a[i] * 1145141919810ull + (uint64_t)b[i] : (uint64_t)a[i]);
            keys.push_back(a[i]);
        }
    }
    const uint32_t m = (uint32_t)firsts.size();
    std::vector<int32_t> nxt(m + 1), bkt(sched_buckets(m) + 1);
    ListSim L{nxt.data(), bkt.data(), pair ? hash.data() : nullptr, keys.data(), m, 0, 1, 0, false};
    L.init();
    for (uint32_t e = 0; e < m; e++) L.insert((int32_t)e);
    if (L.broken) return -1;
    uint32_t k = 0;
    for (int32_t p = nxt[m]; p != kNil && k < m; p = nxt[p]) order[k++] = firsts[p];
    return k == m ? (int64_t)m : -1;
}

extern "C" int asz_set_tsel_mode(asz_ctx *ctx, int mode) {
    if (!ctx || mode < 0 || mode > 2) return ASZ_E_ARG;
    ctx->tsel_mode = mode;
    return ASZ_OK;
}

// ---------------------------------------------------------------------------------------------
// Batched compression: many fields of any shapes with one plan and one error bound. Each field's
// range, default slope and geometry are its own; the rounds run as one sequence for all fields:
// per round, one launch of each selection kernel (a work queue over every field's (block) groups)
// and one launch of the round kernel (a work queue over every field's target lines), captured
// once as a CUDA graph. Each field's result is the single-field result: same kernels per group
// and per target, only the mapping of work to CTAs differs.

namespace {

struct BatchItem {
    const float *d_in = nullptr;
    uint64_t dims[3] = {0, 0, 0};
    u64 N = 0;
    float mn = 0, mx = 0, abs_eb = 0, slope = 0, max_invalid = 0;
    int reason = 0;
    Geometry G;
    std::vector<u64> qb_off, qb_len;
    u64 o_in = 0, o_rec = 0, o_qb = 0, o_tval = 0, o_tint = 0, o_ent = 0, o_prox = 0;
};

constexpr uint32_t kBatchAmbCap = 1024;

// Launch shapes that change no result: CTAs per SM of the persistent selection and round
// kernels, and a shift of the threads per target line (fewer threads per line, more lines per CTA).
using BatchShape = std::array<uint32_t, 3>;

}  // namespace

static int compress_batch_impl(asz_ctx *ctx, uint32_t count, const float *const *in, int in_on_device, const uint64_t *dims,
                               float rel_eb, const asz_params *pp, const char *plan_text, const int64_t *const *t_tables,
                               const uint64_t *t_lens, uint8_t **out, size_t *out_len, asz_report *reps,
                               asz_batch_report *brep) {
    if (!ctx) return ASZ_E_ARG;
    auto t_start = clk::now();
    const uint64_t launches0 = launch_counter();
    ctx->err.clear();
    ctx->have_last = false;
    if (!count || !in || !dims || !plan_text || !out || !out_len) return fail(ctx, ASZ_E_ARG, "null argument");
    for (uint32_t f = 0; f < count; f++) {
        out[f] = nullptr;
        out_len[f] = 0;
    }
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    int rc = validate(ctx, p, true);
    if (rc) return rc;
    if (p.predictor_family == ASZ_FAMILY_AUTO) return fail(ctx, ASZ_E_ARG, "a batch needs a fixed predictor family");
    Plan plan;
    std::string perr;
    if (!parse_plan(plan_text, plan, perr)) return fail(ctx, ASZ_E_ARG, perr);
    if (plan.pred.size() > 63) return fail(ctx, ASZ_E_ARG, "predictor plan cannot contain more than 63 layers");
    const bool quintic = p.predictor_family == ASZ_FAMILY_QUINTIC;
    const u64 L = plan.pred.size();
    const uint32_t nf = count;
    for (uint32_t f = 0; f < nf; f++) {
        rc = validate_dims(ctx, dims + 3 * f, rel_eb);
        if (rc) return fail(ctx, rc, "field " + std::to_string(f) + ": " + ctx->err);
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, ASZ_E_CUDA, "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    CK(ctx->misc.reserve(sizeof(MiscLayout)));
    asz_batch_report BR{};
    std::vector<BatchItem> B(nf);
    // ---- Inputs, ranges, slopes, geometry.
    u64 in_total = 0;
    for (uint32_t f = 0; f < nf; f++) {
        for (int a = 0; a < 3; a++) B[f].dims[a] = dims[3 * f + a];
        B[f].N = B[f].dims[0] * B[f].dims[1] * B[f].dims[2];
        B[f].o_in = in_total;
        if (!in_on_device) in_total += B[f].N;
        if (!in[f]) return fail(ctx, ASZ_E_ARG, "field " + std::to_string(f) + ": null input");
    }
    auto t_h2d = clk::now();
    if (!in_on_device) {
        CK(ctx->b_in.reserve(in_total * sizeof(float)));
        for (uint32_t f = 0; f < nf; f++) {
            CK(cudaMemcpyAsync(ctx->b_in.as<float>() + B[f].o_in, in[f], B[f].N * sizeof(float), cudaMemcpyHostToDevice, st));
            B[f].d_in = ctx->b_in.as<float>() + B[f].o_in;
        }
        CK(cudaStreamSynchronize(st));
    } else {
        for (uint32_t f = 0; f < nf; f++) B[f].d_in = in[f];
    }
    BR.h2d_s = secs(t_h2d, clk::now());
    auto t_prep = clk::now();
    const std::vector<float> cand = candidate_t(p);
    u64 nb_total = 0, ent_total = 0, tint_total = 0, qb_total = 0;
    uint32_t capmax = 1;
    for (uint32_t f = 0; f < nf; f++) {
        BatchItem &b = B[f];
        const std::string tag = "field " + std::to_string(f) + ": ";
        rc = compute_range(ctx, b.d_in, b.N, b.mn, b.mx);
        if (rc) return fail(ctx, rc, tag + ctx->err);
        if (b.mn == b.mx) return fail(ctx, ASZ_E_DATA, tag + "max_val==min_val");
        b.abs_eb = rel_eb * (b.mx - b.mn);
        rc = default_slope(ctx, b.d_in, b.dims, p, b.abs_eb, b.mn, b.mx, cand, b.slope, b.max_invalid, b.reason);
        if (rc) return fail(ctx, rc, tag + ctx->err);
        build_geometry(b.dims, plan, p, b.abs_eb, b.slope, quintic, b.G);
        if (!kernel_limits_ok(b.G)) return fail(ctx, ASZ_E_UNSUPPORTED, tag + "field too large for 32-bit line indexing");
        b.qb_off.assign(L + 1, 0);
        b.qb_len.assign(L + 1, 0);
        b.qb_len[0] = b.G.pivots;
        for (u64 l = 0; l < L; l++) b.qb_len[l + 1] = b.G.rounds[l].qb_total;
        u64 acc = 0;
        for (u64 s2 = 0; s2 <= L; s2++) {
            b.qb_off[s2] = acc;
            acc += b.qb_len[s2];
        }
        if (acc != b.N) return fail(ctx, ASZ_E_DATA, tag + "total_qb_num!=data.size()");
        if (t_tables && t_lens[f] != b.G.nblocks * L)
            return fail(ctx, ASZ_E_ARG, tag + "t table length does not match the plan's blocks and rounds");
        for (u64 l = 0; l < L; l++) {
            for (auto &ci : b.G.classes[l])
                if (ci.n) ci.log2_off = log2_table(ctx, ci.n);
            capmax = std::max(capmax, b.G.cap[l]);
        }
        b.o_rec = b.o_qb = qb_total;
        qb_total += b.N;
        b.o_tval = nb_total;
        b.o_prox = nb_total * L * 10;
        nb_total += b.G.nblocks;
        b.o_tint = tint_total;
        tint_total += b.G.nblocks * L;
        b.o_ent = ent_total;
        ent_total += b.G.ent.size();
    }
    rc = upload_log2(ctx);
    if (rc) return rc;
    // ---- Arenas and tables.
    CK(ctx->b_rec.reserve(qb_total * sizeof(float)));
    CK(ctx->b_qb.reserve(qb_total * sizeof(int32_t)));
    CK(ctx->b_tval.reserve(std::max<u64>(nb_total, 1) * sizeof(float)));
    CK(ctx->b_tint.reserve(std::max<u64>(tint_total, 1) * sizeof(int64_t)));
    CK(ctx->b_ent.reserve(std::max<u64>(ent_total, 1) * sizeof(AxisEntry)));
    CK(ctx->b_cls.reserve((u64)nf * 27 * L * sizeof(ClassInfo)));
    CK(ctx->b_rounds.reserve((u64)nf * L * sizeof(RoundGeom)));
    CK(ctx->b_qoff.reserve((u64)nf * (L + 1) * sizeof(u64)));
    CK(ctx->b_range.reserve((u64)nf * 2 * (L + 1) * sizeof(int32_t)));
    CK(ctx->b_range0.reserve((u64)nf * 2 * (L + 1) * sizeof(int32_t)));
    CK(ctx->b_prox.reserve(std::max<u64>(nb_total * L * 10, 1) * sizeof(float)));
    CK(ctx->b_amb.reserve((u64)nf * kBatchAmbCap * sizeof(AmbiguousRecord)));
    CK(ctx->b_cnt.reserve((u64)nf * sizeof(BatchCounters)));
    CK(ctx->b_fields.reserve((u64)nf * sizeof(BatchField)));
    CK(ctx->b_goff.reserve((u64)(nf + 1) * sizeof(u64)));
    CK(ctx->b_poff.reserve((u64)(nf + 1) * sizeof(u64)));
    CK(ctx->b_ioff.reserve((u64)L * (nf + 1) * sizeof(u64)));
    CK(ctx->b_queue.reserve((u64)L * 5 * sizeof(uint32_t)));
    CK(ctx->b_hand.reserve(std::max<u64>(nb_total, 1) * sizeof(unsigned long long)));
    CK(ctx->b_spill.reserve(std::max<u64>(nb_total, 1) * sizeof(unsigned long long)));
    // Groups above the exact kernel's shared-memory capacity: the same replay with global scratch,
    // a CTA per group (at most 148 CTAs and 512 MiB), then the serial kernel for what is left.
    const u64 gstride = exact_global_stride(capmax);
    unsigned ggrid = 0;
    if (capmax > exact_cap()) {
        ggrid = (unsigned)std::max<u64>(1, std::min<u64>(148, (512ull << 20) / gstride));
        CK(ctx->gscratch.reserve(ggrid * gstride));
        CK(ctx->b_spill2.reserve(std::max<u64>(nb_total, 1) * sizeof(unsigned long long)));
    }
    uint32_t bcap, tcap;
    u64 sstride;
    scratch_dims(capmax, bcap, tcap, sstride);
    const u64 slots = std::min<u64>(nb_total, 2048);
    CK(ctx->scratch.reserve(std::max<u64>(slots, 1) * sstride));
    u64 pivots_total = 0;
    {
        std::vector<ClassInfo> cls;
        std::vector<RoundGeom> rounds;
        std::vector<u64> qoff;
        std::vector<int32_t> range0;
        for (uint32_t f = 0; f < nf; f++) {
            const BatchItem &b = B[f];
            CK(cudaMemcpyAsync(ctx->b_ent.as<AxisEntry>() + b.o_ent, b.G.ent.data(), b.G.ent.size() * sizeof(AxisEntry),
                               cudaMemcpyHostToDevice, st));
            for (u64 l = 0; l < L; l++) cls.insert(cls.end(), b.G.classes[l].begin(), b.G.classes[l].end());
            rounds.insert(rounds.end(), b.G.rounds.begin(), b.G.rounds.end());
            qoff.insert(qoff.end(), b.qb_off.begin(), b.qb_off.end());
            for (u64 s2 = 0; s2 <= L; s2++) {
                range0.push_back(INT32_MAX);
                range0.push_back(INT32_MIN);
            }
        }
        CK(cudaMemcpyAsync(ctx->b_cls.p, cls.data(), cls.size() * sizeof(ClassInfo), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->b_rounds.p, rounds.data(), rounds.size() * sizeof(RoundGeom), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->b_qoff.p, qoff.data(), qoff.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->b_range0.p, range0.data(), range0.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        std::vector<u64> goff(nf + 1, 0), poff(nf + 1, 0);
        for (uint32_t f = 0; f < nf; f++) {
            goff[f + 1] = goff[f] + B[f].G.nblocks;
            poff[f + 1] = poff[f] + B[f].G.pivots;
        }
        pivots_total = poff[nf];
        CK(cudaMemcpyAsync(ctx->b_goff.p, goff.data(), goff.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->b_poff.p, poff.data(), poff.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    if (t_tables)
        for (uint32_t f = 0; f < nf; f++)
            CK(cudaMemcpyAsync(ctx->b_tint.as<int64_t>() + B[f].o_tint, t_tables[f], t_lens[f] * sizeof(int64_t),
                               cudaMemcpyHostToDevice, st));
    // Field table and per-round work-item offsets for a launch shape (threads-per-line shift).
    auto upload_shape = [&](uint32_t tpl_shift) -> int {
        std::vector<BatchField> F(nf);
        std::vector<u64> ioff((u64)L * (nf + 1), 0);
        for (uint32_t f = 0; f < nf; f++) {
            const BatchItem &b = B[f];
            BatchField &x = F[f];
            std::memset(&x, 0, sizeof(x));
            x.fg = b.G.fg;
            x.pg = b.G.pg;
            x.rounds = ctx->b_rounds.as<RoundGeom>() + (u64)f * L;
            x.ent = ctx->b_ent.as<AxisEntry>() + b.o_ent;
            x.classes = ctx->b_cls.as<ClassInfo>() + (u64)f * 27 * L;
            x.in = b.d_in;
            x.rec = ctx->b_rec.as<float>() + b.o_rec;
            x.tval = ctx->b_tval.as<float>() + b.o_tval;
            x.tint = ctx->b_tint.as<int64_t>() + b.o_tint;
            x.qb = ctx->b_qb.as<int32_t>() + b.o_qb;
            x.qoff = ctx->b_qoff.as<u64>() + (u64)f * (L + 1);
            x.qb_range = ctx->b_range.as<int32_t>() + (u64)f * 2 * (L + 1);
            x.proxies = ctx->b_prox.as<float>() + b.o_prox;
            x.amb = ctx->b_amb.as<AmbiguousRecord>() + (u64)f * kBatchAmbCap;
            x.amb_cap = kBatchAmbCap;
            x.cnt = ctx->b_cnt.as<BatchCounters>() + f;
            x.R2 = (b.mx - b.mn) * (b.mx - b.mn);
            for (u64 l = 0; l < L; l++) {
                const uint32_t lg = round_tpl_log2(b.G.rounds[l].tcount[2]);
                x.tpl_log2[l] = lg > tpl_shift ? lg - tpl_shift : 0;
                ioff[l * (nf + 1) + f + 1] = ioff[l * (nf + 1) + f] + round_batch_items(b.G.rounds[l], x.tpl_log2[l]);
            }
        }
        CK(cudaMemcpyAsync(ctx->b_fields.p, F.data(), F.size() * sizeof(BatchField), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->b_ioff.p, ioff.data(), ioff.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
        return ASZ_OK;
    };
    const float t_default = 4.0f / 16;  // insufficient_sample_t (asz_param.hpp:206)
    const BatchField *dF = ctx->b_fields.as<BatchField>();
    const u64 *d_goff = ctx->b_goff.as<u64>(), *d_ioff = ctx->b_ioff.as<u64>();
    uint32_t *d_queue = ctx->b_queue.as<uint32_t>();
    unsigned long long *d_hand = ctx->b_hand.as<unsigned long long>(), *d_spill = ctx->b_spill.as<unsigned long long>();
    // The whole sequence: counters and ranges reset, pivots, then per round the batched fast
    // selection, exact replay, serial spill and prediction.
    auto enqueue = [&](const BatchShape &sh) -> int {
        CK(cudaMemcpyAsync(ctx->b_range.p, ctx->b_range0.p, (u64)nf * 2 * (L + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                           st));
        CK(cudaMemsetAsync(ctx->b_cnt.p, 0, (u64)nf * sizeof(BatchCounters), st));
        CK(cudaMemsetAsync(ctx->b_queue.p, 0, (u64)L * 5 * sizeof(uint32_t), st));
        CK(launch_pivot_compress_batch(dF, ctx->b_poff.as<u64>(), nf, pivots_total, st));
        for (u64 l = 0; l < L; l++) {
            // Per round: fast queue, round queue, hand-off count, spill count, second spill count.
            uint32_t *q = d_queue + 5 * l;
            if (t_tables) {
                // The caller's t codes replace the coefficient selection.
                CK(launch_tval_from_codes_batch(dF, d_goff, nf, nb_total, (uint32_t)l, st));
                CK(launch_round_compress_batch(dF, d_ioff + l * (nf + 1), nf, (uint32_t)l, q + 1, 148 * sh[1], st));
                continue;
            }
            CK(launch_tsel_fast_batch(dF, d_goff, nf, (uint32_t)l, ctx->log2arena.as<float>(), t_default, q, d_hand, q + 2,
                                      148 * sh[0], st));
            CK(launch_tsel_exact_batch(dF, (uint32_t)l, ctx->log2arena.as<float>(), t_default, d_hand, q + 2, d_spill, q + 3,
                                       exact_cap(), 148, st));
            unsigned long long *d_left = d_spill;
            uint32_t *d_lcnt = q + 3;
            if (ggrid) {
                d_left = ctx->b_spill2.as<unsigned long long>();
                d_lcnt = q + 4;
                CK(launch_tsel_exact_global_batch(dF, (uint32_t)l, ctx->log2arena.as<float>(), t_default, d_spill, q + 3, d_left,
                                                  d_lcnt, ctx->gscratch.as<uint8_t>(), gstride, capmax, ggrid, st));
            }
            CK(launch_tsel_v0_batch(dF, (uint32_t)l, ctx->log2arena.as<float>(), t_default, ctx->scratch.as<uint8_t>(), sstride,
                                    capmax, bcap, tcap, d_left, d_lcnt, slots, st));
            CK(launch_round_compress_batch(dF, d_ioff + l * (nf + 1), nf, (uint32_t)l, q + 1, 148 * sh[1], st));
        }
        return ASZ_OK;
    };
    BR.prep_s = secs(t_prep, clk::now());
    // ---- Launch shapes: measured once per batch shape (the autotuner), then reused.
    std::vector<uint64_t> shape_key{nf, L, (uint64_t)quintic, p.block_pivot_ratio, (uint64_t)(t_tables != nullptr)};
    for (uint32_t f = 0; f < nf; f++) shape_key.insert(shape_key.end(), B[f].dims, B[f].dims + 3);
    for (u64 l = 0; l < L; l++) shape_key.push_back((uint64_t)plan.dir[l] * 3 + plan.order[l]);
    BatchShape best{16, 5, 0};
    auto tuned = ctx->batch_tuned.find(shape_key);
    if (tuned != ctx->batch_tuned.end()) {
        best = tuned->second;
    } else {
        auto t_tune = clk::now();
        cudaEvent_t e0 = prof_event(ctx), e1 = prof_event(ctx);
        float best_ms = INFINITY;
        uint32_t last_shift = UINT32_MAX;
        for (uint32_t shift : {0u, 1u})
            for (uint32_t fast : {8u, 16u})
                for (uint32_t round : {3u, 5u}) {
                    if (shift != last_shift) {
                        rc = upload_shape(shift);
                        if (rc) return rc;
                        last_shift = shift;
                    }
                    const BatchShape sh{fast, round, shift};
                    CK(cudaEventRecord(e0, st));
                    rc = enqueue(sh);
                    if (rc) return rc;
                    CK(cudaEventRecord(e1, st));
                    CK(cudaEventSynchronize(e1));
                    float ms = 0;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = sh;
                    }
                }
        ctx->event_pool.push_back(e0);
        ctx->event_pool.push_back(e1);
        ctx->batch_tuned[shape_key] = best;
        BR.tuned_now = 1;
        BR.tune_s = secs(t_tune, clk::now());
    }
    BR.fast_ctas_per_sm = best[0];
    BR.round_ctas_per_sm = best[1];
    BR.tpl_shift = best[2];
    rc = upload_shape(best[2]);
    if (rc) return rc;
    // ---- The round sequence as a CUDA graph (captured once per batch layout).
    std::vector<uint64_t> graph_key = shape_key;
    graph_key.insert(graph_key.end(), best.begin(), best.end());
    for (uint32_t f = 0; f < nf; f++) graph_key.push_back((uint64_t)(uintptr_t)B[f].d_in);
    for (DevBuf *d : {&ctx->b_rec, &ctx->b_qb, &ctx->b_tval, &ctx->b_tint, &ctx->b_ent, &ctx->b_cls, &ctx->b_rounds,
                      &ctx->b_qoff, &ctx->b_range, &ctx->b_range0, &ctx->b_prox, &ctx->b_amb, &ctx->b_cnt, &ctx->b_fields,
                      &ctx->b_goff, &ctx->b_poff, &ctx->b_ioff, &ctx->b_queue, &ctx->b_hand, &ctx->b_spill, &ctx->scratch,
                      &ctx->log2arena, &ctx->b_spill2, &ctx->gscratch})
        graph_key.push_back((uint64_t)(uintptr_t)d->p);
    graph_key.push_back((uint64_t)(uintptr_t)st);
    auto t_rounds = clk::now();
    cudaEvent_t r0 = prof_event(ctx), r1 = prof_event(ctx);
    if (!ctx->batch_graph || ctx->batch_graph_key != graph_key) {
        if (ctx->batch_graph) {
            cudaGraphExecDestroy(ctx->batch_graph);
            ctx->batch_graph = nullptr;
        }
        cudaGraph_t graph = nullptr;
        const bool prof = ctx->prof;
        ctx->prof = false;  // no event records inside the capture
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int erc = enqueue(best);
        const cudaError_t ce = cudaStreamEndCapture(st, &graph);
        ctx->prof = prof;
        if (erc) {
            if (graph) cudaGraphDestroy(graph);
            return erc;
        }
        if (ce != cudaSuccess) return fail(ctx, ASZ_E_CUDA, std::string("stream capture: ") + cudaGetErrorString(ce));
        const cudaError_t ie = cudaGraphInstantiate(&ctx->batch_graph, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            ctx->batch_graph = nullptr;
            return fail(ctx, ASZ_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        }
        ctx->batch_graph_key = graph_key;
    } else {
        BR.graph_reused = 1;
    }
    CK(cudaEventRecord(r0, st));
    CK(cudaGraphLaunch(ctx->batch_graph, st));
    CK(cudaEventRecord(r1, st));
    std::vector<BatchCounters> cnt(nf);
    CK(cudaMemcpyAsync(cnt.data(), ctx->b_cnt.p, nf * sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, r0, r1));
        BR.rounds_ms = ms;
        ctx->event_pool.push_back(r0);
        ctx->event_pool.push_back(r1);
    }
    BR.rounds_s = secs(t_rounds, clk::now());
    for (uint32_t f = 0; f < nf; f++)
        if (cnt[f].err)
            return fail(ctx, ASZ_E_DEVICE, "field " + std::to_string(f) + ": round kernels reported an internal error " +
                                               std::to_string(cnt[f].err));
    // ---- Host replay of the ambiguous coefficient decisions (glibc log10f, compress.tpp:127-142).
    // A field whose replay confirms every provisional choice keeps its batch result; a field whose
    // replay changes one takes the single-field path, which reruns its rounds with the choices.
    std::vector<char> single(nf, 0);
    for (uint32_t f = 0; f < nf; f++) {
        if (!cnt[f].amb_count) continue;
        if (cnt[f].amb_count > kBatchAmbCap) {
            single[f] = 1;
            continue;
        }
        std::vector<AmbiguousRecord> recs(cnt[f].amb_count);
        CK(cudaMemcpyAsync(recs.data(), ctx->b_amb.as<AmbiguousRecord>() + (u64)f * kBatchAmbCap,
                           recs.size() * sizeof(AmbiguousRecord), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (const AmbiguousRecord &r : recs) {
            const float t = replay_decision(r, B[f].G.rounds[r.round].slope);
            if ((int32_t)host_lround_f(t * (float)p.t_precision) != r.provisional) single[f] = 1;
        }
    }
    // ---- Entropy stage in chunks of fields (one set of transfers and syncs per chunk); zstd on
    // host threads from the chunk's pinned buffer while the next chunk is encoded.
    auto t_enc = clk::now();
    std::vector<asz_report> R(nf);
    for (auto &r : R) std::memset(&r, 0, sizeof(r));
    std::vector<std::string> zerr(nf);
    std::vector<double> zsec(nf, 0.0);
    std::vector<std::thread> zth[2];
    auto join_buf = [&](int k) {
        for (auto &t : zth[k]) t.join();
        zth[k].clear();
    };
    int frc = ASZ_OK;
    const uint32_t kChunk = 8;
    std::vector<uint32_t> order;
    for (uint32_t f = 0; f < nf; f++)
        if (!single[f]) order.push_back(f);
    for (size_t c0 = 0, k = 0; c0 < order.size() && !frc; c0 += kChunk, k ^= 1) {
        join_buf((int)k);  // the zstd threads of two chunks ago are done with this buffer
        std::vector<EncodeArgs> ea;
        std::vector<asz_report *> rs;
        const size_t c1 = std::min(order.size(), c0 + kChunk);
        for (size_t i = c0; i < c1; i++) {
            const uint32_t f = order[i];
            const BatchItem &b = B[f];
            ea.push_back(EncodeArgs{&b.G, &b.qb_off, &b.qb_len, ctx->b_qb.as<int32_t>() + b.o_qb,
                                    ctx->b_tint.as<int64_t>() + b.o_tint, ctx->b_range.as<int32_t>() + (u64)f * 2 * (L + 1),
                                    b.mn, b.mx, quintic, &plan, &p, t_tables ? t_tables[f] : nullptr,
                                    t_tables ? t_lens[f] : 0, b.N});
            rs.push_back(&R[f]);
        }
        std::vector<std::pair<u64, u64>> span;
        PinnedBuf &pb = ctx->batch_pre[k];
        const int erc = encode_fields(ctx, ea, rs, span, pb);
        if (erc) {
            frc = erc;
            break;
        }
        for (size_t i = c0; i < c1; i++) {
            const uint32_t f = order[i];
            const uint8_t *src = pb.p + span[i - c0].first;
            const size_t len = span[i - c0].second;
            R[f].pre_zstd_len = len;
            zth[k].emplace_back([&, f, src, len]() {
                auto tz = clk::now();
                size_t bound = ZSTD_compressBound(len);
                uint8_t *z = out_alloc(bound);
                if (!z) {
                    zerr[f] = "out of host memory";
                    return;
                }
                size_t zl = zstd3(ctx, z, bound, src, len);
                if (ZSTD_isError(zl)) {
                    out_release(z);
                    zerr[f] = std::string("ZSTD_compress: ") + ZSTD_getErrorName(zl);
                    return;
                }
                out[f] = z;
                out_len[f] = zl;
                zsec[f] = secs(tz, clk::now());
            });
        }
    }
    join_buf(0);
    join_buf(1);
    for (uint32_t f = 0; f < nf && !frc; f++) {
        BatchItem &b = B[f];
        asz_report &r = R[f];
        if (single[f]) {
            BR.fields_fallback++;
            uint8_t *o1 = nullptr;
            size_t l1 = 0;
            frc = compress_entry(ctx, b.d_in, 1, b.dims, rel_eb, &p, plan_text, t_tables ? t_tables[f] : nullptr,
                                 t_tables ? t_lens[f] : 0, &o1, &l1, &r);
            if (out[f]) out_release(out[f]);
            out[f] = o1;
            out_len[f] = l1;
            continue;
        }
        r.min_val = b.mn;
        r.max_val = b.mx;
        r.abs_eb = b.abs_eb;
        r.default_slope = b.slope;
        r.slope_max_invalid_ratio = b.max_invalid;
        r.slope_fallback_reason = b.reason;
        r.layer_num = L;
        r.quintic = quintic ? 1 : 0;
        r.t_fallback_count = cnt[f].fb;
        r.ambiguous_decisions = cnt[f].amb_count;
        r.exact_window = cnt[f].why[0];
        r.exact_undecided = cnt[f].why[1];
        r.wide_groups = cnt[f].why[2];
        for (int a = 0; a < 3; a++) {
            r.pivot_stride[a] = (uint32_t)b.G.fg.pivot_stride[a];
            r.block_shape[a] = (uint32_t)b.G.fg.block_shape[a];
            r.block_num[a] = (uint32_t)b.G.fg.block_num[a];
        }
        std::snprintf(r.plan, sizeof(r.plan), "%s", plan_text);
    }
    BR.encode_s = secs(t_enc, clk::now());
    if (frc) {
        for (uint32_t f = 0; f < nf; f++) {
            if (out[f]) out_release(out[f]);
            out[f] = nullptr;
            out_len[f] = 0;
        }
        return frc;
    }
    for (uint32_t f = 0; f < nf; f++)
        if (!zerr[f].empty()) {
            for (uint32_t g = 0; g < nf; g++) {
                if (out[g]) out_release(out[g]);
                out[g] = nullptr;
                out_len[g] = 0;
            }
            return fail(ctx, ASZ_E_DATA, "field " + std::to_string(f) + ": " + zerr[f]);
        }
    for (uint32_t f = 0; f < nf; f++) {
        BR.zstd_s += zsec[f];
        if (!R[f].asz_len) {
            R[f].asz_len = out_len[f];
            R[f].zstd_s = zsec[f];
            R[f].cr = (float)B[f].N * sizeof(float) / (float)out_len[f];
            R[f].br = 8 * sizeof(float) / R[f].cr;
        }
        BR.input_bytes += B[f].N * sizeof(float);
        BR.output_bytes += out_len[f];
    }
    BR.kernel_launches = launch_counter() - launches0;
    BR.total_s = secs(t_start, clk::now());
    if (reps)
        for (uint32_t f = 0; f < nf; f++) reps[f] = R[f];
    if (brep) *brep = BR;
    return ASZ_OK;
}

extern "C" int asz_compress_batch(asz_ctx *ctx, uint32_t count, const float *const *in, int in_on_device,
                                  const uint64_t *dims, float rel_eb, const asz_params *pp, const char *plan_text,
                                  uint8_t **out, size_t *out_len, asz_report *reps, asz_batch_report *brep) {
    return compress_batch_impl(ctx, count, in, in_on_device, dims, rel_eb, pp, plan_text, nullptr, nullptr, out, out_len, reps,
                               brep);
}

extern "C" int asz_compress_batch_with_t(asz_ctx *ctx, uint32_t count, const float *const *in, int in_on_device,
                                         const uint64_t *dims, float rel_eb, const asz_params *pp, const char *plan_text,
                                         const int64_t *const *t_tables, const uint64_t *t_lens, uint8_t **out,
                                         size_t *out_len, asz_report *reps, asz_batch_report *brep) {
    if (!ctx) return ASZ_E_ARG;
    ctx->err.clear();
    if (!t_tables || !t_lens) return fail(ctx, ASZ_E_ARG, "null t tables");
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    const int64_t lo = (int64_t)std::llround((double)p.t_min * p.t_precision);
    const int64_t hi = (int64_t)std::llround((double)p.t_max * p.t_precision);
    for (uint32_t f = 0; f < count; f++) {
        if (!t_tables[f]) return fail(ctx, ASZ_E_ARG, "field " + std::to_string(f) + ": null t table");
        for (uint64_t i = 0; i < t_lens[f]; i++)
            if (t_tables[f][i] < lo || t_tables[f][i] > hi)
                return fail(ctx, ASZ_E_ARG, "field " + std::to_string(f) + ": t code outside [t_min, t_max] at index " +
                                                std::to_string(i));
    }
    return compress_batch_impl(ctx, count, in, in_on_device, dims, rel_eb, &p, plan_text, t_tables, t_lens, out, out_len, reps,
                               brep);
}

// ---------------------------------------------------------------------------------------------
// Internal interface for the other C-ABI translation units (host/internal.h).

// ---------------------------------------------------------------------------------------------
// One field over several ranks (asz_compress_slab). Each rank holds a slab of axis-0 blocks and
// runs the single-field core on a frame: [halo planes | the face plane of the slab below | its
// planes], with the frame origin at the face, so blocks, targets, sample boxes and stencil cases
// are those of the same blocks in the whole field (compress.tpp:179-209 walks the blocks in raster
// order; a slab's blocks are contiguous in every stream). The halo is at least two pivot strides
// deep (quintic stencils reach 2.5 strides below a target, cubic 1.5) or reaches plane 0.

namespace {

struct SlabLayout {
    u64 ps0 = 1, bs0 = 1, blocks0 = 0;  // axis 0: pivot stride, block shape, block count
    u64 s0 = 0;                          // global plane of the slab's lower face (block_begin * bs0)
    u64 last = 0;                        // global plane of its upper face (inclusive)
    u64 plane_begin = 0, plane_count = 0;
    u64 halo = 0;                        // planes below the face in the frame (0 for the first slab)
    u64 local0 = 0;                      // frame planes: halo + face + owned
};

int slab_layout(const uint64_t dims[3], const Plan &plan, const asz_params &p, u64 b0, u64 b1, SlabLayout &S,
                std::string &err) {
    S = SlabLayout{};
    for (int d : plan.dir)
        if (d == 0) S.ps0 *= 2;
    S.bs0 = S.ps0 * p.block_pivot_ratio;
    S.blocks0 = (dims[0] + S.bs0 - 1) / S.bs0;
    if (b0 >= b1 || b1 > S.blocks0) {
        err = "slab blocks [" + std::to_string(b0) + ", " + std::to_string(b1) + ") outside the field's " +
              std::to_string(S.blocks0) + " axis-0 blocks";
        return ASZ_E_ARG;
    }
    S.s0 = b0 * S.bs0;
    S.last = b1 == S.blocks0 ? dims[0] - 1 : b1 * S.bs0;
    S.plane_begin = b0 == 0 ? 0 : S.s0 + 1;
    S.plane_count = S.last + 1 - S.plane_begin;
    S.halo = b0 == 0 ? 0 : std::min<u64>(S.s0, 2 * S.ps0);
    S.local0 = b0 == 0 ? S.plane_count : S.halo + 1 + S.plane_count;
    return ASZ_OK;
}

// The caller's collectives (a single rank needs none).
struct SlabComm {
    asz_ctx *ctx;
    const asz_comm *c;
    int allreduce(void *buf, u64 n, int dtype, int op) {
        if (c->size == 1 || n == 0) return ASZ_OK;
        return c->allreduce(c->user, buf, n, dtype, op) ? fail(ctx, ASZ_E_COMM, "slab: allreduce failed") : ASZ_OK;
    }
    int allgather(const void *send, u64 bytes, void *recv) {
        if (c->size == 1) {
            std::memcpy(recv, send, bytes);
            return ASZ_OK;
        }
        return c->allgather(c->user, send, bytes, recv) ? fail(ctx, ASZ_E_COMM, "slab: allgather failed") : ASZ_OK;
    }
    int send(const void *buf, u64 bytes, int dst) {
        return c->send(c->user, buf, bytes, dst) ? fail(ctx, ASZ_E_COMM, "slab: send failed") : ASZ_OK;
    }
    int recv(void *buf, u64 bytes, int src) {
        return c->recv(c->user, buf, bytes, src) ? fail(ctx, ASZ_E_COMM, "slab: recv failed") : ASZ_OK;
    }
    // Every rank learns whether any rank failed (rc nonzero), so that none waits in a later
    // exchange for a rank that returned.
    int agree_ok(int rc) {
        int32_t bad = rc ? 1 : 0;
        const int e = allreduce(&bad, 1, 2, 2);
        if (e) return e;
        if (rc) return rc;
        return bad ? fail(ctx, ASZ_E_COMM, "slab: another rank failed") : ASZ_OK;
    }
};

// The field's range from every slab's: the first smallest and the last largest value in raster
// order (std::minmax_element, s1_compress.cpp:131-137), so equal extremes keep the sign of zero of
// the lowest rank's minimum and the highest rank's maximum.
int slab_range(SlabComm &cm, float mn, float mx, float &gmn, float &gmx) {
    const int R = cm.c->size;
    float mine[2] = {mn, mx};
    std::vector<float> all(2 * R);
    int rc = cm.allgather(mine, sizeof(mine), all.data());
    if (rc) return rc;
    gmn = all[0];
    gmx = all[1];
    for (int r = 1; r < R; r++) {
        if (all[2 * r] < gmn) gmn = all[2 * r];
        if (all[2 * r + 1] >= gmx) gmx = all[2 * r + 1];
    }
    return ASZ_OK;
}

// get_default_slope over the whole field from the slabs: the three global sample boxes
// (slope_boxes) and, per sample, the seven values along the box's direction around it (offsets
// -3..3; the AB map reads -3, -1, 0, 1, 3). Each rank gathers the values in its planes, all ranks
// exchange them, and each evaluates the boxes on one compact array that keeps the samples' order:
// direction d's block holds its samples' lattice with axis d widened seven-fold, the blocks
// stacked along axis 0. Every rank computes the same slope.
int slab_slope(asz_ctx *ctx, SlabComm &cm, const float *d_local, const uint64_t ldims[3], u64 local_first_plane,
               u64 own_lo, u64 own_hi, const uint64_t dims[3], const asz_params &p, float abs_eb, float mn, float mx,
               const std::vector<float> &cand, float &slope, float &max_invalid, int &reason) {
    SampleBox gb[3];
    slope_boxes(dims, p, abs_eb, gb);
    u64 cnt[3][3], D[3][3], off0[3], M1 = 1, M2 = 1, T0 = 0;
    for (int d = 0; d < 3; d++) {
        for (int a = 0; a < 3; a++) {
            cnt[d][a] = gb[d].hi[a] > gb[d].lo[a] ? (gb[d].hi[a] - gb[d].lo[a] + gb[d].step[a] - 1) / gb[d].step[a] : 0;
            D[d][a] = cnt[d][a] * (a == d ? 7 : 1);
        }
        off0[d] = T0;
        T0 += D[d][0];
        M1 = std::max<u64>(M1, D[d][1]);
        M2 = std::max<u64>(M2, D[d][2]);
    }
    const u64 total = std::max<u64>(T0, 1) * M1 * M2;
    // Entries of this rank: compact index and local field index.
    std::vector<u64> cidx, lidx;
    const u64 n1n2 = dims[1] * dims[2];
    for (int d = 0; d < 3; d++)
        for (u64 k0 = 0; k0 < cnt[d][0]; k0++)
            for (u64 k1 = 0; k1 < cnt[d][1]; k1++)
                for (u64 k2 = 0; k2 < cnt[d][2]; k2++)
                    for (int o = 0; o < 7; o++) {
                        const u64 kk[3] = {k0, k1, k2};
                        int64_t g[3];
                        u64 c[3];
                        for (int a = 0; a < 3; a++) {
                            g[a] = (int64_t)(gb[d].lo[a] + kk[a] * gb[d].step[a]) + (a == d ? o - 3 : 0);
                            c[a] = a == d ? 7 * kk[a] + o : kk[a];
                        }
                        if (g[0] < (int64_t)own_lo || g[0] > (int64_t)own_hi) continue;
                        if (g[d] < 0 || g[d] >= (int64_t)dims[d]) continue;
                        cidx.push_back(((off0[d] + c[0]) * M1 + c[1]) * M2 + c[2]);
                        lidx.push_back(((u64)g[0] - local_first_plane) * n1n2 + (u64)g[1] * dims[2] + (u64)g[2]);
                    }
    cudaStream_t st = ctx->stream;
    std::vector<float> vals(cidx.size());
    if (!cidx.empty()) {
        CK(ctx->slab_idx.reserve(lidx.size() * sizeof(u64)));
        CK(ctx->slab_val.reserve(lidx.size() * sizeof(float)));
        CK(cudaMemcpyAsync(ctx->slab_idx.p, lidx.data(), lidx.size() * sizeof(u64), cudaMemcpyHostToDevice, st));
        CK(launch_gather(d_local, ctx->slab_idx.as<u64>(), lidx.size(), ctx->slab_val.as<float>(), st));
        CK(cudaMemcpyAsync(vals.data(), ctx->slab_val.p, vals.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    (void)ldims;
    // Exchange: every rank's (count, then indices and values padded to the largest count).
    const int R = cm.c->size;
    u64 mine = cidx.size();
    std::vector<u64> counts(R);
    int rc = cm.allgather(&mine, sizeof(u64), counts.data());
    if (rc) return rc;
    const u64 cmax = *std::max_element(counts.begin(), counts.end());
    std::vector<u64> sidx(cmax, 0), ridx(cmax * R);
    std::vector<float> sval(cmax, 0.0f), rval(cmax * R);
    std::copy(cidx.begin(), cidx.end(), sidx.begin());
    std::copy(vals.begin(), vals.end(), sval.begin());
    if ((rc = cm.allgather(sidx.data(), cmax * sizeof(u64), ridx.data()))) return rc;
    if ((rc = cm.allgather(sval.data(), cmax * sizeof(float), rval.data()))) return rc;
    std::vector<float> cmp(total, 0.0f);
    for (int r = 0; r < R; r++)
        for (u64 k = 0; k < counts[r]; k++) {
            const u64 ci = ridx[(u64)r * cmax + k];
            if (ci >= total) return fail(ctx, ASZ_E_COMM, "slab: default-slope sample index out of range");
            cmp[ci] = rval[(u64)r * cmax + k];
        }
    CK(ctx->slab_cmp.reserve(total * sizeof(float)));
    CK(cudaMemcpyAsync(ctx->slab_cmp.p, cmp.data(), total * sizeof(float), cudaMemcpyHostToDevice, st));
    SampleBox cb[3];
    const uint64_t cdims[3] = {std::max<u64>(T0, 1), M1, M2};
    for (int d = 0; d < 3; d++) {
        cb[d] = gb[d];
        for (int a = 0; a < 3; a++) {
            const u64 base = a == 0 ? off0[d] : 0;
            cb[d].lo[a] = base + (a == d ? 3 : 0);
            cb[d].step[a] = a == d ? 7 : 1;
            cb[d].hi[a] = cnt[d][a] ? cb[d].lo[a] + (cnt[d][a] - 1) * cb[d].step[a] + 1 : cb[d].lo[a];
        }
        cb[d].dist = d == 0 ? M1 * M2 : d == 1 ? M2 : 1;
    }
    return default_slope_on(ctx, ctx->slab_cmp.as<float>(), cdims, cb, p, abs_eb, mn, mx, cand, slope, max_invalid, reason);
}

}  // namespace

namespace {

// Appends `bits` bits of src (LSB-first, zero past the last bit) to dst at bit offset off; dst is
// zero from off on and holds dst_len bytes.
void bit_append(uint8_t *dst, u64 dst_len, u64 off, const uint8_t *src, u64 bits) {
    const u64 nb = (bits + 7) / 8;
    const unsigned sh = (unsigned)(off & 7);
    const u64 b0 = off / 8;
    for (u64 i = 0; i < nb && b0 + i < dst_len; i++) {
        dst[b0 + i] |= (uint8_t)(src[i] << sh);
        if (sh && b0 + i + 1 < dst_len) dst[b0 + i + 1] |= (uint8_t)(src[i] >> (8 - sh));
    }
}

// The entropy stage of a slab (compress.tpp:233-291 over the whole field): global ranges, counts
// and histograms from every rank's, the same codes on every rank, each rank's pieces encoded on
// its device, and on rank 0 the pieces concatenated bit-exactly in rank order (each stream's
// pieces are consecutive symbols of it) and the stream assembled.
int slab_encode(asz_ctx *ctx, SlabComm &cm, const CoreOut &co, const Plan &plan, const asz_params &p, float mn, float mx,
                bool quintic, asz_report &R) {
    cudaStream_t st = ctx->stream;
    MiscLayout *dm = ctx->misc.as<MiscLayout>();
    const Geometry &G = co.G;
    const u64 L = plan.pred.size(), NS = L + 2;
    const int rank = cm.c->rank, nr = cm.c->size;
    auto t_huff = clk::now();
    // Per stream (0: t codes, 1..L+1: QB streams): local count, global range and count.
    std::vector<StreamOut> so(NS);
    std::vector<u64> local(NS), global(NS);
    std::vector<int32_t> rng(2 * (L + 1));
    CK(cudaMemcpyAsync(rng.data(), dm->qb_range, rng.size() * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<int32_t> rlo(L + 1), rhi(L + 1);
    for (u64 s = 0; s <= L; s++) {
        rlo[s] = rng[2 * s];
        rhi[s] = rng[2 * s + 1];
    }
    int rc;
    if ((rc = cm.allreduce(rlo.data(), L + 1, 2, 1))) return rc;
    if ((rc = cm.allreduce(rhi.data(), L + 1, 2, 2))) return rc;
    local[0] = G.nblocks * L;
    for (u64 s = 0; s <= L; s++) local[s + 1] = co.qb_len[s];
    global = local;
    if ((rc = cm.allreduce(global.data(), NS, 1, 0))) return rc;
    {
        const float t_default = 4.0f / 16;
        const float tv[6] = {t_default, 1.0f / 16, 1.0f / 4, 9.0f / 32, 5.0f / 16, 11.0f / 32};
        int64_t lo = INT64_MAX, hi = INT64_MIN;
        for (float t : tv) {
            const int64_t c = host_lround_f(t * (float)p.t_precision);
            lo = std::min(lo, c);
            hi = std::max(hi, c);
        }
        so[0].lo = lo;
        so[0].hi = hi;
    }
    for (u64 s = 0; s <= L; s++) {
        so[s + 1].lo = rlo[s];
        so[s + 1].hi = rhi[s];
    }
    u64 hist_total = 0;
    for (u64 s = 0; s < NS; s++) {
        so[s].count = global[s];
        if (!global[s]) continue;
        const u64 range = (u64)(so[s].hi - so[s].lo) + 1;
        if (range > (1ull << 27)) return fail(ctx, ASZ_E_UNSUPPORTED, "QB range too wide for the dense histogram");
        so[s].hist_off = hist_total;
        hist_total += range;
    }
    CK(ctx->hist.reserve(std::max<u64>(hist_total, 1) * 8));
    CK(cudaMemsetAsync(ctx->hist.p, 0, std::max<u64>(hist_total, 1) * 8, st));
    unsigned long long *d_hist = ctx->hist.as<unsigned long long>();
    for (u64 s = 0; s < NS; s++) {
        if (!global[s] || !local[s]) continue;
        const u64 range = (u64)(so[s].hi - so[s].lo) + 1;
        if (s == 0) CK(launch_histogram<int64_t>(ctx->tint.as<int64_t>(), local[0], so[0].lo, range, d_hist + so[0].hist_off, st));
        else
            CK(launch_histogram<int32_t>(ctx->qb.as<int32_t>() + co.qb_off[s - 1], local[s], so[s].lo, range,
                                         d_hist + so[s].hist_off, st));
    }
    std::vector<u64> lhist(hist_total), ghist;
    if (hist_total) CK(cudaMemcpyAsync(lhist.data(), d_hist, hist_total * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    ghist = lhist;
    if ((rc = cm.allreduce(ghist.data(), hist_total, 1, 0))) return rc;
    // The same codes on every rank, and this rank's payload bits per stream.
    std::vector<u64> lbits(NS, 0);
    for (u64 s = 0; s < NS; s++) {
        StreamOut &o = so[s];
        if (!o.count) continue;
        const u64 range = (u64)(o.hi - o.lo) + 1;
        const u64 *h = ghist.data() + o.hist_off;
        u64 a0 = 0, b0 = range;
        while (a0 < b0 && h[a0] == 0) a0++;
        while (b0 > a0 && h[b0 - 1] == 0) b0--;
        std::vector<u64> hh(h + a0, h + b0);
        std::string err;
        if (!build_code(hh, o.lo + (int64_t)a0, o.lo + (int64_t)b0 - 1, o.count, s == 0, o.code, err))
            return fail(ctx, ASZ_E_UNSUPPORTED, err);
        const int64_t old_lo = o.lo;
        o.lo += (int64_t)a0;
        if (o.code.maxval == 1) continue;
        const u64 *lh = lhist.data() + o.hist_off;
        for (u64 k = a0; k < b0; k++)
            if (lh[k]) lbits[s] += lh[k] * o.code.table[(u64)(old_lo + (int64_t)k - o.code.offset)].len;
    }
    // Encode this rank's pieces.
    u64 code_total = 0, words_total = 0;
    std::vector<u64> code_off(NS, 0), word_off(NS, 0);
    for (u64 s = 0; s < NS; s++) {
        if (!so[s].count) continue;
        code_off[s] = code_total;
        code_total += so[s].code.table.size();
        word_off[s] = words_total;
        words_total += (lbits[s] + 31) / 32 + 2;
    }
    std::vector<CodeEntry> codes(std::max<u64>(code_total, 1));
    for (u64 s = 0; s < NS; s++)
        if (so[s].count) std::copy(so[s].code.table.begin(), so[s].code.table.end(), codes.begin() + code_off[s]);
    CK(ctx->codes.reserve(codes.size() * sizeof(CodeEntry)));
    CK(cudaMemcpyAsync(ctx->codes.p, codes.data(), codes.size() * sizeof(CodeEntry), cudaMemcpyHostToDevice, st));
    CK(ctx->payload.reserve(std::max<u64>(words_total, 1) * 4));
    CK(cudaMemsetAsync(ctx->payload.p, 0, std::max<u64>(words_total, 1) * 4, st));
    uint32_t *d_pay = ctx->payload.as<uint32_t>();
    CodeEntry *d_codes = ctx->codes.as<CodeEntry>();
    u64 enc_err[2] = {0, 0};  // the encoder's error words, read back with the pieces
    {
        std::vector<EncStream> es[2];
        std::vector<u64> toff[2] = {{0}, {0}};
        for (u64 s = 0; s < NS; s++) {
            if (!so[s].count || so[s].code.maxval == 1 || !local[s]) continue;
            const int k = s == 0 ? 1 : 0;
            const void *sym = s == 0 ? (const void *)ctx->tint.as<int64_t>() : (const void *)(ctx->qb.as<int32_t>() + co.qb_off[s - 1]);
            es[k].push_back(EncStream{sym, local[s], so[s].lo, d_codes + code_off[s], d_pay + word_off[s]});
            const u64 tile = k ? enc_tile<int64_t>() : enc_tile<int32_t>();
            toff[k].push_back(toff[k].back() + (local[s] + tile - 1) / tile);
        }
        u64 off[2][4], bytes = 0;
        auto place = [&](u64 n) {
            const u64 o = bytes;
            bytes += (n + 15) / 16 * 16;
            return o;
        };
        size_t tmp_bytes = 0;
        for (int k = 0; k < 2; k++) {
            const u64 nt = toff[k].back();
            off[k][0] = place(es[k].size() * sizeof(EncStream));
            off[k][1] = place(toff[k].size() * sizeof(u64));
            off[k][2] = place((nt + 1) * sizeof(u64));
            off[k][3] = place((nt + 1) * sizeof(u64));
            size_t tb = 0;
            if (k == 0) CK(launch_encode_tiles<int32_t>(nullptr, 0, nullptr, nt, nullptr, nullptr, nullptr, tb, st));
            else CK(launch_encode_tiles<int64_t>(nullptr, 0, nullptr, nt, nullptr, nullptr, nullptr, tb, st));
            tmp_bytes = std::max(tmp_bytes, tb);
        }
        CK(ctx->enc.reserve(std::max<u64>(bytes, 16)));
        CK(ctx->cubtmp.reserve(std::max<size_t>(tmp_bytes, 16)));
        uint8_t *eb = ctx->enc.as<uint8_t>();
        for (int k = 0; k < 2; k++) {
            const u64 nt = toff[k].back();
            if (!nt) continue;
            CK(cudaMemcpyAsync(eb + off[k][0], es[k].data(), es[k].size() * sizeof(EncStream), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(eb + off[k][1], toff[k].data(), toff[k].size() * sizeof(u64), cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(eb + off[k][2] + nt * sizeof(u64), 0, sizeof(u64), st));
            size_t tb = ctx->cubtmp.cap;
            const EncStream *E = (const EncStream *)(eb + off[k][0]);
            const u64 *T = (const u64 *)(eb + off[k][1]);
            u64 *tbits = (u64 *)(eb + off[k][2]), *tscan = (u64 *)(eb + off[k][3]);
            if (k == 0) CK(launch_encode_tiles<int32_t>(E, (uint32_t)es[k].size(), T, nt, tbits, tscan, ctx->cubtmp.p, tb, st));
            else CK(launch_encode_tiles<int64_t>(E, (uint32_t)es[k].size(), T, nt, tbits, tscan, ctx->cubtmp.p, tb, st));
            CK(cudaMemcpyAsync(&enc_err[k], tscan, sizeof(u64), cudaMemcpyDeviceToHost, st));
        }
    }
    // This rank's pieces, back on the host: per stream its bits, then the bytes.
    u64 piece_bytes = 0;
    for (u64 s = 0; s < NS; s++) piece_bytes += (lbits[s] + 7) / 8;
    std::vector<uint8_t> piece(std::max<u64>(piece_bytes, 1));
    {
        u64 w = 0;
        for (u64 s = 0; s < NS; s++) {
            const u64 nb = (lbits[s] + 7) / 8;
            if (nb) CK(cudaMemcpyAsync(piece.data() + w, d_pay + word_off[s], nb, cudaMemcpyDeviceToHost, st));
            w += nb;
        }
        CK(cudaStreamSynchronize(st));
        if (enc_err[0] | enc_err[1])
            return fail(ctx, ASZ_E_DEVICE, "Huffman encoder: a tile's wait for the tiles before it timed out");
    }
    auto t_d2h = clk::now();
    if (rank != 0) {
        if ((rc = cm.send(lbits.data(), NS * sizeof(u64), 0))) return rc;
        if (piece_bytes && (rc = cm.send(piece.data(), piece_bytes, 0))) return rc;
        R.huffman_s = secs(t_huff, clk::now());
        return ASZ_OK;
    }
    // Rank 0: every stream's payload from the ranks' pieces, then the stream (compress.tpp:233-291).
    std::vector<std::vector<uint8_t>> pay(NS);
    std::vector<u64> at(NS, 0);
    for (u64 s = 0; s < NS; s++)
        if (so[s].count && so[s].code.maxval != 1) pay[s].assign((so[s].code.bits + 7) / 8, 0);
    for (int r = 0; r < nr; r++) {
        std::vector<u64> bits(NS);
        std::vector<uint8_t> in;
        if (r == 0) {
            bits = lbits;
            in = piece;
        } else {
            if ((rc = cm.recv(bits.data(), NS * sizeof(u64), r))) return rc;
            u64 nbytes = 0;
            for (u64 s = 0; s < NS; s++) nbytes += (bits[s] + 7) / 8;
            in.assign(std::max<u64>(nbytes, 1), 0);
            if (nbytes && (rc = cm.recv(in.data(), nbytes, r))) return rc;
        }
        u64 rd = 0;
        for (u64 s = 0; s < NS; s++) {
            const u64 nb = (bits[s] + 7) / 8;
            if (bits[s]) {
                if (pay[s].empty() || at[s] + bits[s] > so[s].code.bits)
                    return fail(ctx, ASZ_E_COMM, "slab: a rank's payload does not fit its stream");
                bit_append(pay[s].data(), pay[s].size(), at[s], in.data() + rd, bits[s]);
                at[s] += bits[s];
            }
            rd += nb;
        }
    }
    for (u64 s = 0; s < NS; s++)
        if (so[s].count && so[s].code.maxval != 1 && at[s] != so[s].code.bits)
            return fail(ctx, ASZ_E_COMM, "slab: the ranks' payload bits do not add up to the stream's");
    u64 total_len = 9 + 2 * L;
    for (auto &o : so) total_len += 8 + (o.count ? o.code.save_size() + o.code.encode_size() : 0);
    PinnedBuf &pb = ctx->pre_zstd;
    CK(pb.reserve(total_len));
    pb.len = total_len;
    uint8_t *w = pb.p;
    std::memcpy(w, &mn, 4);
    std::memcpy(w + 4, &mx, 4);
    w[8] = (uint8_t)(L | 0x40 | (quintic ? 0x80 : 0));
    w += 9;
    for (u64 l = 0; l < L; l++) {
        w[0] = (uint8_t)plan.pred[l][5];
        w[1] = (uint8_t)plan.pred[l][9];
        w += 2;
    }
    for (u64 s = 0; s < NS; s++) {
        const StreamOut &o = so[s];
        for (int i = 0; i < 8; i++) w[i] = (uint8_t)(o.count >> (8 * i));
        w += 8;
        if (!o.count) continue;
        write_tree(o.code, w);
        w += o.code.save_size();
        write_len_word(o.code, w);
        w += 8;
        if (o.code.maxval != 1) {
            std::memcpy(w, pay[s].data(), pay[s].size());
            w += pay[s].size();
        }
    }
    if ((u64)(w - pb.p) != total_len) return fail(ctx, ASZ_E_DEVICE, "Huffman encoded size mismatch");
    R.d2h_s = secs(t_d2h, clk::now());
    R.huffman_s = secs(t_huff, clk::now());
    return ASZ_OK;
}

}  // namespace

extern "C" int asz_slab_planes(const uint64_t dims[3], const asz_params *pp, const char *plan_text, uint64_t block_begin,
                               uint64_t block_end, uint64_t *plane_begin, uint64_t *plane_count, uint64_t *blocks0) {
    if (!dims || !plan_text || !plane_begin || !plane_count) return ASZ_E_ARG;
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    if (p.block_pivot_ratio == 0) return ASZ_E_ARG;
    Plan plan;
    std::string err;
    if (!parse_plan(plan_text, plan, err)) return ASZ_E_ARG;
    SlabLayout S;
    const int rc = slab_layout(dims, plan, p, block_begin, block_end, S, err);
    if (rc) return rc;
    *plane_begin = S.plane_begin;
    *plane_count = S.plane_count;
    if (blocks0) *blocks0 = S.blocks0;
    return ASZ_OK;
}

extern "C" int asz_compress_slab(asz_ctx *ctx, const asz_comm *comm, const float *planes, int on_device,
                                 const uint64_t dims[3], uint64_t block_begin, uint64_t block_end, float rel_eb,
                                 const asz_params *pp, const char *plan_text, uint8_t **out, size_t *out_len,
                                 asz_report *rep) {
    if (!ctx) return ASZ_E_ARG;
    auto t_start = clk::now();
    const uint64_t launches0 = launch_counter();
    ctx->err.clear();
    ctx->have_last = false;
    if (!comm || !planes || !out || !out_len || !plan_text) return fail(ctx, ASZ_E_ARG, "null argument");
    if (comm->size < 1 || comm->rank < 0 || comm->rank >= comm->size ||
        (comm->size > 1 && (!comm->allreduce || !comm->allgather || !comm->send || !comm->recv)))
        return fail(ctx, ASZ_E_ARG, "invalid communicator");
    *out = nullptr;
    *out_len = 0;
    asz_params p;
    if (pp) p = *pp;
    else asz_default_params(&p);
    SlabComm cm{ctx, comm};
    // Argument checks run on every rank before the first exchange, and their outcome is agreed.
    int rc = validate(ctx, p, true);
    if (!rc) rc = validate_dims(ctx, dims, rel_eb);
    Plan plan;
    std::string perr;
    if (!rc && !parse_plan(plan_text, plan, perr)) rc = fail(ctx, ASZ_E_ARG, perr);
    if (!rc && plan.pred.size() > 63) rc = fail(ctx, ASZ_E_ARG, "predictor plan cannot contain more than 63 layers");
    if (!rc && p.predictor_family == ASZ_FAMILY_AUTO)
        rc = fail(ctx, ASZ_E_ARG, "a slab needs the predictor family (the selector samples the whole field)");
    SlabLayout S;
    if (!rc) {
        rc = slab_layout(dims, plan, p, block_begin, block_end, S, perr);
        if (rc) rc = fail(ctx, rc, perr);
    }
    // Blocks of consecutive ranks must follow each other: rank r's first block is rank r-1's end.
    std::vector<u64> bounds(2 * comm->size);
    {
        const u64 mine[2] = {block_begin, block_end};
        const int e = cm.allgather(mine, sizeof(mine), bounds.data());
        if (e) return e;
        if (!rc) {
            if (bounds[0] != 0 || bounds[2 * comm->size - 1] != S.blocks0)
                rc = fail(ctx, ASZ_E_ARG, "the ranks' slabs must cover the axis-0 blocks from the first to the last");
            for (int r = 1; r < comm->size && !rc; r++)
                if (bounds[2 * r] != bounds[2 * r - 1]) rc = fail(ctx, ASZ_E_ARG, "the ranks' slabs must follow each other");
        }
    }
    if (!rc && cudaSetDevice(ctx->device) != cudaSuccess) rc = fail(ctx, ASZ_E_CUDA, "cudaSetDevice");
    if ((rc = cm.agree_ok(rc))) return rc;
    const bool quintic = p.predictor_family == ASZ_FAMILY_QUINTIC;
    const u64 L = plan.pred.size();
    const u64 n1n2 = dims[1] * dims[2];
    const int rank = comm->rank, nr = comm->size;
    cudaStream_t st = ctx->stream;
    asz_report R{};
    // The frame: [halo | face | owned planes] (rank 0: its planes from plane 0).
    const u64 first_plane = rank == 0 || block_begin == 0 ? 0 : S.s0 - S.halo;  // global plane of frame plane 0
    const u64 own_off = block_begin == 0 ? 0 : S.halo + 1;                      // frame plane of the first owned plane
    const uint64_t ldims[3] = {S.local0, dims[1], dims[2]};
    const uint64_t origin[3] = {block_begin == 0 ? 0 : S.halo, 0, 0};
    auto t0 = clk::now();
    rc = ASZ_OK;
    {
        const cudaError_t e1 = ctx->misc.reserve(sizeof(MiscLayout));
        const cudaError_t e2 = ctx->in.reserve(S.local0 * n1n2 * sizeof(float));
        if (e1 != cudaSuccess || e2 != cudaSuccess) rc = fail(ctx, ASZ_E_CUDA, "slab: device allocation failed");
    }
    float *d_local = ctx->in.as<float>();
    if (!rc && own_off) {
        const cudaError_t e = cudaMemsetAsync(d_local, 0, own_off * n1n2 * sizeof(float), st);
        if (e != cudaSuccess) rc = fail(ctx, ASZ_E_CUDA, cudaGetErrorString(e));
    }
    if (!rc) {
        const cudaError_t e = cudaMemcpyAsync(d_local + own_off * n1n2, planes, S.plane_count * n1n2 * sizeof(float),
                                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) rc = fail(ctx, ASZ_E_CUDA, cudaGetErrorString(e));
        else if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(ctx, ASZ_E_CUDA, "slab: input copy failed");
    }
    R.h2d_s = secs(t0, clk::now());
    // Data range over the owned planes, then over the field.
    float mn = 0, mx = 0, gmn = 0, gmx = 0;
    auto t_range = clk::now();
    if (!rc) rc = compute_range(ctx, d_local + own_off * n1n2, S.plane_count * n1n2, mn, mx);
    if ((rc = cm.agree_ok(rc))) return rc;
    if ((rc = slab_range(cm, mn, mx, gmn, gmx))) return rc;
    R.data_range_s = secs(t_range, clk::now());
    if (gmn == gmx) return fail(ctx, ASZ_E_DATA, "max_val==min_val");
    const float abs_eb = rel_eb * (gmx - gmn);
    // Default slope from the whole field's samples.
    auto t_slope = clk::now();
    const std::vector<float> cand = candidate_t(p);
    float slope = 0, max_invalid = 0;
    int reason = 0;
    rc = slab_slope(ctx, cm, d_local, ldims, first_plane, S.plane_begin, S.last, dims, p, abs_eb, gmn, gmx, cand, slope,
                    max_invalid, reason);
    if ((rc = cm.agree_ok(rc))) return rc;
    R.default_slope_s = secs(t_slope, clk::now());
    // Rounds on the frame; before each axis-0 round, the reconstructed planes below each slab
    // come from the rank below (received first, then this rank's top planes go up).
    auto t_core = clk::now();
    SlabGeom sg{block_end - block_begin, block_begin > 0};
    CoreOut co;
    CoreArgs ca{d_local, ldims, origin, &plan, &p, quintic, false, nullptr, gmn, gmx, abs_eb, slope, nullptr, 0};
    ca.slab = &sg;
    ca.before_round = [&](u64 l) -> int {
        if (plan.dir[l] != 0 || nr == 1) return ASZ_OK;
        float *rec = ctx->rec.as<float>();
        int e;
        if (rank > 0) {
            std::vector<float> h((S.halo + 1) * n1n2);
            if ((e = cm.recv(h.data(), h.size() * sizeof(float), rank - 1))) return e;
            CK(cudaMemcpyAsync(rec, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
        if (rank < nr - 1) {
            const u64 up = std::min<u64>(S.last, 2 * S.ps0);  // the halo of the rank above
            std::vector<float> h((up + 1) * n1n2);
            CK(cudaMemcpyAsync(h.data(), rec + (S.last - up - first_plane) * n1n2, h.size() * sizeof(float),
                               cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if ((e = cm.send(h.data(), h.size() * sizeof(float), rank + 1))) return e;
        }
        return ASZ_OK;
    };
    ca.agree = [&](bool &changed) -> int {
        int32_t c = changed ? 1 : 0;
        const int e = cm.allreduce(&c, 1, 2, 2);
        changed = c != 0;
        return e;
    };
    rc = run_core(ctx, ca, co, R);
    if ((rc = cm.agree_ok(rc))) return rc;
    rc = slab_encode(ctx, cm, co, plan, p, gmn, gmx, quintic, R);
    if ((rc = cm.agree_ok(rc))) return rc;
    R.core_s = secs(t_core, clk::now());
    // zstd level 3 on rank 0 (compress.tpp:294-299).
    u64 lens[2] = {0, 0};
    if (rank == 0) {
        auto t_z = clk::now();
        PinnedBuf &pb = ctx->pre_zstd;
        const size_t bound = ZSTD_compressBound(pb.len);
        uint8_t *z = out_alloc(bound);
        size_t zl = 0;
        if (!z) rc = fail(ctx, ASZ_E_DATA, "out of host memory");
        else {
            zl = zstd3(ctx, z, bound, pb.p, pb.len);
            if (ZSTD_isError(zl)) {
                out_release(z);
                rc = fail(ctx, ASZ_E_DATA, std::string("ZSTD_compress: ") + ZSTD_getErrorName(zl));
            } else {
                *out = z;
                *out_len = zl;
                lens[0] = pb.len;
                lens[1] = zl;
            }
        }
        R.zstd_s = secs(t_z, clk::now());
    }
    {
        const int e = cm.agree_ok(rc);
        if (e) {
            if (*out) out_release(*out);
            *out = nullptr;
            *out_len = 0;
            return e;
        }
    }
    // The whole field's figures on every rank.
    u64 sums[8] = {lens[0], lens[1], R.t_fallback_count, R.ambiguous_decisions, R.exact_groups, R.serial_groups,
                   R.exact_undecided, R.wide_groups};
    if ((rc = cm.allreduce(sums, 8, 1, 0))) return rc;
    if (rep) {
        R.min_val = gmn;
        R.max_val = gmx;
        R.abs_eb = abs_eb;
        R.default_slope = slope;
        R.slope_max_invalid_ratio = max_invalid;
        R.slope_fallback_reason = reason;
        R.pre_zstd_len = sums[0];
        R.asz_len = sums[1];
        R.t_fallback_count = sums[2];
        R.ambiguous_decisions = sums[3];
        R.exact_groups = sums[4];
        R.serial_groups = sums[5];
        R.exact_undecided = sums[6];
        R.wide_groups = sums[7];
        R.layer_num = L;
        R.quintic = quintic ? 1 : 0;
        R.pivot_stride[0] = (uint32_t)co.G.fg.pivot_stride[0];
        R.block_shape[0] = (uint32_t)co.G.fg.block_shape[0];
        R.block_num[0] = (uint32_t)S.blocks0;
        for (int a = 1; a < 3; a++) {
            R.pivot_stride[a] = (uint32_t)co.G.fg.pivot_stride[a];
            R.block_shape[a] = (uint32_t)co.G.fg.block_shape[a];
            R.block_num[a] = (uint32_t)co.G.fg.block_num[a];
        }
        std::string pl;
        for (u64 l = 0; l < L; l++) pl += (l ? "," : "") + plan.pred[l];
        std::snprintf(R.plan, sizeof(R.plan), "%s", pl.c_str());
        const u64 N = dims[0] * n1n2;
        if (sums[1]) {
            R.cr = (float)N * sizeof(float) / (float)sums[1];
            R.br = 8 * sizeof(float) / R.cr;
        }
        R.kernel_launches = launch_counter() - launches0;
        R.total_s = secs(t_start, clk::now());
        *rep = R;
    }
    return ASZ_OK;
}

namespace asz::host {

cudaStream_t ctx_stream(asz_ctx *c) { return c->stream; }

int ctx_fail(asz_ctx *c, int code, const std::string &m) { return fail(c, code, m); }

int ctx_range(asz_ctx *ctx, const float *d_in, uint64_t n, bool first_max, float &mn, float &mx) {
    CK(ctx->misc.reserve(sizeof(MiscLayout)));
    return compute_range(ctx, d_in, n, mn, mx, first_max);
}

int ctx_upload(asz_ctx *ctx, const float *in, uint64_t n, const float **d_in) {
    CK(ctx->in.reserve(n * sizeof(float)));
    CK(cudaMemcpyAsync(ctx->in.p, in, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    *d_in = ctx->in.as<float>();
    return ASZ_OK;
}

void *&ctx_sweep_state(asz_ctx *c) { return c->sweep; }

}  // namespace asz::host
