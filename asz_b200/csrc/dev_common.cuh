// Shared device helpers: the reference's floating-point steps spelled with rounding-explicit
// intrinsics, plus the plan geometry every kernel uses.
//
// Every operation that the reference performs is written with a _rn intrinsic or an explicit
// fused multiply-add, and the library is compiled with -fmad=false, so nvcc neither contracts
// nor reassociates. The forms follow the code GCC 13.3 emits for the reference at
// -Ofast -mfma (c_codes/CMakeLists.txt:12); each use site cites the source line it restates.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define ASZ_HD __host__ __device__ __forceinline__
#else
#define ASZ_HD inline
#endif

namespace asz {

#ifdef __CUDACC__
// llround(float) as expanded under -Ofast: truncate x + copysign(0.49999997f, x).
__device__ __forceinline__ int64_t lround_f(float x) {
    float h = copysignf(0x1.fffffep-2f, x);
    return __float2ll_rz(__fadd_rn(x, h));
}
// llround(double): truncate x + copysign(0.49999999999999994, x).
__device__ __forceinline__ int64_t lround_d(double x) {
    double h = copysign(0x1.fffffffffffffp-2, x);
    return __double2ll_rz(__dadd_rn(x, h));
}
#endif

// Quintic 1D6R weights (c_codes/asz_core/asz_param.hpp:72-74): a=3/256, b=-25/256, inner=0.5-a-b.
constexpr double kQuinticA = 3.0 / 256, kQuinticB = -25.0 / 256, kQuinticI = 0.5 - 3.0 / 256 + 25.0 / 256;

// One prediction round of the plan, in global (not per-block) terms. Host-filled.
struct RoundGeom {
    int32_t dir;             // interpolation axis of the round
    int32_t order;           // QB serialisation order: 0 "120", 1 "021", 2 "012"
    uint64_t stride[3];      // lattice strides at the start of the round
    uint64_t hs;             // stride[dir]/2
    uint64_t dist;           // linear distance of one half stride along dir
    uint64_t tcount[3];      // targets per axis (global lattice)
    uint64_t targets;        // product of tcount
    float eb;                // layer error bound (compress.tpp:194)
    float slope;             // layer default slope (compress.tpp:195)
    float stat_eb;           // eb * stat_eb_ratio (compress.tpp:118)
    float neg_2_stat_eb;     // 0.5f / stat_eb (compress.tpp:120 as emitted)
    uint32_t axis_off[3];    // offset of this round's per-block count/prefix arrays, per axis
    uint64_t total[3];       // sum of per-block counts along each axis
    uint64_t qb_total;       // QBs of this round (stream length)
    uint32_t fallback_all;   // 1 when every block falls back to the default t
    uint64_t ent_off[3];     // offset of this round's per-axis AxisEntry tables, per axis
};

// Stencil forms of one target along the round axis (compress.tpp:7-34), decided by its index i,
// the half stride and the block's right bound.
enum StencilCase : uint32_t {
    kStencilCubic = 0,    // interior 1D4R with the block's t
    kStencilQuintic = 1,  // interior 1D6R
    kStencilLeft1 = 2,    // i <= hs, only x-1 inside
    kStencilLeft2 = 3,    // i <= hs, x-1 and x1
    kStencilLeft3 = 4,    // i <= hs, x-1, x1, x3
    kStencilRight1 = 5,   // i + hs >= right
    kStencilRight2 = 6,   // i + 3hs >= right
};

// What a round's target geometry needs along one axis, for lattice index k on that axis: the
// coordinate, the owning block, the index inside the block's QB box, the box extent and the
// exclusive prefix of box extents before the block. Along the round axis, also the stencil case.
struct AxisEntry {
    uint32_t ii, bb, jj, cc;
    uint64_t pre;
    uint32_t stencil, pad;
};

struct FieldGeom {
    uint64_t n[3];
    // Frame origin: blocks and the pivot lattice start here (0 for a whole field). Positions below
    // it are a read-only halo that keeps its input values (the predictor-family probe's local
    // contexts, predictor_family.tpp:40-60).
    uint64_t origin[3];
    uint64_t block_shape[3];
    uint64_t block_num[3];
    uint64_t pivot_stride[3];
    uint32_t layer_num;
    int32_t quintic;
    int32_t t_precision;
};

// The pivot lattice (compress.tpp:162-175) and its quantisation step.
struct PivotGeom {
    uint64_t cnt[3];      // pivots per axis
    uint64_t stride[3];
    uint64_t origin[3];   // first pivot (the frame origin)
    uint64_t n1n2, n2;
    double rp;            // 0.5 / (double)pivot_eb
    double peb2;          // 2 * (double)pivot_eb
};

// ---- Batches: several fields compressed with the same plan, one launch per round for all. ----

struct AmbiguousRecord;
struct ClassInfo;

// Per-field counters of a batch (device): error bits, fallbacks, ambiguous decisions, and the
// fast path's hand-off reasons (as asz_report's exact_window, exact_undecided, wide_groups).
struct BatchCounters {
    uint32_t err, fb, amb_count, why[3];
};

// One field of a batch, as the batched kernels see it (device copy).
struct BatchField {
    FieldGeom fg;
    PivotGeom pg;
    const RoundGeom *rounds;        // layer_num rounds
    const AxisEntry *ent;           // per-axis target tables of all rounds
    const ClassInfo *classes;       // 27 per round
    const float *in;                // original values
    float *rec, *tval;              // reconstruction, this round's t per block
    int64_t *tint;                  // t codes, block-major
    int32_t *qb;                    // QB streams, pivots first
    const uint64_t *qoff;           // stream offsets (layer_num + 1)
    int32_t *qb_range;              // [min, max] per stream
    float *proxies;                 // exact path's proxies, 10 per (block, round)
    AmbiguousRecord *amb;           // ambiguous decisions for the host replay
    uint32_t amb_cap;
    BatchCounters *cnt;
    float R2;                       // (max - min)^2
    uint32_t tpl_log2[64];          // threads per target line (log2), per round
};

#ifdef __CUDACC__
// Field of global item `gi` given the exclusive prefix `off` (nf + 1 entries) of per-field counts.
__device__ __forceinline__ uint32_t field_of(const uint64_t *off, uint32_t nf, uint64_t gi) {
    uint32_t lo = 0, hi = nf;  // off[lo] <= gi < off[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= gi) lo = mid;
        else hi = mid;
    }
    return lo;
}
#endif

ASZ_HD uint64_t owner_block(uint64_t i, uint64_t shape) { return i == 0 ? 0 : (i - 1) / shape; }

// Block of coordinate i in a frame starting at h: a block's upper face belongs to it, its lower face
// to the block below (only the frame's first face at h == 0 starts block 0).
ASZ_HD uint64_t owner_block_at(uint64_t i, uint64_t h, uint64_t shape) { return i <= h ? 0 : (i - h - 1) / shape; }

}  // namespace asz
