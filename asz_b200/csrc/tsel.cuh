// Per-(block, round) coefficient selection and the default-slope proxy: shared declarations.
#pragma once
#include <cstdint>

#include "dev_common.cuh"

namespace asz {

// libstdc++ unordered_map growth (GCC 13 _Prime_rehash_policy, max_load_factor 1): before the
// k-th insertion (1-based) listed here the table is rehashed to the listed bucket count.
// Measured through bucket_count() on this toolchain; the same for every key type.
constexpr int kSchedLen = 21;
constexpr uint64_t kSchedAt[kSchedLen] = {1, 14, 30, 60, 128, 258, 542, 1110, 2358, 5088, 10274, 20754,
                                          42044, 85230, 172934, 351062, 712698, 1447154, 2938680,
                                          5967348, 12117690};
constexpr uint64_t kSchedBkt[kSchedLen] = {13, 29, 59, 127, 257, 541, 1109, 2357, 5087, 10273, 20753,
                                           42043, 85229, 172933, 351061, 712697, 1447153, 2938679,
                                           5967347, 12117689, 24607243};


// One AB map: the sample box of get_AB_map (c_codes/asz_core/get_AB_map.tpp:7-24) after
// sampling_stride is applied. lo/hi bound the coordinates; step = stride * sampling_stride.
struct SampleBox {
    uint64_t lo[3], hi[3], step[3];
    uint64_t dist;
    float neg_2_stat_eb;
    float stat_eb;
    uint32_t n;             // number of samples (product of per-axis counts)
    uint32_t log2_off;      // offset of the log2f table for n (entries 1..n) in the table arena
};

// One evaluation of get_h1_psnr: t and abs_eb (the error bound whose bins are counted).
struct ProxyEval {
    float t, abs_eb;
};

// Per-round table of the up to 27 block classes (first/middle/last along each axis).
struct ClassInfo {
    uint32_t ss;         // sampling_stride (needs glibc cbrt, so computed on the host)
    uint32_t n;          // samples
    uint32_t log2_off;   // log2 table offset for n
    uint32_t fallback;   // 1: the block is too short along the axis (compress.tpp:96)
    uint32_t cnt[3];     // samples per axis (the same for every block of the class)
    uint32_t m2, m12;    // floor((2^32 - 1) / d) + 1 for d = cnt[2] and cnt[1] * cnt[2] (0 when d <= 1)
};

// A per-block t decision that needs the host's glibc log10f to settle.
struct AmbiguousRecord {
    uint32_t block;      // linear block index
    uint32_t round;
    int32_t provisional; // t code chosen on the device
    uint32_t pad;
    float h1[5], x[5];   // proxies for t = 1/16, 1/4, 9/32, 5/16, 11/32
};

}  // namespace asz
