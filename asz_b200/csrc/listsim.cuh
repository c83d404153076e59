// Emulation of libstdc++'s std::unordered_map node list (GCC 13 _Hashtable, unique keys).
//
// The list order is what the reference's proxy sums iterate over. Inserting a node puts it at the
// front of its bucket's run if the bucket is occupied, otherwise at the list head. A rehash walks
// the old list and rebuilds it with the same rule (_M_rehash_aux). Rehashes happen before the
// insertions listed in tsel.cuh (kSchedAt/kSchedBkt).
#pragma once
#include <cstdint>

#include "dev_common.cuh"
#include "tsel.cuh"

namespace asz {

constexpr int32_t kNil = -1;

#ifdef __CUDACC__
// Device copy of the bucket schedule.
static __constant__ uint64_t d_sched_at[kSchedLen] = {1, 14, 30, 60, 128, 258, 542, 1110, 2358, 5088, 10274, 20754,
                                               42044, 85230, 172934, 351062, 712698, 1447154, 2938680,
                                               5967348, 12117690};
static __constant__ uint64_t d_sched_bkt[kSchedLen] = {13, 29, 59, 127, 257, 541, 1109, 2357, 5087, 10273, 20753,
                                                42043, 85229, 172933, 351061, 712697, 1447153, 2938679,
                                                5967347, 12117689, 24607243};

#endif

ASZ_HD uint64_t sched_at(int i) {
#ifdef __CUDA_ARCH__
    return d_sched_at[i];
#else
    return kSchedAt[i];
#endif
}
ASZ_HD uint64_t sched_bkt(int i) {
#ifdef __CUDA_ARCH__
    return d_sched_bkt[i];
#else
    return kSchedBkt[i];
#endif
}

// Bucket count in use after `m` insertions.
ASZ_HD uint64_t sched_buckets(uint64_t m) {
    uint64_t b = 1;
    for (int i = 0; i < kSchedLen; i++)
        if (sched_at(i) <= m) b = sched_bkt(i);
    return b;
}

// Emulated std::unordered_map list: nodes 0..count-1, sentinel (before_begin) at index `cap`.
struct ListSim {
    int32_t *nxt, *bkt;
    const uint64_t *hash;  // NULL: identity hash of the int64 keys in `keys`
    const int64_t *keys;
    uint32_t cap, count;
    uint64_t nbkt;
    int sched;
    bool broken;   // set if a walk exceeds the node count (cannot happen for a consistent list)

    ASZ_HD uint64_t code(int32_t x) const { return hash ? hash[x] : (uint64_t)keys[x]; }

    ASZ_HD void init() {
        count = 0;
        nbkt = 1;
        sched = 0;
        broken = false;
        nxt[cap] = kNil;
    }
    // _Hashtable::_M_rehash_aux (unique keys).
    ASZ_HD void rehash(uint64_t nb) {
        for (uint64_t i = 0; i < nb; i++) bkt[i] = kNil;
        int32_t p = nxt[cap];
        nxt[cap] = kNil;
        uint64_t bbegin = 0;
        const int32_t S = (int32_t)cap;
        uint32_t steps = 0;
        while (p != kNil) {
            if (++steps > count) {  // a well-formed list has exactly `count` nodes
                broken = true;
                break;
            }
            int32_t nx = nxt[p];
            uint64_t b = code(p) % nb;
            if (bkt[b] == kNil) {
                nxt[p] = nxt[S];
                nxt[S] = p;
                bkt[b] = S;
                if (nxt[p] != kNil) bkt[bbegin] = p;
                bbegin = b;
            } else {
                nxt[p] = nxt[bkt[b]];
                nxt[bkt[b]] = p;
            }
            p = nx;
        }
        nbkt = nb;
    }
    // _M_insert_unique_node: rehash check, then _M_insert_bucket_begin.
    ASZ_HD void insert(int32_t x) {
        if (sched < kSchedLen && (uint64_t)count + 1 == sched_at(sched)) {
            rehash(sched_bkt(sched));
            sched++;
        }
        const int32_t S = (int32_t)cap;
        uint64_t b = code(x) % nbkt;
        if (bkt[b] != kNil) {
            nxt[x] = nxt[bkt[b]];
            nxt[bkt[b]] = x;
        } else {
            nxt[x] = nxt[S];
            nxt[S] = x;
            if (nxt[x] != kNil) bkt[code(nxt[x]) % nbkt] = x;
            bkt[b] = S;
        }
        count++;
    }
};

}  // namespace asz
