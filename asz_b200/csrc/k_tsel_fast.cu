// Per-(block, round) coefficient selection, fast path (c_codes/asz_core/compress.tpp:91-144): one
// CTA per group over the field in global memory; the selection itself is fastsel::fast_group.
// The sample positions follow get_AB_map's loops (get_AB_map.tpp:13-15).
#include <cuda_runtime.h>

#include <algorithm>

#include "tsel_fast.cuh"

namespace asz {
using namespace fastsel;
namespace {

// Samples of a group read from the field in global memory.
struct GlobalSrc {
    FastSampleGeo sg;
    const float *rec, *orig;
    uint64_t n1, n2, dist;
    float neg;
    __device__ __forceinline__ void keys(uint32_t s, float &af, float &bf, bool &nz) const {
        sample_keys(rec, orig, fast_sample_pos(sg, s, n1, n2), dist, neg, af, bf, nz);
    }
};

}  // namespace

// Selection of group g of one field and round: the fallbacks and overrides, the sample geometry
// (get_AB_map.tpp:13-15), then fast_group. handoff(g) is called by thread 0 for a group the exact
// path has to settle.
template <int kT, class HandOff>
__device__ void fast_one(GroupShared &sh, const FieldGeom &fg, const RoundGeom &rg, uint32_t l,
                         const ClassInfo *__restrict__ classes, const float *__restrict__ rec, const float *__restrict__ orig,
                         const float *__restrict__ log2arena, float R2, float t_default, float *__restrict__ tval,
                         int64_t *__restrict__ t_int, uint32_t *fb_count, const uint32_t *__restrict__ overrides,
                         uint32_t n_overrides, uint32_t *why, uint64_t g, const HandOff &handoff) {
    const uint32_t tid = threadIdx.x;
    const int d = rg.dir;
    const uint64_t b2 = g % fg.block_num[2], b1 = (g / fg.block_num[2]) % fg.block_num[1],
                   b0 = g / (fg.block_num[1] * fg.block_num[2]);
    const uint64_t bb[3] = {b0, b1, b2};
    const int cls = (class_of(b0, fg.block_num[0]) * 3 + class_of(b1, fg.block_num[1])) * 3 + class_of(b2, fg.block_num[2]);
    const ClassInfo ci = classes[cls];
    bool forced = false;
    float forced_t = 0.0f;
    for (uint32_t i = 0; i < n_overrides; i++)
        if (overrides[3 * i] == (uint32_t)g && overrides[3 * i + 1] == l) {
            forced = true;
            forced_t = __uint_as_float(overrides[3 * i + 2]);
        }
    if (ci.fallback || ci.n == 0 || forced) {
        if (tid == 0) {
            float t = forced ? forced_t : t_default;
            if (!forced) atomicAdd(fb_count, 1u);
            tval[g] = t;
            t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(t, (float)fg.t_precision));
        }
        return;
    }
    const uint32_t n = ci.n;
    if (n > 0xffffu) {  // a bin count could overflow its 16-bit half word
        if (tid == 0) {
            handoff(g);
            atomicAdd(&why[0], 1u);
        }
        return;
    }
    // The per-axis sample counts and their division constants come with the class.
    FastSampleGeo sg;
    for (int a = 0; a < 3; a++) {
        uint64_t lo = fg.origin[a] + bb[a] * fg.block_shape[a];
        if (a != d && lo != 0) lo += rg.stride[a];
        if (a == d) lo += 3 * rg.stride[a] / 2;
        sg.lo[a] = lo;
        sg.step[a] = rg.stride[a] * ci.ss;
    }
    sg.cnt2 = ci.cnt[2];
    sg.c2 = SmallDiv{ci.cnt[2], ci.m2};
    sg.c12 = SmallDiv{ci.cnt[1] * ci.cnt[2], ci.m12};
    const GlobalSrc src{sg, rec, orig, fg.n[1], fg.n[2], rg.dist, rg.neg_2_stat_eb};
    float t = 0.0f;
    const uint32_t code = fast_group<GlobalSrc, kT>(sh, src, n, rg, log2arena + ci.log2_off, R2, why, t);
    if (tid == 0) {
        if (code == kFastDecided) {
            tval[g] = t;
            t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(t, (float)fg.t_precision));
        } else {
            handoff(g);
        }
    }
}

struct ListHandOff {
    uint32_t *list, *count;
    __device__ void operator()(uint64_t g) const { list[atomicAdd(count, 1u)] = (uint32_t)g; }
};

// One CTA per (block, round) group at a time (persistent grid). list_out receives the groups this
// path could not settle; why[0] counts those whose bins span too many windows, why[1] those with an
// undecidable comparison; why[2] counts the groups settled here by window-by-window counting.
template <int kT>
__global__ void __launch_bounds__(kT, kT == 32 ? 20 : kT == 64 ? 16 : 8)
    tsel_fast_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const ClassInfo *__restrict__ classes,
                     const float *__restrict__ rec, const float *__restrict__ orig, const float *__restrict__ log2arena,
                     float R2, float t_default, float *__restrict__ tval, int64_t *__restrict__ t_int,
                     uint32_t *__restrict__ fb_count, uint32_t *__restrict__ list_out, uint32_t *__restrict__ list_count,
                     const uint32_t *__restrict__ overrides, uint32_t n_overrides, uint32_t *__restrict__ why) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupShared &sh = *reinterpret_cast<GroupShared *>(smem_raw);
    const uint64_t nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    for (int i = threadIdx.x; i < 5 * kWinWords; i += kT) (&sh.hist[0][0])[i] = 0;
    __syncthreads();
    const ListHandOff ho{list_out, list_count};
    for (uint64_t g = blockIdx.x; g < nblocks; g += gridDim.x) {
        fast_one<kT>(sh, fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int, fb_count, overrides, n_overrides,
                 why, g, ho);
        __syncthreads();
    }
}

// Batched form: one work queue over the (field, group) pairs of every field of a batch (same
// round of the same plan), fields found by their group-offset prefix. Handed-off groups go to one
// list of (field << 32 | group) entries for the batched exact path.
struct PairHandOff {
    unsigned long long *list;
    uint32_t *count;
    uint32_t f;
    __device__ void operator()(uint64_t g) const { list[atomicAdd(count, 1u)] = ((unsigned long long)f << 32) | g; }
};

__global__ void __launch_bounds__(kThreads, 16)
    tsel_fast_batch_kernel(const BatchField *__restrict__ F, const uint64_t *__restrict__ goff, uint32_t nf, uint32_t l,
                           const float *__restrict__ log2arena, float t_default, uint32_t *queue,
                           unsigned long long *handoff_list, uint32_t *handoff_count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupShared &sh = *reinterpret_cast<GroupShared *>(smem_raw);
    __shared__ uint64_t item;
    const uint64_t total = goff[nf];
    for (int i = threadIdx.x; i < 5 * kWinWords; i += kThreads) (&sh.hist[0][0])[i] = 0;
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(queue, 1u);
        __syncthreads();
        const uint64_t gi = item;
        __syncthreads();
        if (gi >= total) break;
        const uint32_t f = field_of(goff, nf, gi);
        const BatchField &B = F[f];
        const PairHandOff ho{handoff_list, handoff_count, f};
        fast_one<kThreads>(sh, B.fg, B.rounds[l], l, B.classes + 27 * l, B.rec, B.in, log2arena, B.R2, t_default, B.tval, B.tint,
                 &B.cnt->fb, nullptr, 0, B.cnt->why, gi - goff[f], ho);
        __syncthreads();
    }
}

cudaError_t launch_tsel_fast_batch(const BatchField *F, const uint64_t *goff, uint32_t nf, uint32_t l, const float *log2arena,
                                   float t_default, uint32_t *queue, unsigned long long *handoff_list, uint32_t *handoff_count,
                                   uint32_t grid, cudaStream_t st) {
    const int smem = (int)sizeof(GroupShared);
    cudaError_t e = cudaFuncSetAttribute(tsel_fast_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    tsel_fast_batch_kernel<<<grid ? grid : 148 * 8, kThreads, smem, st>>>(F, goff, nf, l, log2arena, t_default, queue,
                                                                          handoff_list, handoff_count);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_tsel_fast(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                             const float *orig, const float *log2arena, float R2, float t_default, float *tval,
                             int64_t *t_int, uint32_t *fb_count, uint32_t *list_out, uint32_t *list_count,
                             const uint32_t *overrides, uint32_t n_overrides, uint32_t *why, cudaStream_t st,
                             uint32_t common_samples) {
    const uint64_t nb = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    const int smem = (int)sizeof(GroupShared);
    // Many groups: 64-thread CTAs, 16 per SM (fewer warps wait at each block barrier), or one-warp
    // CTAs, 20 per SM, when the most common group size (common_samples) is at most 32 samples
    // (measured: one-warp CTAs win at 9 samples a group and lose at 45; any size is handled).
    // Fewer groups than four waves of 64-thread CTAs: 128-thread CTAs, which finish each group sooner.
    const bool wide = nb < 148 * 16 * 4, narrow = !wide && common_samples <= 32;
    cudaError_t e = wide     ? cudaFuncSetAttribute(tsel_fast_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                    : narrow ? cudaFuncSetAttribute(tsel_fast_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                             : cudaFuncSetAttribute(tsel_fast_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    if (wide)
        tsel_fast_kernel<128><<<(unsigned)nb, 128, smem, st>>>(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval,
                                                              t_int, fb_count, list_out, list_count, overrides, n_overrides,
                                                              why);
    else if (narrow)
        tsel_fast_kernel<32><<<(unsigned)std::min<uint64_t>(nb, 148 * 20 * 4), 32, smem, st>>>(
            fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int, fb_count, list_out, list_count, overrides,
            n_overrides, why);
    else
        tsel_fast_kernel<64><<<(unsigned)std::min<uint64_t>(nb, 148 * 16 * 4), 64, smem, st>>>(
            fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval, t_int, fb_count, list_out, list_count, overrides,
            n_overrides, why);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz
