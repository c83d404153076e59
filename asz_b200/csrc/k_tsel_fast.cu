// Per-(block, round) coefficient selection, fast path (c_codes/asz_core/compress.tpp:91-144): one
// CTA per group over the field in global memory; the selection itself is fastsel::fast_group.
// The sample positions follow get_AB_map's loops (get_AB_map.tpp:13-15).
#include <cuda_runtime.h>

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

// One CTA per (block, round) group at a time (persistent grid). list_out receives the groups this
// path could not settle; why[0] counts those whose bins span too many windows, why[1] those with an
// undecidable comparison; why[2] counts the groups settled here by window-by-window counting.
__global__ void __launch_bounds__(kThreads, 8)
    tsel_fast_kernel(FieldGeom fg, RoundGeom rg, uint32_t l, const ClassInfo *__restrict__ classes,
                     const float *__restrict__ rec, const float *__restrict__ orig, const float *__restrict__ log2arena,
                     float R2, float t_default, float *__restrict__ tval, int64_t *__restrict__ t_int,
                     uint32_t *__restrict__ fb_count, uint32_t *__restrict__ list_out, uint32_t *__restrict__ list_count,
                     const uint32_t *__restrict__ overrides, uint32_t n_overrides, uint32_t *__restrict__ why) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupShared &sh = *reinterpret_cast<GroupShared *>(smem_raw);
    const uint32_t tid = threadIdx.x;
    const uint64_t nblocks = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    const int d = rg.dir;
    for (int i = tid; i < 5 * kWinWords; i += kThreads) (&sh.hist[0][0])[i] = 0;
    __syncthreads();
    for (uint64_t g = blockIdx.x; g < nblocks; g += gridDim.x) {
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
            continue;
        }
        const uint32_t n = ci.n;
        if (n > 0xffffu) {  // a bin count could overflow its 16-bit half word
            if (tid == 0) {
                list_out[atomicAdd(list_count, 1u)] = (uint32_t)g;
                atomicAdd(&why[0], 1u);
            }
            continue;
        }
        FastSampleGeo sg;
        uint32_t cnt[3];
        for (int a = 0; a < 3; a++) {
            uint64_t lo = fg.origin[a] + bb[a] * fg.block_shape[a];
            uint64_t hi = min(fg.origin[a] + (bb[a] + 1) * fg.block_shape[a] + 1, fg.n[a]);
            if (a != d && lo != 0) lo += rg.stride[a];
            if (a == d) {
                lo += 3 * rg.stride[a] / 2;
                hi -= 3 * rg.stride[a] / 2;
            }
            sg.lo[a] = lo;
            sg.step[a] = rg.stride[a] * ci.ss;
            cnt[a] = (uint32_t)((hi - lo + sg.step[a] - 1) / sg.step[a]);
        }
        sg.cnt2 = cnt[2];
        sg.c2 = small_div(cnt[2]);
        sg.c12 = small_div(cnt[1] * cnt[2]);
        const GlobalSrc src{sg, rec, orig, fg.n[1], fg.n[2], rg.dist, rg.neg_2_stat_eb};
        float t = 0.0f;
        const uint32_t code = fast_group(sh, src, n, rg, log2arena + ci.log2_off, R2, why, t);
        if (tid == 0) {
            if (code == kFastDecided) {
                tval[g] = t;
                t_int[g * fg.layer_num + l] = lround_f(__fmul_rn(t, (float)fg.t_precision));
            } else {
                list_out[atomicAdd(list_count, 1u)] = (uint32_t)g;
            }
        }
        __syncthreads();
    }
}

cudaError_t launch_tsel_fast(const FieldGeom &fg, const RoundGeom &rg, uint32_t l, const ClassInfo *classes, const float *rec,
                             const float *orig, const float *log2arena, float R2, float t_default, float *tval,
                             int64_t *t_int, uint32_t *fb_count, uint32_t *list_out, uint32_t *list_count,
                             const uint32_t *overrides, uint32_t n_overrides, uint32_t *why, cudaStream_t st) {
    uint64_t nb = fg.block_num[0] * fg.block_num[1] * fg.block_num[2];
    uint64_t blocks = nb < 148 * 8 * 4 ? nb : 148 * 8 * 4;
    const int smem = (int)sizeof(GroupShared);
    cudaError_t e = cudaFuncSetAttribute(tsel_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    tsel_fast_kernel<<<(unsigned)blocks, kThreads, smem, st>>>(fg, rg, l, classes, rec, orig, log2arena, R2, t_default, tval,
                                                              t_int, fb_count, list_out, list_count, overrides, n_overrides,
                                                              why);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz
