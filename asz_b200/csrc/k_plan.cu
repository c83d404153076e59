// Plan search (c_codes/asz_core/generate_config.tpp:444-678) on the device: the sampled open-loop
// compression of every candidate predictor of a layer in one launch, and the candidates' squared
// error sums in the reference's sequential order.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "launch.h"

namespace asz {
namespace {

__device__ __forceinline__ uint32_t cand_of(const PlanCand *__restrict__ c, uint32_t nc, uint64_t k) {
    uint32_t lo = 0, hi = nc;  // last candidate with off <= k
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (c[mid].off <= k) lo = mid;
        else hi = mid;
    }
    return lo;
}

// dot_sample_compress (generate_config.tpp:227-254) as GCC emits it for the reference build: the
// edge stencils below, the interior 1D4R in double with a float product in between, the residual
// quantised in float (diff * neg_2_eb) and e = fmaf(-eb, (float)(2 * qb), diff) for the error sum.
__global__ void plan_sample_kernel(const float *__restrict__ d, uint64_t n1, uint64_t n2, const PlanCand *__restrict__ cands,
                                   uint32_t ncands, uint64_t total, int32_t *__restrict__ qb_out, float *__restrict__ e_out,
                                   int32_t *__restrict__ qb_range) {
    int32_t lo = INT32_MAX, hi = INT32_MIN;
    uint32_t ci_last = 0xffffffffu;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ci = cand_of(cands, ncands, k);
        if (ci != ci_last) {
            if (ci_last != 0xffffffffu && lo <= hi) {
                atomicMin(&qb_range[2 * ci_last], lo);
                atomicMax(&qb_range[2 * ci_last + 1], hi);
            }
            lo = INT32_MAX;
            hi = INT32_MIN;
            ci_last = ci;
        }
        const PlanCand c = cands[ci];
        const uint64_t kl = k - c.off;
        // Loop nest: axes ax[0] (outer) .. ax[2] (inner).
        const uint64_t c2 = c.cnt[c.ax[2]], c1 = c.cnt[c.ax[1]];
        const uint64_t k2 = kl % c2, r = kl / c2, k1 = r % c1, k0 = r / c1;
        uint64_t ii[3];
        ii[c.ax[0]] = c.lo[c.ax[0]] + k0 * c.st[c.ax[0]];
        ii[c.ax[1]] = c.lo[c.ax[1]] + k1 * c.st[c.ax[1]];
        ii[c.ax[2]] = c.lo[c.ax[2]] + k2 * c.st[c.ax[2]];
        const uint64_t pos = (ii[0] * n1 + ii[1]) * n2 + ii[2];
        const uint64_t i = ii[c.dir], hs = c.hs, right = c.right, dist = c.dist;
        const float xm1 = d[pos - dist];
        float pred;
        if (i <= hs) {
            if (i + hs >= right) pred = xm1;
            else if (i + 3 * hs >= right) pred = __fmul_rn(__fadd_rn(d[pos + dist], xm1), 0.5f);
            else pred = __fmul_rn(__fmaf_rn(d[pos + dist], 6.0f, __fmaf_rn(xm1, 3.0f, -d[pos + 3 * dist])), 0.125f);
        } else {
            const float xm3 = d[pos - 3 * dist];
            if (i + hs >= right) {
                pred = __fmul_rn(__fmaf_rn(xm1, 3.0f, -xm3), 0.5f);
            } else if (i + 3 * hs >= right) {
                pred = __fmul_rn(__fsub_rn(__fmaf_rn(xm1, 6.0f, __fmul_rn(d[pos + dist], 3.0f)), xm3), 0.125f);
            } else {
                const float s1 = __fadd_rn(d[pos + dist], xm1), s3 = __fadd_rn(xm3, d[pos + 3 * dist]);
                const double td = (double)c.t;
                const float p1 = __double2float_rn(__dmul_rn((double)s3, __dsub_rn(0.25, td)));
                pred = __double2float_rn(__fma_rn(__dadd_rn(0.25, td), (double)s1, (double)p1));
            }
        }
        const float diff = __fsub_rn(pred, d[pos]);
        const int32_t q = (int32_t)lround_f(__fmul_rn(diff, c.neg_2_eb));
        const float q2 = __int2float_rn((int32_t)((uint32_t)q * 2u));
        qb_out[k] = q;
        e_out[k] = __fmaf_rn(-c.eb, q2, diff);
        lo = min(lo, q);
        hi = max(hi, q);
    }
    if (ci_last != 0xffffffffu && lo <= hi) {
        atomicMin(&qb_range[2 * ci_last], lo);
        atomicMax(&qb_range[2 * ci_last + 1], hi);
    }
}

// mse = fmaf(e, e, mse) over each candidate's samples in loop order (one warp per candidate), the
// reference's float sum (generate_config.tpp:227-254), bit for bit.
//
// Batches of kBatch terms, kPer consecutive ones per lane. While the running sum s stays in one
// binade [2^E, 2^(E+1)), with ulp u = 2^(E-23) and s = m*u (m in [2^23, 2^24)), every step
// s' = RN(s + x*x) equals (m + r)*u with r = x*x/u rounded to the nearest integer, unless the
// fraction of x*x/u is exactly one half (round-half-even then depends on m). The terms are not
// negative, so the partial sums grow: if the batch's total stays below 2^24 no step leaves the
// binade, and the batch adds sum(r)*u in one step. x*x is exact in double and u a power of two,
// so r and the tie test are exact. A batch with a tie, a crossing, or a sum below the normal range
// is replayed term by term (the exact chain).
constexpr uint32_t kPer = 8, kBatch = 32 * kPer;

__global__ void plan_mse_kernel(const PlanCand *__restrict__ cands, uint32_t ncands, const float *__restrict__ e,
                                float *__restrict__ mse_out) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= ncands) return;
    const PlanCand c = cands[warp];
    const uint64_t n = c.cnt[0] * c.cnt[1] * c.cnt[2];
    const float *p = e + c.off;
    float mse = 0.0f;
    for (uint64_t b = 0; b < n; b += kBatch) {
        float v[kPer];
#pragma unroll
        for (uint32_t i = 0; i < kPer; i++) {
            const uint64_t k = b + lane * kPer + i;
            v[i] = k < n ? p[k] : 0.0f;
        }
        if (mse >= 0x1p-100f) {
            int ex;
            frexpf(mse, &ex);  // mse = f * 2^ex, f in [0.5, 1): binade 2^(ex-1), ulp 2^(ex-24)
            const double inv_u = ldexp(1.0, 24 - ex);
            const uint32_t m = (uint32_t)__double2uint_rz((double)mse * inv_u);
            bool ok = true;
            uint32_t sum = 0;
#pragma unroll
            for (uint32_t i = 0; i < kPer; i++) {
                const double t = __dmul_rn(__dmul_rn((double)v[i], (double)v[i]), inv_u);
                const double r = rint(t);
                ok = ok && r < 0x1p24 && fabs(t - r) != 0.5;
                sum += ok ? (uint32_t)r : 0u;
            }
            ok = __all_sync(0xffffffffu, ok);
            const uint32_t tot = __reduce_add_sync(0xffffffffu, sum);
            if (ok && (uint64_t)m + tot < (1ull << 24)) {
                mse = ldexpf((float)(m + tot), ex - 24);
                continue;
            }
        }
        const uint32_t cnt = n - b < kBatch ? (uint32_t)(n - b) : kBatch;
        for (uint32_t j = 0; j < cnt; j++) {
            const uint32_t i = j % kPer;
            float vi = v[0];
#pragma unroll
            for (uint32_t q = 1; q < kPer; q++) vi = i == q ? v[q] : vi;
            const float x = __shfl_sync(0xffffffffu, vi, j / kPer);
            mse = __fmaf_rn(x, x, mse);
        }
    }
    if (lane == 0) mse_out[warp] = mse;
}

}  // namespace

cudaError_t launch_plan_sample(const float *d, uint64_t n1, uint64_t n2, const PlanCand *cands, uint32_t ncands, uint64_t total,
                               int32_t *qb, float *e, int32_t *qb_range, cudaStream_t st) {
    if (total == 0) return cudaSuccess;
    const uint64_t b = (total + 255) / 256;
    plan_sample_kernel<<<(unsigned)(b < 148 * 16 ? b : 148 * 16), 256, 0, st>>>(d, n1, n2, cands, ncands, total, qb, e, qb_range);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_plan_mse(const PlanCand *cands, uint32_t ncands, const float *e, float *mse, cudaStream_t st) {
    if (ncands == 0) return cudaSuccess;
    plan_mse_kernel<<<(ncands * 32 + 127) / 128, 128, 0, st>>>(cands, ncands, e, mse);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz
