// The prediction sweep of the reference's study tool (c_codes/s2_many_prediction.cpp:164-464):
// every target of one predictor's loop nest is predicted from the original data with each of a
// set of coefficients, quantised, and summed into the tool's error figures. The QB streams then
// go through the library's histogram and tiled Huffman kernels.
//
// Floating point follows what GCC 13.3 makes of the reference under -Ofast -mfma (pinned against
// the reference's own dot functions and binary outputs): neighbour pairs summed in float; the
// 1D4R and 2D4R products of those sums with 0.25 -+ t are exact in double; 1D6R is
// fma(w, s1, fma(a, s5, b * s3)) with w = 0.5 - (a + b); e = pred - x; qb = llround(e * neg_2_eb);
// e2 = fma(-2 qb, abs_eb, e); the sums of e^2 and e2^2 are fused steps. The sums run per thread,
// per block and over blocks in a fixed order, so a launch is deterministic; the reference sums one
// target after the other, so the sums agree to rounding, while every QB is identical.
#include <climits>

#include "launch.h"

namespace asz {

namespace {

constexpr unsigned kSweepThreads = 256;
constexpr uint32_t kSeg = 16;  // positions of a line per work item when a thread walks lines

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace

// Running figures of one thread: the three sums and the QB extremes.
struct SweepAcc {
    double se = 0.0, sr = 0.0, sa = 0.0;
    long long lo = LLONG_MAX, hi = LLONG_MIN;
};

// One target (index `it` of the (line, position) space) with one coefficient set.
__device__ __forceinline__ void sweep_one(const float *__restrict__ d, const SweepGeom &g, const SweepCoef &c, double abs_eb,
                                          double neg_2_eb, int64_t *__restrict__ out, uint64_t it, SweepAcc &a) {
    uint64_t i[3], j;
    if (!sweep_target(g, it, i, j)) return;
    const uint64_t pos = i[0] * (g.n[1] * g.n[2]) + i[1] * g.n[2] + i[2];
    const uint64_t d0 = g.dist[0];
    const float x = d[pos];
    double pred;
    if (g.kind == 0) {  // compress_1d4r_dot (s2_many_prediction.cpp:28-45)
        const float s3 = __fadd_rn(d[pos - 3 * d0], d[pos + 3 * d0]);
        const float s1 = __fadd_rn(d[pos - d0], d[pos + d0]);
        pred = __dadd_rn(__dmul_rn(c.lo, (double)s3), __dmul_rn(c.hi, (double)s1));
    } else if (g.kind == 1) {  // compress_2d4r_dot (:47-65)
        const uint64_t d1 = g.dist[1];
        const float sa_ = __fadd_rn(d[pos - d0], d[pos + d0]);
        const float sb_ = __fadd_rn(d[pos - d1], d[pos + d1]);
        pred = __dadd_rn(__dmul_rn(c.hi, (double)sa_), __dmul_rn(c.lo, (double)sb_));
    } else {  // compress_1d6r_dot (:67-87)
        const float s5 = __fadd_rn(d[pos - 5 * d0], d[pos + 5 * d0]);
        const float s3 = __fadd_rn(d[pos - 3 * d0], d[pos + 3 * d0]);
        const float s1 = __fadd_rn(d[pos - d0], d[pos + d0]);
        pred = __fma_rn(c.w, (double)s1, __fma_rn(c.c0, (double)s5, __dmul_rn(c.c1, (double)s3)));
    }
    const double e = __dsub_rn(pred, (double)x);
    a.sr = __fma_rn(e, e, a.sr);
    a.sa = __dadd_rn(a.sa, fabs(e));
    const int64_t q = lround_d(__dmul_rn(e, neg_2_eb));
    out[j] = q;
    const double e2 = __fma_rn(-(double)(q * 2), abs_eb, e);
    a.se = __fma_rn(e2, e2, a.se);
    a.lo = min(a.lo, (long long)q);
    a.hi = max(a.hi, (long long)q);
}

// grid (x: CTAs over the work items, y: coefficient). Writes the QB stream of coefficient y at
// qb + y * qb_stride, the CTA's three partial sums at part[(y * gridDim.x + blockIdx.x) * 3], and
// folds the stream's extremes into mm[2y], mm[2y + 1].
//
// When the QB order runs along the contiguous axis, neighbouring threads take neighbouring
// positions of a line. When it runs along axis 0 or 1, a work item is a segment of kSeg positions
// of one line, with neighbouring items on neighbouring lines: a warp then reads neighbouring lines
// (adjacent along axis 2), and each thread writes its segment's QB run in order.
__global__ void __launch_bounds__(kSweepThreads)
    sweep_predict_kernel(const float *__restrict__ d, SweepGeom g, const SweepCoef *__restrict__ coef, double abs_eb,
                         double neg_2_eb, int64_t *__restrict__ qb, uint64_t qb_stride, double *__restrict__ part,
                         long long *__restrict__ mm) {
    const SweepCoef c = coef[blockIdx.y];
    int64_t *out = qb + (uint64_t)blockIdx.y * qb_stride;
    const uint64_t gtid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, gstride = (uint64_t)gridDim.x * blockDim.x;
    SweepAcc a;
    if (g.line_per_thread) {
        const uint64_t items = g.lines * ((g.per_line + kSeg - 1) / kSeg);
        for (uint64_t item = gtid; item < items; item += gstride) {
            const uint64_t line = item % g.lines, k0 = (item / g.lines) * kSeg;
            const uint64_t k1 = min(k0 + kSeg, g.per_line);
            for (uint64_t k = k0; k < k1; k++) sweep_one(d, g, c, abs_eb, neg_2_eb, out, line * g.per_line + k, a);
        }
    } else {
        const uint64_t total = g.lines * g.per_line;
        for (uint64_t it = gtid; it < total; it += gstride) sweep_one(d, g, c, abs_eb, neg_2_eb, out, it, a);
    }
    double se = a.se, sr = a.sr, sa = a.sa;
    long long lo = a.lo, hi = a.hi;
    __shared__ double red[3][kSweepThreads / 32];
    __shared__ long long rlo[kSweepThreads / 32], rhi[kSweepThreads / 32];
    se = warp_sum(se);
    sr = warp_sum(sr);
    sa = warp_sum(sa);
    for (int o = 16; o; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const unsigned w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = se;
        red[1][w] = sr;
        red[2][w] = sa;
        rlo[w] = lo;
        rhi[w] = hi;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (unsigned k = 0; k < kSweepThreads / 32; k++) s = __dadd_rn(s, red[threadIdx.x][k]);
        part[((uint64_t)blockIdx.y * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = s;
    } else if (threadIdx.x == 32) {
        long long l = LLONG_MAX, h = LLONG_MIN;
        for (unsigned k = 0; k < kSweepThreads / 32; k++) {
            l = min(l, rlo[k]);
            h = max(h, rhi[k]);
        }
        if (l <= h) {
            atomicMin(mm + 2 * blockIdx.y, l);
            atomicMax(mm + 2 * blockIdx.y + 1, h);
        }
    }
}

// One CTA per coefficient: the partial sums of its nparts CTAs, in a fixed order.
__global__ void __launch_bounds__(kSweepThreads)
    sweep_sums_kernel(const double *__restrict__ part, uint32_t nparts, double *__restrict__ sums) {
    __shared__ double red[3][kSweepThreads / 32];
    const double *p = part + (uint64_t)blockIdx.x * nparts * 3;
    double s[3] = {0.0, 0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < nparts; i += kSweepThreads)
        for (int c = 0; c < 3; c++) s[c] = __dadd_rn(s[c], p[(uint64_t)i * 3 + c]);
    for (int c = 0; c < 3; c++) s[c] = warp_sum(s[c]);
    if ((threadIdx.x & 31) == 0)
        for (int c = 0; c < 3; c++) red[c][threadIdx.x >> 5] = s[c];
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (unsigned k = 0; k < kSweepThreads / 32; k++) t = __dadd_rn(t, red[threadIdx.x][k]);
        sums[(uint64_t)blockIdx.x * 3 + threadIdx.x] = t;
    }
}

// Histogram and first position of each symbol of a stream (hist[] preset to zero, first[] to all
// ones). A CTA takes one contiguous chunk of the stream. With at most kStatsShared symbols, it
// counts and keeps first positions (relative to its chunk) in shared memory and folds them into
// the global tables once; a wider alphabet goes to the global tables directly. Reading a first
// position before lowering it skips the atomic for all but the earliest positions of a symbol.
constexpr uint32_t kStatsShared = 4096;

__global__ void __launch_bounds__(kSweepThreads)
    sweep_stats_kernel(const int64_t *__restrict__ s, uint64_t n, int64_t offset, uint64_t range,
                       unsigned long long *__restrict__ hist, unsigned long long *__restrict__ first) {
    __shared__ uint32_t hsh[kStatsShared], fsh[kStatsShared];
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t c0 = blockIdx.x * chunk, c1 = min(n, c0 + chunk);
    if (range <= kStatsShared) {
        for (uint32_t i = threadIdx.x; i < range; i += kSweepThreads) {
            hsh[i] = 0u;
            fsh[i] = 0xffffffffu;
        }
        __syncthreads();
        for (uint64_t j = c0 + threadIdx.x; j < c1; j += kSweepThreads) {
            const uint32_t v = (uint32_t)(s[j] - offset), r = (uint32_t)(j - c0);
            atomicAdd(&hsh[v], 1u);
            if (fsh[v] > r) atomicMin(&fsh[v], r);
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < range; i += kSweepThreads)
            if (hsh[i]) {
                atomicAdd(&hist[i], (unsigned long long)hsh[i]);
                atomicMin(&first[i], (unsigned long long)(c0 + fsh[i]));
            }
        return;
    }
    for (uint64_t j = c0 + threadIdx.x; j < c1; j += kSweepThreads) {
        const uint64_t v = (uint64_t)(s[j] - offset);
        atomicAdd(&hist[v], 1ull);
        unsigned long long *slot = first + v;
        if (__ldcg(slot) > j) atomicMin(slot, (unsigned long long)j);
    }
}

uint32_t sweep_predict_grid(const SweepGeom &g) {
    const uint64_t total = g.line_per_thread ? g.lines * ((g.per_line + kSeg - 1) / kSeg) : g.lines * g.per_line;
    const uint64_t want = (total + kSweepThreads - 1) / kSweepThreads;
    return (uint32_t)(want < 148 * 8 ? (want ? want : 1) : 148 * 8);
}

cudaError_t launch_sweep_predict(const float *d, const SweepGeom &g, const SweepCoef *coef, uint32_t ncoef, double abs_eb,
                                 double neg_2_eb, int64_t *qb, uint64_t qb_stride, double *part, long long *mm,
                                 cudaStream_t st) {
    if (ncoef == 0) return cudaSuccess;
    sweep_predict_kernel<<<dim3(sweep_predict_grid(g), ncoef), kSweepThreads, 0, st>>>(d, g, coef, abs_eb, neg_2_eb, qb,
                                                                                       qb_stride, part, mm);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_sweep_sums(const double *part, uint32_t nparts, uint32_t ncoef, double *sums, cudaStream_t st) {
    if (ncoef == 0) return cudaSuccess;
    sweep_sums_kernel<<<ncoef, kSweepThreads, 0, st>>>(part, nparts, sums);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_sweep_stats(const int64_t *s, uint64_t n, int64_t offset, uint64_t range, unsigned long long *hist,
                               unsigned long long *first, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    // Chunks of at least 4096 symbols, so the shared tables' set-up and fold stay small beside them.
    const uint64_t want = (n + 4095) / 4096;
    sweep_stats_kernel<<<(unsigned)(want < 148 * 8 ? want : 148 * 8), kSweepThreads, 0, st>>>(s, n, offset, range, hist,
                                                                                             first);
    count_launch();
    return cudaGetLastError();
}

}  // namespace asz
