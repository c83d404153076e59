// Per-target steps shared by the round kernels (k_field.cu) and the fused axis-2 rounds
// (k_lines.cu): the stencil predictions, the per-axis table reads, the QB index and the quotient
// of the quantisation step.
#pragma once
#include <cuda_runtime.h>

#include "dev_common.cuh"

namespace asz {

// ---------------------------------------------------------------------------------------------
// Prediction (compress.tpp:7-34, decompress.tpp:6-33) in the emitted form, by stencil case:
//   1D6R:            (float) fma(a*s5, fma(inner*s1, b*s3)) in double
//   left, one ref:   x-1
//   left, two refs:  (x-1 + x1) * 0.5
//   left, three:     (fmaf(x-1, 3, 6*x1) - x3) * 0.125
//   right edge:      fmaf(x-1, 3, -x-3) * 0.5
//   right second:    fmaf(x1, 3, fmaf(x-1, 6, -x-3)) * 0.125
//   interior 1D4R:   p=(float)(s3*(0.25-t)); (float)fma(0.25+t, s1, p) in double
__device__ __forceinline__ float predict_case(const float *__restrict__ c, uint64_t pos, uint64_t dist, uint32_t sc,
                                              float t) {
    switch (sc) {
    case kStencilQuintic: {
        float s1 = __fadd_rn(c[pos - dist], c[pos + dist]);
        float s3 = __fadd_rn(c[pos - 3 * dist], c[pos + 3 * dist]);
        float s5 = __fadd_rn(c[pos - 5 * dist], c[pos + 5 * dist]);
        double acc = __dmul_rn((double)s3, kQuinticB);
        acc = __fma_rn((double)s1, kQuinticI, acc);
        acc = __fma_rn((double)s5, kQuinticA, acc);
        return __double2float_rn(acc);
    }
    case kStencilLeft1:
        return c[pos - dist];
    case kStencilLeft2:
        return __fmul_rn(__fadd_rn(c[pos - dist], c[pos + dist]), 0.5f);
    case kStencilLeft3:
        return __fmul_rn(__fsub_rn(__fmaf_rn(c[pos - dist], 3.0f, __fmul_rn(c[pos + dist], 6.0f)), c[pos + 3 * dist]), 0.125f);
    case kStencilRight1:
        return __fmul_rn(__fmaf_rn(c[pos - dist], 3.0f, -c[pos - 3 * dist]), 0.5f);
    case kStencilRight2:
        return __fmul_rn(__fmaf_rn(c[pos + dist], 3.0f, __fmaf_rn(c[pos - dist], 6.0f, -c[pos - 3 * dist])), 0.125f);
    default: {
        float s3 = __fadd_rn(c[pos - 3 * dist], c[pos + 3 * dist]);
        float s1 = __fadd_rn(c[pos - dist], c[pos + dist]);
        double td = (double)t;
        float p1 = __double2float_rn(__dmul_rn((double)s3, __dsub_rn(0.25, td)));
        return __double2float_rn(__fma_rn(__dadd_rn(0.25, td), (double)s1, (double)p1));
    }
    }
}

// A target's stencil inputs, loaded ahead of its prediction: the neighbours that its stencil case
// uses (others are not read) through the read-only path. Within a round, no target reads a
// position that the round writes, so these loads may run ahead of the round's stores.
struct StencilIn {
    float m1, p1, m3, p3, m5, p5;
};

__device__ __forceinline__ StencilIn load_stencil(const float *__restrict__ c, uint64_t pos, uint64_t dist, uint32_t sc) {
    StencilIn v{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    switch (sc) {
    case kStencilQuintic:
        v.m5 = __ldg(c + pos - 5 * dist);
        v.p5 = __ldg(c + pos + 5 * dist);
        [[fallthrough]];
    case kStencilCubic:
        v.m3 = __ldg(c + pos - 3 * dist);
        v.p3 = __ldg(c + pos + 3 * dist);
        v.m1 = __ldg(c + pos - dist);
        v.p1 = __ldg(c + pos + dist);
        break;
    case kStencilLeft1:
        v.m1 = __ldg(c + pos - dist);
        break;
    case kStencilLeft2:
        v.m1 = __ldg(c + pos - dist);
        v.p1 = __ldg(c + pos + dist);
        break;
    case kStencilLeft3:
        v.m1 = __ldg(c + pos - dist);
        v.p1 = __ldg(c + pos + dist);
        v.p3 = __ldg(c + pos + 3 * dist);
        break;
    case kStencilRight1:
        v.m1 = __ldg(c + pos - dist);
        v.m3 = __ldg(c + pos - 3 * dist);
        break;
    default:  // kStencilRight2
        v.m1 = __ldg(c + pos - dist);
        v.p1 = __ldg(c + pos + dist);
        v.m3 = __ldg(c + pos - 3 * dist);
        break;
    }
    return v;
}

// predict_case on loaded inputs: the same operations in the same order.
__device__ __forceinline__ float predict_loaded(const StencilIn &v, uint32_t sc, float t) {
    switch (sc) {
    case kStencilQuintic: {
        float s1 = __fadd_rn(v.m1, v.p1);
        float s3 = __fadd_rn(v.m3, v.p3);
        float s5 = __fadd_rn(v.m5, v.p5);
        double acc = __dmul_rn((double)s3, kQuinticB);
        acc = __fma_rn((double)s1, kQuinticI, acc);
        acc = __fma_rn((double)s5, kQuinticA, acc);
        return __double2float_rn(acc);
    }
    case kStencilLeft1:
        return v.m1;
    case kStencilLeft2:
        return __fmul_rn(__fadd_rn(v.m1, v.p1), 0.5f);
    case kStencilLeft3:
        return __fmul_rn(__fsub_rn(__fmaf_rn(v.m1, 3.0f, __fmul_rn(v.p1, 6.0f)), v.p3), 0.125f);
    case kStencilRight1:
        return __fmul_rn(__fmaf_rn(v.m1, 3.0f, -v.m3), 0.5f);
    case kStencilRight2:
        return __fmul_rn(__fmaf_rn(v.p1, 3.0f, __fmaf_rn(v.m1, 6.0f, -v.m3)), 0.125f);
    default: {
        float s3 = __fadd_rn(v.m3, v.p3);
        float s1 = __fadd_rn(v.m1, v.p1);
        double td = (double)t;
        float p1 = __double2float_rn(__dmul_rn((double)s3, __dsub_rn(0.25, td)));
        return __double2float_rn(__fma_rn(__dadd_rn(0.25, td), (double)s1, (double)p1));
    }
    }
}

__device__ __forceinline__ AxisEntry load_entry(const AxisEntry *e) {
    const uint4 *p = reinterpret_cast<const uint4 *>(e);
    uint4 a = __ldg(p), b = __ldg(p + 1);
    AxisEntry r;
    r.ii = a.x;
    r.bb = a.y;
    r.jj = a.z;
    r.cc = a.w;
    r.pre = (uint64_t)b.x | ((uint64_t)b.y << 32);
    r.stencil = b.z;
    r.pad = b.w;
    return r;
}

// The parts of qb_index() that depend only on the line (k0, k1); qi = base + mul * e2.pre + local.
struct LineQB {
    uint64_t base, mul;
    uint32_t a, b;  // order 2: local = a * cc2 + jj2; order 0: (jj1 * cc2 + jj2) * cc0 + jj0; order 1 likewise
};

__device__ __forceinline__ LineQB line_qb(const RoundGeom &rg, const AxisEntry &e0, const AxisEntry &e1) {
    LineQB q;
    q.base = e0.pre * rg.total[1] * rg.total[2] + (uint64_t)e0.cc * e1.pre * rg.total[2];
    q.mul = (uint64_t)e0.cc * e1.cc;
    if (rg.order == 2) {
        q.a = e0.jj * e1.cc + e1.jj;
        q.b = 0;
    } else if (rg.order == 0) {
        q.a = e1.jj;  // times cc2, plus jj2, times cc0, plus jj0
        q.b = 0;
    } else {
        q.a = e0.jj;
        q.b = 0;
    }
    return q;
}

__device__ __forceinline__ uint64_t target_qb(const RoundGeom &rg, const LineQB &q, const AxisEntry &e0, const AxisEntry &e1,
                                              const AxisEntry &e2) {
    uint64_t local;
    if (rg.order == 2) local = (uint64_t)q.a * e2.cc + e2.jj;
    else if (rg.order == 0) local = ((uint64_t)q.a * e2.cc + e2.jj) * e0.cc + e0.jj;
    else local = ((uint64_t)q.a * e2.cc + e2.jj) * e1.cc + e1.jj;
    return q.base + q.mul * e2.pre + local;
}

// (diff * 0.5) / eb rounded to nearest, as far as lround of it is concerned: h * (1/eb) is within
// 2^-51.4 relative of the correctly rounded quotient, so unless it lies within 2^-48 relative of a
// rounding boundary of lround (a half-integer) both round to the same integer; the exact division
// runs only in that band.
__device__ __forceinline__ double quot_for_lround(double h, double eb, double rinv) {
    const double qa = __dmul_rn(h, rinv);
    const double aq = fabs(qa);
    const double fr = aq - floor(aq);
    if (aq < 0x1p50 && fabs(fr - 0.5) > aq * 0x1p-48 + 0x1p-60) return qa;
    return __ddiv_rn(h, eb);
}

}  // namespace asz
