// Target geometry of one round, shared by the kernels and the host-side geometry check.
#pragma once
#include "dev_common.cuh"

namespace asz {

// Per-axis block tables of one round: count[b] targets of block b along the axis and prefix[b]
// (exclusive sum), laid out at RoundGeom::axis_off[a].
struct AxisTables {
    const uint64_t *count, *prefix;
};

struct Target {
    uint64_t pos, i, right, qi, block;
};

// Global target k of the round -> position, owning block, stencil bound and QB index.
ASZ_HD Target locate(const FieldGeom &fg, const RoundGeom &rg, AxisTables at, uint64_t k) {
    uint64_t k2 = k % rg.tcount[2], k1 = (k / rg.tcount[2]) % rg.tcount[1], k0 = k / (rg.tcount[1] * rg.tcount[2]);
    const uint64_t kk[3] = {k0, k1, k2};
    uint64_t ii[3], bb[3], jj[3], cc[3];
    for (int a = 0; a < 3; a++) {
        const uint64_t h = fg.origin[a];
        ii[a] = a == rg.dir ? h + rg.hs + 2 * rg.hs * kk[a] : (h == 0 ? rg.stride[a] * kk[a] : h + rg.stride[a] * (kk[a] + 1));
        bb[a] = owner_block_at(ii[a], h, fg.block_shape[a]);
        const uint64_t b0 = h + bb[a] * fg.block_shape[a];
        uint64_t start = b0 + (a == rg.dir ? rg.hs : (b0 == 0 ? 0 : rg.stride[a]));
        jj[a] = (ii[a] - start) / rg.stride[a];
        cc[a] = at.count[rg.axis_off[a] + bb[a]];
    }
    Target t;
    t.pos = (ii[0] * fg.n[1] + ii[1]) * fg.n[2] + ii[2];
    t.i = ii[rg.dir];
    const uint64_t r = fg.origin[rg.dir] + (bb[rg.dir] + 1) * fg.block_shape[rg.dir] + 1;
    t.right = r < fg.n[rg.dir] ? r : fg.n[rg.dir];
    // QB base of the block: per-axis prefix sums of the raster-ordered box sizes.
    uint64_t base = at.prefix[rg.axis_off[0] + bb[0]] * rg.total[1] * rg.total[2] +
                    cc[0] * at.prefix[rg.axis_off[1] + bb[1]] * rg.total[2] +
                    cc[0] * cc[1] * at.prefix[rg.axis_off[2] + bb[2]];
    // get_qb_index (asz_param.hpp:122-129).
    uint64_t local = rg.order == 0 ? (jj[1] * cc[2] + jj[2]) * cc[0] + jj[0]
                   : rg.order == 1 ? (jj[0] * cc[2] + jj[2]) * cc[1] + jj[1]
                                   : (jj[0] * cc[1] + jj[1]) * cc[2] + jj[2];
    t.qi = base + local;
    t.block = (bb[0] * fg.block_num[1] + bb[1]) * fg.block_num[2] + bb[2];
    return t;
}

ASZ_HD uint32_t stencil_case(uint64_t i, uint64_t hs, uint64_t right, bool quintic) {
    if (quintic && i >= 5 * hs && i + 5 * hs < right) return kStencilQuintic;
    if (i <= hs) {
        if (i + hs >= right) return kStencilLeft1;
        if (i + 3 * hs >= right) return kStencilLeft2;
        return kStencilLeft3;
    }
    if (i + hs >= right) return kStencilRight1;
    if (i + 3 * hs >= right) return kStencilRight2;
    return kStencilCubic;
}

// The per-axis part of locate() for lattice index k along axis a.
ASZ_HD AxisEntry axis_entry(const FieldGeom &fg, const RoundGeom &rg, AxisTables at, int a, uint64_t k) {
    AxisEntry e{};
    const uint64_t h = fg.origin[a];
    // Target lattice: odd multiples of hs past the origin along the round axis; on the other axes
    // the stride lattice from the origin, without the origin's face when it is not the field's.
    const uint64_t ii = a == rg.dir ? h + rg.hs + 2 * rg.hs * k : (h == 0 ? rg.stride[a] * k : h + rg.stride[a] * (k + 1));
    const uint64_t bb = owner_block_at(ii, h, fg.block_shape[a]);
    const uint64_t b0 = h + bb * fg.block_shape[a];
    const uint64_t start = b0 + (a == rg.dir ? rg.hs : (b0 == 0 ? 0 : rg.stride[a]));
    e.ii = (uint32_t)ii;
    e.bb = (uint32_t)bb;
    e.jj = (uint32_t)((ii - start) / rg.stride[a]);
    e.cc = (uint32_t)at.count[rg.axis_off[a] + bb];
    e.pre = at.prefix[rg.axis_off[a] + bb];
    if (a == rg.dir) {
        const uint64_t r = b0 + fg.block_shape[a] + 1;
        e.stencil = stencil_case(ii, rg.hs, r < fg.n[a] ? r : fg.n[a], fg.quintic != 0);
    }
    return e;
}

// Serialised QB index of the target with per-axis entries e0, e1, e2 (get_qb_index,
// asz_param.hpp:122-129, after the block's base offset).
ASZ_HD uint64_t qb_index(const RoundGeom &rg, const AxisEntry &e0, const AxisEntry &e1, const AxisEntry &e2) {
    const uint64_t base = e0.pre * rg.total[1] * rg.total[2] + (uint64_t)e0.cc * e1.pre * rg.total[2] +
                          (uint64_t)e0.cc * e1.cc * e2.pre;
    const uint64_t local = rg.order == 0 ? ((uint64_t)e1.jj * e2.cc + e2.jj) * e0.cc + e0.jj
                         : rg.order == 1 ? ((uint64_t)e0.jj * e2.cc + e2.jj) * e1.cc + e1.jj
                                         : ((uint64_t)e0.jj * e1.cc + e1.jj) * e2.cc + e2.jj;
    return base + local;
}

}  // namespace asz
