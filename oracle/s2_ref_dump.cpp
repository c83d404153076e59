// Oracle-side access to the unmodified reference prediction sweep, as a shared library.
//
// Test infrastructure only: oracle/Makefile builds it from the reference sources where they lie,
// with the reference's flags, and the product never links it. It compiles
// c_codes/s2_many_prediction.cpp as is, with `main` renamed, and exports C entry points that call
// the reference's own functions on caller-given inputs:
//   s2ref_dot       -> compress_1d4r_dot / compress_2d4r_dot / compress_1d6r_dot (:28-87) over a
//                      list of target coordinates, returning every QB and the three running sums
//   s2ref_h1        -> get_H1 (c_codes/get_H.hpp)
//   s2ref_grid      -> six_reference_grid (:89-124)
//   s2ref_common    -> for_each_common_target (:126-149) and common_target_count (:151-162)
#define main asz_reference_s2_many_prediction_main
#include "s2_many_prediction.cpp"
#undef main

#include <cstring>

extern "C" {

// kind: 0 = 1d4r (c0 = t), 1 = 2d4r (c0 = t), 2 = 1d6r (c0 = a, c1 = b). coords: n x 3 (i0, i1, i2).
// sums: mse, pred_rmse, pred_mae after the last target (before the reference divides them).
int s2ref_dot(int kind, const float *data, const uint64_t dims[3], const uint64_t dists[2], double abs_eb,
              double neg_2_eb, double c0, double c1, const uint64_t *coords, uint64_t n, int64_t *qb_out,
              double sums[3]) {
    vector<float> d(data, data + dims[0] * dims[1] * dims[2]);
    vector<uint64_t> shape = {dims[0], dims[1], dims[2]};
    vector<uint64_t> dist = {dists[0], dists[1]};
    vector<int64_t> qb;
    qb.reserve(n);
    double mse = 0, rmse = 0, mae = 0;
    for (uint64_t k = 0; k < n; k++) {
        const uint64_t *c = coords + 3 * k;
        if (kind == 0)
            compress_1d4r_dot(qb, mse, rmse, mae, d, shape, dist, abs_eb, neg_2_eb, {c0}, c[0], c[1], c[2]);
        else if (kind == 1)
            compress_2d4r_dot(qb, mse, rmse, mae, d, shape, dist, abs_eb, neg_2_eb, {c0}, c[0], c[1], c[2]);
        else if (kind == 2)
            compress_1d6r_dot(qb, mse, rmse, mae, d, shape, dist, abs_eb, neg_2_eb, {c0, c1}, c[0], c[1], c[2]);
        else
            return -1;
    }
    std::memcpy(qb_out, qb.data(), n * sizeof(int64_t));
    sums[0] = mse;
    sums[1] = rmse;
    sums[2] = mae;
    return 0;
}

double s2ref_h1(const int64_t *qb, uint64_t n) {
    vector<int64_t> v(qb, qb + n);
    return get_H1(v);
}

// Writes up to cap (a, b) pairs; returns the grid size.
uint64_t s2ref_grid(const char *mode, double *out, uint64_t cap) {
    auto g = six_reference_grid(mode);
    for (uint64_t i = 0; i < g.size() && i < cap; i++) {
        out[2 * i] = g[i][0];
        out[2 * i + 1] = g[i][1];
    }
    return g.size();
}

// Writes the common targets of QB order `order` (up to cap, as i0 i1 i2 triples); returns
// common_target_count(dims), and the visited count in *visited.
uint64_t s2ref_common(const uint64_t dims[3], int order, uint64_t *coords, uint64_t cap, uint64_t *visited) {
    vector<uint64_t> shape = {dims[0], dims[1], dims[2]};
    uint64_t k = 0;
    for_each_common_target(shape, order, [&](uint64_t i0, uint64_t i1, uint64_t i2) {
        if (k < cap) {
            coords[3 * k] = i0;
            coords[3 * k + 1] = i1;
            coords[3 * k + 2] = i2;
        }
        k++;
    });
    *visited = k;
    return common_target_count(shape);
}

}  // extern "C"
