// Internal definition of a registration pair: the device constants of one (grid, images, weights, reference).
#pragma once
#include "q1_common.cuh"

struct svp_pair {
    svp_grid grid;
    svp_weights w;
    svp::Q1Const q;
    int device = 0;
    // images and spline
    double *fixed = nullptr;      // (nz, ny, nx)
    double *coeff = nullptr;      // (nz, ny, nx) not-a-knot cubic coefficients
    double *knots[3] = {nullptr, nullptr, nullptr};  // x, y, z knot vectors (n + 4)
    double *spline_rcp[3] = {nullptr, nullptr, nullptr};  // per span, 14 reciprocal knot differences (n x 14)
    double *u_ref = nullptr;      // (nz, ny, nx, 3) frozen reference displacement
    // workspace
    double *loc1 = nullptr, *loc2 = nullptr;  // (24, ncell) per-cell vertex values (SoA)
    double *cellbuf = nullptr;                // (ncell)
    svp::dd *partial = nullptr;               // block partial sums
    long long partial_cap = 0;                // in dd entries
    double *result = nullptr;                 // small device result area (64 doubles)
    long long *counter = nullptr;             // small device counters (8)
    long long *cand = nullptr;                // candidate cells of the T69/T73 node JD extension (ncell)
    uint8_t *flags = nullptr;                 // (ncell) cells the float32 cell kernels hand to the float64 barrier
    // DST-I Poisson metric
    double *dst_half[3] = {nullptr, nullptr, nullptr};  // folded orthonormal DST-I half matrices, x, y, z
    double *dst_pad[3] = {nullptr, nullptr, nullptr};   // the same zero-padded to the passes' tiles (PadF64)
    int dst_n[3] = {0, 0, 0};                               // their transform lengths (free nodes per axis)
    // the same rounded to float32 for the mixed form, as TF32 parts: big parts of H0^T, H1^T, then the small parts
    unsigned *dst_tf32[3] = {nullptr, nullptr, nullptr};
    int precision = 0;                                      // SVP_PRECISION_PLAIN or SVP_PRECISION_MIXED
    double *dst_tmp = nullptr;                          // 2 * 3 * nfree scratch
    double *den = nullptr;                              // (nz-2, ny-2, nx-2) omega (a + b lambda)
    double den_a = -1, den_b = -1;
    int den_metric = -1;
};

namespace svp {
int pair_partials(svp_pair *p, long long blocks, int k);
int pair_locals(svp_pair *p, int n);
int pair_flags(svp_pair *p);
}  // namespace svp
