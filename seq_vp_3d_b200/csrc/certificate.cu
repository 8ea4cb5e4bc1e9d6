// Whole-cell Jacobian-determinant certificate on the GPU, bit-identical to the reference CPU certifier.
//
// Stages (jd_curl/three_d/feasibility.py:623 _certify_map_parallel):
//   1. edge-hull interval enclosure of every cell (compiled_enclosure.py:210 _chunk_hoisted_margins),
//      with the per-tile flag rule (feasibility.py:650);
//   2. float Bernstein prescreen with an a-priori rounding bound (certificate_prescreen.py:66) of the unproven cells;
//   3. interval Bernstein fallback arrays (compiled_fallback.py:63) and lowest-bound-first subdivision
//      (feasibility.py:295 _classify), one warp per cell with the box heap in scratch memory;
//   4. the record: status, reason, counts, bounds and the first witness (feasibility.py:755-771).
// This file is compiled with -fmad=false and uses explicit round-to-nearest intrinsics for every certificate
// operation, so no product can be contracted into an FMA.
#include <cuda.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "svp_common.cuh"

namespace svp {
namespace {

// Division by the spacing, x / h_j correctly rounded.  Where h_j is a power of two, 1/h_j is exact and x * (1/h_j) is
// the same correctly rounded quotient (one rounding of the same exact value, subnormal and overflowing results
// included), for a multiply instead of a division.
struct AxisDiv {
    double h[3], ih[3];
    int pow2[3];
};
AxisDiv axis_div(const double h[3]) {
    AxisDiv d;
    for (int j = 0; j < 3; j++) {
        int e = 0;
        d.h[j] = h[j];
        d.pow2[j] = std::isfinite(h[j]) && h[j] > 0 && std::frexp(h[j], &e) == .5 && e > -1000 && e < 1000;
        d.ih[j] = d.pow2[j] ? 1. / h[j] : 0.;
    }
    return d;
}
__device__ __forceinline__ double div_axis(double x, const AxisDiv &d, int j) {
    return d.pow2[j] ? rmul(x, d.ih[j]) : rdiv(x, d.h[j]);
}

// ---------------------------------------------------------------------------------------- directed rounding
// The directed-rounding arithmetic of the mixed form's certificate: every interval operation rounds its lower end
// toward -inf and its upper end toward +inf (__d*_rd / __d*_ru), one rounding per end.  Each such end lies inside
// the nearest-plus-one-ulp end of the reference's arithmetic (RD(x) >= step_down(RN(x)), RU(x) <= step_up(RN(x))),
// so every enclosure is a valid one at least as tight as the reference's: a cell the reference proves stays proven,
// and a witness (an upper bound <= 0) is a true violation in both.  Validity: both ends finite and lo <= hi.
__device__ __forceinline__ bool dvalid(double lo, double hi) { return finite64(lo) && finite64(hi) && lo <= hi; }
__device__ __forceinline__ bool dadd(double al, double ah, double bl, double bh, double &rl, double &rh) {
    rl = __dadd_rd(al, bl);
    rh = __dadd_ru(ah, bh);
    return dvalid(rl, rh);
}
__device__ __forceinline__ bool dsub(double al, double ah, double bl, double bh, double &rl, double &rh) {
    rl = __dsub_rd(al, bh);
    rh = __dsub_ru(ah, bl);
    return dvalid(rl, rh);
}
__device__ __forceinline__ bool dmul(double al, double ah, double bl, double bh, double &rl, double &rh) {
    rl = nmin(nmin(nmin(__dmul_rd(al, bl), __dmul_rd(al, bh)), __dmul_rd(ah, bl)), __dmul_rd(ah, bh));
    rh = nmax(nmax(nmax(__dmul_ru(al, bl), __dmul_ru(al, bh)), __dmul_ru(ah, bl)), __dmul_ru(ah, bh));
    return dvalid(rl, rh);
}
// interval / h_j with h_j > 0 (a power of two: the exact reciprocal multiply, directed)
__device__ __forceinline__ double div_axis_rd(double x, const AxisDiv &d, int j) {
    return d.pow2[j] ? __dmul_rd(x, d.ih[j]) : __ddiv_rd(x, d.h[j]);
}
__device__ __forceinline__ double div_axis_ru(double x, const AxisDiv &d, int j) {
    return d.pow2[j] ? __dmul_ru(x, d.ih[j]) : __ddiv_ru(x, d.h[j]);
}
// the left-associated cofactor expansion of idet, directed
__device__ __forceinline__ bool ddet(const double fl[3][3], const double fh[3][3], double &jl, double &jh) {
    double p1l, p1h, p2l, p2h, al, ah, bl, bh, cl, ch, t1l, t1h, t2l, t2h, sl, sh, t3l, t3h;
    bool ok = true;
    ok &= dmul(fl[1][1], fh[1][1], fl[2][2], fh[2][2], p1l, p1h);
    ok &= dmul(fl[1][2], fh[1][2], fl[2][1], fh[2][1], p2l, p2h);
    ok &= dsub(p1l, p1h, p2l, p2h, al, ah);
    ok &= dmul(fl[1][2], fh[1][2], fl[2][0], fh[2][0], p1l, p1h);
    ok &= dmul(fl[1][0], fh[1][0], fl[2][2], fh[2][2], p2l, p2h);
    ok &= dsub(p1l, p1h, p2l, p2h, bl, bh);
    ok &= dmul(fl[1][0], fh[1][0], fl[2][1], fh[2][1], p1l, p1h);
    ok &= dmul(fl[1][1], fh[1][1], fl[2][0], fh[2][0], p2l, p2h);
    ok &= dsub(p1l, p1h, p2l, p2h, cl, ch);
    ok &= dmul(fl[0][0], fh[0][0], al, ah, t1l, t1h);
    ok &= dmul(fl[0][1], fh[0][1], bl, bh, t2l, t2h);
    ok &= dadd(t1l, t1h, t2l, t2h, sl, sh);
    ok &= dmul(fl[0][2], fh[0][2], cl, ch, t3l, t3h);
    ok &= dadd(sl, sh, t3l, t3h, jl, jh);
    return ok;
}
// the interval operations of either arithmetic (DIR: directed; else the reference's nearest plus one ulp)
template <bool DIR>
__device__ __forceinline__ bool Iadd(double al, double ah, double bl, double bh, double &rl, double &rh) {
    if constexpr (DIR) return dadd(al, ah, bl, bh, rl, rh);
    else return iadd(al, ah, bl, bh, rl, rh);
}
template <bool DIR>
__device__ __forceinline__ bool Isub(double al, double ah, double bl, double bh, double &rl, double &rh) {
    if constexpr (DIR) return dsub(al, ah, bl, bh, rl, rh);
    else return isub(al, ah, bl, bh, rl, rh);
}
template <bool DIR>
__device__ __forceinline__ bool Imul(double al, double ah, double bl, double bh, double &rl, double &rh) {
    if constexpr (DIR) return dmul(al, ah, bl, bh, rl, rh);
    else return imul(al, ah, bl, bh, rl, rh);
}
template <bool DIR>
__device__ __forceinline__ bool Idet(const double fl[3][3], const double fh[3][3], double &jl, double &jh) {
    if constexpr (DIR) return ddet(fl, fh, jl, jh);
    else return idet(fl, fh, jl, jh);
}

struct CellGrid {
    long long nx, ny, nz, cx, cy, cz, ncell;
    double h[3];
    AxisDiv div;
};

CellGrid cell_grid(const svp_grid *g) {
    CellGrid c;
    c.nx = g->nx; c.ny = g->ny; c.nz = g->nz;
    c.cx = g->nx - 1; c.cy = g->ny - 1; c.cz = g->nz - 1;
    c.ncell = c.cx * c.cy * c.cz;
    c.h[0] = g->hx; c.h[1] = g->hy; c.h[2] = g->hz;
    c.div = axis_div(c.h);
    return c;
}

__device__ __forceinline__ long long cell_base(long long c, const CellGrid &g) {
    long long x0, y0, z0;
    unflatten3(c, g.cx, g.cy, x0, y0, z0);
    return (z0 * g.ny + y0) * g.nx + x0;
}
__device__ __forceinline__ long long vnode(long long base, int a, long long ny, long long nx) {
    return base + (long long)(a >> 2) * ny * nx + (long long)((a >> 1) & 1) * nx + (a & 1);
}
// e-th vertex with bit j clear, in increasing vertex order (the reference's edge loop order)
__device__ __forceinline__ int edge_start(int j, int e) {
    int k = 0;
    for (int a = 0; a < 8; a++) {
        if (a & (1 << j)) continue;
        if (k == e) return a;
        k++;
    }
    return 0;
}

// ============================================================================================== 1. edge hull
// F_rj interval: hull of the 4 edge differences (from +inf / -inf in edge order), outward, /h, outward, + identity.
template <bool DIR>
__device__ __forceinline__ bool hull_entry_v(const double v[8][3], int j, int r, const AxisDiv &dv, double &lo,
                                             double &hi) {
    bool ok = true;
    double lower = __longlong_as_double(0x7FF0000000000000LL), upper = -lower;
    double l, hh;
    if constexpr (DIR) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            int a = edge_start(j, e), b = a | (1 << j);
            double dl = __dsub_rd(v[b][r], v[a][r]), dh = __dsub_ru(v[b][r], v[a][r]);
            ok &= finite64(dl) && finite64(dh);
            lower = nmin(lower, dl);
            upper = nmax(upper, dh);
        }
        l = div_axis_rd(lower, dv, j);
        hh = div_axis_ru(upper, dv, j);
        ok &= dvalid(l, hh);
    } else {
#pragma unroll
        for (int e = 0; e < 4; e++) {
            int a = edge_start(j, e), b = a | (1 << j);
            double d = rsub(v[b][r], v[a][r]);
            ok &= finite64(d);
            lower = nmin(lower, d);
            upper = nmax(upper, d);
        }
        ok &= iout(lower, upper, l, hh);
        ok &= iout(div_axis(l, dv, j), div_axis(hh, dv, j), l, hh);
    }
    double id = (r == j) ? 1.0 : 0.0;
    ok &= Iadd<DIR>(l, hh, id, id, lo, hi);
    return ok;
}

template <bool DIR>
__global__ void __launch_bounds__(256) edge_hull_kernel(const double *__restrict__ u, CellGrid g, double delta,
                                                        double *__restrict__ margin, uint8_t *__restrict__ flag) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long base = cell_base(c, g);
        double v[8][3];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) v[a][r] = __ldg(u + 3 * vnode(base, a, g.ny, g.nx) + r);
        double fl[3][3], fh[3][3];
        bool ok = true;
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int r = 0; r < 3; r++) ok &= hull_entry_v<DIR>(v, j, r, g.div, fl[r][j], fh[r][j]);
        double jl, jh, ml, mh;
        ok &= Idet<DIR>(fl, fh, jl, jh);
        if constexpr (DIR) ok &= dsub(jl, jh, delta, delta, ml, mh);
        else ok &= iout(rsub(jl, delta), rsub(jh, delta), ml, mh);
        margin[c] = ml;
        flag[c] = ok ? 0 : 1;
    }
}

// ============================================================================================== 2. prescreen
struct PrescreenConst {
    double D[3 * 27 * 8];  // closed27 Q1 derivative table (3, 27, 8), passed by value (constant bank)
    double g12, g6, g3, sq27, eta;
    int usable;            // 0: table not finite or has a subnormal entry -> every bound NaN
    int sparse;            // 1: every structurally vanishing entry (table_nonzero false) is exactly zero
};

// D[j][p][a] = (+-1/h_j) f_k f_l over the two axes k, l != j, with f = c (vertex bit 1) or 1 - c (bit 0) and c in
// {0, 1/2, 1} the point's coordinate: the entry vanishes exactly when some factor is 1 - 1 or 0.  Point
// p = x + 3 y + 9 z, vertex a = x + 2 y + 4 z.
__host__ __device__ constexpr bool table_nonzero(int j, int p, int a) {
    const int c[3] = {p % 3, (p / 3) % 3, p / 9};
    for (int k = 0; k < 3; k++) {
        if (k == j) continue;
        const int bit = (a >> k) & 1;
        if ((bit == 1 && c[k] == 0) || (bit == 0 && c[k] == 2)) return false;
    }
    return true;
}

__device__ double prescreen_cell(const double *__restrict__ u, long long base, long long ny, long long nx,
                                 const PrescreenConst &k) {
    long long off[8];
#pragma unroll
    for (int a = 0; a < 8; a++) off[a] = (long long)(a >> 2) * ny * nx + (long long)((a >> 1) & 1) * nx + (a & 1);
    double uv[8][3];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int r = 0; r < 3; r++) uv[a][r] = __ldg(u + 3 * (base + off[a]) + r);
    double b[27];
    double sigma = 0., phi = 0., big = 0.;
    bool finite = true;
    for (int p = 0; p < 27; p++) {
        double F[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
                double acc = 0., mag = 0.;
#pragma unroll
                for (int a = 0; a < 8; a++) {
                    double term = rmul(uv[a][r], k.D[(j * 27 + p) * 8 + a]);
                    acc = radd(acc, term);
                    mag = radd(mag, fabs(term));
                }
                F[r][j] = acc;
                if (mag > sigma) sigma = mag;
            }
            F[r][r] = radd(F[r][r], 1.);
        }
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                if (fabs(F[r][j]) > phi) phi = fabs(F[r][j]);
        double t0 = rmul(F[0][0], rsub(rmul(F[1][1], F[2][2]), rmul(F[1][2], F[2][1])));
        double t1 = rmul(F[0][1], rsub(rmul(F[1][2], F[2][0]), rmul(F[1][0], F[2][2])));
        double t2 = rmul(F[0][2], rsub(rmul(F[1][0], F[2][1]), rmul(F[1][1], F[2][0])));
        double v = radd(radd(t0, t1), t2);
        b[p] = v;
        if (fabs(v) > big) big = fabs(v);
    }
    // separable T along x, y, z: middle entry of each line -> 2 b_m - (b_l + b_r) / 2
#pragma unroll
    for (int s = 0; s < 3; s++) {
        int stride = s == 0 ? 1 : (s == 1 ? 3 : 9);
#pragma unroll
        for (int p = 0; p < 27; p++)
            if ((p / stride) % 3 == 1) b[p] = rsub(rmul(2., b[p]), rmul(.5, radd(b[p - stride], b[p + stride])));
    }
    double e = radd(rmul(k.g12, radd(sigma, phi)), k.eta);
    double P = radd(phi, e);
    double inner = radd(radd(rmul(rmul(3., P), P), rmul(rmul(3., P), e)), rmul(e, e));
    double ej = radd(rmul(rmul(k.sq27, e), inner), rmul(rmul(rmul(rmul(6., k.g6), P), P), P));
    double bound = radd(rmul(1.01, radd(rmul(27., ej), rmul(rmul(135., k.g3), big))), k.eta);
    double low = __longlong_as_double(0x7FF0000000000000LL);
    for (int p = 0; p < 27; p++) {
        double w = b[p];
        if (!(w == w) || !finite64(w)) finite = false;
        else if (w < low) low = w;
    }
    if (!(bound == bound) || !finite64(bound) || !(sigma == sigma) || !finite64(sigma)) finite = false;
    return finite ? rsub(low, bound) : __longlong_as_double(0x7FF8000000000000LL);
}

// The same bound with the 27 points unrolled and the vanishing table entries' terms left out of the 8-term sums
// (about 55% of them).  For a finite u, bitwise prescreen_cell's value: a left-out term is a signed zero, so every
// partial sum keeps its value (only the sign of a zero sum may differ), the magnitude sums add +0, and a zero's sign
// cannot reach the bound (it enters products and sums that end in low - bound with bound > 0, and the min and max
// compare -0 equal to +0).  certify_map runs the prescreen only on finite states.
template <int P>
__device__ __forceinline__ void prescreen_point(const double (&uv)[8][3], const PrescreenConst &k, double &b,
                                                double &sigma, double &phi, double &big) {
    double F[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double acc = 0., mag = 0.;
#pragma unroll
            for (int a = 0; a < 8; a++) {
                if (table_nonzero(j, P, a)) {
                    double term = rmul(uv[a][r], k.D[(j * 27 + P) * 8 + a]);
                    acc = radd(acc, term);
                    mag = radd(mag, fabs(term));
                }
            }
            F[r][j] = acc;
            if (mag > sigma) sigma = mag;
        }
        F[r][r] = radd(F[r][r], 1.);
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            if (fabs(F[r][j]) > phi) phi = fabs(F[r][j]);
    double t0 = rmul(F[0][0], rsub(rmul(F[1][1], F[2][2]), rmul(F[1][2], F[2][1])));
    double t1 = rmul(F[0][1], rsub(rmul(F[1][2], F[2][0]), rmul(F[1][0], F[2][2])));
    double t2 = rmul(F[0][2], rsub(rmul(F[1][0], F[2][1]), rmul(F[1][1], F[2][0])));
    double v = radd(radd(t0, t1), t2);
    b = v;
    if (fabs(v) > big) big = fabs(v);
}
template <int... Ps>
__device__ __forceinline__ void prescreen_points(std::integer_sequence<int, Ps...>, const double (&uv)[8][3],
                                                 const PrescreenConst &k, double *bs, int T, double &sigma,
                                                 double &phi, double &big) {
    double b;
    ((prescreen_point<Ps>(uv, k, b, sigma, phi, big), bs[Ps * T] = b), ...);     // p = 0 .. 26 in order
}
// bs: the thread's 27-entry slice of shared memory (stride T), which holds the point values between the passes
__device__ double prescreen_cell_sparse(const double *__restrict__ u, long long base, long long ny, long long nx,
                                        const PrescreenConst &k, double *bs, int T) {
    double uv[8][3];
#pragma unroll
    for (int a = 0; a < 8; a++) {
        const long long off = (long long)(a >> 2) * ny * nx + (long long)((a >> 1) & 1) * nx + (a & 1);
#pragma unroll
        for (int r = 0; r < 3; r++) uv[a][r] = __ldg(u + 3 * (base + off) + r);
    }
    double sigma = 0., phi = 0., big = 0.;
    prescreen_points(std::make_integer_sequence<int, 27>(), uv, k, bs, T, sigma, phi, big);
    double b[27];
#pragma unroll
    for (int p = 0; p < 27; p++) b[p] = bs[p * T];
#pragma unroll
    for (int s = 0; s < 3; s++) {
        int stride = s == 0 ? 1 : (s == 1 ? 3 : 9);
#pragma unroll
        for (int p = 0; p < 27; p++)
            if ((p / stride) % 3 == 1) b[p] = rsub(rmul(2., b[p]), rmul(.5, radd(b[p - stride], b[p + stride])));
    }
    double e = radd(rmul(k.g12, radd(sigma, phi)), k.eta);
    double P = radd(phi, e);
    double inner = radd(radd(rmul(rmul(3., P), P), rmul(rmul(3., P), e)), rmul(e, e));
    double ej = radd(rmul(rmul(k.sq27, e), inner), rmul(rmul(rmul(rmul(6., k.g6), P), P), P));
    double bound = radd(rmul(1.01, radd(rmul(27., ej), rmul(rmul(135., k.g3), big))), k.eta);
    double low = __longlong_as_double(0x7FF0000000000000LL);
    bool finite = true;
#pragma unroll
    for (int p = 0; p < 27; p++) {
        double w = b[p];
        if (!(w == w) || !finite64(w)) finite = false;
        else if (w < low) low = w;
    }
    if (!(bound == bound) || !finite64(bound) || !(sigma == sigma) || !finite64(sigma)) finite = false;
    return finite ? rsub(low, bound) : __longlong_as_double(0x7FF8000000000000LL);
}

template <bool SPARSE>
__global__ void __launch_bounds__(128) prescreen_kernel(const double *__restrict__ u, CellGrid g,
                                                        const long long *__restrict__ cells, long long n,
                                                        const PrescreenConst k, double *__restrict__ out) {
    __shared__ double slice[27 * 128];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long base = cell_base(cells[i], g);
        out[i] = !k.usable ? __longlong_as_double(0x7FF8000000000000LL)
                 : SPARSE  ? prescreen_cell_sparse(u, base, g.ny, g.nx, k, slice + threadIdx.x, blockDim.x)
                           : prescreen_cell(u, base, g.ny, g.nx, k);
    }
}
void launch_prescreen(const double *u, const CellGrid &g, const long long *cells, long long n,
                      const PrescreenConst &k, double *out, cudaStream_t s) {
    if (k.sparse)
        prescreen_kernel<true><<<blocks_for(n, 128, 8), 128, 0, s>>>(u, g, cells, n, k, out);
    else
        prescreen_kernel<false><<<blocks_for(n, 128, 8), 128, 0, s>>>(u, g, cells, n, k, out);
}

// ============================================================================================== 3a. fallback arrays
__device__ __forceinline__ double edge_weight(int j, int e, int p) {
    int a = edge_start(j, e);
    double coord[3] = {(p % 3) * .5, ((p / 3) % 3) * .5, (p / 9) * .5};
    double w = 1.;
    for (int kk = 0; kk < 3; kk++) {
        if (kk == j) continue;
        w = rmul(w, ((a >> kk) & 1) ? coord[kk] : rsub(1., coord[kk]));
    }
    return w;
}

// One cell per warp (v: its 24 vertex displacements, vertex-major, in every lane; outputs with stride 1, 27 entries
// each; sb: 54 doubles of the warp's shared memory).  Lane p < 27 evaluates closed27 point p: the interval J - delta
// from the outward-rounded edge quotients, and the float sample.  The Lagrange -> Bernstein passes (x, y, z) update
// the middle entries of each line on their own lanes, with a warp barrier between passes.  Bitwise the sequential
// form: each point's arithmetic is the same, and a pass reads only entries it does not write.  Returns ok for the
// whole cell (warp-uniform).
template <bool DIR>
__device__ bool fallback_cell_warp(const double v[24], const AxisDiv &dv, double delta, double *plo, double *phi,
                                   double *clo, double *chi, double *smp, double *sb) {
    const int p = threadIdx.x & 31;
    const bool point = p < 27;
    bool ok = true;
    double elo[3][4][3], ehi[3][4][3];
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            int a = edge_start(j, e), b = a | (1 << j);
#pragma unroll
            for (int r = 0; r < 3; r++) {
                if constexpr (DIR) {
                    // [RD(vb - va), RU(vb - va)] / h_j directed (h_j > 0)
                    double dl = __dsub_rd(v[3 * b + r], v[3 * a + r]), dh = __dsub_ru(v[3 * b + r], v[3 * a + r]);
                    ok &= dvalid(dl, dh);
                    elo[j][e][r] = div_axis_rd(dl, dv, j);
                    ehi[j][e][r] = div_axis_ru(dh, dv, j);
                    ok &= dvalid(elo[j][e][r], ehi[j][e][r]);
                } else {
                    double d = rsub(v[3 * b + r], v[3 * a + r]);
                    double sl, sh;
                    ok &= iout(d, d, sl, sh);
                    double x1 = div_axis(sl, dv, j), x2 = div_axis(sh, dv, j);
                    ok &= iout(nmin(nmin(nmin(x1, x1), x2), x2), nmax(nmax(nmax(x1, x1), x2), x2), elo[j][e][r],
                               ehi[j][e][r]);
                }
            }
        }
    if (point) {
        double fl[3][3], fh[3][3];
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int r = 0; r < 3; r++) {
                double dl = 0., dh = 0.;
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    double w = edge_weight(j, e, p), wl, wh;
                    if constexpr (DIR) ok &= dmul(elo[j][e][r], ehi[j][e][r], w, w, wl, wh);
                    else ok &= iout(rmul(elo[j][e][r], w), rmul(ehi[j][e][r], w), wl, wh);
                    ok &= Iadd<DIR>(dl, dh, wl, wh, dl, dh);
                }
                double c = (r == j) ? 1. : 0.;
                ok &= Iadd<DIR>(dl, dh, c, c, fl[r][j], fh[r][j]);
            }
        double jl, jh, ml, mh;
        ok &= Idet<DIR>(fl, fh, jl, jh);
        ok &= Isub<DIR>(jl, jh, delta, delta, ml, mh);
        plo[p] = ml; phi[p] = mh;
        sb[p] = ml; sb[27 + p] = mh;
    }
    __syncwarp();
    // lagrange_to_bernstein: axes x, y, z; middle <- 2 b - (a + c) * .5, all outward
#pragma unroll
    for (int s = 0; s < 3; s++) {
        const int stride = s == 0 ? 1 : (s == 1 ? 3 : 9);
        const bool mid = point && (p / stride) % 3 == 1;
        double nl = 0., nh = 0.;
        if (mid) {
            int a0 = p - stride, a2 = p + stride;
            double ml1, mh1, sl1, sh1, hl1, hh1;
            ok &= Imul<DIR>(sb[p], sb[27 + p], 2., 2., ml1, mh1);
            ok &= Iadd<DIR>(sb[a0], sb[27 + a0], sb[a2], sb[27 + a2], sl1, sh1);
            ok &= Imul<DIR>(sl1, sh1, .5, .5, hl1, hh1);
            ok &= Isub<DIR>(ml1, mh1, hl1, hh1, nl, nh);
        }
        __syncwarp();
        if (mid) { sb[p] = nl; sb[27 + p] = nh; }
        __syncwarp();
    }
    if (point) {
        clo[p] = sb[p]; chi[p] = sb[27 + p];
        // float64 sample: F = I + sum_(j,e) ((v_b - v_a) / h) w, cofactors, ((0 + t0) + t1) + t2
        double fs[3][3];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int j = 0; j < 3; j++) fs[r][j] = (r == j) ? 1. : 0.;
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                int a = edge_start(j, e), b = a | (1 << j);
                double w = edge_weight(j, e, p);
#pragma unroll
                for (int r = 0; r < 3; r++)
                    fs[r][j] = radd(fs[r][j], rmul(div_axis(rsub(v[3 * b + r], v[3 * a + r]), dv, j), w));
            }
        bool finite = true;
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int j = 0; j < 3; j++) finite = finite && finite64(fs[r][j]);
        double a00 = rsub(rmul(fs[1][1], fs[2][2]), rmul(fs[1][2], fs[2][1]));
        double a01 = rsub(rmul(fs[1][2], fs[2][0]), rmul(fs[1][0], fs[2][2]));
        double a02 = rsub(rmul(fs[1][0], fs[2][1]), rmul(fs[1][1], fs[2][0]));
        double a10 = rsub(rmul(fs[2][1], fs[0][2]), rmul(fs[2][2], fs[0][1]));
        double a11 = rsub(rmul(fs[2][2], fs[0][0]), rmul(fs[2][0], fs[0][2]));
        double a12 = rsub(rmul(fs[2][0], fs[0][1]), rmul(fs[2][1], fs[0][0]));
        double a20 = rsub(rmul(fs[0][1], fs[1][2]), rmul(fs[0][2], fs[1][1]));
        double a21 = rsub(rmul(fs[0][2], fs[1][0]), rmul(fs[0][0], fs[1][2]));
        double a22 = rsub(rmul(fs[0][0], fs[1][1]), rmul(fs[0][1], fs[1][0]));
        finite = finite && finite64(a00) && finite64(a01) && finite64(a02) && finite64(a10) && finite64(a11) &&
                 finite64(a12) && finite64(a20) && finite64(a21) && finite64(a22);
        double t0 = rmul(fs[0][0], a00), t1 = rmul(fs[0][1], a01), t2 = rmul(fs[0][2], a02);
        double sv = radd(radd(radd(0., t0), t1), t2);
        finite = finite && finite64(t0) && finite64(t1) && finite64(t2) && finite64(sv);
        smp[p] = sv;
        ok = ok && finite;
    }
    return __all_sync(0xFFFFFFFFu, ok);
}

constexpr int kFallbackWarps = 4;   // cells per 128-thread block

// Standalone cells: vertices (n, 8, 3), one warp per cell
template <bool DIR>
__global__ void __launch_bounds__(32 * kFallbackWarps) fallback_vertices_kernel(
    const double *__restrict__ vertices, long long n, const AxisDiv dv, double delta, double *plo, double *phi,
    double *clo, double *chi, double *smp, uint8_t *ok) {
    __shared__ double sb[kFallbackWarps][54];
    const int w = threadIdx.x >> 5;
    for (long long i = blockIdx.x * (long long)kFallbackWarps + w; i < n; i += (long long)gridDim.x * kFallbackWarps) {
        double v[24];
#pragma unroll
        for (int k = 0; k < 24; k++) v[k] = vertices[24 * i + k];
        bool good = fallback_cell_warp<DIR>(v, dv, delta, plo + 27 * i, phi + 27 * i, clo + 27 * i, chi + 27 * i,
                                            smp + 27 * i, sb[w]);
        if ((threadIdx.x & 31) == 0) ok[i] = good;
        __syncwarp();
    }
}

// Grid cells from a list: vertices gathered from u, one warp per cell
template <bool DIR>
__global__ void __launch_bounds__(32 * kFallbackWarps) fallback_grid_kernel(
    const double *__restrict__ u, CellGrid g, const long long *__restrict__ cells, long long n, double delta,
    double *plo, double *phi, double *clo, double *chi, double *smp, uint8_t *ok) {
    __shared__ double sb[kFallbackWarps][54];
    const int w = threadIdx.x >> 5;
    for (long long i = blockIdx.x * (long long)kFallbackWarps + w; i < n; i += (long long)gridDim.x * kFallbackWarps) {
        long long base = cell_base(cells[i], g);
        double v[24];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) v[3 * a + r] = __ldg(u + 3 * vnode(base, a, g.ny, g.nx) + r);
        bool good = fallback_cell_warp<DIR>(v, g.div, delta, plo + 27 * i, phi + 27 * i, clo + 27 * i,
                                            chi + 27 * i, smp + 27 * i, sb[w]);
        if ((threadIdx.x & 31) == 0) ok[i] = good;
        __syncwarp();
    }
}

// ============================================================================================== 3b. subdivision
// Status / reason codes: see svp3d.h.
enum { ST_FEASIBLE = 0, ST_INFEASIBLE = 1, ST_UNCERTAIN = 2 };
enum { R_ENCLOSURE = 0, R_BERNSTEIN = 1, R_VIOLATION = 2, R_ARITH = 3, R_SUBDIV_BUDGET = 4, R_NONFINITE = 5,
       R_BOUNDARY = 6, R_DOMAIN = 7, R_SAMPLE_WITNESS = 9, R_SUBDIV_WITNESS = 10, R_BOX_BUDGET = 11,
       R_DEPTH_BUDGET = 12 };

// Per-warp scratch layout for S slots: coefficients (S, 54) doubles, meta (S, 8) doubles (low xyz, high xyz, key),
// serial (S) int64, depth (S) int32, heap (S) int32, free stack (S) int32.  The per-warp stride is rounded up to
// 256 bytes so that every warp's float64/int64 arrays stay 8-byte aligned.
__host__ __device__ inline size_t warp_scratch_bytes(long long slots) {
    size_t b = (size_t)slots * (54 * 8 + 8 * 8 + 8 + 4 + 4 + 4);
    return (b + 255) / 256 * 256;
}

__device__ __forceinline__ double warp_min27(double x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        double y = __shfl_xor_sync(0xFFFFFFFFu, x, o);
        x = y < x ? y : x;
    }
    return x;
}

// Priority queue of the pending boxes of one cell.  Lowest-bound-first (AdaptiveCertificateConfig family): key = the
// box's lowest Bernstein coefficient, ties by creation serial (feasibility.py:319 heap of (lower, serial, box)).
// Depth-first (the bare CertificateConfig's list used as a stack, feasibility.py:353-354): the most recently pushed
// box pops first, i.e. the largest serial, with the left child pushed after the right one.
struct WarpHeap {
    double *coef, *meta;
    long long *serial;
    int *depth, *heap, *freel;
    int size, nfree;
    int depth_first;
    __device__ bool less(int a, int b) const {
        if (depth_first) return serial[a] > serial[b];
        double ka = meta[8 * a + 6], kb = meta[8 * b + 6];
        return ka < kb || (ka == kb && serial[a] < serial[b]);
    }
    __device__ void push(int slot) {  // lane 0 only
        int i = size++;
        heap[i] = slot;
        while (i > 0) {
            int p = (i - 1) / 2;
            if (!less(heap[i], heap[p])) break;
            int t = heap[i]; heap[i] = heap[p]; heap[p] = t;
            i = p;
        }
    }
    __device__ int pop() {  // lane 0 only
        int top = heap[0];
        heap[0] = heap[--size];
        int i = 0;
        for (;;) {
            int l = 2 * i + 1, r = l + 1, m = i;
            if (l < size && less(heap[l], heap[m])) m = l;
            if (r < size && less(heap[r], heap[m])) m = r;
            if (m == i) break;
            int t = heap[i]; heap[i] = heap[m]; heap[m] = t;
            i = m;
        }
        return top;
    }
};

template <bool DIR>
__device__ void verdict_result(svp_cell_verdict &v, int status, double margin, long long boxes, long long depth,
                               const double *w, int reason, double delta) {
    v.boxes = boxes; v.depth = depth;
    v.witness[0] = v.witness[1] = v.witness[2] = __longlong_as_double(0x7FF8000000000000LL);
    if (delta != 0.) {
        double l, h;
        if (DIR ? !dadd(margin, margin, delta, delta, l, h) : !iout(radd(margin, delta), radd(margin, delta), l, h)) {
            v.status = ST_UNCERTAIN; v.reason = R_ARITH; v.has_margin = 0; v.has_witness = 0;
            v.margin = __longlong_as_double(0x7FF8000000000000LL);
            return;
        }
    }
    v.status = status; v.reason = reason; v.margin = margin; v.has_margin = 1;
    v.has_witness = w != nullptr;
    if (w) { v.witness[0] = w[0]; v.witness[1] = w[1]; v.witness[2] = w[2]; }
}

// One warp per cell; rows[i] selects the input row (nullptr: row i).  Lanes 0..26 hold one coefficient each.
template <bool DIR>
__global__ void __launch_bounds__(128) classify_kernel(const double *__restrict__ clo, const double *__restrict__ chi,
                                                       const double *__restrict__ phi, const long long *rows,
                                                       long long n, double delta, long long max_depth,
                                                       long long max_boxes, svp_cell_verdict *out, char *scratch,
                                                       long long slots, int depth_first) {
    const int lane = threadIdx.x & 31;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const bool act = lane < 27;
    const double INF = __longlong_as_double(0x7FF0000000000000LL);
    char *base = scratch + warp_scratch_bytes(slots) * gw;
    WarpHeap H;
    H.coef = (double *)base;
    H.meta = H.coef + 54 * slots;
    H.serial = (long long *)(H.meta + 8 * slots);
    H.depth = (int *)(H.serial + slots);
    H.heap = H.depth + slots;
    H.freel = H.heap + slots;
    H.depth_first = depth_first;
    for (long long i = gw; i < n; i += nw) {
        long long row = rows ? rows[i] : i;
        double lo = act ? clo[27 * row + lane] : INF;
        double hi = act ? chi[27 * row + lane] : INF;
        double ph = act ? phi[27 * row + lane] : INF;
        double root_lower = warp_min27(lo);
        svp_cell_verdict v;
        unsigned sw = __ballot_sync(0xFFFFFFFFu, act && ph <= 0);
        if (sw) {
            int q = __ffs(sw) - 1;
            double w[3] = {(q % 3) / 2., ((q / 3) % 3) / 2., (q / 9) / 2.};
            verdict_result<DIR>(v, ST_INFEASIBLE, root_lower, 1, 0, w, R_SAMPLE_WITNESS, delta);
            if (lane == 0) out[i] = v;
            continue;
        }
        // root box in slot 0; slots 1.. free
        if (act) { H.coef[lane] = lo; H.coef[27 + lane] = hi; }
        if (lane == 0) {
            for (int k = 0; k < 3; k++) { H.meta[k] = 0.; H.meta[3 + k] = 1.; }
            H.meta[6] = root_lower;
            H.serial[0] = 0; H.depth[0] = 0;
            H.size = 0; H.nfree = 0;
            for (long long s = slots - 1; s >= 1; s--) H.freel[H.nfree++] = (int)s;
            H.push(0);
        }
        __syncwarp();
        long long serial = 0, boxes = 0, depth_used = 0;
        bool uncertain = false, done = false;
        double cert_min = INF;
        int size = 1;
        while (size > 0) {
            if (boxes >= max_boxes) {
                verdict_result<DIR>(v, ST_UNCERTAIN, root_lower, boxes, depth_used, nullptr, R_BOX_BUDGET, delta);
                done = true;
                break;
            }
            int slot = 0;
            if (lane == 0) slot = H.pop();
            slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
            __syncwarp();
            double clo_ = act ? H.coef[54 * slot + lane] : INF;
            double chi_ = act ? H.coef[54 * slot + 27 + lane] : INF;
            double low[3], high[3];
            for (int k = 0; k < 3; k++) { low[k] = H.meta[8 * slot + k]; high[k] = H.meta[8 * slot + 3 + k]; }
            int depth = H.depth[slot];
            boxes += 1;
            if (depth > depth_used) depth_used = depth;
            double minimum = warp_min27(clo_);
            __syncwarp();
            if (minimum > 0) {
                if (minimum < cert_min) cert_min = minimum;
                if (lane == 0) { H.freel[H.nfree++] = slot; size = H.size; }
                size = __shfl_sync(0xFFFFFFFFu, size, 0);
                continue;
            }
            bool corner = act && ((lane % 3) % 2 == 0) && (((lane / 3) % 3) % 2 == 0) && ((lane / 9) % 2 == 0);
            unsigned cw = __ballot_sync(0xFFFFFFFFu, corner && chi_ <= 0);
            if (cw) {
                int q = __ffs(cw) - 1;
                int bits[3] = {(q % 3) / 2, ((q / 3) % 3) / 2, (q / 9) / 2};
                double w[3];
                for (int k = 0; k < 3; k++) w[k] = bits[k] ? high[k] : low[k];
                verdict_result<DIR>(v, ST_INFEASIBLE, root_lower, boxes, depth_used, w, R_SUBDIV_WITNESS, delta);
                done = true;
                break;
            }
            if (depth >= max_depth) {
                uncertain = true;
                if (lane == 0) { H.freel[H.nfree++] = slot; size = H.size; }
                size = __shfl_sync(0xFFFFFFFFu, size, 0);
                continue;
            }
            int axis = 0;
            double best = rsub(high[0], low[0]);
            for (int k = 1; k < 3; k++) {
                double ext = rsub(high[k], low[k]);
                if (ext > best) { best = ext; axis = k; }
            }
            int stride = axis == 0 ? 1 : (axis == 1 ? 3 : 9);
            int t = act ? (lane / stride) % 3 : 0;
            int la = act ? lane - t * stride : lane;
            int lb = act ? la + stride : lane, lc = act ? la + 2 * stride : lane;
            double al = __shfl_sync(0xFFFFFFFFu, clo_, la), ah = __shfl_sync(0xFFFFFFFFu, chi_, la);
            double bl = __shfl_sync(0xFFFFFFFFu, clo_, lb), bh = __shfl_sync(0xFFFFFFFFu, chi_, lb);
            double cl = __shfl_sync(0xFFFFFFFFu, clo_, lc), ch = __shfl_sync(0xFFFFFFFFu, chi_, lc);
            double sl, sh, abl, abh, bcl, bch, ml, mh;
            bool ok = true;
            ok &= Iadd<DIR>(al, ah, bl, bh, sl, sh);
            ok &= Imul<DIR>(sl, sh, .5, .5, abl, abh);
            ok &= Iadd<DIR>(bl, bh, cl, ch, sl, sh);
            ok &= Imul<DIR>(sl, sh, .5, .5, bcl, bch);
            ok &= Iadd<DIR>(abl, abh, bcl, bch, sl, sh);
            ok &= Imul<DIR>(sl, sh, .5, .5, ml, mh);
            if (__ballot_sync(0xFFFFFFFFu, act && !ok)) {
                verdict_result<DIR>(v, ST_UNCERTAIN, root_lower, boxes, depth_used, nullptr, R_ARITH, delta);
                done = true;
                break;
            }
            double Ll = t == 0 ? al : (t == 1 ? abl : ml), Lh = t == 0 ? ah : (t == 1 ? abh : mh);
            double Rl = t == 0 ? ml : (t == 1 ? bcl : cl), Rh = t == 0 ? mh : (t == 1 ? bch : ch);
            if (!act) { Ll = INF; Rl = INF; }
            double kl = warp_min27(Ll), kr = warp_min27(Rl);
            double mid = rmul(radd(low[axis], high[axis]), .5);
            int rslot = 0;
            if (lane == 0) rslot = H.freel[--H.nfree];
            rslot = __shfl_sync(0xFFFFFFFFu, rslot, 0);
            if (act) {
                H.coef[54 * slot + lane] = Ll; H.coef[54 * slot + 27 + lane] = Lh;
                H.coef[54 * rslot + lane] = Rl; H.coef[54 * rslot + 27 + lane] = Rh;
            }
            if (lane == 0) {
                for (int k = 0; k < 3; k++) {
                    H.meta[8 * slot + k] = low[k];
                    H.meta[8 * slot + 3 + k] = k == axis ? mid : high[k];
                    H.meta[8 * rslot + k] = k == axis ? mid : low[k];
                    H.meta[8 * rslot + 3 + k] = high[k];
                }
                H.meta[8 * slot + 6] = kl; H.meta[8 * rslot + 6] = kr;
                H.depth[slot] = depth + 1; H.depth[rslot] = depth + 1;
                // the heap pushes left then right; the depth-first stack pushes right then left
                H.serial[slot] = serial + (depth_first ? 2 : 1); H.serial[rslot] = serial + (depth_first ? 1 : 2);
            }
            serial += 2;
            __syncwarp();
            if (lane == 0) { H.push(slot); H.push(rslot); size = H.size; }
            size = __shfl_sync(0xFFFFFFFFu, size, 0);
            __syncwarp();
        }
        if (!done) {
            if (uncertain)
                verdict_result<DIR>(v, ST_UNCERTAIN, root_lower, boxes, depth_used, nullptr, R_DEPTH_BUDGET, delta);
            else
                verdict_result<DIR>(v, ST_FEASIBLE, cert_min, boxes, depth_used, nullptr, R_BERNSTEIN, delta);
        }
        if (lane == 0) out[i] = v;
        __syncwarp();
    }
}

// ============================================================================================== 4. whole map
struct Accum {
    unsigned long long nonfinite, boundary, invalid;   // pre-checks (nodes)
    unsigned long long fast, prescreened, unknown, bad, boxes_extra, fallback_ok_cells;
    long long lowest_key, sampled_key, max_depth, witness_cell;
    int any_margin, arith, has_witness, pad;
    double witness[3];
};

// Sampling-domain and boundary checks per node (interpolation.py:43 check_map_domain, validation zero_boundary).
__global__ void precheck_kernel(const double *__restrict__ u, CellGrid g, double x0, double y0, double z0,
                                Accum *acc) {
    unsigned long long nf = 0, nb = 0, ni = 0;
    long long nn = g.nx * g.ny * g.nz;
    const double org[3] = {x0, y0, z0};
    const long long len[3] = {g.nx, g.ny, g.nz};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        long long x = i % g.nx, y = (i / g.nx) % g.ny, z = i / (g.nx * g.ny);
        long long idx[3] = {x, y, z};
        double q[3] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
        bool nonfin = !(finite64(q[0]) && finite64(q[1]) && finite64(q[2]));
        bool face = z == 0 || z == g.nz - 1 || y == 0 || y == g.ny - 1 || x == 0 || x == g.nx - 1;
        bool interior = !face;
        bool bad = false;
        for (int j = 0; j < 3; j++) {
            double lo = org[j], hi = radd(org[j], rmul(g.h[j], (double)(len[j] - 1)));
            double value = radd(q[j], radd(org[j], rmul(g.h[j], (double)idx[j])));
            if (!finite64(value) || value < lo || value > hi) bad = true;
            if (interior && (value <= lo || value >= hi)) bad = true;
        }
        nf += nonfin;
        nb += face && (q[0] != 0 || q[1] != 0 || q[2] != 0);
        ni += bad;
    }
    for (int o = 16; o; o >>= 1) {
        nf += __shfl_xor_sync(0xFFFFFFFFu, nf, o);
        nb += __shfl_xor_sync(0xFFFFFFFFu, nb, o);
        ni += __shfl_xor_sync(0xFFFFFFFFu, ni, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nf) atomicAdd(&acc->nonfinite, nf);
        if (nb) atomicAdd(&acc->boundary, nb);
        if (ni) atomicAdd(&acc->invalid, ni);
    }
}

__global__ void tile_flag_kernel(const uint8_t *__restrict__ flag, long long ncell, long long tile,
                                 int *__restrict__ tile_bad) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x)
        if (flag[c]) tile_bad[c / tile] = 1;
}

__device__ __forceinline__ void warp_min_key(long long &k) {
    for (int o = 16; o; o >>= 1) {
        long long y = __shfl_xor_sync(0xFFFFFFFFu, k, o);
        k = y < k ? y : k;
    }
}

// hull-proven cells: margin > 0 in an unflagged tile; sel[c] = 1 marks the rest (prescreen/fallback candidates)
__global__ void hull_stage_kernel(const double *__restrict__ margin, const int *__restrict__ tile_bad,
                                  long long ncell, long long tile, uint8_t *__restrict__ sel, Accum *acc) {
    unsigned long long nfast = 0;
    long long key = kKeyPosInf;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        bool proven = !tile_bad[c / tile] && margin[c] > 0;
        sel[c] = proven ? 0 : 1;
        if (proven) {
            nfast++;
            long long k = order_key(margin[c]);
            key = k < key ? k : key;
        }
    }
    for (int o = 16; o; o >>= 1) nfast += __shfl_xor_sync(0xFFFFFFFFu, nfast, o);
    warp_min_key(key);
    if ((threadIdx.x & 31) == 0) {
        if (nfast) {
            atomicAdd(&acc->fast, nfast);
            atomicMin(&acc->lowest_key, key);
            acc->any_margin = 1;
        }
    }
}

// prescreen decision: margin_pre = lower (delta == 0) or nextafter(lower - delta, -inf); proven iff margin_pre > 0
__global__ void prescreen_stage_kernel(const double *__restrict__ lower, long long n, double delta,
                                       uint8_t *__restrict__ sel, Accum *acc) {
    unsigned long long np = 0;
    long long key = kKeyPosInf;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double m = delta == 0. ? lower[i] : step_down(rsub(lower[i], delta));
        bool ok = m > 0;
        sel[i] = ok ? 0 : 1;
        if (ok) {
            np++;
            long long k = order_key(m);
            key = k < key ? k : key;
        }
    }
    for (int o = 16; o; o >>= 1) np += __shfl_xor_sync(0xFFFFFFFFu, np, o);
    warp_min_key(key);
    if ((threadIdx.x & 31) == 0 && np) {
        atomicAdd(&acc->prescreened, np);
        atomicMin(&acc->lowest_key, key);
        acc->any_margin = 1;
    }
}

__global__ void job_fail_kernel(const long long *__restrict__ cells, const uint8_t *__restrict__ ok, long long n,
                                long long tile, int *__restrict__ tile_fail) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (!ok[i]) tile_fail[cells[i] / tile] = 1;
}

// fallback cells in successful jobs: count, sampled min, safe cells' min coefficient; sel marks cells to classify
__global__ void fallback_stage_kernel(const long long *__restrict__ cells, const double *__restrict__ clo,
                                      const double *__restrict__ smp, long long n, long long tile,
                                      const int *__restrict__ tile_fail, uint8_t *__restrict__ sel, Accum *acc) {
    unsigned long long nok = 0, nunk = 0;
    long long key = kKeyPosInf, skey = kKeyPosInf;
    int any_safe = 0, any_fail = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        sel[i] = 0;
        if (tile_fail[cells[i] / tile]) { nunk++; any_fail = 1; continue; }
        nok++;
        double mn = clo[27 * i];
        for (int q = 1; q < 27; q++) { double x = clo[27 * i + q]; if (x < mn) mn = x; }
        for (int q = 0; q < 27; q++) { long long k = order_key(smp[27 * i + q]); skey = k < skey ? k : skey; }
        if (mn > 0) {
            any_safe = 1;
            long long k = order_key(mn);
            key = k < key ? k : key;
        } else {
            sel[i] = 1;
        }
    }
    for (int o = 16; o; o >>= 1) {
        nok += __shfl_xor_sync(0xFFFFFFFFu, nok, o);
        nunk += __shfl_xor_sync(0xFFFFFFFFu, nunk, o);
        any_safe |= __shfl_xor_sync(0xFFFFFFFFu, any_safe, o);
        any_fail |= __shfl_xor_sync(0xFFFFFFFFu, any_fail, o);
    }
    warp_min_key(key);
    warp_min_key(skey);
    if ((threadIdx.x & 31) == 0) {
        if (nok) atomicAdd(&acc->fallback_ok_cells, nok);
        if (nunk) atomicAdd(&acc->unknown, nunk);
        if (any_fail) acc->arith = 1;
        if (skey != kKeyPosInf) atomicMin(&acc->sampled_key, skey);
        if (any_safe) { atomicMin(&acc->lowest_key, key); acc->any_margin = 1; }
    }
}

__global__ void verdict_stage_kernel(const svp_cell_verdict *__restrict__ v, const long long *__restrict__ rows,
                                     const long long *__restrict__ cells, long long n, Accum *acc) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const svp_cell_verdict &r = v[i];
        if (r.has_margin) { atomicMin(&acc->lowest_key, order_key(r.margin)); acc->any_margin = 1; }
        if (r.reason == R_ARITH) acc->arith = 1;
        atomicAdd(&acc->boxes_extra, (unsigned long long)(r.boxes - 1));
        atomicMax(&acc->max_depth, r.depth);
        if (r.status == ST_UNCERTAIN) atomicAdd(&acc->unknown, 1ULL);
        if (r.status == ST_INFEASIBLE) {
            atomicAdd(&acc->bad, 1ULL);
            atomicMin(&acc->witness_cell, cells[rows[i]]);
        }
    }
}

__global__ void witness_kernel(const svp_cell_verdict *__restrict__ v, const long long *__restrict__ rows,
                               const long long *__restrict__ cells, long long n, Accum *acc) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (v[i].status == ST_INFEASIBLE && cells[rows[i]] == acc->witness_cell) {
            acc->has_witness = v[i].has_witness;
            for (int k = 0; k < 3; k++) acc->witness[k] = v[i].witness[k];
        }
    }
}

__global__ void accum_init_kernel(Accum *acc) {
    memset(acc, 0, sizeof(Accum));
    acc->lowest_key = kKeyPosInf;
    acc->sampled_key = kKeyPosInf;
    acc->max_depth = 0;
    acc->witness_cell = 0x7FFFFFFFFFFFFFFFLL;
}

// Host-side table and constants, computed with the reference's expressions (cell_q1.py:101-129,
// certificate_prescreen.py:46-55).
void closed27_table(const double h[3], double *D) {
    const double nodes[3] = {0., .5, 1.};
    for (int a = 0; a < 8; a++) {
        int vertex[3] = {a & 1, (a >> 1) & 1, (a >> 2) & 1};
        for (int p = 0; p < 27; p++) {
            double pt[3] = {nodes[p % 3], nodes[(p / 3) % 3], nodes[p / 9]};
            double f[3];
            for (int j = 0; j < 3; j++) f[j] = vertex[j] ? pt[j] : 1 - pt[j];
            for (int j = 0; j < 3; j++) {
                int o0 = j == 0 ? 1 : 0, o1 = j == 2 ? 1 : 2;
                D[(j * 27 + p) * 8 + a] = (vertex[j] ? 1. : -1.) / h[j] * f[o0] * f[o1];
            }
        }
    }
}

PrescreenConst prescreen_const(const double h[3]) {
    PrescreenConst k;
    closed27_table(h, k.D);
    const double unit = 0x1p-53;
    auto gamma = [&](double n) { return n * unit / (1 - n * unit); };
    k.g12 = gamma(12); k.g6 = gamma(6); k.g3 = gamma(3);
    k.sq27 = 5.196152422706633;
    k.eta = 1e-290;
    k.usable = 1;
    k.sparse = 1;
    for (int i = 0; i < 3 * 27 * 8; i++) {
        double x = k.D[i];
        if (!std::isfinite(x)) k.usable = 0;
        if (x != 0 && std::fabs(x) < 2.2250738585072014e-308) k.usable = 0;
        if (x != 0 && !table_nonzero(i / 216, (i / 8) % 27, i % 8)) k.sparse = 0;
    }
    return k;
}

}  // namespace

// ============================================================================================== C ABI
extern "C" int svp_edge_hull_margins(const svp_grid *g, const double *u, double delta, double *margin,
                                     uint8_t *flag, void *stream) {
    SVP_REQUIRE(grid_ok(g), "svp_edge_hull_margins: invalid grid");
    SVP_REQUIRE(u && margin && flag, "svp_edge_hull_margins: null pointer");
    CellGrid cg = cell_grid(g);
    { svp::KernelTimer _t("edge_hull_kernel", (cudaStream_t)stream); SVP_LAUNCH(edge_hull_kernel<false><<<blocks_for(cg.ncell, 256, 8), 256, 0, (cudaStream_t)stream>>>(u, cg, delta, margin, flag)); }
    SVP_LAUNCH_CHECK("edge_hull_kernel");
    return SVP_OK;
}

extern "C" int svp_edge_hull_margins_directed(const svp_grid *g, const double *u, double delta, double *margin,
                                              uint8_t *flag, void *stream) {
    SVP_REQUIRE(grid_ok(g), "svp_edge_hull_margins_directed: invalid grid");
    SVP_REQUIRE(u && margin && flag, "svp_edge_hull_margins_directed: null pointer");
    CellGrid cg = cell_grid(g);
    { svp::KernelTimer _t("edge_hull_kernel", (cudaStream_t)stream); SVP_LAUNCH(edge_hull_kernel<true><<<blocks_for(cg.ncell, 256, 8), 256, 0, (cudaStream_t)stream>>>(u, cg, delta, margin, flag)); }
    SVP_LAUNCH_CHECK("edge_hull_kernel");
    return SVP_OK;
}

extern "C" int svp_prescreen_lower_bounds(const svp_grid *g, const double *u, const int64_t *cells, int64_t n,
                                          double *out, void *stream) {
    SVP_REQUIRE(grid_ok(g), "svp_prescreen_lower_bounds: invalid grid");
    SVP_REQUIRE(n >= 0, "svp_prescreen_lower_bounds: negative count");
    if (n == 0) return SVP_OK;
    SVP_REQUIRE(u && cells && out, "svp_prescreen_lower_bounds: null pointer");
    CellGrid cg = cell_grid(g);
    PrescreenConst k = prescreen_const(cg.h);
    { svp::KernelTimer _t("prescreen_kernel", (cudaStream_t)stream); SVP_LAUNCH(launch_prescreen(u, cg, (const long long *)cells, n, k, out, (cudaStream_t)stream)); }
    SVP_LAUNCH_CHECK("prescreen_kernel");
    return SVP_OK;
}

static int fallback_arrays(const double *vertices, int64_t n, const double *spacing3, double delta, double *p_lo,
                           double *p_hi, double *c_lo, double *c_hi, double *samples, uint8_t *ok, bool directed,
                           void *stream) {
    SVP_REQUIRE(n >= 0 && spacing3, "svp_fallback_arrays: invalid arguments");
    if (n == 0) return SVP_OK;
    SVP_REQUIRE(vertices && p_lo && p_hi && c_lo && c_hi && samples && ok, "svp_fallback_arrays: null pointer");
    SVP_REQUIRE(spacing3[0] > 0 && spacing3[1] > 0 && spacing3[2] > 0, "svp_fallback_arrays: spacing must be > 0");
    const AxisDiv dv = axis_div(spacing3);
    const unsigned blocks = blocks_for(div_up(n, kFallbackWarps), 1, 16);
    if (directed)
        SVP_LAUNCH(fallback_vertices_kernel<true><<<blocks, 32 * kFallbackWarps, 0, (cudaStream_t)stream>>>(
            vertices, n, dv, delta, p_lo, p_hi, c_lo, c_hi, samples, ok));
    else
        SVP_LAUNCH(fallback_vertices_kernel<false><<<blocks, 32 * kFallbackWarps, 0, (cudaStream_t)stream>>>(
            vertices, n, dv, delta, p_lo, p_hi, c_lo, c_hi, samples, ok));
    SVP_LAUNCH_CHECK("fallback_vertices_kernel");
    return SVP_OK;
}

extern "C" int svp_fallback_arrays(const double *vertices, int64_t n, const double *spacing3, double delta,
                                   double *p_lo, double *p_hi, double *c_lo, double *c_hi, double *samples,
                                   uint8_t *ok, void *stream) {
    return fallback_arrays(vertices, n, spacing3, delta, p_lo, p_hi, c_lo, c_hi, samples, ok, false, stream);
}

extern "C" int svp_fallback_arrays_directed(const double *vertices, int64_t n, const double *spacing3, double delta,
                                            double *p_lo, double *p_hi, double *c_lo, double *c_hi, double *samples,
                                            uint8_t *ok, void *stream) {
    return fallback_arrays(vertices, n, spacing3, delta, p_lo, p_hi, c_lo, c_hi, samples, ok, true, stream);
}

static int classify_launch(const double *c_lo, const double *c_hi, const double *p_hi, const long long *rows,
                           long long n, double delta, long long max_depth, long long max_boxes,
                           svp_cell_verdict *out, char *scratch, long long warps, long long slots,
                           int depth_first, bool directed, cudaStream_t stream) {
    long long threads = 128, blocks = div_up(warps * 32, threads);
    svp::KernelTimer _t("classify_kernel", stream);
    if (directed)
        SVP_LAUNCH(classify_kernel<true><<<(unsigned)blocks, (unsigned)threads, 0, stream>>>(
            c_lo, c_hi, p_hi, rows, n, delta, max_depth, max_boxes, out, scratch, slots, depth_first));
    else
        SVP_LAUNCH(classify_kernel<false><<<(unsigned)blocks, (unsigned)threads, 0, stream>>>(
            c_lo, c_hi, p_hi, rows, n, delta, max_depth, max_boxes, out, scratch, slots, depth_first));
    SVP_LAUNCH_CHECK("classify_kernel");
    return SVP_OK;
}

static int classify_cells(const double *c_lo, const double *c_hi, const double *p_lo, const double *p_hi, int64_t n,
                          double delta, int64_t max_depth, int64_t max_boxes, int depth_first, bool directed,
                          svp_cell_verdict *out, void *stream) {
    SVP_REQUIRE(n >= 0 && max_depth >= 0 && max_boxes >= 1, "svp_classify_cells: invalid arguments");
    if (n == 0) return SVP_OK;
    SVP_REQUIRE(c_lo && c_hi && p_lo && p_hi && out, "svp_classify_cells: null pointer");
    SVP_REQUIRE(max_boxes <= (1LL << 24), "svp_classify_cells: max_boxes above 2^24");
    cudaStream_t s = (cudaStream_t)stream;
    long long slots = max_boxes + 2;
    long long warps = n < (long long)kSMs * 8 ? n : (long long)kSMs * 8;
    warps = (warps + 3) / 4 * 4;  // whole blocks of 4 warps
    char *scratch = nullptr;
    SVP_CUDA(scratch_alloc((void **)&scratch, warp_scratch_bytes(slots) * warps, s));
    int rc = classify_launch(c_lo, c_hi, p_hi, nullptr, n, delta, max_depth, max_boxes, out, scratch, warps, slots,
                             depth_first, directed, s);
    cudaError_t e = scratch_free(scratch, s);
    if (rc != SVP_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaFreeAsync");
    return SVP_OK;
}

}  // namespace svp

extern "C" int svp_classify_cells(const double *c_lo, const double *c_hi, const double *p_lo, const double *p_hi,
                                  int64_t n, double delta, int64_t max_depth, int64_t max_boxes,
                                  svp_cell_verdict *out, void *stream) {
    return svp::classify_cells(c_lo, c_hi, p_lo, p_hi, n, delta, max_depth, max_boxes, 0, false, out, stream);
}

extern "C" int svp_classify_cells_policy(const double *c_lo, const double *c_hi, const double *p_lo,
                                         const double *p_hi, int64_t n, double delta, int64_t max_depth,
                                         int64_t max_boxes, int32_t policy, svp_cell_verdict *out, void *stream) {
    SVP_REQUIRE((policy & ~(SVP_SUBDIVIDE_DEPTH_FIRST | SVP_SUBDIVIDE_DIRECTED)) == 0,
                "svp_classify_cells_policy: unknown subdivision policy");
    return svp::classify_cells(c_lo, c_hi, p_lo, p_hi, n, delta, max_depth, max_boxes,
                               (policy & SVP_SUBDIVIDE_DEPTH_FIRST) ? 1 : 0, (policy & SVP_SUBDIVIDE_DIRECTED) != 0,
                               out, stream);
}

// ---------------------------------------------------------------------------------------------- certifier handle
struct svp_certifier {
    svp_grid grid;
    svp_cert_config cfg;
    svp::CellGrid cg;
    long long ncell, ntiles;
    double *margin = nullptr, *lower = nullptr;
    uint8_t *flag = nullptr, *sel = nullptr;
    int *tile_bad = nullptr, *tile_fail = nullptr;
    long long *list1 = nullptr, *list2 = nullptr, *list3 = nullptr, *counts = nullptr;
    svp::Accum *acc = nullptr;
    long long *sel_cnt = nullptr;    // per-block flag counts of the stage-list compaction
    size_t sel_bytes = 0;
    // fallback workspace (grows on demand)
    long long fb_cap = 0;
    double *fb = nullptr;  // 5 * 27 * cap
    uint8_t *fb_ok = nullptr;
    svp_cell_verdict *verdicts = nullptr;
    char *heap = nullptr;
    long long heap_warps = 0, heap_slots = 0;
    svp::PrescreenConst pk;
};

namespace svp {
namespace {

int ensure_fallback(svp_certifier *c, long long n) {
    if (n <= c->fb_cap) return SVP_OK;
    long long cap = n < 1024 ? 1024 : n;
    if (c->fb_cap) cap = cap < 2 * c->fb_cap ? 2 * c->fb_cap : cap;
    cudaFree(c->fb); cudaFree(c->fb_ok); cudaFree(c->verdicts);
    c->fb = nullptr; c->fb_ok = nullptr; c->verdicts = nullptr; c->fb_cap = 0;
    SVP_CUDA(cudaMalloc((void **)&c->fb, sizeof(double) * 5 * 27 * cap));
    SVP_CUDA(cudaMalloc((void **)&c->fb_ok, cap));
    SVP_CUDA(cudaMalloc((void **)&c->verdicts, sizeof(svp_cell_verdict) * cap));
    c->fb_cap = cap;
    return SVP_OK;
}

// Stage lists: the flagged entries of 0..n-1 (or of a previous list) in their order, in two launches with no
// inter-block waiting.  Block b owns the contiguous chunk [b chunk, (b + 1) chunk); select_count_kernel counts its
// flags, select_scatter_kernel sums the counts of the blocks before it and writes its flagged entries in order, a
// 256-entry tile at a time (warp ballots, then the 8 warps' counts scanned in shared memory).  The last block writes
// the total.
constexpr int kSelThreads = 256;

__global__ void __launch_bounds__(kSelThreads) select_count_kernel(const uint8_t *__restrict__ flags, long long n,
                                                                 long long chunk, long long *__restrict__ cnt) {
    const long long lo = blockIdx.x * chunk, hi = lo + chunk < n ? lo + chunk : n;
    int k = 0;
    for (long long i = lo + threadIdx.x; i < hi; i += kSelThreads) k += flags[i] != 0;
    for (int o = 16; o; o >>= 1) k += __shfl_xor_sync(0xFFFFFFFFu, k, o);
    __shared__ int w[kSelThreads / 32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = k;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int j = 0; j < kSelThreads / 32; j++) t += w[j];
        cnt[blockIdx.x] = t;
    }
}

template <bool LIST>
__global__ void __launch_bounds__(kSelThreads) select_scatter_kernel(const long long *__restrict__ list,
                                                                   const uint8_t *__restrict__ flags, long long n,
                                                                   long long chunk, const long long *__restrict__ cnt,
                                                                   long long *__restrict__ out,
                                                                   long long *__restrict__ count) {
    __shared__ long long red[kSelThreads / 32];
    __shared__ int wsum[kSelThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long before = 0;
    for (long long j = threadIdx.x; j < blockIdx.x; j += kSelThreads) before += cnt[j];
    for (int o = 16; o; o >>= 1) before += __shfl_xor_sync(0xFFFFFFFFu, before, o);
    if (lane == 0) red[warp] = before;
    __syncthreads();
    long long off = 0;
    for (int j = 0; j < kSelThreads / 32; j++) off += red[j];
    const long long lo = blockIdx.x * chunk, hi = lo + chunk < n ? lo + chunk : n;
    for (long long t0 = lo; t0 < hi; t0 += kSelThreads) {
        const long long i = t0 + threadIdx.x;
        const bool on = i < hi && flags[i] != 0;
        const unsigned m = __ballot_sync(0xFFFFFFFFu, on);
        __syncthreads();     // the previous tile's reads of wsum are done
        if (lane == 0) wsum[warp] = __popc(m);
        __syncthreads();
        int wo = 0, tot = 0;
        for (int j = 0; j < kSelThreads / 32; j++) {
            wo += j < warp ? wsum[j] : 0;
            tot += wsum[j];
        }
        if (on) out[off + wo + __popc(m & ((1u << lane) - 1u))] = LIST ? list[i] : i;
        off += tot;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *count = off;
}

template <bool LIST>
int select_flagged(svp_certifier *c, const long long *list, const uint8_t *flags, long long *out, long long *count,
                   long long n, cudaStream_t s) {
    const long long blocks = n < 1 ? 1 : (long long)blocks_for(n, 8 * kSelThreads, 8);
    const long long chunk = (div_up(n < 1 ? 1 : n, blocks) + kSelThreads - 1) / kSelThreads * kSelThreads;
    const size_t need = sizeof(long long) * (size_t)blocks;
    if (need > c->sel_bytes) {
        cudaFree(c->sel_cnt);
        c->sel_cnt = nullptr;
        c->sel_bytes = 0;
        SVP_CUDA(cudaMalloc((void **)&c->sel_cnt, need));
        c->sel_bytes = need;
    }
    SVP_LAUNCH(select_count_kernel<<<(unsigned)blocks, kSelThreads, 0, s>>>(flags, n, chunk, c->sel_cnt));
    SVP_LAUNCH(select_scatter_kernel<LIST><<<(unsigned)blocks, kSelThreads, 0, s>>>(list, flags, n, chunk,
                                                                                   c->sel_cnt, out, count));
    SVP_LAUNCH_CHECK("select_flagged");
    return SVP_OK;
}

}  // namespace
}  // namespace svp

extern "C" int svp_certifier_create(const svp_grid *g, const svp_cert_config *cfg, svp_certifier **out) {
    using namespace svp;
    SVP_REQUIRE(out, "svp_certifier_create: null output");
    *out = nullptr;
    SVP_REQUIRE(grid_ok(g) && cfg, "svp_certifier_create: invalid grid/config");
    SVP_REQUIRE(cfg->delta >= 0 && cfg->delta < 1, "svp_certifier_create: require 0 <= delta < 1");
    SVP_REQUIRE(cfg->max_depth >= 0 && cfg->max_boxes >= 1 && cfg->tile_size >= 1,
                "svp_certifier_create: invalid budgets/tile size");
    SVP_REQUIRE(cfg->max_boxes <= (1LL << 24), "svp_certifier_create: max_boxes above 2^24");
    SVP_REQUIRE((cfg->execution & ~(SVP_CERT_NO_HULL | SVP_CERT_DEPTH_FIRST | SVP_CERT_DIRECTED)) == 0,
                "svp_certifier_create: unknown execution flags");
    SVP_REQUIRE(!(cfg->prescreen && (cfg->execution & SVP_CERT_NO_HULL)),
                "svp_certifier_create: the prescreen runs only after the edge-hull preproof");
    svp_certifier *c = new svp_certifier();
    c->grid = *g;
    c->cfg = *cfg;
    if (c->cfg.delta == 0) c->cfg.delta = 0.0;  // canonical +0
    c->cg = cell_grid(g);
    c->ncell = c->cg.ncell;
    c->ntiles = div_up(c->ncell, cfg->tile_size);
    c->pk = prescreen_const(c->cg.h);
    auto bail = [&](cudaError_t e, const char *what) {
        svp_certifier_destroy(c);
        return cuda_fail(e, what);
    };
    cudaError_t e;
    if ((e = cudaMalloc((void **)&c->margin, sizeof(double) * c->ncell)) != cudaSuccess) return bail(e, "margin");
    if ((e = cudaMalloc((void **)&c->lower, sizeof(double) * c->ncell)) != cudaSuccess) return bail(e, "lower");
    if ((e = cudaMalloc((void **)&c->flag, c->ncell)) != cudaSuccess) return bail(e, "flag");
    if ((e = cudaMalloc((void **)&c->sel, c->ncell)) != cudaSuccess) return bail(e, "sel");
    if ((e = cudaMalloc((void **)&c->tile_bad, sizeof(int) * c->ntiles)) != cudaSuccess) return bail(e, "tiles");
    if ((e = cudaMalloc((void **)&c->tile_fail, sizeof(int) * c->ntiles)) != cudaSuccess) return bail(e, "tiles");
    if ((e = cudaMalloc((void **)&c->list1, sizeof(long long) * c->ncell)) != cudaSuccess) return bail(e, "list1");
    if ((e = cudaMalloc((void **)&c->list2, sizeof(long long) * c->ncell)) != cudaSuccess) return bail(e, "list2");
    if ((e = cudaMalloc((void **)&c->list3, sizeof(long long) * c->ncell)) != cudaSuccess) return bail(e, "list3");
    if ((e = cudaMalloc((void **)&c->counts, sizeof(long long) * 4)) != cudaSuccess) return bail(e, "counts");
    if ((e = cudaMalloc((void **)&c->acc, sizeof(Accum))) != cudaSuccess) return bail(e, "accum");
    c->heap_slots = cfg->max_boxes + 2;
    c->heap_warps = (long long)kSMs * 8;
    if ((e = cudaMalloc((void **)&c->heap, warp_scratch_bytes(c->heap_slots) * c->heap_warps)) != cudaSuccess)
        return bail(e, "subdivision heap");
    *out = c;
    return SVP_OK;
}

extern "C" int svp_certifier_destroy(svp_certifier *c) {
    if (!c) return SVP_OK;
    cudaFree(c->margin); cudaFree(c->lower); cudaFree(c->flag); cudaFree(c->sel);
    cudaFree(c->tile_bad); cudaFree(c->tile_fail); cudaFree(c->list1); cudaFree(c->list2); cudaFree(c->list3);
    cudaFree(c->counts); cudaFree(c->acc); cudaFree(c->sel_cnt); cudaFree(c->fb); cudaFree(c->fb_ok);
    cudaFree(c->verdicts); cudaFree(c->heap);
    delete c;
    return SVP_OK;
}

extern "C" int svp_certify_map(svp_certifier *c, const double *u, svp_cert_result *out, void *stream) {
    using namespace svp;
    SVP_REQUIRE(c && u && out, "svp_certify_map: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = c->ncell, tile = c->cfg.tile_size;
    const double delta = c->cfg.delta;
    const bool hull = !(c->cfg.execution & SVP_CERT_NO_HULL);
    const int depth_first = (c->cfg.execution & SVP_CERT_DEPTH_FIRST) ? 1 : 0;
    const bool directed = (c->cfg.execution & SVP_CERT_DIRECTED) != 0;
    const double nan = std::nan("");
    memset(out, 0, sizeof *out);
    out->status = ST_UNCERTAIN;
    out->reason = 14;  // not_checked
    out->n_uncertain = n;
    out->witness_cell = -1;
    out->min_jd_lower_bound = out->min_margin_lower_bound = out->sampled_min_jd = nan;
    out->witness_point[0] = out->witness_point[1] = out->witness_point[2] = nan;

    SVP_LAUNCH(accum_init_kernel<<<1, 1, 0, s>>>(c->acc));
    { svp::KernelTimer _t("precheck_kernel", s); SVP_LAUNCH(precheck_kernel<<<blocks_for(n_nodes(&c->grid), 256, 8), 256, 0, s>>>(u, c->cg, c->grid.x0, c->grid.y0,
                                                                            c->grid.z0, c->acc)); }
    SVP_LAUNCH_CHECK("precheck_kernel");
    SVP_CUDA(cudaMemsetAsync(c->tile_fail, 0, sizeof(int) * c->ntiles, s));
    if (hull) {
        {
            svp::KernelTimer _t("edge_hull_kernel", s);
            if (directed)
                SVP_LAUNCH(edge_hull_kernel<true><<<blocks_for(n, 256, 8), 256, 0, s>>>(u, c->cg, delta, c->margin,
                                                                                      c->flag));
            else
                SVP_LAUNCH(edge_hull_kernel<false><<<blocks_for(n, 256, 8), 256, 0, s>>>(u, c->cg, delta, c->margin,
                                                                                       c->flag));
        }
        SVP_LAUNCH_CHECK("edge_hull_kernel");
        SVP_CUDA(cudaMemsetAsync(c->tile_bad, 0, sizeof(int) * c->ntiles, s));
        SVP_LAUNCH(tile_flag_kernel<<<blocks_for(n, 256, 8), 256, 0, s>>>(c->flag, n, tile, c->tile_bad));
    } else {
        // the whole-cell Bernstein execution (feasibility.py:447-491): no preproof, every cell to the fallback
        SVP_CUDA(cudaMemsetAsync(c->tile_bad, 1, sizeof(int) * c->ntiles, s));
    }
    SVP_LAUNCH(hull_stage_kernel<<<blocks_for(n, 256, 8), 256, 0, s>>>(c->margin, c->tile_bad, n, tile, c->sel, c->acc));
    SVP_LAUNCH_CHECK("hull stage");
    int rc = select_flagged<false>(c, nullptr, c->sel, c->list1, c->counts, n, s);
    if (rc) return rc;
    Accum acc;
    long long counts[4];
    SVP_CUDA(cudaMemcpyAsync(&acc, c->acc, sizeof acc, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaMemcpyAsync(counts, c->counts, sizeof(long long), cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    // early returns, in certify_map's order (feasibility.py:412-428)
    if (acc.nonfinite) { out->reason = R_NONFINITE; return SVP_OK; }
    if (acc.boundary) { out->status = ST_INFEASIBLE; out->reason = R_BOUNDARY; return SVP_OK; }
    if (acc.invalid) { out->status = ST_INFEASIBLE; out->reason = R_DOMAIN; return SVP_OK; }
    long long n1 = counts[0], n2 = n1;
    const long long *list2 = c->list1;
    const bool staged = n1 != 0;   // a later stage updates acc; with no flagged cell the copy above is final
    if (c->cfg.prescreen && n1) {
        { svp::KernelTimer _t("prescreen_kernel", s); SVP_LAUNCH(launch_prescreen(u, c->cg, c->list1, n1, c->pk, c->lower, s)); }
        SVP_LAUNCH_CHECK("prescreen_kernel");
        SVP_LAUNCH(prescreen_stage_kernel<<<blocks_for(n1, 256, 8), 256, 0, s>>>(c->lower, n1, delta, c->sel, c->acc));
        SVP_LAUNCH_CHECK("prescreen stage");
        rc = select_flagged<true>(c, c->list1, c->sel, c->list2, c->counts + 1, n1, s);
        if (rc) return rc;
        SVP_CUDA(cudaMemcpyAsync(&n2, c->counts + 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
        SVP_CUDA(cudaStreamSynchronize(s));
        list2 = c->list2;
    }
    long long n3 = 0;
    if (n2) {
        rc = ensure_fallback(c, n2);
        if (rc) return rc;
        double *fb = c->fb, *plo = fb, *phi = fb + 27 * n2, *clo = fb + 2 * 27 * n2, *chi = fb + 3 * 27 * n2,
               *smp = fb + 4 * 27 * n2;
        {
            svp::KernelTimer _t("fallback_grid_kernel", s);
            const unsigned fb_blocks = blocks_for(div_up(n2, kFallbackWarps), 1, 16);
            if (directed)
                SVP_LAUNCH(fallback_grid_kernel<true><<<fb_blocks, 32 * kFallbackWarps, 0, s>>>(
                    u, c->cg, list2, n2, delta, plo, phi, clo, chi, smp, c->fb_ok));
            else
                SVP_LAUNCH(fallback_grid_kernel<false><<<fb_blocks, 32 * kFallbackWarps, 0, s>>>(
                    u, c->cg, list2, n2, delta, plo, phi, clo, chi, smp, c->fb_ok));
        }
        SVP_LAUNCH_CHECK("fallback_grid_kernel");
        SVP_LAUNCH(job_fail_kernel<<<blocks_for(n2, 256, 8), 256, 0, s>>>(list2, c->fb_ok, n2, tile, c->tile_fail));
        SVP_LAUNCH(fallback_stage_kernel<<<blocks_for(n2, 256, 8), 256, 0, s>>>(list2, clo, smp, n2, tile, c->tile_fail,
                                                                      c->sel, c->acc));
        SVP_LAUNCH_CHECK("fallback stage");
        rc = select_flagged<false>(c, nullptr, c->sel, c->list3, c->counts + 2, n2, s);
        if (rc) return rc;
        SVP_CUDA(cudaMemcpyAsync(&n3, c->counts + 2, sizeof(long long), cudaMemcpyDeviceToHost, s));
        SVP_CUDA(cudaStreamSynchronize(s));
        if (n3) {
            long long warps = n3 < c->heap_warps ? n3 : c->heap_warps;
            warps = (warps + 3) / 4 * 4;
            if (warps > c->heap_warps) warps = c->heap_warps;
            rc = classify_launch(clo, chi, phi, c->list3, n3, delta, c->cfg.max_depth, c->cfg.max_boxes,
                                 c->verdicts, c->heap, warps, c->heap_slots, depth_first, directed, s);
            if (rc) return rc;
            SVP_LAUNCH(verdict_stage_kernel<<<blocks_for(n3, 256, 8), 256, 0, s>>>(c->verdicts, c->list3, list2, n3, c->acc));
            SVP_LAUNCH(witness_kernel<<<blocks_for(n3, 256, 8), 256, 0, s>>>(c->verdicts, c->list3, list2, n3, c->acc));
            SVP_LAUNCH_CHECK("verdict stage");
        }
    }
    if (staged) {
        SVP_CUDA(cudaMemcpyAsync(&acc, c->acc, sizeof acc, cudaMemcpyDeviceToHost, s));
        SVP_CUDA(cudaStreamSynchronize(s));
    }
    // the record (feasibility.py:755-771)
    long long fallback = n2;
    long long unknown = (long long)acc.unknown, bad = (long long)acc.bad;
    int status = bad ? ST_INFEASIBLE : (unknown ? ST_UNCERTAIN : ST_FEASIBLE);
    int reason = bad ? R_VIOLATION : (acc.arith ? R_ARITH : (unknown ? R_SUBDIV_BUDGET : R_BERNSTEIN));
    long long fast = (long long)acc.fast, pre = (long long)acc.prescreened;
    if ((fast || pre) && status == ST_FEASIBLE) reason = R_ENCLOSURE;
    out->status = status;
    out->reason = reason;
    out->n_cells_checked = n;
    out->n_uncertain = unknown;
    out->n_infeasible = bad;
    out->n_boxes = fast + pre + (long long)acc.fallback_ok_cells + (long long)acc.boxes_extra;
    out->max_depth = acc.max_depth;
    out->witness_cell = bad ? acc.witness_cell : -1;
    out->n_fast_cells = fast;
    out->n_fallback_cells = hull ? fallback : 0;   // the plain FeasibilityResult has no stage counts
    out->n_prescreen_cells = pre;
    if (acc.any_margin && !acc.arith) {
        double lowest = key_value(acc.lowest_key);
        out->min_margin_lower_bound = lowest;
        out->min_jd_lower_bound = delta == 0. ? lowest : std::nextafter(lowest + delta, -INFINITY);
        out->has_min_jd = 1;
    }
    if (!(fast || pre) && acc.sampled_key != kKeyPosInf) {
        double sm = key_value(acc.sampled_key);
        if (std::isfinite(sm)) { out->sampled_min_jd = sm; out->has_sampled_min = 1; }
    }
    if (bad && acc.has_witness)
        for (int k = 0; k < 3; k++) out->witness_point[k] = acc.witness[k];
    return SVP_OK;
}

// ---------------------------------------------------------------------------------------------- allocation-free
// svp_classify_cells_noalloc: the subdivision of svp_classify_cells with its box heaps in a fixed, file-scope device
// array instead of a stream-ordered allocation, for callers that may not allocate device memory after start-up.
// Capacity: 32 warps (cells in flight) with max_boxes <= 255; each warp's region is rewritten from scratch for every
// cell it takes, so nothing carries over between calls.  Every loaded device holds the array until process exit.
namespace svp {
namespace {
constexpr long long kNoAllocWarps = 32;
constexpr long long kNoAllocMaxBoxes = 255;
constexpr size_t kNoAllocWarpBytes = ((size_t)(kNoAllocMaxBoxes + 2) * (54 * 8 + 8 * 8 + 8 + 4 + 4 + 4) + 255) / 256 * 256;
constexpr size_t kNoAllocBytes = (size_t)kNoAllocWarps * kNoAllocWarpBytes;  // 4,317,184 bytes

static __device__ __align__(256) char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[256] = {};
unsigned long long g_noalloc_ctx[256] = {};   // unique id of the context the cached address belongs to

// Unique id of the calling thread's current context (0 when there is none yet), through the driver entry points so
// that the library keeps linking against the runtime alone.  A context created after a cudaDeviceReset gets a new
// id, so an address cached for the old context is never reused.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
int current_context_id(unsigned long long *id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        cudaDriverEntryPointQueryResult q1, q2;
        SVP_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void **)&get_current, 12000, cudaEnableDefault,
                                                  &q1));
        SVP_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetId", (void **)&get_id, 12000, cudaEnableDefault, &q2));
        SVP_REQUIRE(q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess && get_current && get_id,
                    "svp_classify_cells_noalloc: driver context queries unavailable");
    }
    CUcontext ctx = nullptr;
    *id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS) return cuda_fail(cudaErrorUnknown, "cuCtxGetCurrent");
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return cuda_fail(cudaErrorUnknown, "cuCtxGetId");
    return SVP_OK;
}

// Device address of the scratch array in the current device's context.  The first call on a device (and the first
// call after that device's context was replaced) looks it up with cudaGetSymbolAddress; later calls reuse it.
int noalloc_scratch(char **out) {
    int dev = -1;
    SVP_CUDA(cudaGetDevice(&dev));
    SVP_REQUIRE(dev >= 0 && dev < 256, "svp_classify_cells_noalloc: device ordinal out of range");
    unsigned long long ctx = 0;
    int rc = current_context_id(&ctx);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev] || ctx == 0 || g_noalloc_ctx[dev] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // creates the primary context if needed
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(svp classify scratch)");
        rc = current_context_id(&ctx);
        if (rc) return rc;
        g_noalloc_ptr[dev] = p;
        g_noalloc_ctx[dev] = ctx;
    }
    *out = (char *)g_noalloc_ptr[dev];
    return SVP_OK;
}
}  // namespace
}  // namespace svp

extern "C" int svp_classify_cells_noalloc(const double *c_lo, const double *c_hi, const double *p_lo,
                                          const double *p_hi, int64_t n, double delta, int64_t max_depth,
                                          int64_t max_boxes, svp_cell_verdict *out, void *stream) {
    using namespace svp;
    SVP_REQUIRE(n >= 0 && max_depth >= 0 && max_boxes >= 1, "svp_classify_cells_noalloc: invalid arguments");
    SVP_REQUIRE(max_boxes <= kNoAllocMaxBoxes,
                "svp_classify_cells_noalloc: max_boxes above the static scratch limit of 255 boxes per cell");
    if (n == 0) return SVP_OK;
    SVP_REQUIRE(c_lo && c_hi && p_lo && p_hi && out, "svp_classify_cells_noalloc: null pointer");
    char *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    const long long slots = max_boxes + 2;
    long long warps = n < kNoAllocWarps ? n : kNoAllocWarps;
    warps = (warps + 3) / 4 * 4;
    SVP_REQUIRE(warp_scratch_bytes(slots) * (size_t)warps <= kNoAllocBytes,
                "svp_classify_cells_noalloc: scratch capacity exceeded");
    SVP_LAUNCH(classify_kernel<false><<<(unsigned)(warps * 32 / 128), 128, 0, (cudaStream_t)stream>>>(
        c_lo, c_hi, p_hi, nullptr, n, delta, max_depth, max_boxes, out, scratch, slots, 0));
    return SVP_OK;
}
