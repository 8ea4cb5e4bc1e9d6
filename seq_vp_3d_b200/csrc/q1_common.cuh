// Q1 cell geometry on the B200: separable evaluation of grad u at the Gauss27 / closed27 points, its adjoint,
// the localized C2 barrier, and deterministic double-double block reductions.
#pragma once
#include "svp_common.cuh"

namespace svp {

// Constants of one registration pair (passed by value: constant bank, race-free across concurrent pairs).
struct Q1Const {
    long long nx, ny, nz, cx, cy, cz, ncell, nnode;
    long long fx, fy, fz, nfree;   // free (interior) node counts per axis and in total
    double h[3], ih[3];            // spacing and fl(1/h) (cell_q1.py:126 divides +-1 by h)
    double gn[3], gm[3];           // Gauss nodes xi and 1 - xi (cell_q1.py:106)
    double gw[27];                 // Gauss27 weights omega*wx*wy*wz, p = 9 iz + 3 iy + ix (cell_q1.py:115)
    double sqmu[27], sqnu[27];     // sqrt(mu gw[p]), sqrt(nu gw[p]) (stable differences of the Gauss terms)
    double omega;
    double lam, mu, nu, bw;        // weights; bw = kappa omega / 27 (problem.py:310)
    double act, delta;             // localized barrier activation a and delta
    double x0[3];                  // node axis origins (x, y, z)
    float gnf[3], gmf[3], gwf[27], ihf[3];   // the same rule constants rounded to float (the mixed form's kernels)
    // the curl term of the GGN diagonal does not depend on the state: per vertex a and component r,
    // nu sum_p gw[p] sum_(j != r) D_j(p, a)^2 over the Gauss points (index 3 a + r), float copy for the mixed form
    double ggn_curl[24];
    float ggn_curlf[24];
};

// ------------------------------------------------------------------------------------------- double-double
struct dd {
    double hi, lo;
};
__device__ __forceinline__ dd two_sum(double a, double b) {
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd dd_add_d(dd a, double b) {
    dd s = two_sum(a.hi, b);
    s.lo += a.lo;
    return two_sum(s.hi, s.lo);
}
// exact product as an unevaluated pair (FMA)
__device__ __forceinline__ dd two_prod(double a, double b) {
    double p = a * b;
    return {p, fma(a, b, -p)};
}
__device__ __forceinline__ dd dd_shfl_xor(dd a, int o) {
    return {__shfl_xor_sync(0xFFFFFFFFu, a.hi, o), __shfl_xor_sync(0xFFFFFFFFu, a.lo, o)};
}

// Block reduction of K double-double accumulators, fixed tree order; thread 0 writes partial[blockIdx][k].
template <int K>
__device__ void block_reduce_dd(dd (&acc)[K], dd *partial) {
    __shared__ dd sh[32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
        for (int o = 16; o; o >>= 1) acc[k] = dd_add(acc[k], dd_shfl_xor(acc[k], o));
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) sh[warp][k] = acc[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < K; k++) {
            dd v = lane < nw ? sh[lane][k] : dd{0., 0.};
#pragma unroll
            for (int o = 16; o; o >>= 1) v = dd_add(v, dd_shfl_xor(v, o));
            if (lane == 0) partial[(size_t)blockIdx.x * K + k] = v;
        }
    }
}

// ------------------------------------------------------------------------------------------- cell geometry
__device__ __forceinline__ long long cell_node0(long long c, const Q1Const &q) {
    long long x0, y0, z0;
    unflatten3(c, q.cx, q.cy, x0, y0, z0);
    return (z0 * q.ny + y0) * q.nx + x0;
}
__device__ __forceinline__ long long vertex_node(long long n0, int a, const Q1Const &q) {
    return n0 + (long long)(a >> 2) * q.ny * q.nx + (long long)((a >> 1) & 1) * q.nx + (a & 1);
}

template <class T>
__device__ __forceinline__ void load_cell(const T *__restrict__ u, long long n0, const Q1Const &q, T v[8][3]) {
#pragma unroll
    for (int a = 0; a < 8; a++) {
        const T *p = u + 3 * vertex_node(n0, a, q);
        v[a][0] = __ldg(p);
        v[a][1] = __ldg(p + 1);
        v[a][2] = __ldg(p + 2);
    }
}

// Edge differences E[j][e][r]: axis j, edge e over the two other vertex bits in increasing order
// (j = 0: e = y + 2z; j = 1: e = x + 2z; j = 2: e = x + 2y).
template <class T>
__device__ __forceinline__ void cell_edges(const T v[8][3], T E[3][4][3]) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
        int lo = e & 1, hi = e >> 1;
        int ax = 2 * lo + 4 * hi, ay = lo + 4 * hi, az = lo + 2 * hi;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            E[0][e][r] = v[ax | 1][r] - v[ax][r];
            E[1][e][r] = v[ay | 2][r] - v[ay][r];
            E[2][e][r] = v[az | 4][r] - v[az][r];
        }
    }
}

// Derivative tables at a 3-point rule per axis: G[j][s][t][r] = d u_r / d x_j at the point whose two other
// coordinates take nodes s (the lower-numbered other axis) and t (the higher); n[] nodes, m[] = 1 - nodes.
template <class T>
__device__ __forceinline__ void point_derivatives(const T E[3][4][3], const T n[3], const T m[3], const T ih[3],
                                                  T G[3][3][3][3]) {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int s = 0; s < 3; s++)
#pragma unroll
            for (int r = 0; r < 3; r++) {
                // interpolate along the lower other axis first (edges e = b0 + 2 b1)
                T l0 = m[s] * E[j][0][r] + n[s] * E[j][1][r];
                T l1 = m[s] * E[j][2][r] + n[s] * E[j][3][r];
#pragma unroll
                for (int t = 0; t < 3; t++) G[j][s][t][r] = (m[t] * l0 + n[t] * l1) * ih[j];
            }
}

// Column j of grad u at one point, straight from the edges (the same operation sequence as point_derivatives, so
// the values are bitwise those of the tables): s indexes the lower-numbered other axis, t the higher.
template <int J, class T>
__device__ __forceinline__ void column(const T E[3][4][3], T ms, T ns, T mt, T nt, T ih, T out[3]) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
        T l0 = ms * E[J][0][r] + ns * E[J][1][r];
        T l1 = ms * E[J][2][r] + ns * E[J][3][r];
        out[r] = (mt * l0 + nt * l1) * ih;
    }
}

// Point coordinates of the two 3-point rules: Gauss (nodes q.gn, 1 - nodes q.gm) or closed (0, 1/2, 1).
template <bool CLOSED>
__device__ __forceinline__ double rule_n(const Q1Const &q, int i) { return CLOSED ? .5 * i : q.gn[i]; }
template <bool CLOSED>
__device__ __forceinline__ double rule_m(const Q1Const &q, int i) { return CLOSED ? 1. - .5 * i : q.gm[i]; }
// the rule's nodes and 1/h in the arithmetic type R (float: the rounded constants, no conversion in the sweeps)
template <bool CLOSED, class R>
__device__ __forceinline__ R node_n(const Q1Const &q, int i) {
    if constexpr (sizeof(R) == 4) return CLOSED ? .5f * (float)i : q.gnf[i];
    else return rule_n<CLOSED>(q, i);
}
template <bool CLOSED, class R>
__device__ __forceinline__ R node_m(const Q1Const &q, int i) {
    if constexpr (sizeof(R) == 4) return CLOSED ? 1.f - .5f * (float)i : q.gmf[i];
    else return rule_m<CLOSED>(q, i);
}
template <class R>
__device__ __forceinline__ R inv_h(const Q1Const &q, int k) {
    if constexpr (sizeof(R) == 4) return q.ihf[k];
    else return q.ih[k];
}

// Visit the 27 points p = 9 iz + 3 iy + ix of a rule with grad u at each, V[r][j].  Column x depends only on
// (iy, iz) and column y only on (ix, iz), so x is evaluated once per (iy, iz) and y once per (ix, iz): 45 column
// evaluations instead of 81, each bitwise the one of column<J> at that point.  Fields: one (sweep) or two
// (sweep2, same points); body(p, ix, iy, iz, V[, V2]).
template <bool CLOSED, class R = double, class Body>
__device__ __forceinline__ void sweep(const R E[3][4][3], const Q1Const &q, Body &&body) {
    const R ih0 = inv_h<R>(q, 0), ih1 = inv_h<R>(q, 1), ih2 = inv_h<R>(q, 2);
#pragma unroll 1
    for (int iz = 0; iz < 3; iz++) {
        const R nz = node_n<CLOSED, R>(q, iz), mz = node_m<CLOSED, R>(q, iz);
        R Y[3][3];
#pragma unroll
        for (int ix = 0; ix < 3; ix++)
            column<1>(E, node_m<CLOSED, R>(q, ix), node_n<CLOSED, R>(q, ix), mz, nz, ih1, Y[ix]);
#pragma unroll 1
        for (int iy = 0; iy < 3; iy++) {
            const R ny = node_n<CLOSED, R>(q, iy), my = node_m<CLOSED, R>(q, iy);
            R X[3];
            column<0>(E, my, ny, mz, nz, ih0, X);
#pragma unroll
            for (int ix = 0; ix < 3; ix++) {
                R Z[3];
                column<2>(E, node_m<CLOSED, R>(q, ix), node_n<CLOSED, R>(q, ix), my, ny, ih2, Z);
                R V[3][3] = {{X[0], Y[ix][0], Z[0]}, {X[1], Y[ix][1], Z[1]}, {X[2], Y[ix][2], Z[2]}};
                body(9 * iz + 3 * iy + ix, ix, iy, iz, V);
            }
        }
    }
}
template <bool CLOSED, class R = double, class Body>
__device__ __forceinline__ void sweep2(const R E[3][4][3], const R E2[3][4][3], const Q1Const &q, Body &&body) {
    const R ih0 = inv_h<R>(q, 0), ih1 = inv_h<R>(q, 1), ih2 = inv_h<R>(q, 2);
#pragma unroll 1
    for (int iz = 0; iz < 3; iz++) {
        const R nz = node_n<CLOSED, R>(q, iz), mz = node_m<CLOSED, R>(q, iz);
#pragma unroll 1
        for (int iy = 0; iy < 3; iy++) {
            const R ny = node_n<CLOSED, R>(q, iy), my = node_m<CLOSED, R>(q, iy);
            R X[3], X2[3];
            column<0>(E, my, ny, mz, nz, ih0, X);
            column<0>(E2, my, ny, mz, nz, ih0, X2);
#pragma unroll 1
            for (int ix = 0; ix < 3; ix++) {
                const R nx = node_n<CLOSED, R>(q, ix), mx = node_m<CLOSED, R>(q, ix);
                R Y[3], Z[3], Y2[3], Z2[3];
                column<1>(E, mx, nx, mz, nz, ih1, Y);
                column<2>(E, mx, nx, my, ny, ih2, Z);
                column<1>(E2, mx, nx, mz, nz, ih1, Y2);
                column<2>(E2, mx, nx, my, ny, ih2, Z2);
                R V[3][3] = {{X[0], Y[0], Z[0]}, {X[1], Y[1], Z[1]}, {X[2], Y[2], Z[2]}};
                R V2[3][3] = {{X2[0], Y2[0], Z2[0]}, {X2[1], Y2[1], Z2[1]}, {X2[2], Y2[2], Z2[2]}};
                body(9 * iz + 3 * iy + ix, ix, iy, iz, V, V2);
            }
        }
    }
}

// V[r][j] at point (ix, iy, iz) from the tables
template <class T>
__device__ __forceinline__ void grad_at(const T G[3][3][3][3], int ix, int iy, int iz, T V[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
        V[r][0] = G[0][iy][iz][r];
        V[r][1] = G[1][ix][iz][r];
        V[r][2] = G[2][ix][iy][r];
    }
}

// Cofactor rows (cross products of cyclic rows of F = I + V) and J = F0 . A0 (geometry.py:11 cofactor, :26 determinant).
template <class T>
__device__ __forceinline__ void cofactor_det(const T V[3][3], T A[3][3], T &J) {
    T F[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) F[r][c] = V[r][c] + (r == c ? T(1) : T(0));
#pragma unroll
    for (int r = 0; r < 3; r++) {
        int j = (r + 1) % 3, k = (r + 2) % 3;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            int l = (c + 1) % 3, mm = (c + 2) % 3;
            A[r][c] = F[j][l] * F[k][mm] - F[j][mm] * F[k][l];
        }
    }
    J = (F[0][0] * A[0][0] + F[0][1] * A[0][1]) + F[0][2] * A[0][2];
}
template <class T>
__device__ __forceinline__ T det_only(const T V[3][3]) {
    T F[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) F[r][c] = V[r][c] + (r == c ? T(1) : T(0));
    T a0 = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    T a1 = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    T a2 = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    return (F[0][0] * a0 + F[0][1] * a1) + F[0][2] * a2;
}
template <class T>
__device__ __forceinline__ void curl_of(const T V[3][3], T C[3]) {
    C[0] = V[2][1] - V[1][2];
    C[1] = V[0][2] - V[2][0];
    C[2] = V[1][0] - V[0][1];
}

// Adjoint of point_derivatives: accumulate vertex values L[a][r] from per-point fluxes summed over the free axis,
// S[j][s][t][r] (same indexing as G).
template <class T>
__device__ __forceinline__ void scatter_edges(const T S[3][3][3][3], const T n[3], const T m[3], const T ih[3],
                                              T L[8][3]) {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            T e[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
            for (int s = 0; s < 3; s++) {
                T t0 = T(0), t1 = T(0);
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    T v = S[j][s][t][r] * ih[j];
                    t0 += m[t] * v;
                    t1 += n[t] * v;
                }
                e[0] += m[s] * t0;
                e[1] += n[s] * t0;
                e[2] += m[s] * t1;
                e[3] += n[s] * t1;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                int lo = k & 1, hi = k >> 1;
                int a = j == 0 ? 2 * lo + 4 * hi : (j == 1 ? lo + 4 * hi : lo + 2 * hi);
                L[a | (1 << j)][r] += e[k];
                L[a][r] -= e[k];
            }
        }
}

// ------------------------------------------------------------------------------------------- localized barrier
// barrier.py:18-36: b = -w r^2 log t, b' and b'' for J < a (zero above); log t via log1p(-r) when r < 1/2.
__device__ __forceinline__ void barrier_eval(double J, double a, double delta, double w, double &b, double &b1,
                                             double &b2) {
    b = b1 = b2 = 0.;
    if (!(J < a)) return;
    double scale = a - delta;
    double t = (J - delta) / scale;
    double r = (a - J) / scale;
    double logt = r < .5 ? log1p(-r) : log(t);
    b = -w * r * r * logt;
    b1 = w * (2 * r * logt - r * r / t) / scale;
    double rt = r / t;
    b2 = w * (-2 * logt + 4 * r / t + rt * rt) / (scale * scale);
}

}  // namespace svp
