// Fused per-cell Q1 kernels of the certified-registration energy (FP64 plain form):
//   warp_kernel        cubic B-spline value (+ gradient) at X + u, image and proximity energy sums
//   cell_energy_kernel Gauss27 JD/curl penalties against u_ref, closed27 localized barrier
//   cell_grad_kernel   per-cell vertex gradients (soft penalties, barrier) -> SoA locals
//   gather_kernel      atomic-free node gather in fixed vertex order, plus the node terms
//   ggn kernels, stable-difference kernels, node JD measure, global closed27 cubic root
// Reference: jd_curl/three_d/{residuals.py, linearization.py, energy_comparison.py, interpolation.py,
// solvers/jd_affine.py, solvers/global_jd_step.py}.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "pair.cuh"

namespace svp {
namespace {

constexpr int CT = 128;      // threads per block of the cell kernels
constexpr int CELL_PER_SM = 8;

// ============================================================================================== spline sampler
struct SplineRef {
    const double *c;
    const double *t[3];    // x, y, z knots
    const double *rcp[3];  // per span, the reciprocals of the knot differences cubic_basis divides by (14 per span)
    long long n[3];        // nx, ny, nz coefficients per axis
    double x0[3], ih[3];
};

// The span s with t[s] <= x < t[s+1] (clamped to [3, n-1]): a first guess from the uniform node spacing, then the
// knot comparisons decide (so the guess's rounding never matters).
__device__ __forceinline__ int find_span(const double *__restrict__ t, long long n, double x, double x0, double ih) {
    long long i = (long long)floor((x - x0) * ih);
    long long s = i + 2;
    s = s < 3 ? 3 : (s > n - 1 ? n - 1 : s);
    while (s < n - 1 && __ldg(t + s + 1) <= x) s++;
    while (s > 3 && __ldg(t + s) > x) s--;
    return (int)s;
}

// backends/spline.py:12 cubic_basis: Cox-de Boor values and derivatives of the 4 B-splines on the span.  The
// denominators are knot differences (right + left = t[s+r+1] - t[s+1-d+r] up to rounding), so their reciprocals are
// tabled per span and the 14 divisions per axis become multiplies (a relative change of one rounding, inside the
// float64 contract's 1e-12).
__device__ __forceinline__ void cubic_basis(const double *__restrict__ t, const double *__restrict__ rcp, int s,
                                            double x, double B[4], double dB[4]) {
    const double *R = rcp + 14 * (long long)s;
    double b[4] = {1., 0., 0., 0.}, q[3];
#pragma unroll
    for (int degree = 1; degree <= 3; degree++) {
        double nb[4];
        double saved = 0.;
#pragma unroll
        for (int r = 0; r < degree; r++) {
            double right = __ldg(t + s + r + 1) - x;
            double left = x - __ldg(t + s + 1 - degree + r);
            double temp = b[r] * __ldg(R + (degree - 1) * degree / 2 + r);
            nb[r] = saved + right * temp;
            saved = left * temp;
        }
        nb[degree] = saved;
#pragma unroll
        for (int r = 0; r <= degree; r++) b[r] = nb[r];
        if (degree == 2) { q[0] = b[0]; q[1] = b[1]; q[2] = b[2]; }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double left = k == 0 ? 0. : q[k - 1], right = k == 3 ? 0. : q[k];
        dB[k] = 3. * left * __ldg(R + 6 + 2 * k) - 3. * right * __ldg(R + 7 + 2 * k);
        B[k] = b[k];
    }
}

// value and (optionally) xyz gradient at physical point (x, y, z)
template <bool GRAD>
__device__ __forceinline__ double spline_eval(const SplineRef &S, double px, double py, double pz, double g[3]) {
    int sx = find_span(S.t[0], S.n[0], px, S.x0[0], S.ih[0]);
    int sy = find_span(S.t[1], S.n[1], py, S.x0[1], S.ih[1]);
    int sz = find_span(S.t[2], S.n[2], pz, S.x0[2], S.ih[2]);
    double bx[4], dx[4], by[4], dy[4], bz[4], dz[4];
    cubic_basis(S.t[0], S.rcp[0], sx, px, bx, dx);
    cubic_basis(S.t[1], S.rcp[1], sy, py, by, dy);
    cubic_basis(S.t[2], S.rcp[2], sz, pz, bz, dz);
    const long long nx = S.n[0], ny = S.n[1];
    const double *c = S.c + ((long long)(sz - 3) * ny + (sy - 3)) * nx + (sx - 3);
    double val = 0., gx = 0., gy = 0., gz = 0.;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double pv = 0., px_ = 0., py_ = 0.;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const double *row = c + ((long long)i * ny + j) * nx;
            double c0 = __ldg(row), c1 = __ldg(row + 1), c2 = __ldg(row + 2), c3 = __ldg(row + 3);
            double rv = c0 * bx[0] + c1 * bx[1] + c2 * bx[2] + c3 * bx[3];
            pv += by[j] * rv;
            if (GRAD) {
                double rd = c0 * dx[0] + c1 * dx[1] + c2 * dx[2] + c3 * dx[3];
                px_ += by[j] * rd;
                py_ += dy[j] * rv;
            }
        }
        val += bz[i] * pv;
        if (GRAD) {
            gx += bz[i] * px_;
            gy += bz[i] * py_;
            gz += dz[i] * pv;
        }
    }
    if (GRAD) { g[0] = gx; g[1] = gy; g[2] = gz; }
    return val;
}

__device__ __forceinline__ double node_weight(long long x, long long y, long long z, const Q1Const &q) {
    double tx = (x == 0 || x == q.nx - 1) ? .5 : 1.;
    double ty = (y == 0 || y == q.ny - 1) ? .5 : 1.;
    double tz = (z == 0 || z == q.nz - 1) ? .5 : 1.;
    return ((q.omega * tz) * ty) * tx;
}

// warped image at X + u (+ gradient), and the image / proximity energy sums (before the 1/2, lambda/2 factors)
template <bool GRAD>
__global__ void __launch_bounds__(256) warp_kernel(Q1Const q, SplineRef S, const double *__restrict__ u,
                                                   const double *__restrict__ fixed, const double *__restrict__ uref,
                                                   double *__restrict__ warped, double *__restrict__ image_grad,
                                                   dd *partial) {
    dd acc[2] = {{0., 0.}, {0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nnode;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.nx, q.ny, x, y, z);
        double ux = u[3 * i], uy = u[3 * i + 1], uz = u[3 * i + 2];
        double px = (q.x0[0] + q.h[0] * (double)x) + ux;
        double py = (q.x0[1] + q.h[1] * (double)y) + uy;
        double pz = (q.x0[2] + q.h[2] * (double)z) + uz;
        double g[3];
        double w = spline_eval<GRAD>(S, px, py, pz, g);
        warped[i] = w;
        if (GRAD) {
            image_grad[3 * i] = g[0];
            image_grad[3 * i + 1] = g[1];
            image_grad[3 * i + 2] = g[2];
        }
        if (partial) {
            double qw = node_weight(x, y, z, q);
            double d = w - fixed[i];
            double e0 = ux - uref[3 * i], e1 = uy - uref[3 * i + 1], e2 = uz - uref[3 * i + 2];
            acc[0] = dd_add_d(acc[0], qw * d * d);
            acc[1] = dd_add_d(acc[1], qw * (e0 * e0 + e1 * e1 + e2 * e2));
        }
    }
    if (partial) block_reduce_dd<2>(acc, partial);
}

__global__ void __launch_bounds__(256) node_energy_kernel(Q1Const q, const double *__restrict__ u,
                                                          const double *__restrict__ warped,
                                                          const double *__restrict__ fixed,
                                                          const double *__restrict__ uref, dd *partial) {
    dd acc[2] = {{0., 0.}, {0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nnode;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.nx, q.ny, x, y, z);
        double qw = node_weight(x, y, z, q);
        double d = warped[i] - fixed[i];
        double e0 = u[3 * i] - uref[3 * i], e1 = u[3 * i + 1] - uref[3 * i + 1], e2 = u[3 * i + 2] - uref[3 * i + 2];
        acc[0] = dd_add_d(acc[0], qw * d * d);
        acc[1] = dd_add_d(acc[1], qw * (e0 * e0 + e1 * e1 + e2 * e2));
    }
    block_reduce_dd<2>(acc, partial);
}

__global__ void __launch_bounds__(256) sample_points_kernel(SplineRef S, const double *__restrict__ pts, long long n,
                                                            double *__restrict__ value, double *__restrict__ grad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double g[3];
        if (grad) {
            value[i] = spline_eval<true>(S, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], g);
            grad[3 * i] = g[0]; grad[3 * i + 1] = g[1]; grad[3 * i + 2] = g[2];
        } else {
            value[i] = spline_eval<false>(S, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], g);
        }
    }
}

// ============================================================================================== cell helpers
// Kernels with 27-point tables keep them in a per-thread slice of dynamic shared memory (slice k at
// smem[k * blockDim.x + threadIdx.x]: bank-conflict free); the edges of the fields stay in registers and the
// point loops stay rolled, so no kernel touches local memory.
constexpr int CS = 64;     // threads per block of the shared-memory cell kernels

__device__ __forceinline__ void load_edges(const double *__restrict__ u, long long n0, const Q1Const &q,
                                           double E[3][4][3]) {
    double v[8][3];
    load_cell(u, n0, q, v);
    cell_edges(v, E);
}
template <class R>
__device__ __forceinline__ void zero_slice(R *sl, int T, int n) {
    for (int k = 0; k < n; k++) sl[k * T] = R(0);
}
// S[j][s][t][r] += f[r][j] at point (ix, iy, iz): j = 0 -> (iy, iz), j = 1 -> (ix, iz), j = 2 -> (ix, iy)
template <class R>
__device__ __forceinline__ void add_flux(R *sl, int T, int ix, int iy, int iz, const R f[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
        sl[((iy * 3 + iz) * 3 + r) * T] += f[r][0];
        sl[(27 + (ix * 3 + iz) * 3 + r) * T] += f[r][1];
        sl[(54 + (ix * 3 + iy) * 3 + r) * T] += f[r][2];
    }
}
// adjoint of the edge interpolation (scatter_edges) reading S from the slice
template <class R, class C>
__device__ __forceinline__ void scatter_slice(const R *sl, int T, const C n[3], const C m[3], const C ih[3],
                                              R L[8][3]) {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            R e[4] = {R(0), R(0), R(0), R(0)};
#pragma unroll
            for (int s = 0; s < 3; s++) {
                R t0 = R(0), t1 = R(0);
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    R v = sl[(27 * j + (s * 3 + t) * 3 + r) * T] * (R)ih[j];
                    t0 += (R)m[t] * v;
                    t1 += (R)n[t] * v;
                }
                e[0] += (R)m[s] * t0;
                e[1] += (R)n[s] * t0;
                e[2] += (R)m[s] * t1;
                e[3] += (R)n[s] * t1;
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

// ============================================================================================== cell energy
// Reference J and curl at the Gauss points of one cell into the thread's shared slice (4 values per point).
__device__ __forceinline__ void reference_points(const double *__restrict__ uref, long long n0, const Q1Const &q,
                                                 double *sl, int T) {
    double Er[3][4][3];
    load_edges(uref, n0, q, Er);
    sweep<false>(Er, q, [&](int p, int, int, int, const double (&Vr)[3][3]) {
        double Cr[3];
        curl_of(Vr, Cr);
        sl[(4 * p) * T] = det_only(Vr);
        sl[(4 * p + 1) * T] = Cr[0];
        sl[(4 * p + 2) * T] = Cr[1];
        sl[(4 * p + 3) * T] = Cr[2];
    });
}

// partial[block][0..2] = sum w (J - Jr)^2, sum w |C - Cr|^2, sum barrier; violations counted in *bad
__global__ void __launch_bounds__(CS) cell_energy_kernel(Q1Const q, const double *__restrict__ u,
                                                         const double *__restrict__ uref, dd *partial,
                                                         unsigned long long *bad) {
    extern __shared__ double smem[];
    double *sl = smem + threadIdx.x;
    const int T = blockDim.x;
    dd acc[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
    unsigned long long nbad = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        reference_points(uref, n0, q, sl, T);
        double E[3][4][3];
        load_edges(u, n0, q, E);
        double sj = 0., sc = 0., sb = 0.;
        sweep<false>(E, q, [&](int p, int, int, int, const double (&V)[3][3]) {
            double C[3];
            curl_of(V, C);
            double dj = det_only(V) - sl[(4 * p) * T];
            double c0 = C[0] - sl[(4 * p + 1) * T], c1 = C[1] - sl[(4 * p + 2) * T], c2 = C[2] - sl[(4 * p + 3) * T];
            const double w = q.gw[p];
            sj += w * dj * dj;
            sc += w * (c0 * c0 + c1 * c1 + c2 * c2);
        });
        sweep<true>(E, q, [&](int, int, int, int, const double (&V)[3][3]) {
            double J = det_only(V);
            if (!(J > q.delta)) { nbad++; return; }
            if (J < q.act) {
                double b, b1, b2;
                barrier_eval(J, q.act, q.delta, q.bw, b, b1, b2);
                sb += b;
            }
        });
        acc[0] = dd_add_d(acc[0], sj);
        acc[1] = dd_add_d(acc[1], sc);
        acc[2] = dd_add_d(acc[2], sb);
    }
    block_reduce_dd<3>(acc, partial);
    for (int o = 16; o; o >>= 1) nbad += __shfl_xor_sync(0xFFFFFFFFu, nbad, o);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad, nbad);
}

// Per-cell vertex values -> SoA locals L[(a * 3 + r) * ncell + c].
template <class R>
__device__ __forceinline__ void store_locals(R *__restrict__ L, long long c, long long ncell, const R v[8][3]) {
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int r = 0; r < 3; r++) L[(long long)(a * 3 + r) * ncell + c] = v[a][r];
}

// ============================================================================================== cell gradients
// L1 = soft (JD, curl penalties scaled by mu_scale, nu_scale) + barrier; with split, L2 = barrier alone.
__global__ void __launch_bounds__(CS) cell_grad_kernel(Q1Const q, const double *__restrict__ u,
                                                       const double *__restrict__ uref, double mu_scale,
                                                       double nu_scale, bool barrier, bool split,
                                                       double *__restrict__ L1, double *__restrict__ L2,
                                                       const uint8_t *__restrict__ active) {
    extern __shared__ double smem[];
    double *sl = smem + threadIdx.x;
    const int T = blockDim.x;
    const double cn[3] = {0., .5, 1.}, cm[3] = {1., .5, 0.};
    const double mu = q.mu * mu_scale, nu = q.nu * nu_scale;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        double E[3][4][3], L[8][3];
        load_edges(u, n0, q, E);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) L[a][r] = 0.;
        if (mu != 0. || nu != 0.) {
            double Er[3][4][3];
            load_edges(uref, n0, q, Er);
            zero_slice(sl, T, 81);
            sweep2<false>(E, Er, q, [&](int p, int ix, int iy, int iz, const double (&V)[3][3],
                                        const double (&Vr)[3][3]) {
                double A[3][3], J, C[3], Cr[3];
                cofactor_det(V, A, J);
                double Jr = det_only(Vr);
                curl_of(V, C);
                curl_of(Vr, Cr);
                const double gw = q.gw[p];
                double jd = mu * gw * (J - Jr);
                double k0 = nu * gw * (C[0] - Cr[0]), k1 = nu * gw * (C[1] - Cr[1]), k2 = nu * gw * (C[2] - Cr[2]);
                double f[3][3];
#pragma unroll
                for (int r = 0; r < 3; r++)
#pragma unroll
                    for (int jj = 0; jj < 3; jj++) f[r][jj] = A[r][jj] * jd;
                f[2][1] += k0; f[1][2] -= k0;
                f[0][2] += k1; f[2][0] -= k1;
                f[1][0] += k2; f[0][1] -= k2;
                add_flux(sl, T, ix, iy, iz, f);
            });
            scatter_slice(sl, T, q.gn, q.gm, q.ih, L);
        }
        bool any = false;
        // cells whose closed27 J are all above the activation (the state's activity mask) have no barrier term
        if (barrier && (!active || active[c])) {
            zero_slice(sl, T, 81);
            sweep<true>(E, q, [&](int, int ix, int iy, int iz, const double (&V)[3][3]) {
                if (!(det_only(V) < q.act)) return;
                double A[3][3], J, b, b1, b2;
                cofactor_det(V, A, J);
                barrier_eval(J, q.act, q.delta, q.bw, b, b1, b2);
                double f[3][3];
#pragma unroll
                for (int r = 0; r < 3; r++)
#pragma unroll
                    for (int jj = 0; jj < 3; jj++) f[r][jj] = A[r][jj] * b1;
                add_flux(sl, T, ix, iy, iz, f);
                any = true;
            });
        }
        double Lb[8][3];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) Lb[a][r] = 0.;
        if (any) scatter_slice(sl, T, cn, cm, q.ih, Lb);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) L[a][r] += Lb[a][r];
        store_locals(L1, c, q.ncell, L);
        if (split) store_locals(L2, c, q.ncell, Lb);
    }
}

// ============================================================================================== gather
struct GatherSpec {
    int nout;
    double ci[3], cp[3], c1[3], c2[3];  // coefficients of image, proximity, L1, L2 per output
    double *out[3];
};

// Free node (z, y, x): sum of the 8 cells' vertex values in fixed order a = 0..7, plus node terms.
template <class LT>
__global__ void __launch_bounds__(256) gather_kernel(Q1Const q, GatherSpec g, const LT *__restrict__ L1,
                                                     const LT *__restrict__ L2, const double *__restrict__ u,
                                                     const double *__restrict__ uref,
                                                     const double *__restrict__ warped,
                                                     const double *__restrict__ fixed,
                                                     const double *__restrict__ image_grad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nfree;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.fx, q.fy, x, y, z);
        x++; y++; z++;
        long long node = (z * q.ny + y) * q.nx + x;
        double qw = node_weight(x, y, z, q);
        double dimg = warped ? qw * (warped[node] - fixed[node]) : 0.;
        // the 8 cells' vertex values summed in the locals' type (float locals: one conversion per sum, not per term)
        LT t1[3] = {LT(0), LT(0), LT(0)}, t2[3] = {LT(0), LT(0), LT(0)};
#pragma unroll
        for (int a = 0; a < 8; a++) {
            long long c = ((z - (a >> 2)) * q.cy + (y - ((a >> 1) & 1))) * q.cx + (x - (a & 1));
#pragma unroll
            for (int r = 0; r < 3; r++) {
                if (L1) t1[r] += L1[(long long)(a * 3 + r) * q.ncell + c];
                if (L2) t2[r] += L2[(long long)(a * 3 + r) * q.ncell + c];
            }
        }
        const double s1[3] = {(double)t1[0], (double)t1[1], (double)t1[2]};
        const double s2[3] = {(double)t2[0], (double)t2[1], (double)t2[2]};
#pragma unroll
        for (int r = 0; r < 3; r++) {
            double img = image_grad ? dimg * image_grad[3 * node + r] : 0.;
            double prox = uref ? q.lam * qw * (u[3 * node + r] - uref[3 * node + r]) : 0.;
#pragma unroll
            for (int k = 0; k < 3; k++)     // constant indices keep the spec in the parameter bank
                if (k < g.nout)
                    g.out[k][r * q.nfree + i] = ((g.ci[k] * img + g.cp[k] * prox) + g.c1[k] * s1[r]) + g.c2[k] * s2[r];
        }
    }
}

// ============================================================================================== GGN
// Per-cell diagonal contributions: sum_p w (mu lj^2 + nu cs) + sum_closed27 b'' lc^2, lj = sum_j A_rj D_jpa.
template <bool CLOSED>
__device__ __forceinline__ void point_D(const Q1Const &q, int ix, int iy, int iz, int a, double D[3]) {
    const int bx = a & 1, by = (a >> 1) & 1, bz = (a >> 2) & 1;
    const double fx = bx ? rule_n<CLOSED>(q, ix) : rule_m<CLOSED>(q, ix);
    const double fy = by ? rule_n<CLOSED>(q, iy) : rule_m<CLOSED>(q, iy);
    const double fz = bz ? rule_n<CLOSED>(q, iz) : rule_m<CLOSED>(q, iz);
    D[0] = (bx ? q.ih[0] : -q.ih[0]) * fy * fz;
    D[1] = (by ? q.ih[1] : -q.ih[1]) * fx * fz;
    D[2] = (bz ? q.ih[2] : -q.ih[2]) * fx * fy;
}

__global__ void __launch_bounds__(CT) cell_ggn_diag_kernel(Q1Const q, const double *__restrict__ u,
                                                           double *__restrict__ L,
                                                           const uint8_t *__restrict__ active, bool barrier) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        double E[3][4][3], out[8][3];
        load_edges(u, cell_node0(c, q), q, E);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) out[a][r] = 0.;
        // JD part per Gauss point; the curl part is the state-independent q.ggn_curl
        sweep<false>(E, q, [&](int p, int ix, int iy, int iz, const double (&V)[3][3]) {
            double A[3][3], J;
            cofactor_det(V, A, J);
            const double gmu = q.gw[p] * q.mu;
#pragma unroll
            for (int a = 0; a < 8; a++) {
                double D[3];
                point_D<false>(q, ix, iy, iz, a, D);
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    double lj = A[r][0] * D[0] + A[r][1] * D[1] + A[r][2] * D[2];
                    out[a][r] += gmu * (lj * lj);
                }
            }
        });
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) out[a][r] += q.ggn_curl[3 * a + r];
        if (barrier && (!active || active[c]))
        sweep<true>(E, q, [&](int, int ix, int iy, int iz, const double (&V)[3][3]) {
            if (!(det_only(V) < q.act)) return;
            double A[3][3], J, b, b1, b2;
            cofactor_det(V, A, J);
            barrier_eval(J, q.act, q.delta, q.bw, b, b1, b2);
#pragma unroll
            for (int a = 0; a < 8; a++) {
                double D[3];
                point_D<true>(q, ix, iy, iz, a, D);
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    double lc = A[r][0] * D[0] + A[r][1] * D[1] + A[r][2] * D[2];
                    out[a][r] += b2 * lc * lc;
                }
            }
        });
        store_locals(L, c, q.ncell, out);
    }
}

// GGN action on a node field vv (zero faces): Gauss JD/curl linearization + closed27 barrier curvature.
__global__ void __launch_bounds__(CS) cell_ggn_hvp_kernel(Q1Const q, const double *__restrict__ u,
                                                          const double *__restrict__ vv, double *__restrict__ L) {
    extern __shared__ double smem[];
    double *sl = smem + threadIdx.x;
    const int T = blockDim.x;
    const double cn[3] = {0., .5, 1.}, cm[3] = {1., .5, 0.};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        double E[3][4][3], Ev[3][4][3], out[8][3];
        load_edges(u, n0, q, E);
        load_edges(vv, n0, q, Ev);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) out[a][r] = 0.;
        zero_slice(sl, T, 81);
        sweep2<false>(E, Ev, q, [&](int p, int ix, int iy, int iz, const double (&V)[3][3],
                                    const double (&W)[3][3]) {
            double A[3][3], J, K[3];
            cofactor_det(V, A, J);
            double jd = 0.;
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int jj = 0; jj < 3; jj++) jd += A[r][jj] * W[r][jj];
            curl_of(W, K);
            const double gw = q.gw[p];
            jd *= q.mu * gw;
            double k0 = q.nu * gw * K[0], k1 = q.nu * gw * K[1], k2 = q.nu * gw * K[2];
            double f[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int jj = 0; jj < 3; jj++) f[r][jj] = A[r][jj] * jd;
            f[2][1] += k0; f[1][2] -= k0;
            f[0][2] += k1; f[2][0] -= k1;
            f[1][0] += k2; f[0][1] -= k2;
            add_flux(sl, T, ix, iy, iz, f);
        });
        scatter_slice(sl, T, q.gn, q.gm, q.ih, out);
        zero_slice(sl, T, 81);
        bool any = false;
        sweep2<true>(E, Ev, q, [&](int, int ix, int iy, int iz, const double (&V)[3][3], const double (&W)[3][3]) {
            if (!(det_only(V) < q.act)) return;
            double A[3][3], J, b, b1, b2;
            cofactor_det(V, A, J);
            barrier_eval(J, q.act, q.delta, q.bw, b, b1, b2);
            double lj = 0.;
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int jj = 0; jj < 3; jj++) lj += A[r][jj] * W[r][jj];
            lj *= b2;
            double f[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int jj = 0; jj < 3; jj++) f[r][jj] = A[r][jj] * lj;
            add_flux(sl, T, ix, iy, iz, f);
            any = true;
        });
        if (any) scatter_slice(sl, T, cn, cm, q.ih, out);
        store_locals(L, c, q.ncell, out);
    }
}

// node part of the GGN: q |b|^2 + lambda q (diagonal) or q b (b . v) + lambda q v (action)
template <class LT>
__global__ void __launch_bounds__(256) ggn_node_kernel(Q1Const q, const LT *__restrict__ L,
                                                       const double *__restrict__ image_grad,
                                                       const double *__restrict__ vv, double *__restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nfree;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.fx, q.fy, x, y, z);
        x++; y++; z++;
        long long node = (z * q.ny + y) * q.nx + x;
        double qw = node_weight(x, y, z, q);
        double s[3] = {0., 0., 0.};
#pragma unroll
        for (int a = 0; a < 8; a++) {
            long long c = ((z - (a >> 2)) * q.cy + (y - ((a >> 1) & 1))) * q.cx + (x - (a & 1));
#pragma unroll
            for (int r = 0; r < 3; r++) s[r] += (double)L[(long long)(a * 3 + r) * q.ncell + c];
        }
        const double *b = image_grad + 3 * node;
        if (vv) {
            const double *v = vv + 3 * node;
            double bv = b[0] * v[0] + b[1] * v[1] + b[2] * v[2];
#pragma unroll
            for (int r = 0; r < 3; r++) out[r * q.nfree + i] = (qw * b[r] * bv + q.lam * qw * v[r]) + s[r];
        } else {
#pragma unroll
            for (int r = 0; r < 3; r++) out[r * q.nfree + i] = (qw * b[r] * b[r] + q.lam * qw) + s[r];
        }
    }
}

// ============================================================================================== mixed form
// The direction pipeline in float32 (gradient, GGN diagonal): edge differences formed in float64 from the float64
// state and rounded once, grad u, cofactors, fluxes and the separable adjoint in float32, float32 locals gathered in
// float64.  The localized barrier stays float64, in separate kernels that visit only the flagged cells: cells active
// in the state's mask, or (without a mask) cells with some float32 closed27 J within kBarrierGuard of the
// activation.  There the whole closed27 sweep is redone in float64 from the float64 state (the plain form's J,
// cofactors and barrier values) and added to the cell's float32 locals, so the float32 kernels carry neither the
// float64 sweep nor its registers.
constexpr float kBarrierGuard = 1e-3f;
constexpr int CB = 128;               // threads per block of the float64 barrier kernels
constexpr int kFlagChunk = 256;       // consecutive cells a warp scans at a time for flagged cells

// Calls f(c, flags[c]) for the flagged cells (flags[c] != 0).  Warp w of the grid scans the chunks of kFlagChunk
// cells w, w + warps, ...; the flagged cells are queued in the warp's shared queue (64 entries) in cell order and
// handed to the lanes 32 at a time, so the float64 work runs on full warps whatever the flags' pattern, and every cell
// goes to the same lane on every run (the lanes' sums are deterministic).
template <class F>
__device__ __forceinline__ void for_flagged_cells(const Q1Const &q, const uint8_t *__restrict__ flags,
                                                  long long *queue, F &&f) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long nchunk = (q.ncell + kFlagChunk - 1) / kFlagChunk;
    long long k = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    long long b = k * kFlagChunk;
    int qn = 0;
    // a chunk's 256 flags are read once, 8 per lane (one 64-bit load where the chunk is whole and aligned), and the
    // flag of cell chunk + 32 j + l is byte l % 8 of lane 4 j + l / 8's word; cells past the end read as zero
    const bool wide = (reinterpret_cast<uintptr_t>(flags) & 7) == 0;
    unsigned long long word = 0;
    for (;;) {
        // fill the queue to a full warp's worth, or until the warp's chunks are exhausted
        while (qn < 32 && k < nchunk) {
            const long long c0 = k * kFlagChunk, hi = min(c0 + kFlagChunk, q.ncell), c = b + lane;
            if (b == c0) {
                const long long f0 = c0 + 8 * lane;
                if (wide && c0 + kFlagChunk <= q.ncell) {
                    word = *reinterpret_cast<const unsigned long long *>(flags + f0);
                } else {
                    word = 0;
#pragma unroll
                    for (int t = 0; t < 8; t++)
                        if (f0 + t < q.ncell) word |= (unsigned long long)flags[f0 + t] << (8 * t);
                }
            }
            const int j = (int)((b - c0) >> 5);
            const unsigned long long v = __shfl_sync(0xFFFFFFFFu, word, 4 * j + (lane >> 3));
            const bool on = c < hi && ((v >> (8 * (lane & 7))) & 0xFFull) != 0;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, on);
            if (on) queue[qn + __popc(m & ((1u << lane) - 1u))] = c;
            qn += __popc(m);
            b += 32;
            if (b >= hi) {
                k += warps;
                b = k * kFlagChunk;
            }
        }
        __syncwarp();
        if (qn == 0) break;
        const int take = qn < 32 ? qn : 32;
        const long long c = lane < take ? queue[lane] : -1;
        __syncwarp();
        if (lane + 32 < qn) queue[lane] = queue[lane + 32];
        __syncwarp();
        qn -= take;
        if (c >= 0) f(c, flags[c]);
    }
}
unsigned barrier_blocks(const Q1Const &q) {
    const long long nchunk = (q.ncell + kFlagChunk - 1) / kFlagChunk;
    return blocks_for(nchunk * 32, CB, 4);
}

__device__ __forceinline__ void load_edges_f32(const double *__restrict__ u, long long n0, const Q1Const &q,
                                               float E[3][4][3]) {
    double v[8][3];
    load_cell(u, n0, q, v);
    double E64[3][4][3];
    cell_edges(v, E64);
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int e = 0; e < 4; e++)
#pragma unroll
            for (int r = 0; r < 3; r++) E[j][e][r] = (float)E64[j][e][r];
}
// The soft part (JD, curl penalties) of the gradient locals; with split, L2 is zeroed for the barrier kernel.  flags
// (when the state has no mask): 1 for the cells with some float32 closed27 J within the guard.
__global__ void __launch_bounds__(CS, 8) cell_grad32_kernel(Q1Const q, const double *__restrict__ u,
                                                         const double *__restrict__ uref, double mu_scale,
                                                         double nu_scale, bool split, float *__restrict__ L1,
                                                         float *__restrict__ L2, uint8_t *__restrict__ flags) {
    extern __shared__ float smemf[];
    float *sl = smemf + threadIdx.x;
    const int T = blockDim.x;
    const float mu = (float)(q.mu * mu_scale), nu = (float)(q.nu * nu_scale);
    const float guard = (float)q.act + kBarrierGuard;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        float E[3][4][3], L[8][3];
        load_edges_f32(u, n0, q, E);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) L[a][r] = 0.f;
        if (mu != 0.f || nu != 0.f) {
            float Er[3][4][3];
            load_edges_f32(uref, n0, q, Er);
            zero_slice(sl, T, 81);
            sweep2<false, float>(E, Er, q, [&](int p, int ix, int iy, int iz, const float (&V)[3][3],
                                               const float (&Vr)[3][3]) {
                float A[3][3], J, C[3], Cr[3];
                cofactor_det(V, A, J);
                float Jr = det_only(Vr);
                curl_of(V, C);
                curl_of(Vr, Cr);
                const float gw = q.gwf[p];
                float jd = mu * gw * (J - Jr);
                float k0 = nu * gw * (C[0] - Cr[0]), k1 = nu * gw * (C[1] - Cr[1]), k2 = nu * gw * (C[2] - Cr[2]);
                float f[3][3];
#pragma unroll
                for (int r = 0; r < 3; r++)
#pragma unroll
                    for (int jj = 0; jj < 3; jj++) f[r][jj] = A[r][jj] * jd;
                f[2][1] += k0; f[1][2] -= k0;
                f[0][2] += k1; f[2][0] -= k1;
                f[1][0] += k2; f[0][1] -= k2;
                add_flux(sl, T, ix, iy, iz, f);
            });
            scatter_slice(sl, T, q.gnf, q.gmf, q.ihf, L);
        }
        // without a mask, the cells with some float32 closed27 J within the guard are flagged for the barrier kernel
        if (flags) {
            bool near = false;
            sweep<true, float>(E, q, [&](int, int, int, int, const float (&V)[3][3]) {
                near |= det_only(V) < guard;
            });
            flags[c] = near ? 1 : 0;
        }
        store_locals(L1, c, q.ncell, L);
        if (split) {
            float Z[8][3];
#pragma unroll
            for (int a = 0; a < 8; a++)
#pragma unroll
                for (int r = 0; r < 3; r++) Z[a][r] = 0.f;
            store_locals(L2, c, q.ncell, Z);
        }
    }
}

// The barrier's locals of the flagged cells in float64: the closed27 sweep from the float64 state, J, b' and the
// cofactors exactly as the float64 kernel forms them, the flux rounded to the locals' type LT (float32 in the mixed
// form, float64 in the plain one) and scattered as the soft kernel scatters its own; then added to the cell's locals
// (L1 += Lb) and, for the outer triple, stored apart (L2).  In the plain form the values are those of the fused
// float64 kernel (the same sweep of the same edges, the same add).
template <class LT>
__global__ void __launch_bounds__(CB) cell_grad_barrier_kernel(Q1Const q, const double *__restrict__ u,
                                                               const uint8_t *__restrict__ flags, bool split,
                                                               LT *__restrict__ L1, LT *__restrict__ L2) {
    extern __shared__ __align__(16) unsigned char smemb[];
    __shared__ long long queue[CB / 32][64];
    LT *sl = reinterpret_cast<LT *>(smemb) + threadIdx.x;
    const int T = blockDim.x;
    const LT cn[3] = {LT(0), LT(.5), LT(1)}, cm[3] = {LT(1), LT(.5), LT(0)};
    const LT ih[3] = {(LT)q.ih[0], (LT)q.ih[1], (LT)q.ih[2]};
    for_flagged_cells(q, flags, queue[threadIdx.x >> 5], [&](long long c, uint8_t) {
        double E64[3][4][3];
        load_edges(u, cell_node0(c, q), q, E64);
        zero_slice(sl, T, 81);
        bool any = false;
        sweep<true>(E64, q, [&](int, int ix, int iy, int iz, const double (&V)[3][3]) {
            if (!(det_only(V) < q.act)) return;
            double A[3][3], J, b, b1, b2;
            cofactor_det(V, A, J);
            barrier_eval(J, q.act, q.delta, q.bw, b, b1, b2);
            LT f[3][3];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int jj = 0; jj < 3; jj++) f[r][jj] = (LT)(A[r][jj] * b1);
            add_flux(sl, T, ix, iy, iz, f);
            any = true;
        });
        if (!any) return;
        LT Lb[8][3];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) Lb[a][r] = LT(0);
        scatter_slice(sl, T, cn, cm, ih, Lb);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) L1[(size_t)(3 * a + r) * q.ncell + c] += Lb[a][r];
        if (split) store_locals(L2, c, q.ncell, Lb);
    });
}

// GGN diagonal contributions in float32 (Gauss JD/curl part); flags (when the state has no mask) as the gradient's.
__global__ void __launch_bounds__(CT, 4) cell_ggn_diag32_kernel(Q1Const q, const double *__restrict__ u,
                                                             float *__restrict__ L, uint8_t *__restrict__ flags) {
    const float guard = (float)q.act + kBarrierGuard;
    const float mu = (float)q.mu;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const long long n0 = cell_node0(c, q);
        float E[3][4][3], out[8][3];
        load_edges_f32(u, n0, q, E);
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) out[a][r] = 0.f;
        sweep<false, float>(E, q, [&](int p, int ix, int iy, int iz, const float (&V)[3][3]) {
            float A[3][3], J;
            cofactor_det(V, A, J);
            const float gmu = q.gwf[p] * mu;
#pragma unroll
            for (int a = 0; a < 8; a++) {
                const int bx = a & 1, by = (a >> 1) & 1, bz = (a >> 2) & 1;
                const float fx = bx ? q.gnf[ix] : q.gmf[ix];
                const float fy = by ? q.gnf[iy] : q.gmf[iy];
                const float fz = bz ? q.gnf[iz] : q.gmf[iz];
                float D[3];
                D[0] = (bx ? q.ihf[0] : -q.ihf[0]) * fy * fz;
                D[1] = (by ? q.ihf[1] : -q.ihf[1]) * fx * fz;
                D[2] = (bz ? q.ihf[2] : -q.ihf[2]) * fx * fy;
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    float lj = A[r][0] * D[0] + A[r][1] * D[1] + A[r][2] * D[2];
                    out[a][r] += gmu * (lj * lj);
                }
            }
        });
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) out[a][r] += q.ggn_curlf[3 * a + r];
        if (flags) {
            bool near = false;
            sweep<true, float>(E, q, [&](int, int, int, int, const float (&V)[3][3]) { near |= det_only(V) < guard; });
            flags[c] = near ? 1 : 0;
        }
        store_locals(L, c, q.ncell, out);
    }
}

// The barrier curvature b'' lc^2 of the flagged cells in float64 (J, b'' and the cofactors lc from the float64
// state), rounded to the locals' type LT and added point by point in sweep order to the cell's locals (in the plain
// form the additions of the fused float64 kernel).
template <class LT>
__global__ void __launch_bounds__(CB) cell_ggn_barrier_kernel(Q1Const q, const double *__restrict__ u,
                                                              const uint8_t *__restrict__ flags,
                                                              LT *__restrict__ L) {
    __shared__ long long queue[CB / 32][64];
    for_flagged_cells(q, flags, queue[threadIdx.x >> 5], [&](long long c, uint8_t) {
        double E64[3][4][3];
        load_edges(u, cell_node0(c, q), q, E64);
        LT out[8][3];
#pragma unroll
        for (int a = 0; a < 8; a++)
#pragma unroll
            for (int r = 0; r < 3; r++) out[a][r] = L[(size_t)(3 * a + r) * q.ncell + c];
        bool any = false;
        sweep<true>(E64, q, [&](int, int ix, int iy, int iz, const double (&V64)[3][3]) {
            if (!(det_only(V64) < q.act)) return;
            any = true;
            double A[3][3], J, b, b1, b2;
            cofactor_det(V64, A, J);
            barrier_eval(J, q.act, q.delta, q.bw, b, b1, b2);
#pragma unroll
            for (int a = 0; a < 8; a++) {
                double D[3];
                point_D<true>(q, ix, iy, iz, a, D);
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    double lc = A[r][0] * D[0] + A[r][1] * D[1] + A[r][2] * D[2];
                    if constexpr (sizeof(LT) == 8) out[a][r] += b2 * lc * lc;   // the fused kernel's expression
                    else out[a][r] += (LT)(b2 * lc * lc);
                }
            }
        });
        if (any) store_locals(L, c, q.ncell, out);
    });
}

// ============================================================================================== stable differences
// One residual pair: (b - a)(b + a) / 2 accumulated exactly enough in double-double.
__device__ __forceinline__ dd sq_change(double a, double b) {
    dd d = two_sum(b, -a), s = two_sum(b, a);
    dd p = two_prod(d.hi, s.hi);
    p.lo += d.hi * s.lo + d.lo * s.hi;
    return {p.hi * .5, p.lo * .5};
}

// energy_comparison.py:14-62 localized branch (double precision), unweighted
__device__ __forceinline__ double barrier_difference(double ja, double jb, double act, double d) {
    double a = ja < act ? ja : act, b = jb < act ? jb : act;
    double scale = act - d;
    double ra = (act - a) / scale, rb = (act - b) / scale;
    double h = (b - a) / scale;
    double loga = ra < .5 ? log1p(-ra) : log((a - d) / scale);
    double x = (b - a) / (a - d);
    double ratio = x >= -.5 ? log1p(x) : log((b - d) / (a - d));
    return h * (ra + rb) * loga - rb * rb * ratio;
}

__global__ void __launch_bounds__(256) node_diff_kernel(Q1Const q, const double *__restrict__ ua,
                                                        const double *__restrict__ wa,
                                                        const double *__restrict__ ub,
                                                        const double *__restrict__ wb,
                                                        const double *__restrict__ fixed,
                                                        const double *__restrict__ uref, dd *partial) {
    dd acc[2] = {{0., 0.}, {0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nnode;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.nx, q.ny, x, y, z);
        double qw = node_weight(x, y, z, q);
        double sq = sqrt(qw), sl = sqrt(q.lam * qw);
        acc[0] = dd_add(acc[0], sq_change(sq * (wa[i] - fixed[i]), sq * (wb[i] - fixed[i])));
#pragma unroll
        for (int r = 0; r < 3; r++)
            acc[1] = dd_add(acc[1], sq_change(sl * (ua[3 * i + r] - uref[3 * i + r]),
                                              sl * (ub[3 * i + r] - uref[3 * i + r])));
    }
    block_reduce_dd<2>(acc, partial);
}

// Reference J and curl at the Gauss points go to the thread's shared slice first (108 values), so only the two
// compared fields' edges are live in registers during the main pass.  Per-point changes are exact products
// (sq_change) summed with a compensated (hi, lo) accumulator.
__device__ __forceinline__ void acc_add(dd &acc, dd t) {
    dd s = two_sum(acc.hi, t.hi);
    acc.hi = s.hi;
    acc.lo += s.lo + t.lo;
}
__global__ void __launch_bounds__(CS) cell_diff_kernel(Q1Const q, const double *__restrict__ ua,
                                                       const double *__restrict__ ub,
                                                       const double *__restrict__ uref, dd *partial,
                                                       const uint8_t *__restrict__ act_a,
                                                       const uint8_t *__restrict__ act_b,
                                                       uint8_t *__restrict__ flags) {
    extern __shared__ double smem[];
    double *sl = smem + threadIdx.x;
    const int T = blockDim.x;
    dd acc[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        reference_points(uref, n0, q, sl, T);
        double Ea[3][4][3], Eb[3][4][3];
        load_edges(ua, n0, q, Ea);
        load_edges(ub, n0, q, Eb);
        sweep2<false>(Ea, Eb, q, [&](int p, int, int, int, const double (&Va)[3][3], const double (&Vb)[3][3]) {
            double Ca[3], Cb[3];
            const double jr = sl[(4 * p) * T];
            const double smu = q.sqmu[p], snu = q.sqnu[p];
            acc_add(acc[0], sq_change(smu * (det_only(Va) - jr), smu * (det_only(Vb) - jr)));
            curl_of(Va, Ca);
            curl_of(Vb, Cb);
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const double cr = sl[(4 * p + 1 + r) * T];
                acc_add(acc[1], sq_change(snu * (Ca[r] - cr), snu * (Cb[r] - cr)));
            }
        });
        double sb = 0.;
        // with both masks, a cell inactive in both fields has no barrier difference at all; with flags, the cells
        // that have one are handed to cell_trial_diff_kernel (the same per-cell value)
        const bool needs = !(act_a && act_b && !act_a[c] && !act_b[c]);
        if (flags)
            flags[c] = needs ? 1 : 0;
        else if (needs)
            sweep2<true>(Ea, Eb, q, [&](int, int, int, int, const double (&Va)[3][3], const double (&Vb)[3][3]) {
                double ja = det_only(Va), jb = det_only(Vb);
                if (ja < q.act || jb < q.act) sb += barrier_difference(ja, jb, q.act, q.delta);
            });
        acc_add(acc[2], dd{q.bw * sb, 0.});
    }
#pragma unroll
    for (int k = 0; k < 3; k++) acc[k] = two_sum(acc[k].hi, acc[k].lo);
    block_reduce_dd<3>(acc, partial);
}

// ============================================================================================== line-search trial
// A trial evaluated against its base in one node pass and one cell pass: the trial's warped image (and image
// gradient), its energy sums exactly as node_energy_kernel / cell_energy_kernel form them, and the stable base ->
// trial changes exactly as node_diff_kernel / cell_diff_kernel form them (same grids, same per-thread order, so the
// results are bitwise those of the separate passes).
template <bool GRAD>
__global__ void __launch_bounds__(256) warp_trial_kernel(Q1Const q, SplineRef S, const double *__restrict__ ua,
                                                         const double *__restrict__ wa,
                                                         const double *__restrict__ ub,
                                                         const double *__restrict__ fixed,
                                                         const double *__restrict__ uref, double *__restrict__ wb,
                                                         double *__restrict__ image_grad, dd *pe, dd *pd) {
    dd acc[2] = {{0., 0.}, {0., 0.}}, dif[2] = {{0., 0.}, {0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nnode;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.nx, q.ny, x, y, z);
        double ux = ub[3 * i], uy = ub[3 * i + 1], uz = ub[3 * i + 2];
        double px = (q.x0[0] + q.h[0] * (double)x) + ux;
        double py = (q.x0[1] + q.h[1] * (double)y) + uy;
        double pz = (q.x0[2] + q.h[2] * (double)z) + uz;
        double g[3];
        double w = spline_eval<GRAD>(S, px, py, pz, g);
        wb[i] = w;
        if (GRAD) {
            image_grad[3 * i] = g[0];
            image_grad[3 * i + 1] = g[1];
            image_grad[3 * i + 2] = g[2];
        }
        double qw = node_weight(x, y, z, q);
        double f = fixed[i];
        double d = w - f;
        double r0 = uref[3 * i], r1 = uref[3 * i + 1], r2 = uref[3 * i + 2];
        double e0 = ux - r0, e1 = uy - r1, e2 = uz - r2;
        acc[0] = dd_add_d(acc[0], qw * d * d);
        acc[1] = dd_add_d(acc[1], qw * (e0 * e0 + e1 * e1 + e2 * e2));
        double sq = sqrt(qw), sl = sqrt(q.lam * qw);
        dif[0] = dd_add(dif[0], sq_change(sq * (wa[i] - f), sq * d));
        dif[1] = dd_add(dif[1], sq_change(sl * (ua[3 * i] - r0), sl * e0));
        dif[1] = dd_add(dif[1], sq_change(sl * (ua[3 * i + 1] - r1), sl * e1));
        dif[1] = dd_add(dif[1], sq_change(sl * (ua[3 * i + 2] - r2), sl * e2));
    }
    block_reduce_dd<2>(acc, pe);
    __syncthreads();     // the two reductions share block_reduce_dd's shared array
    block_reduce_dd<2>(dif, pd);
}

// Barrier activity mask: act[c] = 1 when some closed27 J of cell c is below the activation; trial_act (optional)
// receives the trial's mask, which later calls on that state use to skip barrier sweeps that contribute nothing.
//
// The closed27 part runs the trial's sweep alone first (its J values parked in the thread's slice, whose reference
// values are dead after the Gauss sweep); the base's sweep and the barrier differences follow only where some point
// of either state is below the activation: the trial's (just found) or the base's (base_act, its mask from its own
// evaluation; NULL: unknown, always sweep).  Elsewhere every difference term is zero.  Same values in the same
// order per accumulator as one two-field sweep.
__global__ void __launch_bounds__(CS) cell_trial_kernel(Q1Const q, const double *__restrict__ ua,
                                                        const double *__restrict__ ub,
                                                        const double *__restrict__ uref, dd *pe, dd *pd,
                                                        unsigned long long *bad, uint8_t *__restrict__ trial_act,
                                                        const uint8_t *__restrict__ base_act,
                                                        uint8_t *__restrict__ flags) {
    extern __shared__ double smem[];
    double *sl = smem + threadIdx.x;
    const int T = blockDim.x;
    dd acc[3] = {{0., 0.}, {0., 0.}, {0., 0.}}, dif[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
    unsigned long long nbad = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        reference_points(uref, n0, q, sl, T);
        double Ea[3][4][3], Eb[3][4][3];
        load_edges(ua, n0, q, Ea);
        load_edges(ub, n0, q, Eb);
        double sj = 0., sc = 0., sb = 0., sbd = 0.;
        sweep2<false>(Ea, Eb, q, [&](int p, int, int, int, const double (&Va)[3][3], const double (&Vb)[3][3]) {
            double Ca[3], Cb[3];
            const double jr = sl[(4 * p) * T];
            const double smu = q.sqmu[p], snu = q.sqnu[p];
            const double jb = det_only(Vb);
            acc_add(dif[0], sq_change(smu * (det_only(Va) - jr), smu * (jb - jr)));
            curl_of(Va, Ca);
            curl_of(Vb, Cb);
            double cd[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const double cr = sl[(4 * p + 1 + r) * T];
                cd[r] = Cb[r] - cr;
                acc_add(dif[1], sq_change(snu * (Ca[r] - cr), snu * cd[r]));
            }
            const double w = q.gw[p], dj = jb - jr;
            sj += w * dj * dj;
            sc += w * (cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
        });
        bool active = false;
        sweep<true>(Eb, q, [&](int p, int, int, int, const double (&Vb)[3][3]) {
            const double jb = det_only(Vb);
            sl[p * T] = jb;
            active |= jb < q.act;
            if (!(jb > q.delta)) { nbad++; return; }
            if (jb < q.act) {
                double b, b1, b2;
                barrier_eval(jb, q.act, q.delta, q.bw, b, b1, b2);
                sb += b;
            }
        });
        // the barrier differences of the cells where the trial or the base is active: here, or (flags) in
        // cell_trial_diff_kernel over those cells alone
        const bool needs = active || !base_act || base_act[c];
        if (flags) {
            flags[c] = needs ? 1 : 0;
        } else if (needs) {
            load_edges(ua, n0, q, Ea);
            sweep<true>(Ea, q, [&](int p, int, int, int, const double (&Va)[3][3]) {
                const double ja = det_only(Va), jb = sl[p * T];
                if (ja < q.act || jb < q.act) sbd += barrier_difference(ja, jb, q.act, q.delta);
            });
        }
        if (trial_act) trial_act[c] = active ? 1 : 0;
        acc[0] = dd_add_d(acc[0], sj);
        acc[1] = dd_add_d(acc[1], sc);
        acc[2] = dd_add_d(acc[2], sb);
        acc_add(dif[2], dd{q.bw * sbd, 0.});
    }
#pragma unroll
    for (int k = 0; k < 3; k++) dif[k] = two_sum(dif[k].hi, dif[k].lo);
    block_reduce_dd<3>(acc, pe);
    __syncthreads();     // the two reductions share block_reduce_dd's shared array
    block_reduce_dd<3>(dif, pd);
    for (int o = 16; o; o >>= 1) nbad += __shfl_xor_sync(0xFFFFFFFFu, nbad, o);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad, nbad);
}

// The float64 trial's barrier differences of the flagged cells (trial or base active), as cell_trial_kernel forms
// them per cell: the trial's closed27 J from its edges, the base's, psi differences where either is below the
// activation.  pd: per block, the barrier difference sum.
__global__ void __launch_bounds__(CB) cell_trial_diff_kernel(Q1Const q, const double *__restrict__ ua,
                                                             const double *__restrict__ ub,
                                                             const uint8_t *__restrict__ flags, dd *pd) {
    extern __shared__ double smem[];
    __shared__ long long queue[CB / 32][64];
    double *dsl = smem + threadIdx.x;
    const int T = blockDim.x;
    dd dif[1] = {{0., 0.}};
    for_flagged_cells(q, flags, queue[threadIdx.x >> 5], [&](long long c, uint8_t) {
        const long long n0 = cell_node0(c, q);
        double E[3][4][3];
        load_edges(ub, n0, q, E);
        sweep<true>(E, q, [&](int p, int, int, int, const double (&Vb)[3][3]) { dsl[p * T] = det_only(Vb); });
        load_edges(ua, n0, q, E);
        double sbd = 0.;
        sweep<true>(E, q, [&](int p, int, int, int, const double (&Va)[3][3]) {
            const double ja = det_only(Va), jb = dsl[p * T];
            if (ja < q.act || jb < q.act) sbd += barrier_difference(ja, jb, q.act, q.delta);
        });
        acc_add(dif[0], dd{q.bw * sbd, 0.});
    });
    dif[0] = two_sum(dif[0].hi, dif[0].lo);
    block_reduce_dd<1>(dif, pd);
}

// ============================================================================================== screened trial
// The mixed form's line-search trial: the JD and curl penalties at the Gauss points in float32 (reference J and curl
// in a float slice, both fields' float edges), their per-cell sums in float and the block sums in double-double; the
// localized barrier and its difference as cell_trial_kernel forms them in float64 (a cell with some float32 closed27 J
// within kBarrierGuard of the activation takes the float64 closed27 sweep; elsewhere every J is above the activation
// in both arithmetics, where the barrier and its difference vanish).  So the violation count and the activity mask
// are cell_trial_kernel's, the barrier sums equal within rounding, and only the JD/curl sums carry float32 error,
// which the host screens against a band (the reference's float32 energy screen, backends/accelerated.py:66-77).
__device__ __forceinline__ void reference_points32(const double *__restrict__ uref, long long n0, const Q1Const &q,
                                                   float *sl, int T) {
    float Er[3][4][3];
    load_edges_f32(uref, n0, q, Er);
    sweep<false, float>(Er, q, [&](int p, int, int, int, const float (&Vr)[3][3]) {
        float Cr[3];
        curl_of(Vr, Cr);
        sl[(4 * p) * T] = det_only(Vr);
        sl[(4 * p + 1) * T] = Cr[0];
        sl[(4 * p + 2) * T] = Cr[1];
        sl[(4 * p + 3) * T] = Cr[2];
    });
}
// The soft part of the screened trial (JD and curl penalty sums and differences) in float32; the barrier part runs in
// cell_trial_barrier_kernel over the cells this kernel flags.  pe, pd: per block, the two soft sums and their two
// differences; pb (the screen's error-bound sums): sum w (|ra| + |rb|) of the JD residuals, the same of the curl
// residual components, sum w ra^2 and sum w |xa|^2 (the base's soft sums), all from the float32 residuals.
__global__ void __launch_bounds__(CS) cell_trial32_kernel(Q1Const q, const double *__restrict__ ua,
                                                          const double *__restrict__ ub,
                                                          const double *__restrict__ uref, dd *pe, dd *pd, dd *pb,
                                                          uint8_t *__restrict__ flags,
                                                          uint8_t *__restrict__ trial_act,
                                                          const uint8_t *__restrict__ base_act) {
    extern __shared__ float smemf[];
    const int T = blockDim.x;
    // per thread: 108 floats (reference J and curl at the Gauss points), strided by the block size
    float *fsl = smemf + threadIdx.x;
    const float guard = (float)q.act + kBarrierGuard;
    dd acc[2] = {{0., 0.}, {0., 0.}}, dif[2] = {{0., 0.}, {0., 0.}};
    dd bnd[4] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        reference_points32(uref, n0, q, fsl, T);
        float Ea[3][4][3], Eb[3][4][3];
        load_edges_f32(ua, n0, q, Ea);
        load_edges_f32(ub, n0, q, Eb);
        float sj = 0.f, sc = 0.f, dj = 0.f, dc = 0.f, mj = 0.f, mc = 0.f, aj = 0.f, ac = 0.f;
        sweep2<false, float>(Ea, Eb, q, [&](int p, int, int, int, const float (&Va)[3][3], const float (&Vb)[3][3]) {
            float Ca[3], Cb[3];
            const float jr = fsl[(4 * p) * T];
            const float ja = det_only(Va) - jr, jb = det_only(Vb) - jr;
            curl_of(Va, Ca);
            curl_of(Vb, Cb);
            const float w = q.gwf[p];
            float cb2 = 0.f, ca2 = 0.f, cd = 0.f, cm = 0.f;
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const float cr = fsl[(4 * p + 1 + r) * T];
                const float xa = Ca[r] - cr, xb = Cb[r] - cr;
                cb2 += xb * xb;
                ca2 += xa * xa;
                cd += (xb - xa) * (xb + xa);
                cm += fabsf(xa) + fabsf(xb);
            }
            sj += w * jb * jb;
            sc += w * cb2;
            dj += w * ((jb - ja) * (jb + ja));
            dc += w * cd;
            mj += w * (fabsf(ja) + fabsf(jb));
            mc += w * cm;
            aj += w * ja * ja;
            ac += w * ca2;
        });
        // the closed27 J in float32: a cell with some trial point within the guard (bit 0), or some base point within
        // the guard where the base may be active (bit 1), is flagged for the float64 barrier kernel; elsewhere every
        // J is above the activation in both arithmetics (no barrier, no difference, no violation)
        bool near_b = false, near_a = false;
        sweep<true, float>(Eb, q, [&](int, int, int, int, const float (&Vb)[3][3]) {
            near_b |= det_only(Vb) < guard;
        });
        if (near_b || !base_act || base_act[c])
            sweep<true, float>(Ea, q, [&](int, int, int, int, const float (&Va)[3][3]) {
                near_a |= det_only(Va) < guard;
            });
        flags[c] = (near_b ? 1 : 0) | (near_a ? 2 : 0);
        if (trial_act) trial_act[c] = 0;
        acc[0] = dd_add_d(acc[0], (double)sj);
        acc[1] = dd_add_d(acc[1], (double)sc);
        acc_add(dif[0], dd{.5 * q.mu * (double)dj, 0.});
        acc_add(dif[1], dd{.5 * q.nu * (double)dc, 0.});
        bnd[0] = dd_add_d(bnd[0], (double)mj);
        bnd[1] = dd_add_d(bnd[1], (double)mc);
        bnd[2] = dd_add_d(bnd[2], (double)aj);
        bnd[3] = dd_add_d(bnd[3], (double)ac);
    }
#pragma unroll
    for (int k = 0; k < 2; k++) dif[k] = two_sum(dif[k].hi, dif[k].lo);
    block_reduce_dd<2>(acc, pe);
    __syncthreads();     // the reductions share block_reduce_dd's shared array
    block_reduce_dd<2>(dif, pd);
    __syncthreads();
    block_reduce_dd<4>(bnd, pb);
}

// The barrier part of the screened trial in float64 over the flagged cells, exactly as the float64 trial kernel forms
// it per cell: the trial's closed27 sweep (barrier, violations, the trial's mask bit; its J kept in the thread's
// shared slice), then the stable barrier differences against the base where the trial is active or the base may be.
// pe, pd: per block, the barrier sum and the barrier difference sum.
__global__ void __launch_bounds__(CB) cell_trial_barrier_kernel(Q1Const q, const double *__restrict__ ua,
                                                                const double *__restrict__ ub,
                                                                const uint8_t *__restrict__ flags, dd *pe, dd *pd,
                                                                unsigned long long *bad,
                                                                uint8_t *__restrict__ trial_act,
                                                                const uint8_t *__restrict__ base_act) {
    extern __shared__ double smem[];
    __shared__ long long queue[CB / 32][64];
    double *dsl = smem + threadIdx.x;
    const int T = blockDim.x;
    dd acc[1] = {{0., 0.}}, dif[1] = {{0., 0.}};
    unsigned long long nbad = 0;
    for_flagged_cells(q, flags, queue[threadIdx.x >> 5], [&](long long c, uint8_t flag) {
        const long long n0 = cell_node0(c, q);
        const bool near_b = flag & 1;
        bool active = false;
        double sb = 0., sbd = 0.;
        if (near_b) {
            double E64[3][4][3];
            load_edges(ub, n0, q, E64);
            sweep<true>(E64, q, [&](int p, int, int, int, const double (&Vb)[3][3]) {
                const double jb = det_only(Vb);
                dsl[p * T] = jb;
                active |= jb < q.act;
                if (!(jb > q.delta)) { nbad++; return; }
                if (jb < q.act) {
                    double b, b1, b2;
                    barrier_eval(jb, q.act, q.delta, q.bw, b, b1, b2);
                    sb += b;
                }
            });
        }
        if (active || !base_act || base_act[c]) {
            if (flag & 2) {
                double E64[3][4][3];
                load_edges(ua, n0, q, E64);
                sweep<true>(E64, q, [&](int p, int, int, int, const double (&Va)[3][3]) {
                    // a trial J above the guard stands for "above the activation": min(J, a) is then a
                    const double ja = det_only(Va), jb = near_b ? dsl[p * T] : (double)q.act;
                    if (ja < q.act || jb < q.act) sbd += barrier_difference(ja, jb, q.act, q.delta);
                });
            } else if (active) {
                // the base is above the activation at every point: each difference is psi(jb) - psi(a)
                for (int p = 0; p < 27; p++) {
                    const double jb = dsl[p * T];
                    if (jb < q.act) sbd += barrier_difference((double)q.act, jb, q.act, q.delta);
                }
            }
        }
        if (trial_act && active) trial_act[c] = 1;
        acc[0] = dd_add_d(acc[0], sb);
        acc_add(dif[0], dd{q.bw * sbd, 0.});
    });
    dif[0] = two_sum(dif[0].hi, dif[0].lo);
    block_reduce_dd<1>(acc, pe);
    __syncthreads();     // the reductions share block_reduce_dd's shared array
    block_reduce_dd<1>(dif, pd);
    for (int o = 16; o; o >>= 1) nbad += __shfl_xor_sync(0xFFFFFFFFu, nbad, o);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad, nbad);
}

// ============================================================================================== node JD measure
// ext_act > 0 (T69/T73): cells whose closed27 Bernstein coefficients allow a value below min(m_c, ext_act) are
// appended to cand (order of arrival; each is then estimated independently, so the order does not matter).
__global__ void __launch_bounds__(CS) cell_min_jd_kernel(Q1Const q, const double *__restrict__ u,
                                                         double *__restrict__ m, double ext_act,
                                                         unsigned long long *__restrict__ ncand,
                                                         long long *__restrict__ cand) {
    extern __shared__ double smem[];
    double *J = smem + threadIdx.x;
    const int T = blockDim.x;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        double E[3][4][3];
        load_edges(u, cell_node0(c, q), q, E);
        double mn = __longlong_as_double(0x7FF0000000000000LL);
        sweep<true>(E, q, [&](int p, int, int, int, const double (&V)[3][3]) {
            double j = det_only(V);
            J[p * T] = j;
            mn = fmin(mn, j);
        });
        // exact interior minima of the edge quadratics through t = 0, 1/2, 1 (solvers/jd_affine.py:24)
#pragma unroll 1
        for (int e = 0; e < 12; e++) {
            int f0, st;
            if (e < 4) {            // x edges: iz, iy in {0, 2}
                f0 = 9 * ((e >> 1) * 2) + 3 * ((e & 1) * 2); st = 1;
            } else if (e < 8) {     // y edges: iz, ix in {0, 2}
                int k = e - 4;
                f0 = 9 * ((k >> 1) * 2) + (k & 1) * 2; st = 3;
            } else {                // z edges: iy, ix in {0, 2}
                int k = e - 8;
                f0 = 3 * ((k >> 1) * 2) + (k & 1) * 2; st = 9;
            }
            double j0 = J[f0 * T], j1 = J[(f0 + st) * T], j2 = J[(f0 + 2 * st) * T];
            double a = 2 * (j0 - 2 * j1 + j2);
            double b = -3 * j0 + 4 * j1 - j2;
            if (a > 0 && b < 0 && -b < 2 * a) mn = fmin(mn, j0 - b * b / (4 * a));
        }
        m[c] = mn;
        if (ext_act > 0.) {
            // closed27 values -> Bernstein coefficients in place: per axis x, y, z the middle entry becomes
            // 2 b - (a + c) / 2 (bernstein_barrier.py:26 to_bernstein)
#pragma unroll 1
            for (int axis = 0; axis < 3; axis++) {
                const int st = axis == 0 ? 1 : (axis == 1 ? 3 : 9);
#pragma unroll 1
                for (int l = 0; l < 9; l++) {
                    const int o = axis == 0 ? 3 * l : (axis == 1 ? (l / 3) * 9 + (l % 3) : l);
                    const double v0 = J[o * T], v1 = J[(o + st) * T], v2 = J[(o + 2 * st) * T];
                    J[(o + st) * T] = 2. * v1 - .5 * (v0 + v2);
                }
            }
            double bmin = J[0];
#pragma unroll 1
            for (int k = 1; k < 27; k++) bmin = fmin(bmin, J[k * T]);
            if (bmin < fmin(mn, ext_act)) cand[atomicAdd(ncand, 1ull)] = c;
        }
    }
}

// ---- T69/T73 face/interior estimate mu_c on candidate cells (solvers/jd_affine.py:45-150) ----
// J on a cell is triquadratic; mu_c = min of its values on the 9^3 grid {0, 1/8, .., 1}^3 and of a bounded Newton
// descent (30 iterations, halving backtracking <= 40, strict decrease only) from the 4 lowest grid points (stable
// order).  A value J attains, so an estimate for the metric, never a bound.  One warp per candidate cell.
struct Tri {
    double c[27];    // monomial coefficients C[k][j][i] of z^k y^j x^i
};
// NumPy's add-reduce order for a contiguous length-27 axis (eight accumulators; jd_affine_compiled.py:_sum27)
__device__ __forceinline__ double sum27(const double *a) {
    double r[8];
#pragma unroll
    for (int i = 0; i < 8; i++) r[i] = a[i];
#pragma unroll
    for (int b = 8; b < 24; b += 8)
#pragma unroll
        for (int i = 0; i < 8; i++) r[i] += a[b + i];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    res += a[24];
    res += a[25];
    res += a[26];
    return 0.0 + res;
}
// sum C[k][j][i] (Z_k Y_j) X_i
__device__ __forceinline__ double tri_e(const Tri &T, const double Z[3], const double Y[3], const double X[3]) {
    double tmp[27];
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double zy = Z[k] * Y[j];
#pragma unroll
            for (int i = 0; i < 3; i++) tmp[9 * k + 3 * j + i] = T.c[9 * k + 3 * j + i] * (zy * X[i]);
        }
    return sum27(tmp);
}
__device__ __forceinline__ void tri_powers(double t, double P[3][3]) {
    P[0][0] = 1.; P[0][1] = t; P[0][2] = t * t;
    P[1][0] = 0.; P[1][1] = 1.; P[1][2] = 2. * t;
    P[2][0] = 0.; P[2][1] = 0.; P[2][2] = 2.;
}
__device__ __forceinline__ double tri_value(const Tri &T, const double x[3]) {
    double px[3][3], py[3][3], pz[3][3];
    tri_powers(x[0], px); tri_powers(x[1], py); tri_powers(x[2], pz);
    return tri_e(T, pz[0], py[0], px[0]);
}
__device__ __forceinline__ double clip01(double v) {
    if (v != v) return v;
    const double w = v > 0. ? v : 0.;
    return w < 1. ? w : 1.;
}
// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations: A = Q diag(w) Q^T (columns of Q).
__device__ void sym3_eigen(double A[3][3], double w[3], double Q[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) Q[i][j] = i == j ? 1. : 0.;
#pragma unroll 1
    for (int sweep = 0; sweep < 64; sweep++) {
        const double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
        const double dia = fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]);
        if (off == 0. || off <= 1e-300 + 1e-18 * dia) break;
#pragma unroll 1
        for (int pq = 0; pq < 3; pq++) {
            const int p = pq == 2 ? 1 : 0, qq = pq == 0 ? 1 : 2;
            const double apq = A[p][qq];
            if (apq == 0.) continue;
            // rotation zeroing A[p][q] (symmetric Schur decomposition of the 2x2 block)
            const double tau = (A[qq][qq] - A[p][p]) / (2. * apq);
            const double t = (tau >= 0. ? 1. : -1.) / (fabs(tau) + sqrt(1. + tau * tau));
            const double cs = 1. / sqrt(1. + t * t), sn = t * cs;
#pragma unroll
            for (int k = 0; k < 3; k++) {     // A <- A J
                const double akp = A[k][p], akq = A[k][qq];
                A[k][p] = cs * akp - sn * akq;
                A[k][qq] = sn * akp + cs * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {     // A <- J^T A
                const double apk = A[p][k], aqk = A[qq][k];
                A[p][k] = cs * apk - sn * aqk;
                A[qq][k] = sn * apk + cs * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {     // Q <- Q J
                const double qkp = Q[k][p], qkq = Q[k][qq];
                Q[k][p] = cs * qkp - sn * qkq;
                Q[k][qq] = sn * qkp + cs * qkq;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) w[i] = A[i][i];
}
// jd_affine.py:_bounded_newton for one start; returns the lowest value reached
__device__ double bounded_newton(const Tri &T, double x[3], double best) {
#pragma unroll 1
    for (int it = 0; it < 30; it++) {
        double px[3][3], py[3][3], pz[3][3];
        tri_powers(x[0], px); tri_powers(x[1], py); tri_powers(x[2], pz);
        double g[3], H[3][3];
        g[0] = tri_e(T, pz[0], py[0], px[1]);
        g[1] = tri_e(T, pz[0], py[1], px[0]);
        g[2] = tri_e(T, pz[1], py[0], px[0]);
        H[0][0] = tri_e(T, pz[0], py[0], px[2]);
        H[1][1] = tri_e(T, pz[0], py[2], px[0]);
        H[2][2] = tri_e(T, pz[2], py[0], px[0]);
        H[0][1] = H[1][0] = tri_e(T, pz[0], py[1], px[1]);
        H[0][2] = H[2][0] = tri_e(T, pz[1], py[0], px[1]);
        H[1][2] = H[2][1] = tri_e(T, pz[1], py[1], px[0]);
        bool free_[3];
        double gf[3], Hf[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            free_[a] = !((x[a] <= 0. && g[a] > 0.) || (x[a] >= 1. && g[a] < 0.));
            gf[a] = free_[a] ? g[a] : 0.;
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++)
                Hf[a][b] = (free_[a] && free_[b]) ? H[a][b] : (a == b && !free_[a] ? 1. : 0.);
        double w[3], Q[3][3];
        sym3_eigen(Hf, w, Q);
        const double scale = fmax(1., fmax(fabs(w[0]), fmax(fabs(w[1]), fabs(w[2]))));
        const bool ok = w[0] > 1e-12 * scale && w[1] > 1e-12 * scale && w[2] > 1e-12 * scale;
        double d[3];
        if (ok) {
            double proj[3];
#pragma unroll
            for (int j = 0; j < 3; j++) proj[j] = (Q[0][j] * gf[0] + Q[1][j] * gf[1] + Q[2][j] * gf[2]) / w[j];
#pragma unroll
            for (int i = 0; i < 3; i++) d[i] = -(Q[i][0] * proj[0] + Q[i][1] * proj[1] + Q[i][2] * proj[2]);
        } else {
#pragma unroll
            for (int i = 0; i < 3; i++) d[i] = -gf[i] / scale;
        }
        double step = 1.;
        bool done = false;
#pragma unroll 1
        for (int bt = 0; bt < 40; bt++) {
            double xt[3];
#pragma unroll
            for (int a = 0; a < 3; a++) xt[a] = clip01(x[a] + step * d[a]);
            const double ft = tri_value(T, xt);
            if (ft < best) {
                x[0] = xt[0]; x[1] = xt[1]; x[2] = xt[2];
                best = ft;
                done = true;
                break;
            }
            step = .5 * step;
        }
        if (!done) break;       // no strict decrease: converged to rounding (or stuck)
    }
    return best;
}

__device__ __forceinline__ double lagrange3(int a, double t) {
    return a == 0 ? 2. * (t - .5) * (t - 1.) : (a == 1 ? -4. * t * (t - 1.) : 2. * t * (t - .5));
}
// (value, index) lexicographic order: the stable ascending sort of the grid values (NaN last)
__device__ __forceinline__ bool vi_less(double v, int i, double w, int j) {
    if (v < w) return true;
    if (w != w && v == v) return true;
    if (v == w || (v != v && w != w)) return i < j;
    return false;
}

__global__ void __launch_bounds__(128) jd_extension_kernel(Q1Const q, const double *__restrict__ u,
                                                           const unsigned long long *__restrict__ ncand,
                                                           const long long *__restrict__ cand,
                                                           double *__restrict__ m) {
    __shared__ double sJ[4][27];
    __shared__ Tri sT[4];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long n = (long long)*ncand;
    for (long long w = blockIdx.x * 4LL + wib; w < n; w += (long long)gridDim.x * 4) {
        const long long c = cand[w];
        double E[3][4][3];
        load_edges(u, cell_node0(c, q), q, E);
        if (lane == 0)
            sweep<true>(E, q, [&](int p, int, int, int, const double (&V)[3][3]) { sJ[wib][p] = det_only(V); });
        __syncwarp();
        // monomial coefficients C[k][j][i] = sum_cba J[c][b][a] M[c][k] M[b][j] M[a][i], M the Lagrange-to-power map
        if (lane < 27) {
            const double M[3][3] = {{1., -3., 2.}, {0., 4., -4.}, {0., -1., 2.}};
            const int k = lane / 9, j = (lane / 3) % 3, i = lane % 3;
            double acc = 0.;
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
#pragma unroll
                for (int b = 0; b < 3; b++)
#pragma unroll
                    for (int a = 0; a < 3; a++)
                        acc += sJ[wib][9 * cc + 3 * b + a] * (M[cc][k] * (M[b][j] * M[a][i]));
            sT[wib].c[lane] = acc;
        }
        __syncwarp();
        // 9^3 grid values (z-major, x fastest), each lane keeping its 4 lowest in stable order
        double tv[4];
        int ti[4];
#pragma unroll
        for (int r = 0; r < 4; r++) { tv[r] = __longlong_as_double(0x7FF8000000000000LL); ti[r] = 0x7FFFFFFF; }
        for (int pnt = lane; pnt < 729; pnt += 32) {
            const int ix = pnt % 9, iy = (pnt / 9) % 9, iz = pnt / 81;
            const double tx = .125 * ix, ty = .125 * iy, tz = .125 * iz;
            double val = 0.;
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
#pragma unroll
                for (int b = 0; b < 3; b++)
#pragma unroll
                    for (int a = 0; a < 3; a++)
                        val += sJ[wib][9 * cc + 3 * b + a] * (lagrange3(cc, tz) * (lagrange3(b, ty) * lagrange3(a, tx)));
            if (vi_less(val, pnt, tv[3], ti[3])) {
                int pos = 3;
                while (pos > 0 && vi_less(val, pnt, tv[pos - 1], ti[pos - 1])) {
                    tv[pos] = tv[pos - 1]; ti[pos] = ti[pos - 1];
                    pos--;
                }
                tv[pos] = val; ti[pos] = pnt;
            }
        }
        // butterfly merge of the lanes' sorted lists
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            double ov[4];
            int oi[4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                ov[r] = __shfl_xor_sync(0xFFFFFFFFu, tv[r], o);
                oi[r] = __shfl_xor_sync(0xFFFFFFFFu, ti[r], o);
            }
            double nv[4];
            int ni[4];
            int a = 0, b = 0;
#pragma unroll
            for (int r = 0; r < 4; r++) {
                if (vi_less(tv[a], ti[a], ov[b], oi[b])) { nv[r] = tv[a]; ni[r] = ti[a]; a++; }
                else { nv[r] = ov[b]; ni[r] = oi[b]; b++; }
            }
#pragma unroll
            for (int r = 0; r < 4; r++) { tv[r] = nv[r]; ti[r] = ni[r]; }
        }
        // bounded Newton from the 4 lowest grid points, lanes 0..3
        double found = __longlong_as_double(0x7FF0000000000000LL);
        if (lane < 4) {
            const int s0 = lane == 0 ? ti[0] : (lane == 1 ? ti[1] : (lane == 2 ? ti[2] : ti[3]));
            double x[3] = {.125 * (s0 % 9), .125 * ((s0 / 9) % 9), .125 * (s0 / 81)};
            found = bounded_newton(sT[wib], x, tri_value(sT[wib], x));
        }
#pragma unroll
        for (int o = 2; o; o >>= 1) found = fmin(found, __shfl_xor_sync(0xFFFFFFFFu, found, o));
        if (lane == 0) {
            const double mu = fmin(tv[0], found);       // grid minimum and the Newton descents
            const double mc = m[c];
            m[c] = (mu < mc || mu != mu) ? mu : mc;     // np.minimum
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(256) node_min_kernel(Q1Const q, const double *__restrict__ m,
                                                       double *__restrict__ node) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nnode;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.nx, q.ny, x, y, z);
        double mn = __longlong_as_double(0x7FF0000000000000LL);
#pragma unroll
        for (int a = 0; a < 8; a++) {
            long long cz = z - (a >> 2), cy = y - ((a >> 1) & 1), cx = x - (a & 1);
            if (cz < 0 || cy < 0 || cx < 0 || cz >= q.cz || cy >= q.cy || cx >= q.cx) continue;
            mn = fmin(mn, m[(cz * q.cy + cy) * q.cx + cx]);
        }
        node[i] = mn;
    }
}

// ============================================================================================== global JD root
// solvers/global_jd_step.py:52 first_roots for one point (b0 > 0), normalized s in (0, 1]; +inf if none
__device__ double first_root(double b0, double b1, double b2, double b3) {
    const double INF = __longlong_as_double(0x7FF0000000000000LL);
    if (b0 > fabs(b1) + fabs(b2) + fabs(b3)) return INF;
    const double nan = __longlong_as_double(0x7FF8000000000000LL);
    double a = 3 * b3, b = 2 * b2, c = b1;
    bool linear = a == 0;
    double r_lin = (linear && b != 0) ? -c / b : nan;
    double disc = b * b - 4 * a * c;
    double sq = sqrt(disc >= 0 ? disc : 0.);
    double qq = -(b + (b >= 0 ? sq : -sq)) / 2;
    double r1 = (!linear && disc >= 0 && a != 0) ? qq / a : nan;
    double r2 = (!linear && disc >= 0 && qq != 0) ? c / qq : nan;
    if (linear) { r1 = r_lin; r2 = nan; }
    r1 = (r1 > 0 && r1 < 1) ? r1 : 1.;
    r2 = (r2 > 0 && r2 < 1) ? r2 : 1.;
    double t1 = fmin(r1, r2), t2 = fmax(r1, r2);
    auto qv = [&](double s) { return b0 + s * (b1 + s * (b2 + s * b3)); };
    const double eps4 = 4 * 2.220446049250313e-16;
    auto touch = [&](double s) { return eps4 * (fabs(b0) + s * (fabs(b1) + s * (fabs(b2) + s * fabs(b3)))); };
    double lo, hi;
    if (qv(t1) <= touch(t1)) { lo = 0.; hi = t1; }
    else if (qv(t2) <= touch(t2)) { lo = t1; hi = t2; }
    else if (qv(1.) <= 0) { lo = t2; hi = 1.; }
    else return INF;
    for (int k = 0; k < 50; k++) {
        double mid = .5 * (lo + hi);
        if (qv(mid) <= 0) hi = mid;
        else lo = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(CT) jd_root_kernel(Q1Const q, const double *__restrict__ u,
                                                     const double *__restrict__ pv, double limit,
                                                     long long *__restrict__ best_key,
                                                     unsigned long long *__restrict__ invalid) {
    long long key = kKeyPosInf;
    unsigned long long nbad = 0;
    const double L2 = limit * limit, L3 = limit * limit * limit;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < q.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        long long n0 = cell_node0(c, q);
        double E[3][4][3], Ep[3][4][3];
        load_edges(u, n0, q, E);
        load_edges(pv, n0, q, Ep);
        sweep2<true>(E, Ep, q, [&](int, int, int, int, const double (&V)[3][3], const double (&W)[3][3]) {
            double AF[3][3], AV[3][3], J, JV;
            cofactor_det(V, AF, J);
#pragma unroll
            for (int r = 0; r < 3; r++) {
                int j = (r + 1) % 3, k = (r + 2) % 3;
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    int l = (cc + 1) % 3, mm = (cc + 2) % 3;
                    AV[r][cc] = W[j][l] * W[k][mm] - W[j][mm] * W[k][l];
                }
            }
            JV = (W[0][0] * AV[0][0] + W[0][1] * AV[0][1]) + W[0][2] * AV[0][2];
            double c0 = J - q.delta, c1 = 0., c2 = 0.;
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    c1 += AF[r][cc] * W[r][cc];
                    c2 += (V[r][cc] + (r == cc ? 1. : 0.)) * AV[r][cc];
                }
            if (!(c0 > 0)) { nbad++; return; }
            double s = first_root(c0, c1 * limit, c2 * L2, JV * L3);
            long long k = order_key(s);
            key = k < key ? k : key;
        });
    }
    for (int o = 16; o; o >>= 1) {
        long long y = __shfl_xor_sync(0xFFFFFFFFu, key, o);
        key = y < key ? y : key;
        nbad += __shfl_xor_sync(0xFFFFFFFFu, nbad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(best_key, key);
        if (nbad) atomicAdd(invalid, nbad);
    }
}

// ============================================================================================== PG metric pieces
__global__ void __launch_bounds__(256) shift_kernel(Q1Const q, const double *__restrict__ image_grad, dd *partial) {
    dd acc[1] = {{0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nfree;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.fx, q.fy, x, y, z);
        x++; y++; z++;
        const double *b = image_grad + 3 * ((z * q.ny + y) * q.nx + x);
        double qo = node_weight(x, y, z, q) / q.omega;
        acc[0] = dd_add_d(acc[0], qo * ((b[0] * b[0] + b[1] * b[1]) + b[2] * b[2]));
    }
    block_reduce_dd<1>(acc, partial);
}

__global__ void __launch_bounds__(256) pg_scale_kernel(Q1Const q, const double *__restrict__ diag,
                                                       const double *__restrict__ node, double sm, double act,
                                                       double floor_, double *__restrict__ scale,
                                                       unsigned long long *bad) {
    unsigned long long nb = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < q.nfree;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, q.fx, q.fy, x, y, z);
        x++; y++; z++;
        double ja = node[(z * q.ny + y) * q.nx + x];
        double r = fmin(1., fmax(ja, floor_) / act);
        if (!(ja == ja) || !(ja < INFINITY) || !(ja > -INFINITY)) nb++;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double d = diag[c * q.nfree + i];
            double s = (sm / sqrt(d)) * r;
            if (!(d > 0) || !(s > 0) || !(s < INFINITY)) nb++;
            scale[c * q.nfree + i] = s;
        }
    }
    for (int o = 16; o; o >>= 1) nb += __shfl_xor_sync(0xFFFFFFFFu, nb, o);
    if ((threadIdx.x & 31) == 0 && nb) atomicAdd(bad, nb);
}

// ============================================================================================== final reduction
__global__ void final_reduce_kernel(const dd *__restrict__ partial, long long blocks, int K, double *out) {
    // one block; thread t reduces blocks t, t + 256, ... in order, then a fixed tree
    __shared__ dd sh[256];
    for (int k = 0; k < K; k++) {
        dd acc = {0., 0.};
        for (long long b = threadIdx.x; b < blocks; b += blockDim.x) acc = dd_add(acc, partial[b * K + k]);
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s; s >>= 1) {
            if ((int)threadIdx.x < s) sh[threadIdx.x] = dd_add(sh[threadIdx.x], sh[threadIdx.x + s]);
            __syncthreads();
        }
        if (threadIdx.x == 0) { out[2 * k] = sh[0].hi; out[2 * k + 1] = sh[0].lo; }
        __syncthreads();
    }
}

SplineRef spline_ref(const svp_pair *p) {
    SplineRef S;
    S.c = p->coeff;
    for (int k = 0; k < 3; k++) {
        S.t[k] = p->knots[k];
        S.rcp[k] = p->spline_rcp[k];
        S.x0[k] = p->q.x0[k];
        S.ih[k] = 1. / p->q.h[k];
    }
    S.n[0] = p->q.nx; S.n[1] = p->q.ny; S.n[2] = p->q.nz;
    return S;
}

unsigned cell_blocks(const svp_pair *p) { return blocks_for(p->q.ncell, CT, CELL_PER_SM); }
unsigned slice_blocks(const svp_pair *p) { return blocks_for(p->q.ncell, CS, 2 * CELL_PER_SM); }
// dynamic shared memory of the slice kernels: k doubles per thread
constexpr size_t slice_bytes(int k) { return sizeof(double) * (size_t)k * CS; }
int allow_slices() {
    // the 108-value slices are above the 48 KB default.  The attribute belongs to the device's context (the primary
    // context torch and this library share), so it is set on the first call per device, not on every launch: a
    // cudaFuncSetAttribute costs host time that the GPU then spends idle.
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    SVP_CUDA(cudaGetDevice(&dev));
    SVP_REQUIRE(dev >= 0 && dev < 64, "allow_slices: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return SVP_OK;
    SVP_CUDA(cudaFuncSetAttribute(cell_diff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)slice_bytes(108)));
    SVP_CUDA(cudaFuncSetAttribute(cell_energy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)slice_bytes(108)));
    SVP_CUDA(cudaFuncSetAttribute(cell_trial_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)slice_bytes(108)));
    SVP_CUDA(cudaFuncSetAttribute(cell_grad_barrier_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * 81 * CB)));
    done[dev] = true;
    return SVP_OK;
}
unsigned node_blocks(long long n) { return blocks_for(n, 256, 8); }

}  // namespace

int pair_partials(svp_pair *p, long long blocks, int k) {
    long long need = blocks * k;
    if (need <= p->partial_cap) return SVP_OK;
    cudaFree(p->partial);
    p->partial = nullptr;
    p->partial_cap = 0;
    SVP_CUDA(cudaMalloc((void **)&p->partial, sizeof(dd) * need));
    p->partial_cap = need;
    return SVP_OK;
}

int pair_locals(svp_pair *p, int n) {
    size_t bytes = sizeof(double) * 24 * (size_t)p->q.ncell;
    if (n >= 1 && !p->loc1) SVP_CUDA(cudaMalloc((void **)&p->loc1, bytes));
    if (n >= 2 && !p->loc2) SVP_CUDA(cudaMalloc((void **)&p->loc2, bytes));
    return SVP_OK;
}

int pair_flags(svp_pair *p) {
    if (!p->flags) SVP_CUDA(cudaMalloc((void **)&p->flags, (size_t)p->q.ncell));
    return SVP_OK;
}

}  // namespace svp

using namespace svp;

extern "C" int svp_pair_set_precision(svp_pair *p, int32_t precision) {
    SVP_REQUIRE(p && (precision == SVP_PRECISION_PLAIN || precision == SVP_PRECISION_MIXED),
                "svp_pair_set_precision: SVP_PRECISION_PLAIN or SVP_PRECISION_MIXED");
    p->precision = precision;
    return SVP_OK;
}

extern "C" int svp_warp(const svp_pair *p, const double *u, double *warped, double *image_grad, void *stream) {
    SVP_REQUIRE(p && u && warped, "svp_warp: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    SplineRef S = spline_ref(p);
    unsigned nb = node_blocks(p->q.nnode);
    if (image_grad)
        { svp::KernelTimer _t("warp_kernel_grad", s); SVP_LAUNCH(warp_kernel<true><<<nb, 256, 0, s>>>(p->q, S, u, p->fixed, p->u_ref, warped, image_grad, nullptr)); }
    else
        { svp::KernelTimer _t("warp_kernel", s); SVP_LAUNCH(warp_kernel<false><<<nb, 256, 0, s>>>(p->q, S, u, p->fixed, p->u_ref, warped, nullptr, nullptr)); }
    SVP_LAUNCH_CHECK("warp_kernel");
    return SVP_OK;
}

extern "C" int svp_sample_points(const svp_pair *p, const double *points, int64_t n, double *value,
                                 double *gradient, void *stream) {
    SVP_REQUIRE(p && n >= 0, "svp_sample_points: invalid arguments");
    if (!n) return SVP_OK;
    SVP_REQUIRE(points && value, "svp_sample_points: null pointer");
    SVP_LAUNCH(sample_points_kernel<<<node_blocks(n), 256, 0, (cudaStream_t)stream>>>(spline_ref(p), points, n, value,
                                                                           gradient));
    SVP_LAUNCH_CHECK("sample_points_kernel");
    return SVP_OK;
}

extern "C" int svp_energy(svp_pair *p, const double *u, const double *warped, double *terms5,
                          int64_t *barrier_violations, void *stream) {
    SVP_REQUIRE(p && u && warped && terms5, "svp_energy: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = node_blocks(p->q.nnode), cb = slice_blocks(p);
    int rc = pair_partials(p, (long long)nb * 2 + (long long)cb * 3, 1);
    if (rc) return rc;
    if ((rc = allow_slices())) return rc;
    SVP_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(long long) * 8, s));
    { svp::KernelTimer _t("node_energy_kernel", s); SVP_LAUNCH(node_energy_kernel<<<nb, 256, 0, s>>>(p->q, u, warped, p->fixed, p->u_ref, p->partial)); }
    SVP_LAUNCH_CHECK("node_energy_kernel");
    dd *pc = p->partial + (long long)nb * 2;
    { svp::KernelTimer _t("cell_energy_kernel", s); SVP_LAUNCH(cell_energy_kernel<<<cb, CS, slice_bytes(108), s>>>(p->q, u, p->u_ref, pc, (unsigned long long *)p->counter)); }
    SVP_LAUNCH_CHECK("cell_energy_kernel");
    double node2[2], cell3[3];
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(p->partial, nb, 2, p->result));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pc, cb, 3, p->result + 4));
    SVP_LAUNCH_CHECK("final_reduce_kernel");
    double tmp[10];
    long long bad = 0;
    SVP_CUDA(cudaMemcpyAsync(tmp, p->result, sizeof tmp, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaMemcpyAsync(&bad, p->counter, sizeof bad, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < 2; k++) node2[k] = tmp[2 * k] + tmp[2 * k + 1];
    for (int k = 0; k < 3; k++) cell3[k] = tmp[4 + 2 * k] + tmp[4 + 2 * k + 1];
    terms5[0] = .5 * node2[0];
    terms5[1] = .5 * p->q.lam * node2[1];
    terms5[2] = .5 * p->q.mu * cell3[0];
    terms5[3] = .5 * p->q.nu * cell3[1];
    terms5[4] = cell3[2];
    if (barrier_violations) *barrier_violations = bad;
    return SVP_OK;
}

extern "C" int svp_energy_difference_masked(svp_pair *p, const double *base_u, const double *base_warped,
                                            const double *trial_u, const double *trial_warped,
                                            const uint8_t *base_active, const uint8_t *trial_active, double *diff2,
                                            void *stream) {
    SVP_REQUIRE(p && base_u && base_warped && trial_u && trial_warped && diff2, "svp_energy_difference: null");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = node_blocks(p->q.nnode), cb = slice_blocks(p), bb = barrier_blocks(p->q);
    int rc = pair_partials(p, (long long)nb * 2 + (long long)cb * 3 + bb, 1);
    if (rc) return rc;
    rc = allow_slices();
    if (rc) return rc;
    // with both states' masks, the barrier differences of the cells active in either run in cell_trial_diff_kernel
    // over those cells alone (per cell the same value)
    const bool apart = base_active && trial_active;
    if (apart && (rc = pair_flags(p))) return rc;
    { svp::KernelTimer _t("node_diff_kernel", s); SVP_LAUNCH(node_diff_kernel<<<nb, 256, 0, s>>>(p->q, base_u, base_warped, trial_u, trial_warped, p->fixed, p->u_ref,
                                        p->partial)); }
    dd *pc = p->partial + (long long)nb * 2, *pb = pc + (long long)cb * 3;
    {
        svp::KernelTimer _t("cell_diff_kernel", s);
        SVP_LAUNCH(cell_diff_kernel<<<cb, CS, slice_bytes(108), s>>>(p->q, base_u, trial_u, p->u_ref, pc, base_active,
                                                                    trial_active, apart ? p->flags : nullptr));
    }
    if (apart) {
        svp::KernelTimer _t("cell_trial_diff_kernel", s);
        SVP_LAUNCH(cell_trial_diff_kernel<<<bb, CB, sizeof(double) * 27 * CB, s>>>(p->q, base_u, trial_u, p->flags,
                                                                                 pb));
    }
    SVP_LAUNCH_CHECK("difference kernels");
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(p->partial, nb, 2, p->result));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pc, cb, 3, p->result + 4));
    if (apart) SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pb, bb, 1, p->result + 8));
    SVP_LAUNCH_CHECK("final_reduce_kernel");
    double tmp[10];
    SVP_CUDA(cudaMemcpyAsync(tmp, p->result, sizeof tmp, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    // E = image + proximity + jd + curl + barrier; F = image + barrier (sums of double-double pieces)
    double img = tmp[0] + tmp[1], prox = tmp[2] + tmp[3];
    double jd = tmp[4] + tmp[5], curl = tmp[6] + tmp[7], bar = tmp[8] + tmp[9];
    diff2[0] = (((img + prox) + jd) + curl) + bar;
    diff2[1] = img + bar;
    return SVP_OK;
}

extern "C" int svp_energy_difference(svp_pair *p, const double *base_u, const double *base_warped,
                                     const double *trial_u, const double *trial_warped, double *diff2,
                                     void *stream) {
    return svp_energy_difference_masked(p, base_u, base_warped, trial_u, trial_warped, nullptr, nullptr, diff2,
                                        stream);
}

// Absolute error estimates of float32 quantities in the screened trial, in units of the float32 unit roundoff
// 2^-24: a Gauss-point J of I + V and its reference J (cofactor products and a 3-term dot product of entries of size
// up to ~2, both rounded), a curl component (one rounded difference of each field's derivatives); and the relative
// rounding of the squared-residual sums.
constexpr double kScreenJ = 256., kScreenCurl = 32., kScreenSum = 64.;

// |error of the E difference| <= mu dJ sum w (|ra| + |rb|) + nu dC sum w (|xa| + |xb|) + 2 dS (soft_a + soft_b): the
// residuals' absolute errors times the summed residual magnitudes, plus the rounding of the squares.  sums: the
// trial's JD and curl sums (unweighted by mu/2, nu/2), then the four pb sums of cell_trial32_kernel.
static double screen_band(const svp_pair *p, const double sums[6]) {
    const double u32 = std::ldexp(1., -24);
    const double soft = .5 * p->q.mu * (sums[0] + sums[4]) + .5 * p->q.nu * (sums[1] + sums[5]);
    return p->q.mu * kScreenJ * u32 * sums[2] + p->q.nu * kScreenCurl * u32 * sums[3] + 2. * kScreenSum * u32 * soft;
}

// The mixed form's screened E/F difference of two evaluated states: node terms float64 (node_diff_kernel), the JD and
// curl penalty differences float32 (cell_trial32_kernel, with the error band), the barrier differences float64 over
// the flagged cells; F (image + barrier) is float64 throughout.
extern "C" int svp_energy_difference_screened(svp_pair *p, const double *base_u, const double *base_warped,
                                              const double *trial_u, const double *trial_warped,
                                              const uint8_t *base_active, double *diff2, double *band,
                                              void *stream) {
    SVP_REQUIRE(p && base_u && base_warped && trial_u && trial_warped && diff2 && band,
                "svp_energy_difference_screened: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = node_blocks(p->q.nnode), cb = slice_blocks(p), bb = barrier_blocks(p->q);
    int rc = pair_partials(p, (long long)nb * 2 + (long long)cb * 8 + (long long)bb * 2, 1);
    if (rc) return rc;
    if ((rc = allow_slices())) return rc;
    if ((rc = pair_flags(p))) return rc;
    SVP_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(long long) * 8, s));
    dd *pn = p->partial, *pce = pn + (long long)nb * 2, *pcd = pce + (long long)cb * 2, *pcb = pcd + (long long)cb * 2;
    dd *pbe = pcb + (long long)cb * 4, *pbd = pbe + bb;
    {
        svp::KernelTimer _t("node_diff_kernel", s);
        SVP_LAUNCH(node_diff_kernel<<<nb, 256, 0, s>>>(p->q, base_u, base_warped, trial_u, trial_warped, p->fixed,
                                                       p->u_ref, pn));
    }
    {
        svp::KernelTimer _t("cell_trial32_kernel", s);
        SVP_LAUNCH(cell_trial32_kernel<<<cb, CS, sizeof(float) * 108 * CS, s>>>(
            p->q, base_u, trial_u, p->u_ref, pce, pcd, pcb, p->flags, nullptr, base_active));
    }
    {
        svp::KernelTimer _t("cell_trial_barrier_kernel", s);
        SVP_LAUNCH(cell_trial_barrier_kernel<<<bb, CB, sizeof(double) * 27 * CB, s>>>(
            p->q, base_u, trial_u, p->flags, pbe, pbd, (unsigned long long *)p->counter, nullptr, base_active));
    }
    SVP_LAUNCH_CHECK("screened difference kernels");
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pn, nb, 2, p->result));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pcd, cb, 2, p->result + 4));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pbd, bb, 1, p->result + 8));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pce, cb, 2, p->result + 10));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pcb, cb, 4, p->result + 14));
    SVP_LAUNCH_CHECK("final_reduce_kernel");
    double tmp[22];
    SVP_CUDA(cudaMemcpyAsync(tmp, p->result, sizeof tmp, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    // E = image + proximity + jd + curl + barrier; F = image + barrier, as svp_energy_difference combines them
    double img = tmp[0] + tmp[1], prox = tmp[2] + tmp[3];
    double jd = tmp[4] + tmp[5], curl = tmp[6] + tmp[7], bar = tmp[8] + tmp[9];
    diff2[0] = (((img + prox) + jd) + curl) + bar;
    diff2[1] = img + bar;
    double sums[6];
    for (int k = 0; k < 6; k++) sums[k] = tmp[10 + 2 * k] + tmp[11 + 2 * k];
    *band = screen_band(p, sums);
    return SVP_OK;
}

static int trial_energy(svp_pair *p, const double *base_u, const double *base_warped, const double *trial_u,
                        double *trial_warped, double *trial_image_grad, const uint8_t *base_active,
                        uint8_t *trial_active, double *terms5, double *diff2, int64_t *barrier_violations,
                        bool screened, double *band, void *stream) {
    SVP_REQUIRE(p && base_u && base_warped && trial_u && trial_warped && terms5 && diff2,
                "svp_trial_energy: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = node_blocks(p->q.nnode), cb = slice_blocks(p), bb = barrier_blocks(p->q);
    int rc = pair_partials(p, (long long)nb * 4 + (long long)cb * 10 + (long long)bb * 2, 1);
    if (rc) return rc;
    if ((rc = allow_slices())) return rc;
    if (screened && (rc = pair_flags(p))) return rc;
    SVP_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(long long) * 8, s));
    dd *pne = p->partial, *pnd = pne + (long long)nb * 2, *pce = pnd + (long long)nb * 2, *pcd = pce + (long long)cb * 3;
    dd *pcb = pcd + (long long)cb * 3, *pbe = pcb + (long long)cb * 4, *pbd = pbe + bb;
    SplineRef S = spline_ref(p);
    if (trial_image_grad) {
        svp::KernelTimer _t("warp_trial_kernel_grad", s);
        SVP_LAUNCH(warp_trial_kernel<true><<<nb, 256, 0, s>>>(p->q, S, base_u, base_warped, trial_u, p->fixed,
                                                                p->u_ref, trial_warped, trial_image_grad, pne, pnd));
    } else {
        svp::KernelTimer _t("warp_trial_kernel", s);
        SVP_LAUNCH(warp_trial_kernel<false><<<nb, 256, 0, s>>>(p->q, S, base_u, base_warped, trial_u, p->fixed,
                                                                 p->u_ref, trial_warped, nullptr, pne, pnd));
    }
    SVP_LAUNCH_CHECK("warp_trial_kernel");
    if (screened) {
        {
            svp::KernelTimer _t("cell_trial32_kernel", s);
            SVP_LAUNCH(cell_trial32_kernel<<<cb, CS, sizeof(float) * 108 * CS, s>>>(
                p->q, base_u, trial_u, p->u_ref, pce, pcd, pcb, p->flags, trial_active, base_active));
        }
        svp::KernelTimer _t("cell_trial_barrier_kernel", s);
        SVP_LAUNCH(cell_trial_barrier_kernel<<<bb, CB, sizeof(double) * 27 * CB, s>>>(
            p->q, base_u, trial_u, p->flags, pbe, pbd, (unsigned long long *)p->counter, trial_active, base_active));
    } else {
        // with the base's mask, the barrier differences of the cells where the trial or the base is active run in
        // cell_trial_diff_kernel over those cells alone (per cell the fused kernel's values)
        const bool apart = base_active != nullptr;
        if (apart && (rc = pair_flags(p))) return rc;
        {
            svp::KernelTimer _t("cell_trial_kernel", s);
            SVP_LAUNCH(cell_trial_kernel<<<cb, CS, slice_bytes(108), s>>>(
                p->q, base_u, trial_u, p->u_ref, pce, pcd, (unsigned long long *)p->counter, trial_active,
                base_active, apart ? p->flags : nullptr));
        }
        if (apart) {
            svp::KernelTimer _t("cell_trial_diff_kernel", s);
            SVP_LAUNCH(cell_trial_diff_kernel<<<bb, CB, sizeof(double) * 27 * CB, s>>>(p->q, base_u, trial_u,
                                                                                     p->flags, pbd));
        }
    }
    SVP_LAUNCH_CHECK("cell_trial_kernel");
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pne, nb, 2, p->result));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pnd, nb, 2, p->result + 10));
    if (screened) {
        // soft sums and differences from the float32 kernel, the barrier's from the float64 barrier kernel
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pce, cb, 2, p->result + 4));
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pbe, bb, 1, p->result + 8));
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pcd, cb, 2, p->result + 14));
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pbd, bb, 1, p->result + 18));
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pcb, cb, 4, p->result + 20));
    } else {
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pce, cb, 3, p->result + 4));
        SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pcd, cb, 3, p->result + 14));
        // the barrier difference from its own kernel in place of the fused kernel's (zero) one
        if (base_active) SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(pbd, bb, 1, p->result + 18));
    }
    SVP_LAUNCH_CHECK("final_reduce_kernel");
    double tmp[28];
    long long bad = 0;
    SVP_CUDA(cudaMemcpyAsync(tmp, p->result, sizeof(double) * (screened ? 28 : 20), cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaMemcpyAsync(&bad, p->counter, sizeof bad, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    // energy terms exactly as svp_energy
    double node2[2], cell3[3];
    for (int k = 0; k < 2; k++) node2[k] = tmp[2 * k] + tmp[2 * k + 1];
    for (int k = 0; k < 3; k++) cell3[k] = tmp[4 + 2 * k] + tmp[4 + 2 * k + 1];
    terms5[0] = .5 * node2[0];
    terms5[1] = .5 * p->q.lam * node2[1];
    terms5[2] = .5 * p->q.mu * cell3[0];
    terms5[3] = .5 * p->q.nu * cell3[1];
    terms5[4] = cell3[2];
    if (barrier_violations) *barrier_violations = bad;
    // differences exactly as svp_energy_difference
    double img = tmp[10] + tmp[11], prox = tmp[12] + tmp[13];
    double jd = tmp[14] + tmp[15], curl = tmp[16] + tmp[17], bar = tmp[18] + tmp[19];
    diff2[0] = (((img + prox) + jd) + curl) + bar;
    diff2[1] = img + bar;
    if (band) {
        *band = 0.;
        if (screened) {
            const double sums[6] = {cell3[0], cell3[1], tmp[20] + tmp[21], tmp[22] + tmp[23], tmp[24] + tmp[25],
                                    tmp[26] + tmp[27]};
            *band = screen_band(p, sums);
        }
    }
    return SVP_OK;
}

extern "C" int svp_trial_energy_active(svp_pair *p, const double *base_u, const double *base_warped,
                                       const double *trial_u, double *trial_warped, double *trial_image_grad,
                                       const uint8_t *base_active, uint8_t *trial_active, double *terms5,
                                       double *diff2, int64_t *barrier_violations, void *stream) {
    return trial_energy(p, base_u, base_warped, trial_u, trial_warped, trial_image_grad, base_active, trial_active,
                        terms5, diff2, barrier_violations, false, nullptr, stream);
}

extern "C" int svp_trial_energy_screened(svp_pair *p, const double *base_u, const double *base_warped,
                                         const double *trial_u, double *trial_warped, double *trial_image_grad,
                                         const uint8_t *base_active, uint8_t *trial_active, double *terms5,
                                         double *diff2, double *band, int64_t *barrier_violations, void *stream) {
    return trial_energy(p, base_u, base_warped, trial_u, trial_warped, trial_image_grad, base_active, trial_active,
                        terms5, diff2, barrier_violations, true, band, stream);
}

extern "C" int svp_trial_energy_masked(svp_pair *p, const double *base_u, const double *base_warped,
                                       const double *trial_u, double *trial_warped, double *trial_image_grad,
                                       uint8_t *trial_active, double *terms5, double *diff2,
                                       int64_t *barrier_violations, void *stream) {
    return svp_trial_energy_active(p, base_u, base_warped, trial_u, trial_warped, trial_image_grad, nullptr,
                                   trial_active, terms5, diff2, barrier_violations, stream);
}

extern "C" int svp_trial_energy(svp_pair *p, const double *base_u, const double *base_warped,
                                const double *trial_u, double *trial_warped, double *trial_image_grad,
                                double *terms5, double *diff2, int64_t *barrier_violations, void *stream) {
    return svp_trial_energy_masked(p, base_u, base_warped, trial_u, trial_warped, trial_image_grad, nullptr, terms5,
                                   diff2, barrier_violations, stream);
}

template <class LT>
static int run_gather(svp_pair *p, const GatherSpec &g, const LT *L1, const LT *L2, const double *u,
                      const double *uref, const double *warped, const double *image_grad, cudaStream_t s) {
    { svp::KernelTimer _t("gather_kernel", s); SVP_LAUNCH(gather_kernel<LT><<<node_blocks(p->q.nfree), 256, 0, s>>>(p->q, g, L1, L2, u, uref, warped, p->fixed, image_grad)); }
    SVP_LAUNCH_CHECK("gather_kernel");
    return SVP_OK;
}

// The plain form's gradient locals: with the state's activity mask, the soft float64 kernel and then the barrier
// kernel over the active cells (the values of the fused kernel: the same sweep, the same add); without a mask the
// fused kernel sweeps the barrier of every cell.
static int grad64(svp_pair *p, const double *u, double mu_scale, double nu_scale, bool barrier, bool split,
                  const uint8_t *active, cudaStream_t s) {
    const bool apart = barrier && active;
    int rc = allow_slices();
    if (rc) return rc;
    {
        svp::KernelTimer _t("cell_grad_kernel", s);
        SVP_LAUNCH(cell_grad_kernel<<<slice_blocks(p), CS, slice_bytes(81), s>>>(
            p->q, u, p->u_ref, mu_scale, nu_scale, barrier && !apart, split, p->loc1, split ? p->loc2 : nullptr,
            active));
    }
    if (apart) {
        svp::KernelTimer _t("cell_grad_barrier_kernel", s);
        SVP_LAUNCH(cell_grad_barrier_kernel<double><<<barrier_blocks(p->q), CB, sizeof(double) * 81 * CB, s>>>(
            p->q, u, active, split, p->loc1, split ? p->loc2 : nullptr));
    }
    return SVP_OK;
}

// The mixed form's gradient locals: the float32 soft kernel, then the float64 barrier kernel over the flagged cells
// (the state's mask, or without one the cells the soft kernel flags from its float32 closed27 J).
static int grad32(svp_pair *p, const double *u, double mu_scale, double nu_scale, bool barrier, bool split,
                  const uint8_t *active, cudaStream_t s) {
    int rc;
    if (barrier && !active && (rc = pair_flags(p))) return rc;
    uint8_t *flags = barrier && !active ? p->flags : nullptr;
    {
        svp::KernelTimer _t("cell_grad32_kernel", s);
        SVP_LAUNCH(cell_grad32_kernel<<<slice_blocks(p), CS, sizeof(float) * 81 * CS, s>>>(
            p->q, u, p->u_ref, mu_scale, nu_scale, split, (float *)p->loc1, (float *)p->loc2, flags));
    }
    if (barrier) {
        svp::KernelTimer _t("cell_grad_barrier32_kernel", s);
        SVP_LAUNCH(cell_grad_barrier_kernel<float><<<barrier_blocks(p->q), CB, sizeof(float) * 81 * CB, s>>>(
            p->q, u, active ? active : flags, split, (float *)p->loc1, (float *)p->loc2));
    }
    return SVP_OK;
}

extern "C" int svp_gradient_masked(svp_pair *p, const double *u, const double *warped, const double *image_grad,
                                   int32_t terms, const uint8_t *active, double *out, void *stream) {
    SVP_REQUIRE(p && u && out, "svp_gradient: null argument");
    SVP_REQUIRE((terms & ~SVP_TERM_TOTAL) == 0 && terms, "svp_gradient: invalid term mask");
    bool img = terms & SVP_TERM_IMAGE;
    SVP_REQUIRE(!img || (warped && image_grad), "svp_gradient: the image term needs warped and image_grad");
    cudaStream_t s = (cudaStream_t)stream;
    const bool mixed = p->precision == SVP_PRECISION_MIXED;
    bool cellwork = terms & (SVP_TERM_JD | SVP_TERM_CURL | SVP_TERM_BARRIER);
    if (cellwork) {
        int rc = pair_locals(p, 1);
        if (rc) return rc;
        if (mixed) {
            if ((rc = grad32(p, u, (terms & SVP_TERM_JD) ? 1. : 0., (terms & SVP_TERM_CURL) ? 1. : 0.,
                             (terms & SVP_TERM_BARRIER) != 0, false, active, s)))
                return rc;
        } else {
            if ((rc = grad64(p, u, (terms & SVP_TERM_JD) ? 1. : 0., (terms & SVP_TERM_CURL) ? 1. : 0.,
                             (terms & SVP_TERM_BARRIER) != 0, false, active, s)))
                return rc;
        }
        SVP_LAUNCH_CHECK("cell_grad_kernel");
    }
    GatherSpec g{};
    g.nout = 1;
    g.ci[0] = img ? 1. : 0.;
    g.cp[0] = (terms & SVP_TERM_PROXIMITY) ? 1. : 0.;
    g.c1[0] = cellwork ? 1. : 0.;
    g.out[0] = out;
    if (mixed)
        return run_gather<float>(p, g, cellwork ? (const float *)p->loc1 : nullptr, nullptr, u, p->u_ref,
                                 img ? warped : nullptr, img ? image_grad : nullptr, s);
    return run_gather<double>(p, g, cellwork ? p->loc1 : nullptr, nullptr, u, p->u_ref, img ? warped : nullptr,
                              img ? image_grad : nullptr, s);
}

extern "C" int svp_outer_gradients_masked(svp_pair *p, const double *u, const double *warped,
                                          const double *image_grad, const uint8_t *active, double *gF, double *gD,
                                          double *gE, void *stream) {
    SVP_REQUIRE(p && u && warped && image_grad && gF && gD && gE, "svp_outer_gradients: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = pair_locals(p, 2);
    if (rc) return rc;
    const bool mixed = p->precision == SVP_PRECISION_MIXED;
    if (mixed) {
        if ((rc = grad32(p, u, 1., 1., true, true, active, s))) return rc;
    } else {
        if ((rc = grad64(p, u, 1., 1., true, true, active, s))) return rc;
    }
    SVP_LAUNCH_CHECK("cell_grad_kernel");
    GatherSpec g{};
    g.nout = 3;
    // gF = image + barrier; gD = image; gE = image + proximity + soft + barrier
    g.ci[0] = 1.; g.cp[0] = 0.; g.c1[0] = 0.; g.c2[0] = 1.; g.out[0] = gF;
    g.ci[1] = 1.; g.cp[1] = 0.; g.c1[1] = 0.; g.c2[1] = 0.; g.out[1] = gD;
    g.ci[2] = 1.; g.cp[2] = 1.; g.c1[2] = 1.; g.c2[2] = 0.; g.out[2] = gE;
    if (mixed) return run_gather<float>(p, g, (const float *)p->loc1, (const float *)p->loc2, u, p->u_ref, warped, image_grad, s);
    return run_gather<double>(p, g, p->loc1, p->loc2, u, p->u_ref, warped, image_grad, s);
}

extern "C" int svp_ggn_diagonal_masked(svp_pair *p, const double *u, const double *image_grad,
                                       const uint8_t *active, double *out, void *stream) {
    SVP_REQUIRE(p && u && image_grad && out, "svp_ggn_diagonal: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = pair_locals(p, 1);
    if (rc) return rc;
    if (p->precision == SVP_PRECISION_MIXED) {
        if (!active && (rc = pair_flags(p))) return rc;
        {
            svp::KernelTimer _t("cell_ggn_diag32_kernel", s);
            SVP_LAUNCH(cell_ggn_diag32_kernel<<<cell_blocks(p), CT, 0, s>>>(p->q, u, (float *)p->loc1,
                                                                           active ? nullptr : p->flags));
        }
        {
            svp::KernelTimer _t("cell_ggn_barrier32_kernel", s);
            SVP_LAUNCH(cell_ggn_barrier_kernel<float><<<barrier_blocks(p->q), CB, 0, s>>>(
                p->q, u, active ? active : p->flags, (float *)p->loc1));
        }
        SVP_LAUNCH(ggn_node_kernel<float><<<node_blocks(p->q.nfree), 256, 0, s>>>(p->q, (const float *)p->loc1, image_grad, nullptr, out));
    } else {
        // with the state's mask, the barrier curvature of the active cells in its own kernel (the same values)
        {
            svp::KernelTimer _t("cell_ggn_diag_kernel", s);
            SVP_LAUNCH(cell_ggn_diag_kernel<<<cell_blocks(p), CT, 0, s>>>(p->q, u, p->loc1, active, active == nullptr));
        }
        if (active) {
            svp::KernelTimer _t("cell_ggn_barrier_kernel", s);
            SVP_LAUNCH(cell_ggn_barrier_kernel<double><<<barrier_blocks(p->q), CB, 0, s>>>(p->q, u, active, p->loc1));
        }
        SVP_LAUNCH(ggn_node_kernel<double><<<node_blocks(p->q.nfree), 256, 0, s>>>(p->q, p->loc1, image_grad, nullptr, out));
    }
    SVP_LAUNCH_CHECK("ggn diagonal");
    return SVP_OK;
}

extern "C" int svp_gradient(svp_pair *p, const double *u, const double *warped, const double *image_grad,
                            int32_t terms, double *out, void *stream) {
    return svp_gradient_masked(p, u, warped, image_grad, terms, nullptr, out, stream);
}
extern "C" int svp_outer_gradients(svp_pair *p, const double *u, const double *warped, const double *image_grad,
                                   double *gF, double *gD, double *gE, void *stream) {
    return svp_outer_gradients_masked(p, u, warped, image_grad, nullptr, gF, gD, gE, stream);
}
extern "C" int svp_ggn_diagonal(svp_pair *p, const double *u, const double *image_grad, double *out,
                                void *stream) {
    return svp_ggn_diagonal_masked(p, u, image_grad, nullptr, out, stream);
}

extern "C" int svp_ggn_hvp(svp_pair *p, const double *u, const double *image_grad, const double *pvec,
                           double *out, void *stream) {
    SVP_REQUIRE(p && u && image_grad && pvec && out, "svp_ggn_hvp: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = pair_locals(p, 2);
    if (rc) return rc;
    // inject p into a node field (zero faces) held in loc2's storage
    double *vv = p->loc2;
    rc = svp_inject(&p->grid, pvec, vv, stream);
    if (rc) return rc;
    { svp::KernelTimer _t("cell_ggn_hvp_kernel", s); SVP_LAUNCH(cell_ggn_hvp_kernel<<<slice_blocks(p), CS, slice_bytes(81), s>>>(p->q, u, vv, p->loc1)); }
    SVP_LAUNCH(ggn_node_kernel<double><<<node_blocks(p->q.nfree), 256, 0, s>>>(p->q, p->loc1, image_grad, vv, out));
    SVP_LAUNCH_CHECK("ggn hvp");
    return SVP_OK;
}

extern "C" int svp_node_min_jd_extended(svp_pair *p, const double *u, double extension_activation, double *node,
                                        int64_t *candidates, void *stream) {
    SVP_REQUIRE(p && u && node, "svp_node_min_jd: null argument");
    SVP_REQUIRE(!(extension_activation < 0.) && extension_activation == extension_activation,
                "svp_node_min_jd: extension activation must be >= 0 (0: no extension)");
    cudaStream_t s = (cudaStream_t)stream;
    const bool ext = extension_activation > 0.;
    if (ext && !p->cand) SVP_CUDA(cudaMalloc((void **)&p->cand, sizeof(long long) * p->q.ncell));
    unsigned long long *ncand = (unsigned long long *)(p->counter + 4);
    if (ext) SVP_CUDA(cudaMemsetAsync(ncand, 0, sizeof(unsigned long long), s));
    { svp::KernelTimer _t("cell_min_jd_kernel", s); SVP_LAUNCH(cell_min_jd_kernel<<<slice_blocks(p), CS, slice_bytes(27), s>>>(p->q, u, p->cellbuf, ext ? extension_activation : 0., ncand, p->cand)); }
    if (ext) {
        svp::KernelTimer _t("jd_extension_kernel", s);
        SVP_LAUNCH(jd_extension_kernel<<<148 * 4, 128, 0, s>>>(p->q, u, ncand, p->cand, p->cellbuf));
    }
    SVP_LAUNCH(node_min_kernel<<<node_blocks(p->q.nnode), 256, 0, s>>>(p->q, p->cellbuf, node));
    SVP_LAUNCH_CHECK("node_min_jd");
    if (candidates) {
        unsigned long long nc = 0;
        if (ext) {
            SVP_CUDA(cudaMemcpyAsync(&nc, ncand, sizeof nc, cudaMemcpyDeviceToHost, s));
            SVP_CUDA(cudaStreamSynchronize(s));
        }
        *candidates = (int64_t)nc;
    }
    return SVP_OK;
}

extern "C" int svp_node_min_jd(svp_pair *p, const double *u, double *node, void *stream) {
    return svp_node_min_jd_extended(p, u, 0., node, nullptr, stream);
}

extern "C" int svp_jd_root(svp_pair *p, const double *u, const double *pvec, double limit, double *root,
                           int64_t *invalid, void *stream) {
    SVP_REQUIRE(p && u && pvec && root && limit > 0, "svp_jd_root: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = pair_locals(p, 2);
    if (rc) return rc;
    double *vv = p->loc2;
    rc = svp_inject(&p->grid, pvec, vv, stream);
    if (rc) return rc;
    long long init[2] = {kKeyPosInf, 0};
    SVP_CUDA(cudaMemcpyAsync(p->counter, init, sizeof init, cudaMemcpyHostToDevice, s));
    { svp::KernelTimer _t("jd_root_kernel", s); SVP_LAUNCH(jd_root_kernel<<<cell_blocks(p), CT, 0, s>>>(p->q, u, vv, limit, p->counter,
                                                 (unsigned long long *)(p->counter + 1))); }
    SVP_LAUNCH_CHECK("jd_root_kernel");
    long long out[2];
    SVP_CUDA(cudaMemcpyAsync(out, p->counter, sizeof out, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    double sv = key_value(out[0]);
    *root = std::isfinite(sv) ? sv * limit : INFINITY;
    if (invalid) *invalid = out[1];
    return SVP_OK;
}

extern "C" int svp_image_shift(svp_pair *p, const double *image_grad, double factor, double *alpha, void *stream) {
    SVP_REQUIRE(p && image_grad && alpha, "svp_image_shift: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = node_blocks(p->q.nfree);
    int rc = pair_partials(p, nb, 1);
    if (rc) return rc;
    SVP_LAUNCH(shift_kernel<<<nb, 256, 0, s>>>(p->q, image_grad, p->partial));
    SVP_LAUNCH(final_reduce_kernel<<<1, 256, 0, s>>>(p->partial, nb, 1, p->result));
    SVP_LAUNCH_CHECK("shift kernels");
    double tmp[2];
    SVP_CUDA(cudaMemcpyAsync(tmp, p->result, sizeof tmp, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    *alpha = factor * ((tmp[0] + tmp[1]) / (double)p->q.nfree) / 3;
    return SVP_OK;
}

extern "C" int svp_pg_scale(svp_pair *p, const double *diag, const double *node_jd, double m, double activation,
                            double floor_, double *scale, int64_t *bad, void *stream) {
    SVP_REQUIRE(p && diag && node_jd && scale && m > 0 && activation > 0, "svp_pg_scale: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    SVP_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(long long), s));
    SVP_LAUNCH(pg_scale_kernel<<<node_blocks(p->q.nfree), 256, 0, s>>>(p->q, diag, node_jd, std::sqrt(m), activation, floor_,
                                                            scale, (unsigned long long *)p->counter));
    SVP_LAUNCH_CHECK("pg_scale_kernel");
    long long host = 0;
    SVP_CUDA(cudaMemcpyAsync(&host, p->counter, sizeof host, cudaMemcpyDeviceToHost, s));
    SVP_CUDA(cudaStreamSynchronize(s));
    if (bad) *bad = host;
    return SVP_OK;
}
