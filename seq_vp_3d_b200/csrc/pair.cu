// Registration-pair handle: device constants (fixed image, spline of the moving image, u_ref, weights) and the
// workspace of the Q1 kernels.  The not-a-knot spline prefilter runs on the device as one dense per-axis transform
// with the inverse collocation matrix (interpolation.py:29 build_image_sampler, SciPy make_interp_spline k=3).
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "pair.cuh"

namespace svp {
int apply_axis(const double *M, int axis, long long batch, long long n2, long long n1, long long n0,
               const double *in, double *out, cudaStream_t s);
int pair_dst_setup(svp_pair *p);

namespace {

// Not-a-knot knot vector of a cubic spline through the nodes x: x0 (x4), x[2 .. n-3], x[n-1] (x4).
std::vector<double> not_a_knot(const std::vector<double> &x) {
    size_t n = x.size();
    std::vector<double> t;
    for (int k = 0; k < 4; k++) t.push_back(x[0]);
    for (size_t i = 2; i + 2 < n; i++) t.push_back(x[i]);
    for (int k = 0; k < 4; k++) t.push_back(x[n - 1]);
    return t;
}

// The reciprocals cubic_basis multiplies by, per span s in [3, n-1] (row s of 14): the Cox-de Boor denominators
// t[s+r+1] - t[s+1-d+r] for d = 1..3, r < d (6), then for each basis function k = 0..3 of the span the two derivative
// denominators a = t[i+3] - t[i], b = t[i+4] - t[i+1] with i = s - 3 + k (1 where a difference is zero, the
// reference's guard).  Rows below 3 are unused (zero).
std::vector<double> spline_reciprocals(const std::vector<double> &t, long long n) {
    std::vector<double> R((size_t)n * 14, 0.);
    for (long long s = 3; s <= n - 1; s++) {
        double *row = R.data() + 14 * s;
        int k = 0;
        for (int d = 1; d <= 3; d++)
            for (int r = 0; r < d; r++) {
                double len = t[(size_t)(s + r + 1)] - t[(size_t)(s + 1 - d + r)];
                row[k++] = len != 0. ? 1. / len : 0.;
            }
        for (int b = 0; b < 4; b++) {
            long long i = s - 3 + b;
            double a = t[(size_t)(i + 3)] - t[(size_t)i], bb = t[(size_t)(i + 4)] - t[(size_t)(i + 1)];
            row[6 + 2 * b] = 1. / (a != 0. ? a : 1.);
            row[7 + 2 * b] = 1. / (bb != 0. ? bb : 1.);
        }
    }
    return R;
}

// Cox-de Boor values of the 4 cubic B-splines on span s at x (backends/spline.py:12 cubic_basis)
void basis4(const std::vector<double> &t, int s, double x, double B[4]) {
    double b[4] = {1., 0., 0., 0.};
    for (int degree = 1; degree <= 3; degree++) {
        double nb[4], saved = 0.;
        for (int r = 0; r < degree; r++) {
            double right = t[s + r + 1] - x, left = x - t[s + 1 - degree + r];
            double temp = b[r] / (right + left);
            nb[r] = saved + right * temp;
            saved = left * temp;
        }
        nb[degree] = saved;
        for (int r = 0; r <= degree; r++) b[r] = nb[r];
    }
    for (int k = 0; k < 4; k++) B[k] = b[k];
}

// Inverse of the collocation matrix B[i][j] = B_j(x_i) (Gauss-Jordan, partial pivoting, long double)
std::vector<double> inverse_collocation(const std::vector<double> &x) {
    int n = (int)x.size();
    std::vector<double> t = not_a_knot(x);
    std::vector<long double> A((size_t)n * n, 0.L), I((size_t)n * n, 0.L);
    for (int i = 0; i < n; i++) {
        int s = 3;
        for (int k = 3; k <= n - 1; k++)
            if (t[k] <= x[i]) s = k;
        double B[4];
        basis4(t, s, x[i], B);
        for (int k = 0; k < 4; k++) A[(size_t)i * n + s - 3 + k] = B[k];
        I[(size_t)i * n + i] = 1.L;
    }
    for (int c = 0; c < n; c++) {
        int piv = c;
        for (int r = c + 1; r < n; r++)
            if (fabsl(A[(size_t)r * n + c]) > fabsl(A[(size_t)piv * n + c])) piv = r;
        if (piv != c)
            for (int k = 0; k < n; k++) {
                std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
                std::swap(I[(size_t)c * n + k], I[(size_t)piv * n + k]);
            }
        long double d = A[(size_t)c * n + c];
        for (int k = 0; k < n; k++) { A[(size_t)c * n + k] /= d; I[(size_t)c * n + k] /= d; }
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            long double f = A[(size_t)r * n + c];
            if (f == 0.L) continue;
            for (int k = 0; k < n; k++) {
                A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
                I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
            }
        }
    }
    std::vector<double> out((size_t)n * n);
    for (size_t k = 0; k < out.size(); k++) out[k] = (double)I[k];
    return out;
}

// The inverse depends only on the axis nodes; registrations on one grid share it (it is O(n^3) in long double, tens
// of milliseconds of host time per axis on a native grid).
std::vector<double> cached_inverse_collocation(const std::vector<double> &x) {
    static std::mutex mu;
    static std::map<std::vector<double>, std::vector<double>> cache;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(x);
        if (it != cache.end()) return it->second;
    }
    std::vector<double> inv = inverse_collocation(x);
    std::lock_guard<std::mutex> lock(mu);
    if (cache.size() >= 32) cache.clear();
    cache.emplace(x, inv);
    return inv;
}

Q1Const make_const(const svp_grid *g, const svp_weights *w) {
    Q1Const q;
    memset(&q, 0, sizeof q);
    q.nx = g->nx; q.ny = g->ny; q.nz = g->nz;
    q.cx = g->nx - 1; q.cy = g->ny - 1; q.cz = g->nz - 1;
    q.ncell = q.cx * q.cy * q.cz;
    q.nnode = q.nx * q.ny * q.nz;
    q.fx = g->nx - 2; q.fy = g->ny - 2; q.fz = g->nz - 2;
    q.nfree = q.fx * q.fy * q.fz;
    q.h[0] = g->hx; q.h[1] = g->hy; q.h[2] = g->hz;
    for (int k = 0; k < 3; k++) q.ih[k] = 1. / q.h[k];
    q.x0[0] = g->x0; q.x0[1] = g->y0; q.x0[2] = g->z0;
    // Gauss nodes .5 -+ sqrt(15)/10 and weights 5/18, 4/9, 5/18 (cell_q1.py:106-107)
    const double r15 = std::sqrt(15.) / 10;
    q.gn[0] = .5 - r15; q.gn[1] = .5; q.gn[2] = .5 + r15;
    for (int k = 0; k < 3; k++) q.gm[k] = 1 - q.gn[k];
    const double w1[3] = {5. / 18, 4. / 9, 5. / 18};
    q.omega = (g->hx * g->hy) * g->hz;
    for (int p = 0; p < 27; p++) q.gw[p] = ((q.omega * w1[p % 3]) * w1[(p / 3) % 3]) * w1[p / 9];
    q.lam = w->lam; q.mu = w->mu; q.nu = w->nu;
    for (int p = 0; p < 27; p++) {       // IEEE square roots: the values the device's sqrt gives
        q.sqmu[p] = std::sqrt(q.mu * q.gw[p]);
        q.sqnu[p] = std::sqrt(q.nu * q.gw[p]);
    }
    for (int k = 0; k < 3; k++) {
        q.gnf[k] = (float)q.gn[k];
        q.gmf[k] = (float)q.gm[k];
        q.ihf[k] = (float)q.ih[k];
    }
    for (int p = 0; p < 27; p++) q.gwf[p] = (float)q.gw[p];
    for (int a = 0; a < 8; a++) {
        const int b[3] = {a & 1, (a >> 1) & 1, (a >> 2) & 1};
        for (int r = 0; r < 3; r++) {
            double sum = 0.;
            for (int p = 0; p < 27; p++) {
                const int idx[3] = {p % 3, (p / 3) % 3, p / 9};
                double f[3], D[3];
                for (int k = 0; k < 3; k++) f[k] = b[k] ? q.gn[idx[k]] : q.gm[idx[k]];
                for (int k = 0; k < 3; k++) {
                    const int k1 = k == 0 ? 1 : 0, k2 = k == 2 ? 1 : 2;
                    D[k] = (b[k] ? q.ih[k] : -q.ih[k]) * f[k1] * f[k2];
                }
                double cs = 0.;
                for (int j = 0; j < 3; j++)
                    if (j != r) cs += D[j] * D[j];
                sum += q.gw[p] * (w->nu * cs);
            }
            q.ggn_curl[3 * a + r] = sum;
            q.ggn_curlf[3 * a + r] = (float)sum;
        }
    }
    q.bw = w->kappa * q.omega / 27;
    q.act = w->activation;
    q.delta = w->delta;
    return q;
}

}  // namespace
}  // namespace svp

using namespace svp;

extern "C" int svp_pair_destroy(svp_pair *p) {
    if (!p) return SVP_OK;
    cudaFree(p->fixed); cudaFree(p->coeff); cudaFree(p->u_ref);
    for (int k = 0; k < 3; k++) {
        cudaFree(p->knots[k]); cudaFree(p->spline_rcp[k]); cudaFree(p->dst_half[k]); cudaFree(p->dst_pad[k]); cudaFree(p->dst_tf32[k]);
    }
    cudaFree(p->loc1); cudaFree(p->loc2); cudaFree(p->cellbuf); cudaFree(p->partial); cudaFree(p->result);
    cudaFree(p->counter); cudaFree(p->cand); cudaFree(p->flags); cudaFree(p->dst_tmp); cudaFree(p->den);
    delete p;
    return SVP_OK;
}

extern "C" int svp_pair_create(const svp_grid *g, const svp_weights *w, const double *fixed, const double *moving,
                               const double *u_ref, svp_pair **out, void *stream) {
    SVP_REQUIRE(out, "svp_pair_create: null output");
    *out = nullptr;
    SVP_REQUIRE(grid_ok(g) && g->nx >= 5 && g->ny >= 5 && g->nz >= 5, "svp_pair_create: grid needs >= 5 nodes/axis");
    SVP_REQUIRE(w && fixed && moving && u_ref, "svp_pair_create: null argument");
    SVP_REQUIRE(w->lam > 0 && w->mu >= 0 && w->nu >= 0 && w->kappa > 0, "svp_pair_create: invalid weights");
    SVP_REQUIRE(w->delta >= 0 && w->delta < w->activation && w->activation <= 1,
                "svp_pair_create: require 0 <= delta < activation <= 1");
    cudaStream_t s = (cudaStream_t)stream;
    svp_pair *p = new svp_pair();
    p->grid = *g;
    p->w = *w;
    p->q = make_const(g, w);
    cudaGetDevice(&p->device);
    const long long nn = p->q.nnode;
    auto bail = [&](int rc) {
        svp_pair_destroy(p);
        return rc;
    };
    cudaError_t e;
    if ((e = cudaMalloc((void **)&p->fixed, sizeof(double) * nn)) != cudaSuccess) return bail(cuda_fail(e, "fixed"));
    if ((e = cudaMalloc((void **)&p->coeff, sizeof(double) * nn)) != cudaSuccess) return bail(cuda_fail(e, "coeff"));
    if ((e = cudaMalloc((void **)&p->u_ref, sizeof(double) * 3 * nn)) != cudaSuccess) return bail(cuda_fail(e, "uref"));
    if ((e = cudaMalloc((void **)&p->cellbuf, sizeof(double) * p->q.ncell)) != cudaSuccess)
        return bail(cuda_fail(e, "cellbuf"));
    if ((e = cudaMalloc((void **)&p->result, sizeof(double) * 64)) != cudaSuccess) return bail(cuda_fail(e, "result"));
    if ((e = cudaMalloc((void **)&p->counter, sizeof(long long) * 8)) != cudaSuccess)
        return bail(cuda_fail(e, "counter"));
    if ((e = cudaMemcpyAsync(p->fixed, fixed, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return bail(cuda_fail(e, "fixed copy"));
    if ((e = cudaMemcpyAsync(p->u_ref, u_ref, sizeof(double) * 3 * nn, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return bail(cuda_fail(e, "u_ref copy"));
    // knots and spline coefficients: prefilter z, then y, then x (the reference's axis order)
    const long long len[3] = {g->nx, g->ny, g->nz};
    const double org[3] = {g->x0, g->y0, g->z0}, h[3] = {g->hx, g->hy, g->hz};
    std::vector<double> inv[3];
    for (int k = 0; k < 3; k++) {
        std::vector<double> x((size_t)len[k]);
        for (long long i = 0; i < len[k]; i++) x[(size_t)i] = org[k] + h[k] * (double)i;
        std::vector<double> t = not_a_knot(x);
        if ((e = cudaMalloc((void **)&p->knots[k], sizeof(double) * t.size())) != cudaSuccess)
            return bail(cuda_fail(e, "knots"));
        if ((e = cudaMemcpy(p->knots[k], t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(e, "knots copy"));
        std::vector<double> rcp = spline_reciprocals(t, len[k]);
        if ((e = cudaMalloc((void **)&p->spline_rcp[k], sizeof(double) * rcp.size())) != cudaSuccess)
            return bail(cuda_fail(e, "spline reciprocals"));
        if ((e = cudaMemcpy(p->spline_rcp[k], rcp.data(), sizeof(double) * rcp.size(), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return bail(cuda_fail(e, "spline reciprocals copy"));
        inv[k] = cached_inverse_collocation(x);
    }
    // the prefilter's matrices and intermediate live in the stream-ordered scratch pool: freeing them does not
    // synchronize the device (registrations on other streams keep running)
    double *mats[3] = {nullptr, nullptr, nullptr}, *tmp = nullptr;
    int rc = SVP_OK;
    for (int k = 0; k < 3 && !rc; k++) {
        if ((e = scratch_alloc((void **)&mats[k], sizeof(double) * inv[k].size(), s)) != cudaSuccess)
            rc = cuda_fail(e, "prefilter matrix");
        else if ((e = cudaMemcpyAsync(mats[k], inv[k].data(), sizeof(double) * inv[k].size(), cudaMemcpyHostToDevice,
                                      s)) != cudaSuccess)
            rc = cuda_fail(e, "prefilter matrix copy");
    }
    if (!rc && (e = scratch_alloc((void **)&tmp, sizeof(double) * nn, s)) != cudaSuccess)
        rc = cuda_fail(e, "prefilter tmp");
    if (!rc) rc = apply_axis(mats[2], 2, 1, g->nz, g->ny, g->nx, moving, tmp, s);
    if (!rc) rc = apply_axis(mats[1], 1, 1, g->nz, g->ny, g->nx, tmp, p->coeff, s);
    if (!rc) rc = apply_axis(mats[0], 0, 1, g->nz, g->ny, g->nx, p->coeff, tmp, s);
    if (!rc) {
        e = cudaMemcpyAsync(p->coeff, tmp, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) rc = cuda_fail(e, "coeff copy");
    }
    for (int k = 0; k < 3; k++)
        if (mats[k]) scratch_free(mats[k], s);
    if (tmp) scratch_free(tmp, s);
    cudaStreamSynchronize(s);      // the host matrices above must outlive their copies
    if (rc) return bail(rc);
    if ((rc = pair_dst_setup(p))) return bail(rc);
    *out = p;
    return SVP_OK;
}

extern "C" int svp_pair_set_reference(svp_pair *p, const double *u_ref, void *stream) {
    SVP_REQUIRE(p && u_ref, "svp_pair_set_reference: null argument");
    SVP_CUDA(cudaMemcpyAsync(p->u_ref, u_ref, sizeof(double) * 3 * p->q.nnode, cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream));
    return SVP_OK;
}

extern "C" int svp_pair_set_spline_coefficients(svp_pair *p, const double *coeff, void *stream) {
    SVP_REQUIRE(p && coeff, "svp_pair_set_spline_coefficients: null argument");
    SVP_CUDA(cudaMemcpyAsync(p->coeff, coeff, sizeof(double) * p->q.nnode, cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream));
    return SVP_OK;
}

extern "C" int svp_pair_spline_coefficients(const svp_pair *p, double *out, void *stream) {
    SVP_REQUIRE(p && out, "svp_pair_spline_coefficients: null argument");
    SVP_CUDA(cudaMemcpyAsync(out, p->coeff, sizeof(double) * p->q.nnode, cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream));
    return SVP_OK;
}
