// Vector kernels of the PG solver on free-node vectors: deterministic dot products, the trial axpy with the
// reference's two roundings, inject/restrict between node fields and free vectors, and the domain step bound.
#include <cmath>
#include <cstring>

#include "pair.cuh"

namespace svp {
namespace {

__global__ void __launch_bounds__(256) dot_kernel(const double *__restrict__ a, const double *__restrict__ b,
                                                  long long n, dd *partial) {
    dd acc[1] = {{0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        acc[0] = dd_add(acc[0], two_prod(a[i], b[i]));
    block_reduce_dd<1>(acc, partial);
}

__global__ void dot_final_kernel(const dd *__restrict__ partial, long long blocks, double *out) {
    __shared__ dd sh[256];
    dd acc = {0., 0.};
    for (long long b = threadIdx.x; b < blocks; b += blockDim.x) acc = dd_add(acc, partial[b]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = dd_add(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0].hi + sh[0].lo;
}

// y = fl(x + fl(tau * p)): the trial step's two roundings (no FMA), as base.theta + tau * direction
__global__ void axpy_kernel(const double *__restrict__ x, double tau, const double *__restrict__ p, long long n,
                            double *__restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = __dadd_rn(x[i], __dmul_rn(tau, p[i]));
}

__global__ void inject_kernel(long long nx, long long ny, long long nz, const double *__restrict__ theta,
                              double *__restrict__ u) {
    const long long fx = nx - 2, fy = ny - 2, fz = nz - 2, nf = fx * fy * fz, nn = nx * ny * nz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, nx, ny, x, y, z);
        bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
        long long f = ((z - 1) * fy + (y - 1)) * fx + (x - 1);
#pragma unroll
        for (int r = 0; r < 3; r++) u[3 * i + r] = face ? 0. : theta[r * nf + f];
    }
}

__global__ void restrict_kernel(long long nx, long long ny, long long nz, const double *__restrict__ u,
                                double *__restrict__ theta) {
    const long long fx = nx - 2, fy = ny - 2, fz = nz - 2, nf = fx * fy * fz;
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf;
         f += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(f, fx, fy, x, y, z);
        x++; y++; z++;
        long long i = (z * ny + y) * nx + x;
#pragma unroll
        for (int r = 0; r < 3; r++) theta[r * nf + f] = u[3 * i + r];
    }
}

// fast_checks.py:85 _step_bound_xu: min over free nodes and components with d != 0 of
// ((d > 0 ? top : bottom) - fl(axis + u)) / d; order-independent min via integer keys
__global__ void step_bound_kernel(long long nx, long long ny, long long nz, double hx, double hy, double hz,
                                  double x0, double y0, double z0, const double *__restrict__ u,
                                  const double *__restrict__ p, long long *best) {
    const long long fx = nx - 2, fy = ny - 2, fz = nz - 2, nf = fx * fy * fz;
    const double h[3] = {hx, hy, hz}, o[3] = {x0, y0, z0};
    const long long len[3] = {nx, ny, nz};
    long long key = kKeyPosInf;
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf;
         f += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(f, fx, fy, x, y, z);
        x++; y++; z++;
        long long idx[3] = {x, y, z};
        long long i = (z * ny + y) * nx + x;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            double d = p[r * nf + f];
            if (d > 0 || d < 0) {
                double base = __dadd_rn(o[r], __dmul_rn(h[r], (double)idx[r]));
                double pt = __dadd_rn(base, u[3 * i + r]);
                double lim = d > 0 ? __dadd_rn(o[r], __dmul_rn(h[r], (double)(len[r] - 1))) : o[r];
                double qv = __ddiv_rn(__dsub_rn(lim, pt), d);
                long long k = order_key(qv);
                key = k < key ? k : key;
            }
        }
    }
    for (int s = 16; s; s >>= 1) {
        long long y = __shfl_xor_sync(0xFFFFFFFFu, key, s);
        key = y < key ? y : key;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(best, key);
}

__global__ void __launch_bounds__(256) bb2_kernel(const double *__restrict__ th, const double *__restrict__ th0,
                                                  const double *__restrict__ g, const double *__restrict__ g0,
                                                  const double *__restrict__ p0, const double *__restrict__ p,
                                                  long long n, dd *partial) {
    dd acc[4] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double s = th[i] - th0[i], y = g[i] - g0[i], iy = p0[i] - p[i];
        acc[0] = dd_add(acc[0], two_prod(s, y));
        acc[1] = dd_add(acc[1], two_prod(s, s));
        acc[2] = dd_add(acc[2], two_prod(y, y));
        acc[3] = dd_add(acc[3], two_prod(y, iy));
    }
    block_reduce_dd<4>(acc, partial);
}

// The scalars of one PG step in one pass: g.g, g.p and, with the previous step, the four BB2 products of bb2_kernel.
// Same grid, per-thread order and reductions as dot_kernel and bb2_kernel, so each value is bitwise theirs.
template <int K>
__global__ void __launch_bounds__(256) step_dots_kernel(const double *__restrict__ g, const double *__restrict__ p,
                                                        const double *__restrict__ th, const double *__restrict__ th0,
                                                        const double *__restrict__ g0, const double *__restrict__ p0,
                                                        long long n, dd *partial) {
    dd acc[K];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] = {0., 0.};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double gi = g[i], pi = p[i];
        acc[0] = dd_add(acc[0], two_prod(gi, gi));
        acc[1] = dd_add(acc[1], two_prod(gi, pi));
        if constexpr (K == 6) {
            double s = th[i] - th0[i], y = gi - g0[i], iy = p0[i] - pi;
            acc[2] = dd_add(acc[2], two_prod(s, y));
            acc[3] = dd_add(acc[3], two_prod(s, s));
            acc[4] = dd_add(acc[4], two_prod(y, y));
            acc[5] = dd_add(acc[5], two_prod(y, iy));
        }
    }
    block_reduce_dd<K>(acc, partial);
}

__global__ void multi_final_kernel(const dd *__restrict__ partial, long long blocks, int K, double *out) {
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
        if (threadIdx.x == 0) out[k] = sh[0].hi + sh[0].lo;
        __syncthreads();
    }
}

// max |a - b| and max |b| as order keys of non-negative values; a NaN maps above +inf (propagates)
__global__ void max_abs_diff_kernel(const double *__restrict__ a, const double *__restrict__ b, long long n,
                                    long long *keys) {
    long long k0 = 0, k1 = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double d = fabs(a[i] - b[i]), m = fabs(b[i]);
        long long x = d != d ? 0x7FF8000000000000LL : __double_as_longlong(d);
        long long y = m != m ? 0x7FF8000000000000LL : __double_as_longlong(m);
        k0 = x > k0 ? x : k0;
        k1 = y > k1 ? y : k1;
    }
    for (int s = 16; s; s >>= 1) {
        long long x = __shfl_xor_sync(0xFFFFFFFFu, k0, s), y = __shfl_xor_sync(0xFFFFFFFFu, k1, s);
        k0 = x > k0 ? x : k0;
        k1 = y > k1 ? y : k1;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(keys, k0);
        atomicMax(keys + 1, k1);
    }
}

// The trial point of a line-search attempt in one pass over the nodes: candidate = fl(theta + fl(tau p)) (axpy_kernel's
// roundings), u = inject(candidate) (zero faces) and the keys of max |candidate - theta|, max |theta|
// (max_abs_diff_kernel's), so the step ratio needs no second pass.
__global__ void trial_point_kernel(long long nx, long long ny, long long nz, const double *__restrict__ theta,
                                   double tau, const double *__restrict__ p, double *__restrict__ cand,
                                   double *__restrict__ u, long long *keys) {
    const long long fx = nx - 2, fy = ny - 2, fz = nz - 2, nf = fx * fy * fz, nn = nx * ny * nz;
    long long k0 = 0, k1 = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nn;
         i += (long long)gridDim.x * blockDim.x) {
        long long x, y, z;
        unflatten3(i, nx, ny, x, y, z);
        bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
        long long f = ((z - 1) * fy + (y - 1)) * fx + (x - 1);
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (face) {
                u[3 * i + r] = 0.;
                continue;
            }
            const double t = theta[r * nf + f];
            const double c = __dadd_rn(t, __dmul_rn(tau, p[r * nf + f]));
            cand[r * nf + f] = c;
            u[3 * i + r] = c;
            double d = fabs(c - t), m = fabs(t);
            long long kx = d != d ? 0x7FF8000000000000LL : __double_as_longlong(d);
            long long ky = m != m ? 0x7FF8000000000000LL : __double_as_longlong(m);
            k0 = kx > k0 ? kx : k0;
            k1 = ky > k1 ? ky : k1;
        }
    }
    for (int s = 16; s; s >>= 1) {
        long long x = __shfl_xor_sync(0xFFFFFFFFu, k0, s), y = __shfl_xor_sync(0xFFFFFFFFu, k1, s);
        k0 = x > k0 ? x : k0;
        k1 = y > k1 ? y : k1;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(keys, k0);
        atomicMax(keys + 1, k1);
    }
}

// order keys -> doubles in place (the deferred form of the step-bound reduction)
__global__ void keys_to_double_kernel(long long *keys, int n) {
    if (threadIdx.x < n) keys[threadIdx.x] = __double_as_longlong(key_value(keys[threadIdx.x]));
}
__global__ void set_key_kernel(long long *key, long long value) { *key = value; }

}  // namespace
}  // namespace svp

using namespace svp;

// ---- deferred forms: results into device memory, no synchronisation (gather several scalars with one copy) ----
extern "C" int svp_dot_dev(const double *a, const double *b, int64_t n, double *out_dev, void *stream) {
    SVP_REQUIRE(a && b && out_dev && n >= 0, "svp_dot_dev: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = blocks_for(n, 256, 4);
    dd *part = nullptr;
    SVP_CUDA(scratch_alloc((void **)&part, sizeof(dd) * nb, s));
    SVP_LAUNCH_KEEP(dot_kernel<<<nb, 256, 0, s>>>(a, b, n, part));
    SVP_LAUNCH_KEEP(dot_final_kernel<<<1, 256, 0, s>>>(part, nb, out_dev));
    cudaError_t le = cudaGetLastError();
    cudaError_t fe = scratch_free(part, s);
    if (le != cudaSuccess) return cuda_fail(le, "dot kernels");
    if (fe != cudaSuccess) return cuda_fail(fe, "dot free");
    return SVP_OK;
}

extern "C" int svp_bb2_dots_dev(const double *theta, const double *theta_old, const double *g, const double *g_old,
                                const double *p_old, const double *pvec, int64_t n, double *out4_dev, void *stream) {
    SVP_REQUIRE(theta && theta_old && g && g_old && p_old && pvec && out4_dev && n >= 0, "svp_bb2_dots_dev: invalid");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = blocks_for(n, 256, 4);
    dd *part = nullptr;
    SVP_CUDA(scratch_alloc((void **)&part, sizeof(dd) * 4 * nb, s));
    SVP_LAUNCH_KEEP(bb2_kernel<<<nb, 256, 0, s>>>(theta, theta_old, g, g_old, p_old, pvec, n, part));
    SVP_LAUNCH_KEEP(multi_final_kernel<<<1, 256, 0, s>>>(part, nb, 4, out4_dev));
    cudaError_t le = cudaGetLastError();
    cudaError_t fe = scratch_free(part, s);
    if (le != cudaSuccess) return cuda_fail(le, "bb2 kernels");
    if (fe != cudaSuccess) return cuda_fail(fe, "bb2 free");
    return SVP_OK;
}

extern "C" int svp_step_dots_dev(const double *g, const double *pvec, const double *theta, const double *theta_old,
                                 const double *g_old, const double *p_old, int64_t n, double *out_dev, void *stream) {
    SVP_REQUIRE(g && pvec && out_dev && n >= 0, "svp_step_dots_dev: invalid argument");
    const bool bb2 = theta && theta_old && g_old && p_old;
    SVP_REQUIRE(bb2 || !(theta || theta_old || g_old || p_old), "svp_step_dots_dev: previous step given in part");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = blocks_for(n, 256, 4);
    const int K = bb2 ? 6 : 2;
    dd *part = nullptr;
    SVP_CUDA(scratch_alloc((void **)&part, sizeof(dd) * K * nb, s));
    if (bb2)
        SVP_LAUNCH_KEEP(step_dots_kernel<6><<<nb, 256, 0, s>>>(g, pvec, theta, theta_old, g_old, p_old, n, part));
    else
        SVP_LAUNCH_KEEP(step_dots_kernel<2><<<nb, 256, 0, s>>>(g, pvec, nullptr, nullptr, nullptr, nullptr, n, part));
    SVP_LAUNCH_KEEP(multi_final_kernel<<<1, 256, 0, s>>>(part, nb, K, out_dev));
    cudaError_t le = cudaGetLastError();
    cudaError_t fe = scratch_free(part, s);
    if (le != cudaSuccess) return cuda_fail(le, "step dots kernels");
    if (fe != cudaSuccess) return cuda_fail(fe, "step dots free");
    return SVP_OK;
}

extern "C" int svp_max_abs_diff_dev(const double *a, const double *b, int64_t n, double *out2_dev, void *stream) {
    SVP_REQUIRE(a && b && out2_dev && n >= 0, "svp_max_abs_diff_dev: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    long long *keys = (long long *)out2_dev;
    SVP_CUDA(cudaMemsetAsync(keys, 0, 2 * sizeof(long long), s));
    // the keys are the bits of the nonnegative maxima (NaN canonical): already the doubles
    SVP_LAUNCH(max_abs_diff_kernel<<<blocks_for(n, 256, 8), 256, 0, s>>>(a, b, n, keys));
    SVP_LAUNCH_CHECK("max_abs_diff");
    return SVP_OK;
}

extern "C" int svp_trial_point(const svp_grid *g, const double *theta, double tau, const double *pvec,
                               double *candidate, double *u, double *out2_dev, void *stream) {
    SVP_REQUIRE(grid_ok(g) && theta && pvec && candidate && u && out2_dev, "svp_trial_point: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    long long *keys = (long long *)out2_dev;
    SVP_CUDA(cudaMemsetAsync(keys, 0, 2 * sizeof(long long), s));
    SVP_LAUNCH(trial_point_kernel<<<blocks_for(n_nodes(g), 256, 8), 256, 0, s>>>(g->nx, g->ny, g->nz, theta, tau, pvec,
                                                                                candidate, u, keys));
    SVP_LAUNCH_CHECK("trial_point_kernel");
    return SVP_OK;
}

extern "C" int svp_step_bound_dev(const svp_grid *g, const double *u, const double *pvec, double *bound_dev,
                                  void *stream) {
    SVP_REQUIRE(grid_ok(g) && u && pvec && bound_dev, "svp_step_bound_dev: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    long long *best = (long long *)bound_dev;
    SVP_LAUNCH(set_key_kernel<<<1, 1, 0, s>>>(best, kKeyPosInf));
    SVP_LAUNCH(step_bound_kernel<<<blocks_for(n_free(g), 256, 8), 256, 0, s>>>(g->nx, g->ny, g->nz, g->hx, g->hy, g->hz, g->x0,
                                                                    g->y0, g->z0, u, pvec, best));
    SVP_LAUNCH(keys_to_double_kernel<<<1, 32, 0, s>>>(best, 1));
    SVP_LAUNCH_CHECK("step_bound");
    return SVP_OK;
}

extern "C" int svp_bb2_dots(const double *theta, const double *theta_old, const double *g, const double *g_old,
                            const double *p_old, const double *pvec, int64_t n, double *out4, void *stream) {
    SVP_REQUIRE(theta && theta_old && g && g_old && p_old && pvec && out4 && n >= 0, "svp_bb2_dots: invalid");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = blocks_for(n, 256, 4);
    dd *part = nullptr;
    SVP_CUDA(scratch_alloc((void **)&part, sizeof(dd) * 4 * nb + 4 * sizeof(double), s));
    double *res = (double *)(part + 4 * nb);
    SVP_LAUNCH_KEEP(bb2_kernel<<<nb, 256, 0, s>>>(theta, theta_old, g, g_old, p_old, pvec, n, part));
    SVP_LAUNCH_KEEP(multi_final_kernel<<<1, 256, 0, s>>>(part, nb, 4, res));
    cudaError_t le = cudaGetLastError();
    double host[4];
    cudaError_t ce = cudaMemcpyAsync(host, res, sizeof host, cudaMemcpyDeviceToHost, s);
    cudaError_t fe = scratch_free(part, s);
    if (le != cudaSuccess) return cuda_fail(le, "bb2 kernels");
    if (ce != cudaSuccess) return cuda_fail(ce, "bb2 copy");
    if (fe != cudaSuccess) return cuda_fail(fe, "bb2 free");
    SVP_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < 4; k++) out4[k] = host[k];
    return SVP_OK;
}

extern "C" int svp_max_abs_diff(const double *a, const double *b, int64_t n, double *out2, void *stream) {
    SVP_REQUIRE(a && b && out2 && n >= 0, "svp_max_abs_diff: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    long long *keys = nullptr;
    SVP_CUDA(scratch_alloc((void **)&keys, 2 * sizeof(long long), s));
    cudaError_t e0 = cudaMemsetAsync(keys, 0, 2 * sizeof(long long), s);
    SVP_LAUNCH_KEEP(max_abs_diff_kernel<<<blocks_for(n, 256, 8), 256, 0, s>>>(a, b, n, keys));
    cudaError_t le = cudaGetLastError();
    long long host[2] = {0, 0};
    cudaError_t ce = cudaMemcpyAsync(host, keys, sizeof host, cudaMemcpyDeviceToHost, s);
    cudaError_t fe = scratch_free(keys, s);
    if (e0 != cudaSuccess) return cuda_fail(e0, "max abs init");
    if (le != cudaSuccess) return cuda_fail(le, "max_abs_diff_kernel");
    if (ce != cudaSuccess) return cuda_fail(ce, "max abs copy");
    if (fe != cudaSuccess) return cuda_fail(fe, "max abs free");
    SVP_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < 2; k++) memcpy(&out2[k], &host[k], sizeof(double));
    return SVP_OK;
}

extern "C" int svp_dot(const double *a, const double *b, int64_t n, double *out, void *stream) {
    SVP_REQUIRE(a && b && out && n >= 0, "svp_dot: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned nb = blocks_for(n, 256, 4);
    dd *part = nullptr;
    SVP_CUDA(scratch_alloc((void **)&part, sizeof(dd) * nb + sizeof(double), s));
    double *res = (double *)(part + nb);
    SVP_LAUNCH_KEEP(dot_kernel<<<nb, 256, 0, s>>>(a, b, n, part));
    SVP_LAUNCH_KEEP(dot_final_kernel<<<1, 256, 0, s>>>(part, nb, res));
    cudaError_t le = cudaGetLastError();
    double host = 0.;
    cudaError_t ce = cudaMemcpyAsync(&host, res, sizeof host, cudaMemcpyDeviceToHost, s);
    cudaError_t fe = scratch_free(part, s);
    if (le != cudaSuccess) return cuda_fail(le, "dot kernels");
    if (ce != cudaSuccess) return cuda_fail(ce, "dot copy");
    if (fe != cudaSuccess) return cuda_fail(fe, "dot free");
    SVP_CUDA(cudaStreamSynchronize(s));
    *out = host;
    return SVP_OK;
}

extern "C" int svp_axpy(const double *x, double tau, const double *pvec, int64_t n, double *y, void *stream) {
    SVP_REQUIRE(x && pvec && y && n >= 0, "svp_axpy: invalid argument");
    if (!n) return SVP_OK;
    SVP_LAUNCH(axpy_kernel<<<blocks_for(n, 256, 8), 256, 0, (cudaStream_t)stream>>>(x, tau, pvec, n, y));
    SVP_LAUNCH_CHECK("axpy_kernel");
    return SVP_OK;
}

extern "C" int svp_inject(const svp_grid *g, const double *theta, double *u, void *stream) {
    SVP_REQUIRE(grid_ok(g) && theta && u, "svp_inject: invalid argument");
    SVP_LAUNCH(inject_kernel<<<blocks_for(n_nodes(g), 256, 8), 256, 0, (cudaStream_t)stream>>>(g->nx, g->ny, g->nz, theta, u));
    SVP_LAUNCH_CHECK("inject_kernel");
    return SVP_OK;
}

extern "C" int svp_restrict(const svp_grid *g, const double *field, double *theta, void *stream) {
    SVP_REQUIRE(grid_ok(g) && field && theta, "svp_restrict: invalid argument");
    SVP_LAUNCH(restrict_kernel<<<blocks_for(n_free(g), 256, 8), 256, 0, (cudaStream_t)stream>>>(g->nx, g->ny, g->nz, field,
                                                                                      theta));
    SVP_LAUNCH_CHECK("restrict_kernel");
    return SVP_OK;
}

extern "C" int svp_step_bound(const svp_grid *g, const double *u, const double *pvec, double *bound, void *stream) {
    SVP_REQUIRE(grid_ok(g) && u && pvec && bound, "svp_step_bound: invalid argument");
    cudaStream_t s = (cudaStream_t)stream;
    long long *best = nullptr;
    SVP_CUDA(scratch_alloc((void **)&best, sizeof(long long), s));
    long long init = kKeyPosInf, host = 0;
    cudaError_t e1 = cudaMemcpyAsync(best, &init, sizeof init, cudaMemcpyHostToDevice, s);
    SVP_LAUNCH_KEEP(step_bound_kernel<<<blocks_for(n_free(g), 256, 8), 256, 0, s>>>(g->nx, g->ny, g->nz, g->hx, g->hy, g->hz, g->x0,
                                                                    g->y0, g->z0, u, pvec, best));
    cudaError_t le = cudaGetLastError();
    cudaError_t e2 = cudaMemcpyAsync(&host, best, sizeof host, cudaMemcpyDeviceToHost, s);
    cudaError_t e3 = scratch_free(best, s);
    if (e1 != cudaSuccess) return cuda_fail(e1, "step bound init");
    if (le != cudaSuccess) return cuda_fail(le, "step_bound_kernel");
    if (e2 != cudaSuccess) return cuda_fail(e2, "step bound copy");
    if (e3 != cudaSuccess) return cuda_fail(e3, "step bound free");
    SVP_CUDA(cudaStreamSynchronize(s));
    *bound = key_value(host);
    return SVP_OK;
}
