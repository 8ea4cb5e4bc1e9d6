// Dense per-axis transforms of (batch, nz, ny, nx) float64 fields: the orthonormal DST-I of the Q1 Poisson metric
// (jd_curl/three_d/poisson.py:99, scipy dstn type=1 norm='ortho') and the not-a-knot spline prefilter
// (interpolation.py:29).  Each axis pass is a batched GEMM with a small square matrix.
#include <cmath>
#include <vector>

#include "pair.cuh"

namespace svp {
namespace {

constexpr int TM = 64, TN = 64, TK = 16;  // output tile 64 x 64, K step 16, 256 threads x (4 x 4) outputs

// C[b][i][w] = sum_j M[i][j] X[b][j][w]  (M: n x n row-major; X rows of length W with stride ldx, batch stride bs)
__global__ void __launch_bounds__(256) gemm_left_kernel(const double *__restrict__ M, int n,
                                                        const double *__restrict__ X, long long W, long long ldx,
                                                        long long bs, double *__restrict__ C) {
    __shared__ double sM[TK][TM + 1];
    __shared__ double sX[TK][TN];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const long long b = blockIdx.z;
    const int i0 = blockIdx.y * TM;
    const long long w0 = (long long)blockIdx.x * TN;
    const double *Xb = X + b * bs;
    double *Cb = C + b * bs;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < n; k0 += TK) {
        for (int e = threadIdx.x; e < TK * TM; e += 256) {
            int kk = e % TK, ii = e / TK;
            int i = i0 + ii, k = k0 + kk;
            sM[kk][ii] = (i < n && k < n) ? M[(long long)i * n + k] : 0.;
        }
        for (int e = threadIdx.x; e < TK * TN; e += 256) {
            int ww = e % TN, kk = e / TN;
            long long w = w0 + ww;
            int k = k0 + kk;
            sX[kk][ww] = (k < n && w < W) ? Xb[(long long)k * ldx + w] : 0.;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk++) {
            double a[4], x[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = sM[kk][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; c++) x[c] = sX[kk][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[r][c] = fma(a[r], x[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        int i = i0 + ty + 16 * r;
        if (i >= n) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            long long w = w0 + tx + 16 * c;
            if (w < W) Cb[(long long)i * ldx + w] = acc[r][c];
        }
    }
}

// C[r][i] = sum_j X[r][j] M[i][j]  (rows of length n, contiguous; R rows)
__global__ void __launch_bounds__(256) gemm_right_kernel(const double *__restrict__ M, int n,
                                                         const double *__restrict__ X, long long R,
                                                         double *__restrict__ C) {
    __shared__ double sX[TK][TM + 1];
    __shared__ double sM[TK][TN + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const long long r0 = (long long)blockIdx.x * TM;
    const int i0 = blockIdx.y * TN;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < n; k0 += TK) {
        for (int e = threadIdx.x; e < TK * TM; e += 256) {
            int kk = e % TK, rr = e / TK;
            long long r = r0 + rr;
            int k = k0 + kk;
            sX[kk][rr] = (r < R && k < n) ? X[r * n + k] : 0.;
        }
        for (int e = threadIdx.x; e < TK * TN; e += 256) {
            int kk = e % TK, ii = e / TK;
            int i = i0 + ii, k = k0 + kk;
            sM[kk][ii] = (i < n && k < n) ? M[(long long)i * n + k] : 0.;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk++) {
            double a[4], m[4];
#pragma unroll
            for (int q = 0; q < 4; q++) a[q] = sX[kk][ty + 16 * q];
#pragma unroll
            for (int c = 0; c < 4; c++) m[c] = sM[kk][tx + 16 * c];
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[q][c] = fma(a[q], m[c], acc[q][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        long long r = r0 + ty + 16 * q;
        if (r >= R) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            int i = i0 + tx + 16 * c;
            if (i < n) C[r * n + i] = acc[q][c];
        }
    }
}

__global__ void scale_kernel(const double *__restrict__ x, const double *__restrict__ s, double sign, long long n,
                             double *__restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = s ? sign * (s[i] * x[i]) : sign * x[i];
}

__global__ void divide_kernel(double *__restrict__ x, const double *__restrict__ den, long long per, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] = x[i] / den[i % per];
}

__global__ void den_kernel(double *__restrict__ den, long long f0, long long f1, long long f2,
                           const double *__restrict__ ex, const double *__restrict__ ey, const double *__restrict__ ez,
                           const double *__restrict__ mx, const double *__restrict__ my, const double *__restrict__ mz,
                           double omega, double a, double b, int metric) {
    long long n = f0 * f1 * f2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        long long x = i % f0, y = (i / f0) % f1, z = i / (f0 * f1);
        double lam = metric == 1 ? (ex[x] + ey[y]) + ez[z]
                                 : ((ex[x] * my[y]) * mz[z] + (mx[x] * ey[y]) * mz[z]) + (mx[x] * my[y]) * ez[z];
        den[i] = omega * (a + b * lam);
    }
}

}  // namespace

// Apply the n x n matrix M along one axis of `batch` fields of dims (n2, n1, n0) (z, y, x); in and out distinct.
int apply_axis(const double *M, int axis, long long batch, long long n2, long long n1, long long n0,
               const double *in, double *out, cudaStream_t s) {
    if (axis == 0) {
        long long R = batch * n2 * n1;
        dim3 grid((unsigned)div_up(R, TM), (unsigned)div_up(n0, TN));
        { svp::KernelTimer _t("gemm_right_kernel", s); SVP_LAUNCH(gemm_right_kernel<<<grid, 256, 0, s>>>(M, (int)n0, in, R, out)); }
    } else if (axis == 1) {
        dim3 grid((unsigned)div_up(n0, TN), (unsigned)div_up(n1, TM), (unsigned)(batch * n2));
        { svp::KernelTimer _t("gemm_left_kernel", s); SVP_LAUNCH(gemm_left_kernel<<<grid, 256, 0, s>>>(M, (int)n1, in, n0, n0, n1 * n0, out)); }
    } else {
        dim3 grid((unsigned)div_up(n1 * n0, TN), (unsigned)div_up(n2, TM), (unsigned)batch);
        { svp::KernelTimer _t("gemm_left_kernel", s); SVP_LAUNCH(gemm_left_kernel<<<grid, 256, 0, s>>>(M, (int)n2, in, n1 * n0, n1 * n0, n2 * n1 * n0, out)); }
    }
    SVP_LAUNCH_CHECK("axis GEMM");
    return SVP_OK;
}

// Orthonormal DST-I matrix S[j][k] = sqrt(2/(n+1)) sin(pi (j+1)(k+1)/(n+1)), evaluated in long double.
std::vector<double> dst1_matrix(int n) {
    std::vector<double> S((size_t)n * n);
    const long double pi = 3.141592653589793238462643383279502884L;
    const long double c = sqrtl(2.0L / (n + 1));
    for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) {
            long long m = ((long long)(j + 1) * (k + 1)) % (2LL * (n + 1));
            S[(size_t)j * n + k] = (double)(c * sinl(pi * (long double)m / (long double)(n + 1)));
        }
    return S;
}

int pair_dst_setup(svp_pair *p) {
    const long long f[3] = {p->q.fx, p->q.fy, p->q.fz};
    for (int k = 0; k < 3; k++) {
        std::vector<double> S = dst1_matrix((int)f[k]);
        SVP_CUDA(cudaMalloc((void **)&p->dst_mat[k], sizeof(double) * S.size()));
        SVP_CUDA(cudaMemcpy(p->dst_mat[k], S.data(), sizeof(double) * S.size(), cudaMemcpyHostToDevice));
    }
    SVP_CUDA(cudaMalloc((void **)&p->dst_tmp, sizeof(double) * 2 * 3 * p->q.nfree));
    SVP_CUDA(cudaMalloc((void **)&p->den, sizeof(double) * p->q.nfree));
    return SVP_OK;
}

// poisson.py:16 poisson_spectrum per axis: ell = (2 sin(theta/2)/h)^2, mass = (2 + cos theta)/3,
// theta = pi k/(n-1), k = 1..n-2 (host, double, the reference's expressions).
static int set_denominator(svp_pair *p, double a, double b, int metric, cudaStream_t s) {
    if (p->den_a == a && p->den_b == b && p->den_metric == metric) return SVP_OK;
    const long long nn[3] = {p->q.nx, p->q.ny, p->q.nz};
    std::vector<double> host;
    long long off[7] = {0};
    for (int k = 0; k < 3; k++) off[k + 1] = off[k] + (nn[k] - 2);
    for (int k = 0; k < 3; k++) off[k + 4] = off[k + 3] + (nn[k] - 2);
    host.resize((size_t)off[6]);
    const double pi = 3.141592653589793;
    for (int k = 0; k < 3; k++) {
        long long n = nn[k];
        for (long long i = 1; i < n - 1; i++) {
            double theta = pi * (double)i / (double)(n - 1);
            double e = 2 * sin(theta / 2) / p->q.h[k];
            host[off[k] + i - 1] = e * e;
            host[off[k + 3] + i - 1] = (2 + cos(theta)) / 3;
        }
    }
    double *dev = nullptr;
    SVP_CUDA(cudaMallocAsync((void **)&dev, sizeof(double) * host.size(), s));
    SVP_CUDA(cudaMemcpyAsync(dev, host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice, s));
    SVP_LAUNCH(den_kernel<<<blocks_for(p->q.nfree, 256, 8), 256, 0, s>>>(p->den, p->q.fx, p->q.fy, p->q.fz, dev + off[0],
                                                              dev + off[1], dev + off[2], dev + off[3], dev + off[4],
                                                              dev + off[5], p->q.omega, a, b, metric));
    SVP_LAUNCH_CHECK("den_kernel");
    SVP_CUDA(cudaFreeAsync(dev, s));
    p->den_a = a;
    p->den_b = b;
    p->den_metric = metric;
    return SVP_OK;
}

}  // namespace svp

using namespace svp;

extern "C" int svp_poisson_apply(svp_pair *p, double a, double b, int32_t metric, const double *scale,
                                 const double *rhs, double sign, double *out, void *stream) {
    SVP_REQUIRE(p && rhs && out, "svp_poisson_apply: null argument");
    SVP_REQUIRE(metric == 0 || metric == 1, "svp_poisson_apply: metric 0 (q1) or 1 (seven_point)");
    SVP_REQUIRE(std::isfinite(a) && a >= 0 && std::isfinite(b) && b > 0, "svp_poisson_apply: a >= 0, b > 0");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = set_denominator(p, a, b, metric, s);
    if (rc) return rc;
    const long long nf = p->q.nfree, n3 = 3 * nf;
    const long long f0 = p->q.fx, f1 = p->q.fy, f2 = p->q.fz;
    double *t0 = p->dst_tmp, *t1 = p->dst_tmp + n3;
    unsigned eb = blocks_for(n3, 256, 8);
    SVP_LAUNCH(scale_kernel<<<eb, 256, 0, s>>>(rhs, scale, 1., n3, t0));
    SVP_LAUNCH_CHECK("scale_kernel");
    if ((rc = apply_axis(p->dst_mat[0], 0, 3, f2, f1, f0, t0, t1, s))) return rc;
    if ((rc = apply_axis(p->dst_mat[1], 1, 3, f2, f1, f0, t1, t0, s))) return rc;
    if ((rc = apply_axis(p->dst_mat[2], 2, 3, f2, f1, f0, t0, t1, s))) return rc;
    SVP_LAUNCH(divide_kernel<<<eb, 256, 0, s>>>(t1, p->den, nf, n3));
    if ((rc = apply_axis(p->dst_mat[0], 0, 3, f2, f1, f0, t1, t0, s))) return rc;
    if ((rc = apply_axis(p->dst_mat[1], 1, 3, f2, f1, f0, t0, t1, s))) return rc;
    if ((rc = apply_axis(p->dst_mat[2], 2, 3, f2, f1, f0, t1, t0, s))) return rc;
    SVP_LAUNCH(scale_kernel<<<eb, 256, 0, s>>>(t0, scale, sign, n3, out));
    SVP_LAUNCH_CHECK("scale_kernel");
    return SVP_OK;
}
