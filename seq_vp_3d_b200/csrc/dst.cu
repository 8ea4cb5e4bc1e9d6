// Dense per-axis transforms of (batch, nz, ny, nx) float64 fields: the orthonormal DST-I of the Q1 Poisson metric
// (jd_curl/three_d/poisson.py:99, scipy dstn type=1 norm='ortho') and the not-a-knot spline prefilter
// (interpolation.py:29).  Each axis pass is a batched GEMM with a small square matrix.
#include <cmath>
#include <map>
#include <mutex>
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

// ------------------------------------------------------------------------------------------- DST-I passes
// The orthonormal DST-I matrix is centro-symmetric along columns: S[i][n-1-k] = (-1)^i S[i][k] (0-indexed).  So
// output rows of one parity need only half the columns, against the folded input u_k = x_k + x_(n-1-k) (even i;
// u_mid = x_mid when n is odd) or v_k = x_k - x_(n-1-k) (odd i): half the FLOPs of the dense product.  The folded
// half matrices are stored per parity, H0 (ceil(n/2) x ceil(n/2)) then H1 (floor(n/2) x floor(n/2)), row-major.
// FP64 tensor-core product D = A B + D on one 8x8x4 tile (mma.sync m8n8k4 f64): lane (g = lane / 4, t = lane % 4)
// holds A[g][t], B[t][g] and D[g][2t], D[g][2t + 1].  FP64 has no tcgen05 kind on sm_100a; this is B200's FP64
// tensor path, one instruction per 256 fused multiply-adds.
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// The mixed form's passes: float32 operands on the tensor cores as 3xTF32 (mma.sync m16n8k8 .tf32, float32
// accumulate).  Each operand x splits into big = tf32(x) and small = tf32(x - big); the product sums
// small*big + big*small + big*big, which keeps float32-level accuracy (the small*small term is below float32
// rounding).  Fragment layout of m16n8k8 (lane: gid = lane / 4, tig = lane % 4): A a0 = A[gid][tig],
// a1 = A[gid + 8][tig], a2 = A[gid][tig + 4], a3 = A[gid + 8][tig + 4]; B b0 = B[tig][gid], b1 = B[tig + 4][gid];
// D d0, d1 = D[gid][2 tig + {0, 1}], d2, d3 = D[gid + 8][2 tig + {0, 1}].
__device__ __forceinline__ unsigned tf32_of(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void tf32_split(float x, unsigned &big, unsigned &small) {
    big = tf32_of(x);
    small = tf32_of(x - __uint_as_float(big));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The float64 half matrices of one axis (the plain form's passes; the mixed form's are HalfTf32 below).
struct HalfDst {
    const double *h0, *h1;
    int n, k0, k1;     // n, ceil(n/2), floor(n/2)
};
// Tile product of one K block held in shared memory on the FP64 tensor path: 8 warps x 16 x 32 outputs, 2 x 4 DMMA
// 8x8x4 tiles per warp (A fragments from sA[k][row], B from sB[k][col]).
__device__ __forceinline__ void tile_product(const double (*sA)[TM + 4], const double (*sB)[TN + 4], int lane,
                                             int warp, double (&dacc)[2][4][2]) {
    const int gid = lane >> 2, tig = lane & 3;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
#pragma unroll
    for (int kb = 0; kb < TK; kb += 4) {
        double a[2], x[4];
#pragma unroll
        for (int fr = 0; fr < 2; fr++) a[fr] = sA[kb + tig][wr + 8 * fr + gid];
#pragma unroll
        for (int fc = 0; fc < 4; fc++) x[fc] = sB[kb + tig][wc + 8 * fc + gid];
#pragma unroll
        for (int fr = 0; fr < 2; fr++)
#pragma unroll
            for (int fc = 0; fc < 4; fc++) dmma_8x8x4(dacc[fr][fc], a[fr], x[fc]);
    }
}

// One K block of the folded operand: the raw pair (x_k, x_(n-1-k)) of each of a thread's 4 entries is fetched into
// registers one block ahead (the loads fly while the previous block's products run) and folded when it is stored
// to shared memory.  fold = x_k (middle row of odd n), x_k + x_m (parity 0) or x_k - x_m (parity 1), formed in
// float64 (with the optional pre-scale) and rounded once to the pass's type; entries outside the operand are +0.
template <class TC>
__device__ __forceinline__ TC fold_value(double xa, double xb, bool mid, int g) {
    return (TC)(mid ? xa : (g ? xa - xb : xa + xb));
}

// Left pass: C[b][i][w] = sum_k S[i][k] X[b][k][w] (rows of length W, stride ldx, batch stride bs).  blockIdx.x
// enumerates the 64-row tiles of parity 0, then of parity 1 (the blocks that read the same X run together).  EPI 1
// divides by den[flat % per], EPI 2 multiplies by sign * post[flat] (the same operation order as the separate
// elementwise passes).  Two shared-memory buffers: block k + 1 is stored while block k is multiplied.
template <int EPI, class TI, class TO>
__global__ void __launch_bounds__(256) dst_left_kernel(HalfDst D, const TI *__restrict__ X, long long W,
                                                       long long ldx, long long bs, TO *__restrict__ C,
                                                       const double *__restrict__ den, long long per,
                                                       const double *__restrict__ post, double sign) {
    __shared__ double sM[2][TK][TM + 4];
    __shared__ double sX[2][TK][TN + 4];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;   // a warp's 16 x 32 block of the 64 x 64 tile
    double dacc[2][4][2] = {};
    const int t0 = (D.k0 + TM - 1) / TM;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int rows = g ? D.k1 : D.k0, K = rows;
    const double *H = g ? D.h1 : D.h0;
    const int i0 = (g ? (int)blockIdx.x - t0 : (int)blockIdx.x) * TM;
    const long long b = blockIdx.z;
    const long long w0 = (long long)blockIdx.y * TN;
    const TI *Xb = X + b * bs;
    double rm[4];
    double ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            {
                const int kk = e % TK, ii = e / TK, i = i0 + ii, k = k0 + kk;
                rm[t] = (i < rows && k < K) ? H[(long long)i * K + k] : 0.;
            }
            const int ww = e % TN, kk = e / TN, k = k0 + kk;
            const long long w = w0 + ww;
            const bool ok = k < K && w < W;
            ra[t] = ok ? (double)Xb[(long long)k * ldx + w] : 0.;
            rb[t] = ok ? (double)Xb[(long long)(D.n - 1 - k) * ldx + w] : 0.;
        }
    };
    auto stash = [&](int buf, int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            sM[buf][e % TK][e / TK] = rm[t];
            const int ww = e % TN, kk = e / TN, k = k0 + kk;
            sX[buf][kk][ww] = fold_value<double>(ra[t], rb[t], k == D.n - 1 - k, g);
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += TK) {
        const bool more = k0 + TK < K;
        if (more) fetch(k0 + TK);
        tile_product(sM[buf], sX[buf], lane, warp, dacc);
        if (more) stash(buf ^ 1, k0 + TK);
        __syncthreads();
        buf ^= 1;
    }
    auto store = [&](int ii, long long w, double v) {
        if (ii >= rows || w >= W) return;
        long long i = 2 * ii + g;
        long long o = b * bs + i * ldx + w;
        if (EPI == 1) v = v / den[o % per];
        if (EPI == 2) v = sign * (post[o] * v);
        C[o] = (TO)v;
    };
#pragma unroll
    for (int fr = 0; fr < 2; fr++)
#pragma unroll
        for (int fc = 0; fc < 4; fc++)
#pragma unroll
            for (int e = 0; e < 2; e++) store(i0 + wr + 8 * fr + gid, w0 + wc + 8 * fc + 2 * tig + e, dacc[fr][fc][e]);
}

// Right pass over contiguous rows of length n: C[r][i] = sum_k X[r][k] S[i][k]; pre (optional) scales X first.
template <class TI, class TO>
__global__ void __launch_bounds__(256) dst_right_kernel(HalfDst D, const TI *__restrict__ X, long long R,
                                                        const double *__restrict__ pre, TO *__restrict__ C) {
    __shared__ double sX[2][TK][TM + 4];
    __shared__ double sM[2][TK][TN + 4];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
    double dacc[2][4][2] = {};
    const int t0 = (D.k0 + TN - 1) / TN;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int cols = g ? D.k1 : D.k0, K = cols;
    const double *H = g ? D.h1 : D.h0;
    const int i0 = (g ? (int)blockIdx.x - t0 : (int)blockIdx.x) * TN;
    const long long r0 = (long long)blockIdx.y * TM;
    const int n = D.n;
    double rm[4];
    double ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            {
                const int kk = e % TK, rr = e / TK, k = k0 + kk;
                const long long r = r0 + rr;
                const bool ok = r < R && k < K;
                const long long a = r * n + k, m = r * n + (n - 1 - k);
                ra[t] = ok ? (pre ? pre[a] * (double)X[a] : (double)X[a]) : 0.;
                rb[t] = ok ? (pre ? pre[m] * (double)X[m] : (double)X[m]) : 0.;
            }
            const int kk = e % TK, ii = e / TK, i = i0 + ii, k = k0 + kk;
            rm[t] = (i < cols && k < K) ? H[(long long)i * K + k] : 0.;
        }
    };
    auto stash = [&](int buf, int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            const int kk = e % TK, k = k0 + kk;
            sX[buf][kk][e / TK] = fold_value<double>(ra[t], rb[t], k == n - 1 - k, g);
            sM[buf][kk][e / TK] = rm[t];
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += TK) {
        const bool more = k0 + TK < K;
        if (more) fetch(k0 + TK);
        tile_product(sX[buf], sM[buf], lane, warp, dacc);
        if (more) stash(buf ^ 1, k0 + TK);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int fr = 0; fr < 2; fr++)
#pragma unroll
        for (int fc = 0; fc < 4; fc++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const long long r = r0 + wr + 8 * fr + gid;
                const int ii = i0 + wc + 8 * fc + 2 * tig + e;
                if (r < R && ii < cols) C[r * n + 2 * ii + g] = (TO)dacc[fr][fc][e];
            }
}

// ---------------------------------------------------------------------------------------- mixed form (3xTF32)
// The float32 passes keep each operand as its two TF32 parts in shared memory: the half matrices are split once per
// grid (split_half_kernel), the folded fields once when a K block is staged, so a fragment is loaded, never split.
// Rows of the staged blocks are padded to TM + 8 words: the fragment loads (rows tig, tig + 4 x columns gid) fall in
// 32 distinct banks.  The products are those of the per-fragment split (same parts, same mma order), bitwise.
constexpr int TP = TM + 8;

struct HalfTf32 {
    const unsigned *b0, *s0, *b1, *s1;   // parity 0 / 1, big / small parts, each k_g x k_g with T[k][a] = H_g[a][k]
    int n, k0, k1;
};

// h: H0 (k0 x k0) then H1 (k1 x k1), row-major float32; out: the big parts of H0^T, H1^T, then the small parts.
__global__ void split_half_kernel(const float *__restrict__ h, int k0, int k1, unsigned *__restrict__ out) {
    const long long n0 = (long long)k0 * k0, total = n0 + (long long)k1 * k1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const bool odd = e >= n0;
        const int kg = odd ? k1 : k0;
        const long long l = odd ? e - n0 : e;
        const long long t = (odd ? n0 : 0) + (l % kg) * kg + l / kg;
        unsigned big, small;
        tf32_split(h[e], big, small);
        out[t] = big;
        out[total + t] = small;
    }
}

// One K block: 8 warps x 16 x 32 outputs, facc[fc] rows gid and gid + 8 of n-tile fc (m16n8k8 layout).
__device__ __forceinline__ void tf32_tile_product(const unsigned (*Ab)[TP], const unsigned (*As)[TP],
                                                  const unsigned (*Bb)[TP], const unsigned (*Bs)[TP], int lane,
                                                  int warp, float (&facc)[4][4]) {
    const int gid = lane >> 2, tig = lane & 3;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
#pragma unroll
    for (int kb = 0; kb < TK; kb += 8) {
        const unsigned ab[4] = {Ab[kb + tig][wr + gid], Ab[kb + tig][wr + gid + 8], Ab[kb + tig + 4][wr + gid],
                                Ab[kb + tig + 4][wr + gid + 8]};
        const unsigned as[4] = {As[kb + tig][wr + gid], As[kb + tig][wr + gid + 8], As[kb + tig + 4][wr + gid],
                                As[kb + tig + 4][wr + gid + 8]};
#pragma unroll
        for (int fc = 0; fc < 4; fc++) {
            const int col = wc + 8 * fc + gid;
            const unsigned b0b = Bb[kb + tig][col], b0s = Bs[kb + tig][col];
            const unsigned b1b = Bb[kb + tig + 4][col], b1s = Bs[kb + tig + 4][col];
            mma_tf32(facc[fc], as, b0b, b1b);
            mma_tf32(facc[fc], ab, b0s, b1s);
            mma_tf32(facc[fc], ab, b0b, b1b);
        }
    }
}

// Left pass in float32 (see dst_left_kernel): A = H_g from its split parts, B = the folded field split on staging.
template <int EPI, class TI, class TO>
__global__ void __launch_bounds__(256) dst_left_tf32_kernel(HalfTf32 D, const TI *__restrict__ X, long long W,
                                                            long long ldx, long long bs, TO *__restrict__ C,
                                                            const double *__restrict__ den, long long per,
                                                            const double *__restrict__ post, double sign) {
    __shared__ unsigned sAb[2][TK][TP], sAs[2][TK][TP], sBb[2][TK][TP], sBs[2][TK][TP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
    const int t0 = (D.k0 + TM - 1) / TM;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int rows = g ? D.k1 : D.k0, K = rows;
    const unsigned *Hb = g ? D.b1 : D.b0, *Hs = g ? D.s1 : D.s0;
    const int i0 = (g ? (int)blockIdx.x - t0 : (int)blockIdx.x) * TM;
    const long long b = blockIdx.z;
    const long long w0 = (long long)blockIdx.y * TN;
    const TI *Xb = X + b * bs;
    float facc[4][4] = {};
    unsigned rhb[4], rhs[4];
    double ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            {
                const int ii = e % TM, kk = e / TM, i = i0 + ii, k = k0 + kk;
                const bool ok = i < rows && k < K;
                rhb[t] = ok ? Hb[(long long)k * rows + i] : 0u;
                rhs[t] = ok ? Hs[(long long)k * rows + i] : 0u;
            }
            const int ww = e % TN, kk = e / TN, k = k0 + kk;
            const long long w = w0 + ww;
            const bool ok = k < K && w < W;
            ra[t] = ok ? (double)Xb[(long long)k * ldx + w] : 0.;
            rb[t] = ok ? (double)Xb[(long long)(D.n - 1 - k) * ldx + w] : 0.;
        }
    };
    auto stash = [&](int buf, int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            sAb[buf][e / TM][e % TM] = rhb[t];
            sAs[buf][e / TM][e % TM] = rhs[t];
            const int ww = e % TN, kk = e / TN, k = k0 + kk;
            unsigned big, small;
            tf32_split(fold_value<float>(ra[t], rb[t], k == D.n - 1 - k, g), big, small);
            sBb[buf][kk][ww] = big;
            sBs[buf][kk][ww] = small;
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += TK) {
        const bool more = k0 + TK < K;
        if (more) fetch(k0 + TK);
        tf32_tile_product(sAb[buf], sAs[buf], sBb[buf], sBs[buf], lane, warp, facc);
        if (more) stash(buf ^ 1, k0 + TK);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int fc = 0; fc < 4; fc++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int ii = i0 + wr + gid + 8 * (e >> 1);
            const long long w = w0 + wc + 8 * fc + 2 * tig + (e & 1);
            if (ii >= rows || w >= W) continue;
            const long long o = b * bs + (long long)(2 * ii + g) * ldx + w;
            double v = (double)facc[fc][e];
            if (EPI == 1) v = v / den[o % per];
            if (EPI == 2) v = sign * (post[o] * v);
            C[o] = (TO)v;
        }
}

// Right pass in float32 (see dst_right_kernel): A = the folded rows split on staging, B = H_g^T from its parts.
template <class TI, class TO>
__global__ void __launch_bounds__(256) dst_right_tf32_kernel(HalfTf32 D, const TI *__restrict__ X, long long R,
                                                             const double *__restrict__ pre, TO *__restrict__ C) {
    __shared__ unsigned sAb[2][TK][TP], sAs[2][TK][TP], sBb[2][TK][TP], sBs[2][TK][TP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
    const int t0 = (D.k0 + TN - 1) / TN;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int cols = g ? D.k1 : D.k0, K = cols;
    const unsigned *Hb = g ? D.b1 : D.b0, *Hs = g ? D.s1 : D.s0;
    const int i0 = (g ? (int)blockIdx.x - t0 : (int)blockIdx.x) * TN;
    const long long r0 = (long long)blockIdx.y * TM;
    const int n = D.n;
    float facc[4][4] = {};
    unsigned rhb[4], rhs[4];
    double ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            {
                const int kk = e % TK, rr = e / TK, k = k0 + kk;
                const long long r = r0 + rr;
                const bool ok = r < R && k < K;
                const long long a = r * n + k, m = r * n + (n - 1 - k);
                ra[t] = ok ? (pre ? pre[a] * (double)X[a] : (double)X[a]) : 0.;
                rb[t] = ok ? (pre ? pre[m] * (double)X[m] : (double)X[m]) : 0.;
            }
            const int ii = e % TN, kk = e / TN, i = i0 + ii, k = k0 + kk;
            const bool ok = i < cols && k < K;
            rhb[t] = ok ? Hb[(long long)k * cols + i] : 0u;
            rhs[t] = ok ? Hs[(long long)k * cols + i] : 0u;
        }
    };
    auto stash = [&](int buf, int k0) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int e = threadIdx.x + 256 * t;
            const int kk = e % TK, k = k0 + kk;
            unsigned big, small;
            tf32_split(fold_value<float>(ra[t], rb[t], k == n - 1 - k, g), big, small);
            sAb[buf][kk][e / TK] = big;
            sAs[buf][kk][e / TK] = small;
            sBb[buf][e / TN][e % TN] = rhb[t];
            sBs[buf][e / TN][e % TN] = rhs[t];
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += TK) {
        const bool more = k0 + TK < K;
        if (more) fetch(k0 + TK);
        tf32_tile_product(sAb[buf], sAs[buf], sBb[buf], sBs[buf], lane, warp, facc);
        if (more) stash(buf ^ 1, k0 + TK);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int fc = 0; fc < 4; fc++)
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const long long r = r0 + wr + gid + 8 * (e >> 1);
            const int ii = i0 + wc + 8 * fc + 2 * tig + (e & 1);
            if (r < R && ii < cols) C[r * n + 2 * ii + g] = (TO)facc[fc][e];
        }
}

__global__ void scale_kernel(const double *__restrict__ x, const double *__restrict__ s, double sign, long long n,
                             double *__restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = s ? sign * (s[i] * x[i]) : sign * x[i];
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

std::vector<double> dst1_matrix(int n);

// One DST-I pass along `axis` of (3, n2, n1, n0) fields with the folded half matrices; see dst_left_kernel for
// pre / EPI.
template <class TC, class TI, class TO>
static int dst_pass(const svp_pair *p, int axis, const TI *in, TO *out, const double *pre, int epi, double sign,
                    const double *post, cudaStream_t s) {
    const long long n0 = p->q.fx, n1 = p->q.fy, n2 = p->q.fz;
    const int n = p->dst_n[axis], k0 = (n + 1) / 2, k1 = n / 2;
    const unsigned tiles = (unsigned)(div_up(k0, TM) + div_up(k1, TM));
    const long long nf = p->q.nfree;
    constexpr bool kDouble = sizeof(TC) == 8;
    HalfDst D{p->dst_half[axis], p->dst_half[axis] + (size_t)k0 * k0, n, k0, k1};
    const unsigned *t = p->dst_tf32[axis];
    const long long tot = (long long)k0 * k0 + (long long)k1 * k1;
    HalfTf32 T{t, t + tot, t + (long long)k0 * k0, t + tot + (long long)k0 * k0, n, k0, k1};
    if (axis == 0) {
        SVP_REQUIRE(epi == 0, "dst_pass: x pass has no epilogue");
        long long R = 3 * n2 * n1;
        dim3 grid(tiles, (unsigned)div_up(R, TM));      // the blocks that share rows run together (L2 reuse)
        svp::KernelTimer _t("dst_right_kernel", s);
        if constexpr (kDouble) SVP_LAUNCH((dst_right_kernel<TI, TO><<<grid, 256, 0, s>>>(D, in, R, pre, out)));
        else SVP_LAUNCH((dst_right_tf32_kernel<TI, TO><<<grid, 256, 0, s>>>(T, in, R, pre, out)));
    } else {
        SVP_REQUIRE(!pre, "dst_pass: pre-scale only on the x pass");
        long long W = axis == 1 ? n0 : n1 * n0;
        long long ldx = W, bs = axis == 1 ? n1 * n0 : n2 * n1 * n0;
        dim3 grid(tiles, (unsigned)div_up(W, TN), (unsigned)(axis == 1 ? 3 * n2 : 3));
        svp::KernelTimer _t("dst_left_kernel", s);
        if constexpr (kDouble) {
            if (epi == 0) SVP_LAUNCH((dst_left_kernel<0, TI, TO><<<grid, 256, 0, s>>>(D, in, W, ldx, bs, out, nullptr, 1, nullptr, 1.)));
            else if (epi == 1) SVP_LAUNCH((dst_left_kernel<1, TI, TO><<<grid, 256, 0, s>>>(D, in, W, ldx, bs, out, p->den, nf, nullptr, 1.)));
            else SVP_LAUNCH((dst_left_kernel<2, TI, TO><<<grid, 256, 0, s>>>(D, in, W, ldx, bs, out, nullptr, 1, post, sign)));
        } else {
            if (epi == 0) SVP_LAUNCH((dst_left_tf32_kernel<0, TI, TO><<<grid, 256, 0, s>>>(T, in, W, ldx, bs, out, nullptr, 1, nullptr, 1.)));
            else if (epi == 1) SVP_LAUNCH((dst_left_tf32_kernel<1, TI, TO><<<grid, 256, 0, s>>>(T, in, W, ldx, bs, out, p->den, nf, nullptr, 1.)));
            else SVP_LAUNCH((dst_left_tf32_kernel<2, TI, TO><<<grid, 256, 0, s>>>(T, in, W, ldx, bs, out, nullptr, 1, post, sign)));
        }
    }
    SVP_LAUNCH_CHECK("dst pass");
    return SVP_OK;
}

// Folded half matrices of the orthonormal DST-I (see HalfDst): H_g[a][k] = S[2a + g][k], k < ceil(n/2) (g = 0) or
// floor(n/2) (g = 1).
std::vector<double> dst1_half(int n) {
    std::vector<double> S = dst1_matrix(n);
    const int k0 = (n + 1) / 2, k1 = n / 2;
    std::vector<double> H((size_t)k0 * k0 + (size_t)k1 * k1);
    for (int a = 0; a < k0; a++)
        for (int k = 0; k < k0; k++) H[(size_t)a * k0 + k] = S[(size_t)(2 * a) * n + k];
    double *H1 = H.data() + (size_t)k0 * k0;
    for (int a = 0; a < k1; a++)
        for (int k = 0; k < k1; k++) H1[(size_t)a * k1 + k] = S[(size_t)(2 * a + 1) * n + k];
    return H;
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

// The folded matrices depend only on n; registrations on one grid share them (n^2 long double sines per axis).
static std::vector<double> cached_dst1_half(int n) {
    static std::mutex mu;
    static std::map<int, std::vector<double>> cache;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(n);
        if (it != cache.end()) return it->second;
    }
    std::vector<double> H = dst1_half(n);
    std::lock_guard<std::mutex> lock(mu);
    if (cache.size() >= 32) cache.clear();
    cache.emplace(n, H);
    return H;
}

int pair_dst_setup(svp_pair *p) {
    const long long f[3] = {p->q.fx, p->q.fy, p->q.fz};
    for (int k = 0; k < 3; k++) {
        std::vector<double> H = cached_dst1_half((int)f[k]);
        SVP_CUDA(cudaMalloc((void **)&p->dst_half[k], sizeof(double) * H.size()));
        SVP_CUDA(cudaMemcpy(p->dst_half[k], H.data(), sizeof(double) * H.size(), cudaMemcpyHostToDevice));
        // the mixed form's matrices: rounded once to float32, then split into TF32 parts on the device (the same
        // cvt.rna the passes use for their staged operands)
        std::vector<float> H32(H.begin(), H.end());
        float *h32 = nullptr;
        SVP_CUDA(cudaMalloc((void **)&h32, sizeof(float) * H32.size()));
        cudaError_t e = cudaMemcpy(h32, H32.data(), sizeof(float) * H32.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc((void **)&p->dst_tf32[k], sizeof(unsigned) * 2 * H32.size());
        if (e == cudaSuccess) {
            split_half_kernel<<<blocks_for((long long)H32.size(), 256, 4), 256>>>(h32, (int)(f[k] + 1) / 2,
                                                                                 (int)f[k] / 2, p->dst_tf32[k]);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        cudaFree(h32);
        if (e != cudaSuccess) return cuda_fail(e, "dst tf32 split");
        p->dst_n[k] = (int)f[k];
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
    SVP_CUDA(scratch_alloc((void **)&dev, sizeof(double) * host.size(), s));
    cudaError_t ce = cudaMemcpyAsync(dev, host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        SVP_LAUNCH_KEEP(den_kernel<<<blocks_for(p->q.nfree, 256, 8), 256, 0, s>>>(
            p->den, p->q.fx, p->q.fy, p->q.fz, dev + off[0], dev + off[1], dev + off[2], dev + off[3], dev + off[4],
            dev + off[5], p->q.omega, a, b, metric));
    cudaError_t le = cudaGetLastError();
    cudaError_t fe = scratch_free(dev, s);
    if (ce != cudaSuccess) return cuda_fail(ce, "den copy");
    if (le != cudaSuccess) return cuda_fail(le, "den_kernel");
    if (fe != cudaSuccess) return cuda_fail(fe, "den free");
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
    const long long n3 = 3 * p->q.nfree;
    if (p->precision == SVP_PRECISION_MIXED) {
        // the same six passes in float32 (the fold and the epilogues formed in float64, rounded once)
        float *f0 = (float *)p->dst_tmp, *f1 = f0 + n3;
        if ((rc = dst_pass<float>(p, 0, rhs, f0, scale, 0, 1., nullptr, s))) return rc;
        if ((rc = dst_pass<float>(p, 1, f0, f1, nullptr, 0, 1., nullptr, s))) return rc;
        if ((rc = dst_pass<float>(p, 2, f1, f0, nullptr, 1, 1., nullptr, s))) return rc;
        if ((rc = dst_pass<float>(p, 0, f0, f1, nullptr, 0, 1., nullptr, s))) return rc;
        if ((rc = dst_pass<float>(p, 1, f1, f0, nullptr, 0, 1., nullptr, s))) return rc;
        if (scale) return dst_pass<float>(p, 2, f0, out, nullptr, 2, sign, scale, s);
        if ((rc = dst_pass<float>(p, 2, f0, out, nullptr, 0, 1., nullptr, s))) return rc;
        SVP_LAUNCH(scale_kernel<<<blocks_for(n3, 256, 8), 256, 0, s>>>(out, nullptr, sign, n3, out));
        SVP_LAUNCH_CHECK("scale_kernel");
        return SVP_OK;
    }
    double *t0 = p->dst_tmp, *t1 = p->dst_tmp + n3;
    // scale -> DST(x, y, z) -> / den -> DST(x, y, z) -> sign * scale; the elementwise steps ride in the passes
    if ((rc = dst_pass<double>(p, 0, rhs, t0, scale, 0, 1., nullptr, s))) return rc;
    if ((rc = dst_pass<double>(p, 1, t0, t1, nullptr, 0, 1., nullptr, s))) return rc;
    if ((rc = dst_pass<double>(p, 2, t1, t0, nullptr, 1, 1., nullptr, s))) return rc;
    if ((rc = dst_pass<double>(p, 0, t0, t1, nullptr, 0, 1., nullptr, s))) return rc;
    if ((rc = dst_pass<double>(p, 1, t1, t0, nullptr, 0, 1., nullptr, s))) return rc;
    if (scale) return dst_pass<double>(p, 2, t0, out, nullptr, 2, sign, scale, s);
    if ((rc = dst_pass<double>(p, 2, t0, t1, nullptr, 0, 1., nullptr, s))) return rc;
    unsigned eb = blocks_for(n3, 256, 8);
    SVP_LAUNCH(scale_kernel<<<eb, 256, 0, s>>>(t1, nullptr, sign, n3, out));
    SVP_LAUNCH_CHECK("scale_kernel");
    return SVP_OK;
}
