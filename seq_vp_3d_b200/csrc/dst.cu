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

// One K block of the folded operand: the raw pair (x_k, x_(n-1-k)) of each of a thread's entries is fetched into
// registers one block ahead (the loads fly while the previous block's products run) and folded when it is stored
// to shared memory.  fold = x_k (middle row of odd n), x_k + x_m (parity 0) or x_k - x_m (parity 1), formed in
// float64 (with the optional pre-scale) and rounded once to the pass's type; entries outside the operand are +0.
template <class TC>
__device__ __forceinline__ TC fold_value(double xa, double xb, bool mid, int g) {
    return (TC)(mid ? xa : (g ? xa - xb : xa + xb));
}

// ---------------------------------------------------------------------------------------- mixed form (3xTF32)
// The float32 passes keep each operand as its two TF32 parts in shared memory: the half matrices are split once per
// grid into zero-padded tiles (split_pad_kernel), the folded fields once when a K block is staged, so a fragment is
// loaded, never split, and the staging loads need no bounds checks on the matrix side.  A block computes a 128-row x
// 64-column (left pass) or 128-row x 16 NT-column (right pass) output tile with 8 warps of 32 x 32 (32 x 8 NT), each
// K block of 16 staged twice-buffered through registers.  Every output is accumulated in k order, three mma per k8
// step (small x big, big x small, big x big), so any tiling gives the same bits.
constexpr int QR = 128, QK = 16;           // output rows per block, K block
constexpr int QC = 64;                     // output columns per block of the left pass
constexpr int QPA = QR + 8, QPB = QC + 8;  // left pass: [k][row] and [k][col] rows padded to 8 mod 32 words
constexpr int QPK = QK + 4;                // right pass: [row][k] rows padded to 4 mod 32 words

struct PadTf32 {
    const unsigned *b[2], *s[2];   // per parity: big / small parts, zero-padded to kpad x ipad (left) or ipad x kpad
    int n, kg[2], ipad[2], kpad[2];
};

// h: H0 (k0 x k0) then H1 (k1 x k1), row-major float32.  out, per parity g: big parts then small parts of H_g in the
// pass's layout, kmajor: T[k][a] = H_g[a][k] (kpad x ipad), else T[a][k] = H_g[a][k] (ipad x kpad), zeros outside.
__global__ void split_pad_kernel(const float *__restrict__ h, int kg, long long src, int kmajor, int ipad, int kpad,
                                 unsigned *__restrict__ big, unsigned *__restrict__ small) {
    const long long total = (long long)ipad * kpad;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int a = kmajor ? (int)(e % ipad) : (int)(e / kpad), k = kmajor ? (int)(e / ipad) : (int)(e % kpad);
        unsigned b = 0u, s = 0u;
        if (a < kg && k < kg) tf32_split(h[src + (long long)a * kg + k], b, s);
        big[e] = b;
        small[e] = s;
    }
}

template <class TI>
__device__ __forceinline__ float fold_tf32(TI xa, TI xb, bool mid, int g) {
    // formed in the input type and rounded once: a float32 sum or difference is the rounded exact value either way
    return (float)(mid ? xa : (g ? xa - xb : xa + xb));
}

// Left pass along y or z: C[b][2i + g][w] = sum_k H_g[i][k] fold_g(X)[b][k][w] (rows of length W, stride ldx, batch
// stride bs).  EPI 1 divides by den[index within the batch] (den is one component's array: the z pass's batch stride
// is its length), EPI 2 multiplies by sign * post[flat] (the operation order of the separate elementwise passes).
// 3xTF32: A = H_g^T tile [k][row], B = the folded field [k][col].
template <int EPI, class TI, class TO>
__global__ void __launch_bounds__(256) dst_left_tf32_kernel(PadTf32 D, const TI *__restrict__ X, long long W,
                                                            long long ldx, long long bs, TO *__restrict__ C,
                                                            const double *__restrict__ den,
                                                            const double *__restrict__ post, double sign) {
    extern __shared__ __align__(16) unsigned qsm[];
    unsigned(*sAb)[QK][QPA] = reinterpret_cast<unsigned(*)[QK][QPA]>(qsm);
    unsigned(*sAs)[QK][QPA] = reinterpret_cast<unsigned(*)[QK][QPA]>(qsm + 2 * QK * QPA);
    unsigned(*sBb)[QK][QPB] = reinterpret_cast<unsigned(*)[QK][QPB]>(qsm + 4 * QK * QPA);
    unsigned(*sBs)[QK][QPB] = reinterpret_cast<unsigned(*)[QK][QPB]>(qsm + 4 * QK * QPA + 2 * QK * QPB);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wm = warp >> 1, wn = warp & 1;
    const int t0 = D.ipad[0] / QR;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int rows = g ? D.kg[1] : D.kg[0], K = rows, ip = g ? D.ipad[1] : D.ipad[0];
    const int i0 = ((int)blockIdx.x - (g ? t0 : 0)) * QR;
    const unsigned *Hb = g ? D.b[1] : D.b[0], *Hs = g ? D.s[1] : D.s[0];
    const long long w0 = (long long)blockIdx.y * QC;
    const TI *Xb = X + (long long)blockIdx.z * bs;
    float facc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
            for (int e = 0; e < 4; e++) facc[a][c][e] = 0.f;
    // staging: the matrix block (16 x 128 words per part) as two uint4 per thread, the field block (16 rows x 64
    // columns, each with its mirror row) as two column pairs per thread
    const int hr = threadIdx.x >> 5, hc = (threadIdx.x & 31) * 4;
    const int xr = threadIdx.x >> 5, xc = (threadIdx.x & 31) * 2;
    const bool ok0 = w0 + xc < W, ok1 = w0 + xc + 1 < W;
    uint4 hb[2], hs[2];
    TI xa[2][2], xb[2][2];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < 2; t++) {
            const long long hk = (long long)(k0 + hr + 8 * t) * ip + i0 + hc;
            hb[t] = *reinterpret_cast<const uint4 *>(Hb + hk);
            hs[t] = *reinterpret_cast<const uint4 *>(Hs + hk);
            const int k = k0 + xr + 8 * t;
            const bool ok = k < K;
            const TI *ra = Xb + (long long)k * ldx + w0 + xc, *rb = Xb + (long long)(D.n - 1 - k) * ldx + w0 + xc;
            xa[t][0] = ok && ok0 ? ra[0] : TI(0);
            xa[t][1] = ok && ok1 ? ra[1] : TI(0);
            xb[t][0] = ok && ok0 ? rb[0] : TI(0);
            xb[t][1] = ok && ok1 ? rb[1] : TI(0);
        }
    };
    auto stash = [&](int buf, int k0) {
#pragma unroll
        for (int t = 0; t < 2; t++) {
            *reinterpret_cast<uint4 *>(&sAb[buf][hr + 8 * t][hc]) = hb[t];
            *reinterpret_cast<uint4 *>(&sAs[buf][hr + 8 * t][hc]) = hs[t];
            const int k = k0 + xr + 8 * t;
            const bool mid = k == D.n - 1 - k;
            unsigned b0, s0, b1, s1;
            tf32_split(fold_tf32<TI>(xa[t][0], xb[t][0], mid, g), b0, s0);
            tf32_split(fold_tf32<TI>(xa[t][1], xb[t][1], mid, g), b1, s1);
            *reinterpret_cast<uint2 *>(&sBb[buf][xr + 8 * t][xc]) = make_uint2(b0, b1);
            *reinterpret_cast<uint2 *>(&sBs[buf][xr + 8 * t][xc]) = make_uint2(s0, s1);
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += QK) {
        const bool more = k0 + QK < K;
        if (more) fetch(k0 + QK);
#pragma unroll
        for (int kb = 0; kb < QK; kb += 8) {
            unsigned ab[2][4], as[2][4];
#pragma unroll
            for (int a = 0; a < 2; a++) {
                const int r = wm * 32 + a * 16 + gid;
                ab[a][0] = sAb[buf][kb + tig][r];
                ab[a][1] = sAb[buf][kb + tig][r + 8];
                ab[a][2] = sAb[buf][kb + tig + 4][r];
                ab[a][3] = sAb[buf][kb + tig + 4][r + 8];
                as[a][0] = sAs[buf][kb + tig][r];
                as[a][1] = sAs[buf][kb + tig][r + 8];
                as[a][2] = sAs[buf][kb + tig + 4][r];
                as[a][3] = sAs[buf][kb + tig + 4][r + 8];
            }
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int col = wn * 32 + 8 * c + gid;
                const unsigned b0b = sBb[buf][kb + tig][col], b0s = sBs[buf][kb + tig][col];
                const unsigned b1b = sBb[buf][kb + tig + 4][col], b1s = sBs[buf][kb + tig + 4][col];
#pragma unroll
                for (int a = 0; a < 2; a++) {
                    mma_tf32(facc[a][c], as[a], b0b, b1b);
                    mma_tf32(facc[a][c], ab[a], b0s, b1s);
                    mma_tf32(facc[a][c], ab[a], b0b, b1b);
                }
            }
        }
        if (more) stash(buf ^ 1, k0 + QK);
        __syncthreads();
        buf ^= 1;
    }
    const long long cb = (long long)blockIdx.z * bs;
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int ii = i0 + wm * 32 + a * 16 + gid + 8 * (e >> 1);
                const long long w = w0 + wn * 32 + 8 * c + 2 * tig + (e & 1);
                if (ii >= rows || w >= W) continue;
                const long long io = (long long)(2 * ii + g) * ldx + w, o = cb + io;
                double v = (double)facc[a][c][e];
                if (EPI == 1) v = v / den[io];
                if (EPI == 2) v = sign * (post[o] * v);
                C[o] = (TO)v;
            }
}

// Right pass along x over contiguous rows of length n: C[r][2i + g] = sum_k fold_g(pre X)[r][k] H_g[i][k], pre an
// optional scale applied first.  3xTF32: A = the folded rows [row][k],
// B = H_g tile [col][k] with 16 NT columns (NT n8 tiles per warp along the 2 column warps).
template <int NT, class TI, class TO>
__global__ void __launch_bounds__(256) dst_right_tf32_kernel(PadTf32 D, const TI *__restrict__ X, long long R,
                                                             const double *__restrict__ pre, TO *__restrict__ C) {
    constexpr int QN = 16 * NT;
    extern __shared__ __align__(16) unsigned qsm[];
    unsigned(*sAb)[QR][QPK] = reinterpret_cast<unsigned(*)[QR][QPK]>(qsm);
    unsigned(*sAs)[QR][QPK] = reinterpret_cast<unsigned(*)[QR][QPK]>(qsm + 2 * QR * QPK);
    unsigned(*sBb)[QN][QPK] = reinterpret_cast<unsigned(*)[QN][QPK]>(qsm + 4 * QR * QPK);
    unsigned(*sBs)[QN][QPK] = reinterpret_cast<unsigned(*)[QN][QPK]>(qsm + 4 * QR * QPK + 2 * QN * QPK);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wm = warp >> 1, wn = warp & 1;
    const int t0 = D.ipad[0] / QN;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int cols = g ? D.kg[1] : D.kg[0], K = cols, kp = g ? D.kpad[1] : D.kpad[0];
    const int i0 = ((int)blockIdx.x - (g ? t0 : 0)) * QN;
    const unsigned *Hb = g ? D.b[1] : D.b[0], *Hs = g ? D.s[1] : D.s[0];
    const long long r0 = (long long)blockIdx.y * QR;
    const int n = D.n;
    float facc[2][NT][4];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int c = 0; c < NT; c++)
#pragma unroll
            for (int e = 0; e < 4; e++) facc[a][c][e] = 0.f;
    // staging: the field block (128 rows x 16 k, each with its mirror) as 8 entries per thread, 16 consecutive k of
    // a row per half warp; the matrix block (16 NT rows x 16 k per part) as uint4 along k
    const int xk = threadIdx.x & 15, xr = threadIdx.x >> 4;
    constexpr int HV = QN * QK / 4, HT = (HV + 255) / 256;
    TI xa[8], xb[8];
    uint4 hb[HT], hs[HT];
    auto fetch = [&](int k0) {
        const int k = k0 + xk;
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const long long r = r0 + xr + 16 * t;
            const bool ok = r < R && k < K;
            const long long a = r * n + k, m = r * n + (n - 1 - k);
            if (pre) {
                xa[t] = ok ? (TI)(pre[a] * (double)X[a]) : TI(0);
                xb[t] = ok ? (TI)(pre[m] * (double)X[m]) : TI(0);
            } else {
                xa[t] = ok ? X[a] : TI(0);
                xb[t] = ok ? X[m] : TI(0);
            }
        }
#pragma unroll
        for (int t = 0; t < HT; t++) {
            const int v = threadIdx.x + 256 * t;
            if (v < HV) {
                const long long hk = (long long)(i0 + v / (QK / 4)) * kp + k0 + (v % (QK / 4)) * 4;
                hb[t] = *reinterpret_cast<const uint4 *>(Hb + hk);
                hs[t] = *reinterpret_cast<const uint4 *>(Hs + hk);
            }
        }
    };
    auto stash = [&](int buf, int k0) {
        const int k = k0 + xk;
        const bool mid = k == n - 1 - k;
#pragma unroll
        for (int t = 0; t < 8; t++) {
            unsigned b, s;
            tf32_split(fold_tf32<TI>(xa[t], xb[t], mid, g), b, s);
            sAb[buf][xr + 16 * t][xk] = b;
            sAs[buf][xr + 16 * t][xk] = s;
        }
#pragma unroll
        for (int t = 0; t < HT; t++) {
            const int v = threadIdx.x + 256 * t;
            if (v < HV) {
                *reinterpret_cast<uint4 *>(&sBb[buf][v / (QK / 4)][(v % (QK / 4)) * 4]) = hb[t];
                *reinterpret_cast<uint4 *>(&sBs[buf][v / (QK / 4)][(v % (QK / 4)) * 4]) = hs[t];
            }
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += QK) {
        const bool more = k0 + QK < K;
        if (more) fetch(k0 + QK);
#pragma unroll
        for (int kb = 0; kb < QK; kb += 8) {
            unsigned ab[2][4], as[2][4];
#pragma unroll
            for (int a = 0; a < 2; a++) {
                const int r = wm * 32 + a * 16 + gid;
                ab[a][0] = sAb[buf][r][kb + tig];
                ab[a][1] = sAb[buf][r + 8][kb + tig];
                ab[a][2] = sAb[buf][r][kb + tig + 4];
                ab[a][3] = sAb[buf][r + 8][kb + tig + 4];
                as[a][0] = sAs[buf][r][kb + tig];
                as[a][1] = sAs[buf][r + 8][kb + tig];
                as[a][2] = sAs[buf][r][kb + tig + 4];
                as[a][3] = sAs[buf][r + 8][kb + tig + 4];
            }
#pragma unroll
            for (int c = 0; c < NT; c++) {
                const int col = wn * 8 * NT + 8 * c + gid;
                const unsigned b0b = sBb[buf][col][kb + tig], b0s = sBs[buf][col][kb + tig];
                const unsigned b1b = sBb[buf][col][kb + tig + 4], b1s = sBs[buf][col][kb + tig + 4];
#pragma unroll
                for (int a = 0; a < 2; a++) {
                    mma_tf32(facc[a][c], as[a], b0b, b1b);
                    mma_tf32(facc[a][c], ab[a], b0s, b1s);
                    mma_tf32(facc[a][c], ab[a], b0b, b1b);
                }
            }
        }
        if (more) stash(buf ^ 1, k0 + QK);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int c = 0; c < NT; c++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const long long r = r0 + wm * 32 + a * 16 + gid + 8 * (e >> 1);
                const int ii = i0 + wn * 8 * NT + 8 * c + 2 * tig + (e & 1);
                if (r < R && ii < cols) C[r * n + 2 * ii + g] = (TO)facc[a][c][e];
            }
}

// right-pass column tile: 16 NT columns with NT = ceil(k0 / 16) in 3..8 (one tile per parity up to 128 columns)
inline int right_nt(int k0) {
    const int nt = (k0 + 15) / 16;
    return nt < 3 ? 3 : (nt > 8 ? 8 : nt);
}
inline size_t left_tf32_smem() { return sizeof(unsigned) * 4 * QK * (QPA + QPB); }
inline size_t right_tf32_smem(int nt) { return sizeof(unsigned) * 4 * QPK * (QR + 16 * nt); }

// Padded TF32 tiles of one axis: the right pass (x) stores H_g row-major padded to column tiles of its width, the left
// passes (y, z) H_g^T padded to 128-row tiles; K is padded to the K block.  Buffer: big g0, big g1, small g0, small g1.
inline long long pad_geometry(int axis, int n, int kg[2], int ipad[2], int kpad[2]) {
    kg[0] = (n + 1) / 2;
    kg[1] = n / 2;
    const int tile = axis == 0 ? 16 * right_nt(kg[0]) : QR;
    for (int g = 0; g < 2; g++) {
        ipad[g] = (kg[g] + tile - 1) / tile * tile;
        kpad[g] = (kg[g] + QK - 1) / QK * QK;
    }
    return 2LL * ((long long)ipad[0] * kpad[0] + (long long)ipad[1] * kpad[1]);
}
inline PadTf32 pad_tf32(const unsigned *t, int axis, int n) {
    PadTf32 T;
    T.n = n;
    pad_geometry(axis, n, T.kg, T.ipad, T.kpad);
    const long long a0 = (long long)T.ipad[0] * T.kpad[0], a1 = (long long)T.ipad[1] * T.kpad[1];
    T.b[0] = t;
    T.b[1] = t + a0;
    T.s[0] = t + a0 + a1;
    T.s[1] = t + 2 * a0 + a1;
    return T;
}

// the TF32 passes' shared memory is above the 48 KB default: set once per device (see allow_slices in q1.cu)
template <int NT>
int allow_right_tf32() {
    SVP_CUDA(cudaFuncSetAttribute(dst_right_tf32_kernel<NT, double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)right_tf32_smem(NT)));
    SVP_CUDA(cudaFuncSetAttribute(dst_right_tf32_kernel<NT, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)right_tf32_smem(NT)));
    return SVP_OK;
}
int allow_tf32() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    SVP_CUDA(cudaGetDevice(&dev));
    SVP_REQUIRE(dev >= 0 && dev < 64, "allow_tf32: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return SVP_OK;
    const int ls = (int)left_tf32_smem();
    SVP_CUDA(cudaFuncSetAttribute(dst_left_tf32_kernel<0, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    SVP_CUDA(cudaFuncSetAttribute(dst_left_tf32_kernel<1, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    SVP_CUDA(cudaFuncSetAttribute(dst_left_tf32_kernel<0, float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    SVP_CUDA(cudaFuncSetAttribute(dst_left_tf32_kernel<2, float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    int rc;
    if ((rc = allow_right_tf32<3>()) || (rc = allow_right_tf32<4>()) || (rc = allow_right_tf32<5>()) ||
        (rc = allow_right_tf32<6>()) || (rc = allow_right_tf32<7>()) || (rc = allow_right_tf32<8>()))
        return rc;
    done[dev] = true;
    return SVP_OK;
}
template <class TI, class TO>
int launch_right_tf32(int nt, dim3 grid, const PadTf32 &T, const TI *in, long long R, const double *pre, TO *out,
                      cudaStream_t s) {
    const size_t sm = right_tf32_smem(nt);
    switch (nt) {
        case 3: SVP_LAUNCH((dst_right_tf32_kernel<3, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 4: SVP_LAUNCH((dst_right_tf32_kernel<4, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 5: SVP_LAUNCH((dst_right_tf32_kernel<5, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 6: SVP_LAUNCH((dst_right_tf32_kernel<6, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 7: SVP_LAUNCH((dst_right_tf32_kernel<7, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        default: SVP_LAUNCH((dst_right_tf32_kernel<8, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
    }
    return SVP_OK;
}

// ------------------------------------------------------------------------------- plain form (FP64 DMMA), tiled
// The float64 passes with the tiling of the 3xTF32 ones: zero-padded half matrices (pad_half_kernel, the same
// geometry), a 128 x 64 (left) or 64 x 16 NT (right) output tile per block, 8 warps of 32 x 32 (16 x 8 NT) = 4 x 4
// (2 x NT) DMMA 8x8x4 tiles, K blocks of 16 staged twice-buffered through registers.  Rows of the staged blocks are
// padded to 4 mod 16 doubles, so the 64-bit fragment loads of each half warp fall in distinct bank pairs.  Every
// output is the DMMA sequence over k in order (kb = 0, 4, 8, ...), the accumulation of a plain 8x8x4 tiling, so the
// values do not depend on the tile shape.
constexpr int DPB = QC + 4, DPK = QK + 4;

struct PadF64 {
    const double *h[2];   // per parity, zero-padded to kpad x ipad (left, k-major) or ipad x kpad (right)
    int n, kg[2], ipad[2], kpad[2];
};

__global__ void pad_half_kernel(const double *__restrict__ h, int kg, long long src, int kmajor, int ipad, int kpad,
                                double *__restrict__ out) {
    const long long total = (long long)ipad * kpad;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int a = kmajor ? (int)(e % ipad) : (int)(e / kpad), k = kmajor ? (int)(e / ipad) : (int)(e % kpad);
        out[e] = (a < kg && k < kg) ? h[src + (long long)a * kg + k] : 0.;
    }
}

// MR m8 row tiles per warp: a block covers 32 MR rows (4 row warps) x 64 columns (2 column warps).
template <int MR, int EPI, class TI, class TO>
__global__ void __launch_bounds__(256) dst_left_dmma_kernel(PadF64 D, const TI *__restrict__ X, long long W,
                                                            long long ldx, long long bs, TO *__restrict__ C,
                                                            const double *__restrict__ den,
                                                            const double *__restrict__ post, double sign) {
    constexpr int RB = 32 * MR, PA = RB + 4;
    extern __shared__ __align__(16) double dsm[];
    double(*sA)[QK][PA] = reinterpret_cast<double(*)[QK][PA]>(dsm);
    double(*sB)[QK][DPB] = reinterpret_cast<double(*)[QK][DPB]>(dsm + 2 * QK * PA);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wm = warp >> 1, wn = warp & 1;
    const int t0 = D.ipad[0] / RB;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int rows = g ? D.kg[1] : D.kg[0], K = rows, ip = g ? D.ipad[1] : D.ipad[0];
    const int i0 = ((int)blockIdx.x - (g ? t0 : 0)) * RB;
    const double *H = g ? D.h[1] : D.h[0];
    const long long w0 = (long long)blockIdx.y * QC;
    const TI *Xb = X + (long long)blockIdx.z * bs;
    double dacc[MR][4][2];
#pragma unroll
    for (int a = 0; a < MR; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) dacc[a][c][0] = dacc[a][c][1] = 0.;
    // staging: the matrix block (16 x 32 MR) as MR double2 per thread (16 MR per row), the field block (16 x 64,
    // with mirrors) as four entries per thread
    const int xr = threadIdx.x >> 6, xc = threadIdx.x & 63;
    const bool okw = w0 + xc < W;
    double2 hv[MR];
    TI xa[4], xb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < MR; t++) {
            const int v = threadIdx.x + 256 * t;
            hv[t] = *reinterpret_cast<const double2 *>(H + (long long)(k0 + v / (16 * MR)) * ip + i0 +
                                                       (v % (16 * MR)) * 2);
        }
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int k = k0 + xr + 4 * t;
            const bool ok = okw && k < K;
            xa[t] = ok ? Xb[(long long)k * ldx + w0 + xc] : TI(0);
            xb[t] = ok ? Xb[(long long)(D.n - 1 - k) * ldx + w0 + xc] : TI(0);
        }
    };
    auto stash = [&](int buf, int k0) {
#pragma unroll
        for (int t = 0; t < MR; t++) {
            const int v = threadIdx.x + 256 * t;
            *reinterpret_cast<double2 *>(&sA[buf][v / (16 * MR)][(v % (16 * MR)) * 2]) = hv[t];
        }
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int k = k0 + xr + 4 * t;
            sB[buf][xr + 4 * t][xc] = fold_value<double>((double)xa[t], (double)xb[t], k == D.n - 1 - k, g);
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += QK) {
        const bool more = k0 + QK < K;
        if (more) fetch(k0 + QK);
#pragma unroll
        for (int kb = 0; kb < QK; kb += 4) {
            double a[MR], x[4];
#pragma unroll
            for (int m = 0; m < MR; m++) a[m] = sA[buf][kb + tig][wm * 8 * MR + 8 * m + gid];
#pragma unroll
            for (int c = 0; c < 4; c++) x[c] = sB[buf][kb + tig][wn * 32 + 8 * c + gid];
#pragma unroll
            for (int m = 0; m < MR; m++)
#pragma unroll
                for (int c = 0; c < 4; c++) dmma_8x8x4(dacc[m][c], a[m], x[c]);
        }
        if (more) stash(buf ^ 1, k0 + QK);
        __syncthreads();
        buf ^= 1;
    }
    const long long cb = (long long)blockIdx.z * bs;
#pragma unroll
    for (int m = 0; m < MR; m++)
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int ii = i0 + wm * 8 * MR + 8 * m + gid;
                const long long w = w0 + wn * 32 + 8 * c + 2 * tig + e;
                if (ii >= rows || w >= W) continue;
                const long long io = (long long)(2 * ii + g) * ldx + w, o = cb + io;
                double v = dacc[m][c][e];
                if (EPI == 1) v = v / den[io];
                if (EPI == 2) v = sign * (post[o] * v);
                C[o] = (TO)v;
            }
}

// MR m8 row tiles per warp: a block covers 32 MR rows (4 row warps) x 16 NT columns (2 column warps).
template <int MR, int NT, class TI, class TO>
__global__ void __launch_bounds__(256) dst_right_dmma_kernel(PadF64 D, const TI *__restrict__ X, long long R,
                                                             const double *__restrict__ pre, TO *__restrict__ C) {
    constexpr int QN = 16 * NT, RB = 32 * MR, XT = RB / 16;
    extern __shared__ __align__(16) double dsm[];
    double(*sA)[RB][DPK] = reinterpret_cast<double(*)[RB][DPK]>(dsm);
    double(*sB)[QN][DPK] = reinterpret_cast<double(*)[QN][DPK]>(dsm + 2 * RB * DPK);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int wm = warp >> 1, wn = warp & 1;
    const int t0 = D.ipad[0] / QN;
    const int g = (int)blockIdx.x < t0 ? 0 : 1;
    const int cols = g ? D.kg[1] : D.kg[0], K = cols, kp = g ? D.kpad[1] : D.kpad[0];
    const int i0 = ((int)blockIdx.x - (g ? t0 : 0)) * QN;
    const double *H = g ? D.h[1] : D.h[0];
    const long long r0 = (long long)blockIdx.y * RB;
    const int n = D.n;
    double dacc[MR][NT][2];
#pragma unroll
    for (int a = 0; a < MR; a++)
#pragma unroll
        for (int c = 0; c < NT; c++) dacc[a][c][0] = dacc[a][c][1] = 0.;
    const int xk = threadIdx.x & 15, xr = threadIdx.x >> 4;
    constexpr int HV = QN * QK / 2, HT = (HV + 255) / 256;
    double xa[XT], xb[XT];
    double2 hv[HT];
    auto fetch = [&](int k0) {
        const int k = k0 + xk;
#pragma unroll
        for (int t = 0; t < XT; t++) {
            const long long r = r0 + xr + 16 * t;
            const bool ok = r < R && k < K;
            const long long a = r * n + k, m = r * n + (n - 1 - k);
            xa[t] = ok ? (pre ? pre[a] * (double)X[a] : (double)X[a]) : 0.;
            xb[t] = ok ? (pre ? pre[m] * (double)X[m] : (double)X[m]) : 0.;
        }
#pragma unroll
        for (int t = 0; t < HT; t++) {
            const int v = threadIdx.x + 256 * t;
            if (v < HV)
                hv[t] = *reinterpret_cast<const double2 *>(H + (long long)(i0 + v / (QK / 2)) * kp + k0 +
                                                           (v % (QK / 2)) * 2);
        }
    };
    auto stash = [&](int buf, int k0) {
        const int k = k0 + xk;
        const bool mid = k == n - 1 - k;
#pragma unroll
        for (int t = 0; t < XT; t++) sA[buf][xr + 16 * t][xk] = fold_value<double>(xa[t], xb[t], mid, g);
#pragma unroll
        for (int t = 0; t < HT; t++) {
            const int v = threadIdx.x + 256 * t;
            if (v < HV) *reinterpret_cast<double2 *>(&sB[buf][v / (QK / 2)][(v % (QK / 2)) * 2]) = hv[t];
        }
    };
    fetch(0);
    stash(0, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += QK) {
        const bool more = k0 + QK < K;
        if (more) fetch(k0 + QK);
#pragma unroll
        for (int kb = 0; kb < QK; kb += 4) {
            double a[MR], x[NT];
#pragma unroll
            for (int m = 0; m < MR; m++) a[m] = sA[buf][wm * 8 * MR + 8 * m + gid][kb + tig];
#pragma unroll
            for (int c = 0; c < NT; c++) x[c] = sB[buf][wn * 8 * NT + 8 * c + gid][kb + tig];
#pragma unroll
            for (int m = 0; m < MR; m++)
#pragma unroll
                for (int c = 0; c < NT; c++) dmma_8x8x4(dacc[m][c], a[m], x[c]);
        }
        if (more) stash(buf ^ 1, k0 + QK);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int m = 0; m < MR; m++)
#pragma unroll
        for (int c = 0; c < NT; c++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const long long r = r0 + wm * 8 * MR + 8 * m + gid;
                const int ii = i0 + wn * 8 * NT + 8 * c + 2 * tig + e;
                if (r < R && ii < cols) C[r * n + 2 * ii + g] = (TO)dacc[m][c][e];
            }
}

// the left float64 passes: DML m8 row tiles per warp (blocks of 32 DML rows)
constexpr int DML = 4;
inline size_t left_dmma_smem() { return sizeof(double) * 2 * QK * (32 * DML + 4 + DPB); }
// the right float64 pass: 64-row blocks (2 m8 tiles per warp) keep two 256-thread blocks resident per SM
constexpr int DMR = 2;
inline size_t right_dmma_smem(int nt) { return sizeof(double) * 2 * DPK * (32 * DMR + 16 * nt); }
inline PadF64 pad_f64(const double *t, int axis, int n) {
    PadF64 T;
    T.n = n;
    pad_geometry(axis, n, T.kg, T.ipad, T.kpad);
    T.h[0] = t;
    T.h[1] = t + (long long)T.ipad[0] * T.kpad[0];
    return T;
}
template <int NT>
int allow_right_dmma() {
    SVP_CUDA(cudaFuncSetAttribute(dst_right_dmma_kernel<DMR, NT, double, double>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)right_dmma_smem(NT)));
    return SVP_OK;
}
int allow_dmma() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    SVP_CUDA(cudaGetDevice(&dev));
    SVP_REQUIRE(dev >= 0 && dev < 64, "allow_dmma: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return SVP_OK;
    const int ls = (int)left_dmma_smem();
    SVP_CUDA(cudaFuncSetAttribute(dst_left_dmma_kernel<DML, 0, double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    SVP_CUDA(cudaFuncSetAttribute(dst_left_dmma_kernel<DML, 1, double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    SVP_CUDA(cudaFuncSetAttribute(dst_left_dmma_kernel<DML, 2, double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ls));
    int rc;
    if ((rc = allow_right_dmma<3>()) || (rc = allow_right_dmma<4>()) || (rc = allow_right_dmma<5>()) ||
        (rc = allow_right_dmma<6>()) || (rc = allow_right_dmma<7>()) || (rc = allow_right_dmma<8>()))
        return rc;
    done[dev] = true;
    return SVP_OK;
}
template <class TI, class TO>
int launch_right_dmma(int nt, dim3 grid, const PadF64 &T, const TI *in, long long R, const double *pre, TO *out,
                      cudaStream_t s) {
    const size_t sm = right_dmma_smem(nt);
    switch (nt) {
        case 3: SVP_LAUNCH((dst_right_dmma_kernel<DMR, 3, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 4: SVP_LAUNCH((dst_right_dmma_kernel<DMR, 4, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 5: SVP_LAUNCH((dst_right_dmma_kernel<DMR, 5, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 6: SVP_LAUNCH((dst_right_dmma_kernel<DMR, 6, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        case 7: SVP_LAUNCH((dst_right_dmma_kernel<DMR, 7, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
        default: SVP_LAUNCH((dst_right_dmma_kernel<DMR, 8, TI, TO><<<grid, 256, sm, s>>>(T, in, R, pre, out))); break;
    }
    return SVP_OK;
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

// One DST-I pass along `axis` of (3, n2, n1, n0) fields with the folded half matrices; see dst_left_tf32_kernel for
// pre / EPI.
template <class TC, class TI, class TO>
static int dst_pass(const svp_pair *p, int axis, const TI *in, TO *out, const double *pre, int epi, double sign,
                    const double *post, cudaStream_t s) {
    const long long n0 = p->q.fx, n1 = p->q.fy, n2 = p->q.fz;
    const int n = p->dst_n[axis], k0 = (n + 1) / 2;
    constexpr bool kDouble = sizeof(TC) == 8;
    PadF64 D = pad_f64(p->dst_pad[axis], axis, n);
    PadTf32 T = pad_tf32(p->dst_tf32[axis], axis, n);
    {
        int rc = kDouble ? allow_dmma() : allow_tf32();
        if (rc) return rc;
    }
    if (axis == 0) {
        SVP_REQUIRE(epi == 0, "dst_pass: x pass has no epilogue");
        long long R = 3 * n2 * n1;
        svp::KernelTimer _t("dst_right_kernel", s);
        // the column tiles of one row block lead the grid: the blocks that share rows run together (L2 reuse)
        const int nt = right_nt(k0);
        dim3 grid((unsigned)((T.ipad[0] + T.ipad[1]) / (16 * nt)), (unsigned)div_up(R, kDouble ? 32 * DMR : QR));
        int rc;
        if constexpr (kDouble) rc = launch_right_dmma<TI, TO>(nt, grid, D, in, R, pre, out, s);
        else rc = launch_right_tf32<TI, TO>(nt, grid, T, in, R, pre, out, s);
        if (rc) return rc;
    } else {
        SVP_REQUIRE(!pre, "dst_pass: pre-scale only on the x pass");
        SVP_REQUIRE(epi != 1 || axis == 2, "dst_pass: the 1/den epilogue rides in the z pass (batch stride = nfree)");
        long long W = axis == 1 ? n0 : n1 * n0;
        long long ldx = W, bs = axis == 1 ? n1 * n0 : n2 * n1 * n0;
        // the row tiles of both parities lead the grid: the blocks that read the same field columns run together
        dim3 qgrid((unsigned)((T.ipad[0] + T.ipad[1]) / QR), (unsigned)div_up(W, QC), (unsigned)(axis == 1 ? 3 * n2 : 3));
        svp::KernelTimer _t("dst_left_kernel", s);
        if constexpr (kDouble) {
            const size_t ds = left_dmma_smem();
            dim3 dgrid((unsigned)((D.ipad[0] + D.ipad[1]) / (32 * DML)), qgrid.y, qgrid.z);
            if (epi == 0) SVP_LAUNCH((dst_left_dmma_kernel<DML, 0, TI, TO><<<dgrid, 256, ds, s>>>(D, in, W, ldx, bs, out, nullptr, nullptr, 1.)));
            else if (epi == 1) SVP_LAUNCH((dst_left_dmma_kernel<DML, 1, TI, TO><<<dgrid, 256, ds, s>>>(D, in, W, ldx, bs, out, p->den, nullptr, 1.)));
            else SVP_LAUNCH((dst_left_dmma_kernel<DML, 2, TI, TO><<<dgrid, 256, ds, s>>>(D, in, W, ldx, bs, out, nullptr, post, sign)));
        } else {
            const size_t qs = left_tf32_smem();
            if (epi == 0) SVP_LAUNCH((dst_left_tf32_kernel<0, TI, TO><<<qgrid, 256, qs, s>>>(T, in, W, ldx, bs, out, nullptr, nullptr, 1.)));
            else if (epi == 1) SVP_LAUNCH((dst_left_tf32_kernel<1, TI, TO><<<qgrid, 256, qs, s>>>(T, in, W, ldx, bs, out, p->den, nullptr, 1.)));
            else SVP_LAUNCH((dst_left_tf32_kernel<2, TI, TO><<<qgrid, 256, qs, s>>>(T, in, W, ldx, bs, out, nullptr, post, sign)));
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
        {
            int kg[2], ipad[2], kpad[2];
            const long long words = pad_geometry(k, (int)f[k], kg, ipad, kpad) / 2;
            SVP_CUDA(cudaMalloc((void **)&p->dst_pad[k], sizeof(double) * words));
            const PadF64 T = pad_f64(p->dst_pad[k], k, (int)f[k]);
            for (int g = 0; g < 2; g++) {
                pad_half_kernel<<<blocks_for((long long)ipad[g] * kpad[g], 256, 4), 256>>>(
                    p->dst_half[k], kg[g], g ? (long long)kg[0] * kg[0] : 0, k != 0, ipad[g], kpad[g],
                    const_cast<double *>(T.h[g]));
                SVP_CUDA(cudaGetLastError());
            }
            SVP_CUDA(cudaStreamSynchronize(0));
        }
        // the mixed form's matrices: rounded once to float32, then split into TF32 parts on the device (the same
        // cvt.rna the passes use for their staged operands)
        std::vector<float> H32(H.begin(), H.end());
        float *h32 = nullptr;
        SVP_CUDA(cudaMalloc((void **)&h32, sizeof(float) * H32.size()));
        cudaError_t e = cudaMemcpy(h32, H32.data(), sizeof(float) * H32.size(), cudaMemcpyHostToDevice);
        int kg[2], ipad[2], kpad[2];
        const long long words = pad_geometry(k, (int)f[k], kg, ipad, kpad);
        if (e == cudaSuccess) e = cudaMalloc((void **)&p->dst_tf32[k], sizeof(unsigned) * words);
        if (e == cudaSuccess) {
            const PadTf32 T = pad_tf32(p->dst_tf32[k], k, (int)f[k]);
            for (int g = 0; g < 2 && e == cudaSuccess; g++) {
                const long long src = g ? (long long)kg[0] * kg[0] : 0;
                split_pad_kernel<<<blocks_for((long long)ipad[g] * kpad[g], 256, 4), 256>>>(
                    h32, kg[g], src, k != 0, ipad[g], kpad[g], const_cast<unsigned *>(T.b[g]),
                    const_cast<unsigned *>(T.s[g]));
                e = cudaGetLastError();
            }
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
