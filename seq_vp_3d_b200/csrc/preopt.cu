// The float32 pyramid pre-optimizer (an uncertified initializer of the native certified solve) and the pyramid's
// resampling, on the device.
//
// Pre-objective of the interior displacement u_int (3, D-2, H-2, W-2) in voxel units, zero faces (preopt.py:157
// _pre_energy_tensors; preopt_grad.py:1-25 for the analytic gradient):
//   P(u) = 1/2 sum_x (T(x + u) - F)^2                       T trilinear in M, align_corners, border padding
//        + mu/2 sum_cells [(det - 1)^2 + |curl|^2]           cell-centre F = I + (h_c/h_d) mean of 4 edge differences
//        + kappa sum_cells relu(j0 - det)^2
//        + alpha/2 sum_interior |h_c Delta_h u_c|^2
// One Adam iteration (preopt.py:217 _run_level_default): g = Gaussian(sigma_grad) * grad P; m, v moments; step =
// lr m^ / (sqrt(v^) + eps); the step is scaled so that its largest entry is at most `cap` voxels; u -= step; then
// optionally u = Gaussian(sigma_field) * u.  Everything stays on the device; the cap's scale is computed there.
#include <cmath>
#include <vector>

#include "svp_common.cuh"

namespace svp {
namespace {

constexpr int PT = 256;

struct Level {
    int D, H, W;                 // level grid (z, y, x)
    float rx, ry, rz;            // h_c / h_d ratios are formed per use from h
    double h[3];                 // spacing x, y, z
};

__device__ __forceinline__ long long interior_index(int c, int z, int y, int x, int D, int H, int W) {
    return (((long long)c * (D - 2) + (z - 1)) * (H - 2) + (y - 1)) * (W - 2) + (x - 1);
}
// displacement component c at node (z, y, x) in voxels; zero on the faces
__device__ __forceinline__ float node_u(const float *__restrict__ u, int c, int z, int y, int x, int D, int H, int W) {
    if (z <= 0 || y <= 0 || x <= 0 || z >= D - 1 || y >= H - 1 || x >= W - 1) return 0.f;
    return u[interior_index(c, z, y, x, D, H, W)];
}

// float block reduction of K sums (fixed order) -> partial[block * K + k]
template <int K>
__device__ void block_sum_f(float (&v)[K], float *partial) {
    __shared__ float sh[PT / 32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
        for (int o = 16; o; o >>= 1) v[k] += __shfl_xor_sync(0xFFFFFFFFu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) sh[warp][k] = v[k];
    __syncthreads();
    if (threadIdx.x < K) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w][threadIdx.x];
        partial[(size_t)blockIdx.x * K + threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------------------------- data term
// Sample coordinate of one axis with the autograd path's operations: g = 2 (x + u) / max(n - 1, 1) - 1, then
// grid_sample's unnormalisation ((g + 1) / 2) (n - 1); clipped to [0, n - 1] with chi = 0 where clipped
// (PyTorch's clip_coordinates_set_grad: <= 0 or >= n - 1).
__device__ __forceinline__ float sample_coord(float xi, float u, int n, float &chi) {
    const float den = (float)(n - 1 > 1 ? n - 1 : 1);
    const float g = __fsub_rn(__fdiv_rn(__fmul_rn(2.f, __fadd_rn(xi, u)), den), 1.f);
    const float c = __fmul_rn(__fmul_rn(__fadd_rn(g, 1.f), .5f), (float)(n - 1));
    if (c <= 0.f) { chi = 0.f; return 0.f; }
    if (c >= (float)(n - 1)) { chi = 0.f; return (float)(n - 1); }
    chi = 1.f;
    return c;
}

// residual r = T(x + u) - F at every node; data gradient r dT/di chi on interior nodes into grad; sums 1/2 r^2
__global__ void __launch_bounds__(PT) pre_data_kernel(const float *__restrict__ F, const float *__restrict__ M,
                                                      int D, int H, int W, const float *__restrict__ u,
                                                      float *__restrict__ grad, float *partial) {
    float acc[1] = {0.f};
    const long long n = (long long)D * H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % W), y = (int)((i / W) % H), z = (int)(i / ((long long)W * H));
        float cx, cy, cz;
        const float ix = sample_coord((float)x, node_u(u, 0, z, y, x, D, H, W), W, cx);
        const float iy = sample_coord((float)y, node_u(u, 1, z, y, x, D, H, W), H, cy);
        const float iz = sample_coord((float)z, node_u(u, 2, z, y, x, D, H, W), D, cz);
        const float x0f = floorf(ix), y0f = floorf(iy), z0f = floorf(iz);
        const float wx1 = ix - x0f, wy1 = iy - y0f, wz1 = iz - z0f;
        const float wx0 = (x0f + 1.f) - ix, wy0 = (y0f + 1.f) - iy, wz0 = (z0f + 1.f) - iz;
        const int x0 = (int)x0f, y0 = (int)y0f, z0 = (int)z0f;
        float c[2][2][2];
#pragma unroll
        for (int dz = 0; dz < 2; dz++)
#pragma unroll
            for (int dy = 0; dy < 2; dy++)
#pragma unroll
                for (int dx = 0; dx < 2; dx++) {
                    const int zz = z0 + dz, yy = y0 + dy, xx = x0 + dx;
                    c[dz][dy][dx] = (zz <= D - 1 && yy <= H - 1 && xx <= W - 1)
                                        ? __ldg(M + ((long long)zz * H + yy) * W + xx) : 0.f;
                }
        const float wx[2] = {wx0, wx1}, wy[2] = {wy0, wy1}, wz[2] = {wz0, wz1};
        float T = 0.f;
#pragma unroll
        for (int dz = 0; dz < 2; dz++)
#pragma unroll
            for (int dy = 0; dy < 2; dy++)
#pragma unroll
                for (int dx = 0; dx < 2; dx++) T += c[dz][dy][dx] * ((wx[dx] * wy[dy]) * wz[dz]);
        const float r = T - __ldg(F + i);
        acc[0] += .5f * r * r;
        if (z > 0 && y > 0 && x > 0 && z < D - 1 && y < H - 1 && x < W - 1) {
            float dtx = 0.f, dty = 0.f, dtz = 0.f;
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 2; b++) {
                    dtx += (c[a][b][1] - c[a][b][0]) * wy[b] * wz[a];
                    dty += (c[a][1][b] - c[a][0][b]) * wx[b] * wz[a];
                    dtz += (c[1][a][b] - c[0][a][b]) * wx[b] * wy[a];
                }
            grad[interior_index(0, z, y, x, D, H, W)] = r * dtx * cx;
            grad[interior_index(1, z, y, x, D, H, W)] = r * dty * cy;
            grad[interior_index(2, z, y, x, D, H, W)] = r * dtz * cz;
        }
    }
    block_sum_f<1>(acc, partial);
}

// ---------------------------------------------------------------------------------------------- cell terms
// Per cell: cell-centre F, det, curl, geometry and floor energies, and G_cd = dE_cell / d(voxel derivative of u_c
// along d) (preopt_grad.py:103 cell_geometry), stored SoA G[(3 c + d) * ncell + cell]; min det reduced.
__global__ void __launch_bounds__(PT) pre_cell_kernel(int D, int H, int W, float r01, float r02, float r10,
                                                      float r12, float r20, float r21, float mu, float kappa,
                                                      float j0, const float *__restrict__ u, float *__restrict__ G,
                                                      float *partial) {
    float acc[3] = {0.f, 0.f, 0.f};     // geometry, floor, -min det (as max of -det)
    float mndet = __int_as_float(0x7F800000);
    const long long cx = W - 1, cy = H - 1, cz = D - 1, ncell = cx * cy * cz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncell; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % cx), y = (int)((i / cx) % cy), z = (int)(i / (cx * cy));
        float v[3][2][2][2];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 2; b++)
#pragma unroll
                    for (int e = 0; e < 2; e++) v[c][a][b][e] = node_u(u, c, z + a, y + b, x + e, D, H, W);
        // derivative along an axis: the edge differences averaged over the lower-numbered other axis first
        float der[3][3];    // der[d][c], d = 0 x, 1 y, 2 z
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float e00, e01, e10, e11;
            // along z: diffs over (y, x); average over y then x
            e00 = v[c][1][0][0] - v[c][0][0][0]; e01 = v[c][1][0][1] - v[c][0][0][1];
            e10 = v[c][1][1][0] - v[c][0][1][0]; e11 = v[c][1][1][1] - v[c][0][1][1];
            der[2][c] = .5f * (.5f * (e00 + e10) + .5f * (e01 + e11));
            // along y: diffs over (z, x); average over z then x
            e00 = v[c][0][1][0] - v[c][0][0][0]; e01 = v[c][0][1][1] - v[c][0][0][1];
            e10 = v[c][1][1][0] - v[c][1][0][0]; e11 = v[c][1][1][1] - v[c][1][0][1];
            der[1][c] = .5f * (.5f * (e00 + e10) + .5f * (e01 + e11));
            // along x: diffs over (z, y); average over z then y
            e00 = v[c][0][0][1] - v[c][0][0][0]; e01 = v[c][0][1][1] - v[c][0][1][0];
            e10 = v[c][1][0][1] - v[c][1][0][0]; e11 = v[c][1][1][1] - v[c][1][1][0];
            der[0][c] = .5f * (.5f * (e00 + e10) + .5f * (e01 + e11));
        }
        const float F00 = 1.f + der[0][0], F01 = der[1][0] * r01, F02 = der[2][0] * r02;
        const float F10 = der[0][1] * r10, F11 = 1.f + der[1][1], F12 = der[2][1] * r12;
        const float F20 = der[0][2] * r20, F21 = der[1][2] * r21, F22 = 1.f + der[2][2];
        const float det = F00 * (F11 * F22 - F12 * F21) - F01 * (F10 * F22 - F12 * F20) + F02 * (F10 * F21 - F11 * F20);
        const float c0 = F21 - F12, c1 = F02 - F20, c2 = F10 - F01;
        const float dm = det - 1.f, low = j0 - det > 0.f ? j0 - det : 0.f;
        acc[0] += dm * dm + (c0 * c0 + c1 * c1 + c2 * c2);
        acc[1] += low * low;
        mndet = fminf(mndet, det);
        const float A = mu * dm - 2.f * kappa * low;
        const float cof[3][3] = {{F11 * F22 - F12 * F21, -(F10 * F22 - F12 * F20), F10 * F21 - F11 * F20},
                                 {-(F01 * F22 - F02 * F21), F00 * F22 - F02 * F20, -(F00 * F21 - F01 * F20)},
                                 {F01 * F12 - F02 * F11, -(F00 * F12 - F02 * F10), F00 * F11 - F01 * F10}};
        const float adj[3][3] = {{0.f, -c2, c1}, {c2, 0.f, -c0}, {-c1, c0, 0.f}};
        const float ratio[3][3] = {{1.f, r01, r02}, {r10, 1.f, r12}, {r20, r21, 1.f}};
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int d = 0; d < 3; d++) G[(3 * c + d) * ncell + i] = (A * cof[c][d] + mu * adj[c][d]) * ratio[c][d];
    }
    acc[2] = -mndet;
    // block reductions: the first two are sums, the third a max (done by hand below)
    __shared__ float shm[PT / 32];
    float s2[2] = {acc[0], acc[1]};
    float mx = acc[2];
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = mx;
    block_sum_f<2>(s2, partial);         // contains a __syncthreads
    if (threadIdx.x == 0) {
        float m = shm[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, shm[w]);
        partial[(size_t)gridDim.x * 2 + blockIdx.x] = m;
    }
}

// seven-point Laplacian (physical) of u, times h_c, on interior nodes (zero faces); sums 1/2 lap^2
__global__ void __launch_bounds__(PT) pre_lap_kernel(int D, int H, int W, float ihx2, float ihy2, float ihz2,
                                                     float hx, float hy, float hz, const float *__restrict__ u,
                                                     float *__restrict__ lap, float *partial) {
    float acc[1] = {0.f};
    const long long n = 3LL * (D - 2) * (H - 2) * (W - 2);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % (W - 2)) + 1, y = (int)((i / (W - 2)) % (H - 2)) + 1;
        const int z = (int)((i / ((long long)(W - 2) * (H - 2))) % (D - 2)) + 1, c = (int)(i / ((long long)(W - 2) * (H - 2) * (D - 2)));
        const float ui = u[i];
        const float lz = (node_u(u, c, z + 1, y, x, D, H, W) - 2.f * ui + node_u(u, c, z - 1, y, x, D, H, W)) * ihz2;
        const float ly = (node_u(u, c, z, y + 1, x, D, H, W) - 2.f * ui + node_u(u, c, z, y - 1, x, D, H, W)) * ihy2;
        const float lx = (node_u(u, c, z, y, x + 1, D, H, W) - 2.f * ui + node_u(u, c, z, y, x - 1, D, H, W)) * ihx2;
        const float l = ((lz + ly) + lx) * (c == 0 ? hx : (c == 1 ? hy : hz));
        lap[i] = l;
        acc[0] += .5f * l * l;
    }
    block_sum_f<1>(acc, partial);
}

// interior-node gradient: data part (already in grad) + the 8 cells' G (+-1/4 per axis) + alpha h_c Delta_h lap
__global__ void __launch_bounds__(PT) pre_node_kernel(int D, int H, int W, const float *__restrict__ G,
                                                      const float *__restrict__ lap, float alpha, float ihx2,
                                                      float ihy2, float ihz2, float hx, float hy, float hz,
                                                      float *__restrict__ grad) {
    const long long n = 3LL * (D - 2) * (H - 2) * (W - 2);
    const long long cx = W - 1, cy = H - 1, ncell = cx * cy * (D - 1);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % (W - 2)) + 1, y = (int)((i / (W - 2)) % (H - 2)) + 1;
        const int z = (int)((i / ((long long)(W - 2) * (H - 2))) % (D - 2)) + 1, c = (int)(i / ((long long)(W - 2) * (H - 2) * (D - 2)));
        float g = 0.f;
#pragma unroll
        for (int a = 0; a < 8; a++) {
            const int bx = a & 1, by = (a >> 1) & 1, bz = a >> 2;
            const long long cell = ((long long)(z - bz) * cy + (y - by)) * cx + (x - bx);
            g += G[(3 * c + 0) * ncell + cell] * (bx ? .25f : -.25f);
            g += G[(3 * c + 1) * ncell + cell] * (by ? .25f : -.25f);
            g += G[(3 * c + 2) * ncell + cell] * (bz ? .25f : -.25f);
        }
        float out = grad[i] + g;
        if (alpha > 0.f) {
            auto L = [&](int zz, int yy, int xx) -> float {
                if (zz <= 0 || yy <= 0 || xx <= 0 || zz >= D - 1 || yy >= H - 1 || xx >= W - 1) return 0.f;
                return lap[interior_index(c, zz, yy, xx, D, H, W)];
            };
            const float li = lap[i];
            const float d2 = ((L(z + 1, y, x) - 2.f * li + L(z - 1, y, x)) * ihz2 +
                              (L(z, y + 1, x) - 2.f * li + L(z, y - 1, x)) * ihy2) +
                             (L(z, y, x + 1) - 2.f * li + L(z, y, x - 1)) * ihx2;
            out += alpha * (c == 0 ? hx : (c == 1 ? hy : hz)) * d2;
        }
        grad[i] = out;
    }
}

// ---------------------------------------------------------------------------------------------- smoothing, Adam
// one axis of the separable Gaussian over a (3, d0, d1, d2) array, replicate padding (preopt.py:134 _smooth)
__global__ void __launch_bounds__(PT) gauss_axis_kernel(const float *__restrict__ in, float *__restrict__ out,
                                                        int d0, int d1, int d2, int axis, const float *__restrict__ k,
                                                        int r) {
    const long long n = 3LL * d0 * d1 * d2;
    const long long st = axis == 0 ? (long long)d1 * d2 : (axis == 1 ? d2 : 1);
    const int len = axis == 0 ? d0 : (axis == 1 ? d1 : d2);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int pos = (int)((i / st) % len);
        const long long base = i - (long long)pos * st;
        float s = 0.f;
        for (int j = -r; j <= r; j++) {
            int q = pos + j;
            q = q < 0 ? 0 : (q > len - 1 ? len - 1 : q);
            s += k[j + r] * in[base + (long long)q * st];
        }
        out[i] = s;
    }
}

// Adam moments and step (the update itself waits for the largest entry): step into `step`, block maxima of |step|
__global__ void __launch_bounds__(PT) adam_kernel(long long n, const float *__restrict__ g, float *__restrict__ m,
                                                  float *__restrict__ v, float b1, float ob1, float b2, float ob2,
                                                  float lr, float rc1, float rc2, float eps, float *__restrict__ step,
                                                  float *partial) {
    float mx = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = m[i] * b1 + gi * ob1;
        const float vi = v[i] * b2 + ob2 * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float s = lr * (mi * rc1) / (sqrtf(vi * rc2) + eps);
        step[i] = s;
        mx = fmaxf(mx, fabsf(s));
    }
    __shared__ float sh[PT / 32];
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = fmaxf(r, sh[w]);
        partial[blockIdx.x] = r;
    }
}

// scale = 1 if largest <= cap else cap / largest (double, then float as PyTorch's float32 scalar); counts cap hits
__global__ void cap_kernel(const float *partial, int blocks, double cap, float *scale, unsigned long long *hits) {
    __shared__ float sh[PT];
    float m = 0.f;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) m = fmaxf(m, partial[b]);
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] = fmaxf(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double largest = (double)sh[0];
        const double sc = largest <= cap ? 1. : cap / largest;
        *scale = (float)sc;
        if (sc < 1.) *hits += 1;
    }
}

__global__ void __launch_bounds__(PT) update_kernel(long long n, const float *__restrict__ step,
                                                    const float *__restrict__ scale, float *__restrict__ u) {
    const float s = *scale;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        u[i] = u[i] - step[i] * s;
}

// terms[it * 6 + k] = data, geometry, floor, curvature, min det, total (from the block partials of one iteration)
__global__ void terms_kernel(const float *pd, int bd, const float *pc, int bc, const float *pl, int bl, float mu,
                             float kappa, float alpha, float *terms) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float data = 0.f, geo = 0.f, flo = 0.f, cur = 0.f, mneg = -__int_as_float(0x7F800000);
    for (int b = 0; b < bd; b++) data += pd[b];
    for (int b = 0; b < bc; b++) { geo += pc[2 * b]; flo += pc[2 * b + 1]; mneg = fmaxf(mneg, pc[2 * bc + b]); }
    for (int b = 0; b < bl; b++) cur += pl[b];
    geo = .5f * mu * geo;
    flo = kappa * flo;
    cur = alpha > 0.f ? alpha * cur : 0.f;
    terms[0] = data; terms[1] = geo; terms[2] = flo; terms[3] = cur; terms[4] = -mneg;
    terms[5] = ((data + geo) + flo) + cur;
}

// ---------------------------------------------------------------------------------------------- pyramid
// separable Gaussian (double) along one axis of a (nz, ny, nx) image, mode 'nearest' (scipy gaussian_filter1d)
__global__ void __launch_bounds__(PT) image_gauss_kernel(const double *__restrict__ in, double *__restrict__ out,
                                                         int nz, int ny, int nx, int axis, const double *__restrict__ k,
                                                         int r) {
    const long long n = (long long)nz * ny * nx;
    const long long st = axis == 0 ? (long long)ny * nx : (axis == 1 ? nx : 1);
    const int len = axis == 0 ? nz : (axis == 1 ? ny : nx);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int pos = (int)((i / st) % len);
        const long long base = i - (long long)pos * st;
        double s = 0.;
        for (int j = -r; j <= r; j++) {
            int q = pos + j;
            q = q < 0 ? 0 : (q > len - 1 ? len - 1 : q);
            s += k[j + r] * in[base + (long long)q * st];
        }
        out[i] = s;
    }
}

// separable linear resampling of a (nz, ny, nx, C) field: out(k2, k1, k0) = sum of the 8 corner weights; per axis
// (left index, weight) tables; C = 1 (images: map_coordinates order 1) or 3 (displacements: Q1 prolongation)
__global__ void __launch_bounds__(PT) resample_kernel(const double *__restrict__ in, int sz, int sy, int sx, int C,
                                                      double *__restrict__ out, int tz, int ty, int tx,
                                                      const int *__restrict__ lz, const double *__restrict__ wz,
                                                      const int *__restrict__ ly, const double *__restrict__ wy,
                                                      const int *__restrict__ lx, const double *__restrict__ wx) {
    const long long n = (long long)tz * ty * tx;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % tx), y = (int)((i / tx) % ty), z = (int)(i / ((long long)tx * ty));
        const int x0 = lx[x], y0 = ly[y], z0 = lz[z];
        const double ax = wx[x], ay = wy[y], az = wz[z];
        const int x1 = x0 + 1 < sx ? x0 + 1 : sx - 1, y1 = y0 + 1 < sy ? y0 + 1 : sy - 1, z1 = z0 + 1 < sz ? z0 + 1 : sz - 1;
        for (int c = 0; c < C; c++) {
            auto at = [&](int zz, int yy, int xx) { return in[(((long long)zz * sy + yy) * sx + xx) * C + c]; };
            // z first, then y, then x (the reference's axis order of the Q1 transfer); (1 - w) a + w b rounded
            // per operation (no contraction), as NumPy evaluates it
            auto lerp = [](double w, double a, double b) {
                return __dadd_rn(__dmul_rn(__dsub_rn(1., w), a), __dmul_rn(w, b));
            };
            const double p00 = lerp(az, at(z0, y0, x0), at(z1, y0, x0));
            const double p01 = lerp(az, at(z0, y0, x1), at(z1, y0, x1));
            const double p10 = lerp(az, at(z0, y1, x0), at(z1, y1, x0));
            const double p11 = lerp(az, at(z0, y1, x1), at(z1, y1, x1));
            out[i * C + c] = lerp(ax, lerp(ay, p00, p10), lerp(ay, p01, p11));
        }
    }
}

unsigned grid_for(long long n) { return blocks_for(n, PT, 8); }

}  // namespace
}  // namespace svp

using namespace svp;

extern "C" int svp_pre_energy_grad(const float *fixed, const float *moving, int32_t D, int32_t H, int32_t W,
                                   double hx, double hy, double hz, const float *u_int, double mu, double alpha,
                                   double kappa, double j0, float *grad, float *terms6, void *stream);

namespace {
struct PreWork {
    float *G = nullptr, *lap = nullptr, *partial = nullptr;
    unsigned bd = 0, bc = 0, bl = 0;
};

// one evaluation of the pre-objective's gradient (and its terms into terms_dev[6], device)
int pre_gradient(const float *F, const float *M, int D, int H, int W, const double h[3], const float *u, double mu,
                 double alpha, double kappa, double j0, float *grad, float *terms_dev, PreWork &w, cudaStream_t s) {
    const long long nn = (long long)D * H * W, nc = (long long)(D - 1) * (H - 1) * (W - 1);
    const long long ni = 3LL * (D - 2) * (H - 2) * (W - 2);
    float *pd = w.partial, *pc = pd + w.bd, *pl = pc + 3 * w.bc;
    const float r01 = (float)(h[0] / h[1]), r02 = (float)(h[0] / h[2]), r10 = (float)(h[1] / h[0]);
    const float r12 = (float)(h[1] / h[2]), r20 = (float)(h[2] / h[0]), r21 = (float)(h[2] / h[1]);
    const float ihx2 = (float)(1. / (h[0] * h[0])), ihy2 = (float)(1. / (h[1] * h[1])), ihz2 = (float)(1. / (h[2] * h[2]));
    { svp::KernelTimer _t("pre_data_kernel", s); SVP_LAUNCH(pre_data_kernel<<<w.bd, PT, 0, s>>>(F, M, D, H, W, u, grad, pd)); }
    { svp::KernelTimer _t("pre_cell_kernel", s); SVP_LAUNCH(pre_cell_kernel<<<w.bc, PT, 0, s>>>(D, H, W, r01, r02, r10, r12, r20, r21, (float)mu, (float)kappa, (float)j0, u, w.G, pc)); }
    if (alpha > 0) SVP_LAUNCH(pre_lap_kernel<<<w.bl, PT, 0, s>>>(D, H, W, ihx2, ihy2, ihz2, (float)h[0], (float)h[1], (float)h[2], u, w.lap, pl));
    { svp::KernelTimer _t("pre_node_kernel", s); SVP_LAUNCH(pre_node_kernel<<<grid_for(ni), PT, 0, s>>>(D, H, W, w.G, w.lap, (float)alpha, ihx2, ihy2, ihz2, (float)h[0], (float)h[1], (float)h[2], grad)); }
    SVP_LAUNCH(terms_kernel<<<1, 1, 0, s>>>(pd, w.bd, pc, w.bc, pl, alpha > 0 ? w.bl : 0, (float)mu, (float)kappa, (float)alpha, terms_dev));
    SVP_LAUNCH_CHECK("pre-objective gradient");
    (void)nn; (void)nc;
    return SVP_OK;
}

int pre_alloc(int D, int H, int W, PreWork &w, cudaStream_t s) {
    const long long nn = (long long)D * H * W, nc = (long long)(D - 1) * (H - 1) * (W - 1);
    const long long ni = 3LL * (D - 2) * (H - 2) * (W - 2);
    w.bd = grid_for(nn); w.bc = grid_for(nc); w.bl = grid_for(ni);
    SVP_CUDA(scratch_alloc((void **)&w.G, sizeof(float) * 9 * nc, s));
    SVP_CUDA(scratch_alloc((void **)&w.lap, sizeof(float) * ni, s));
    SVP_CUDA(scratch_alloc((void **)&w.partial, sizeof(float) * (w.bd + 3 * w.bc + w.bl), s));
    return SVP_OK;
}
void pre_free(PreWork &w, cudaStream_t s) {
    if (w.G) scratch_free(w.G, s);
    if (w.lap) scratch_free(w.lap, s);
    if (w.partial) scratch_free(w.partial, s);
}

// normalised float32 Gaussian taps exp(-x^2/(2 sigma^2)), radius ceil(3 sigma) (preopt.py:128 _gaussian_1d)
std::vector<float> gauss_taps(double sigma) {
    const int r = (int)std::ceil(3 * sigma);
    std::vector<float> k(2 * r + 1);
    float sum = 0.f;
    for (int j = -r; j <= r; j++) {
        const float x = (float)j / (float)sigma;
        k[j + r] = std::exp(-.5f * x * x);
    }
    for (float v : k) sum += v;
    for (float &v : k) v = v / sum;
    return k;
}
}  // namespace

extern "C" int svp_pre_energy_grad(const float *fixed, const float *moving, int32_t D, int32_t H, int32_t W,
                                   double hx, double hy, double hz, const float *u_int, double mu, double alpha,
                                   double kappa, double j0, float *grad, float *terms6, void *stream) {
    SVP_REQUIRE(fixed && moving && u_int && grad && terms6, "svp_pre_energy_grad: null argument");
    SVP_REQUIRE(D >= 3 && H >= 3 && W >= 3, "svp_pre_energy_grad: at least 3 nodes per axis");
    cudaStream_t s = (cudaStream_t)stream;
    const double h[3] = {hx, hy, hz};
    PreWork w;
    int rc = pre_alloc(D, H, W, w, s);
    float *tdev = nullptr;
    if (!rc && scratch_alloc((void **)&tdev, sizeof(float) * 6, s) != cudaSuccess) rc = fail(SVP_ENOMEM, "terms");
    if (!rc) rc = pre_gradient(fixed, moving, D, H, W, h, u_int, mu, alpha, kappa, j0, grad, tdev, w, s);
    if (!rc && cudaMemcpyAsync(terms6, tdev, sizeof(float) * 6, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = fail(SVP_ECUDA, "terms copy");
    if (tdev) scratch_free(tdev, s);
    pre_free(w, s);
    if (!rc) SVP_CUDA(cudaStreamSynchronize(s));
    return rc;
}

extern "C" int svp_pre_level(const float *fixed, const float *moving, int32_t D, int32_t H, int32_t W, double hx,
                             double hy, double hz, const svp_pre_params *prm, int32_t first_iteration,
                             int32_t iterations, float *u_int, float *m, float *v, float *terms_first,
                             float *terms_last, int64_t *cap_hits, void *stream) {
    SVP_REQUIRE(fixed && moving && prm && u_int && m && v, "svp_pre_level: null argument");
    SVP_REQUIRE(D >= 3 && H >= 3 && W >= 3 && iterations >= 0 && first_iteration >= 0, "svp_pre_level: bad sizes");
    SVP_REQUIRE(prm->beta1 < 1 && prm->beta2 < 1 && prm->lr > 0 && prm->cap > 0 && prm->eps > 0,
                "svp_pre_level: invalid Adam parameters");
    cudaStream_t s = (cudaStream_t)stream;
    const double h[3] = {hx, hy, hz};
    const long long ni = 3LL * (D - 2) * (H - 2) * (W - 2);
    PreWork w;
    int rc = pre_alloc(D, H, W, w, s);
    if (rc) return rc;
    float *grad = nullptr, *tmp = nullptr, *step = nullptr, *taps = nullptr, *scale = nullptr, *terms = nullptr;
    float *apart = nullptr;
    unsigned long long *hits = nullptr;
    const unsigned ab = grid_for(ni);
    std::vector<float> kg = gauss_taps(prm->sigma_grad > 0 ? prm->sigma_grad : 1.);
    std::vector<float> kf = gauss_taps(prm->sigma_field > 0 ? prm->sigma_field : 1.);
    const int rg = (int)(kg.size() / 2), rf = (int)(kf.size() / 2);
    auto bail = [&](int code) {
        for (void *p : {(void *)grad, (void *)tmp, (void *)step, (void *)taps, (void *)scale, (void *)terms,
                        (void *)apart, (void *)hits})
            if (p) scratch_free(p, s);
        pre_free(w, s);
        return code;
    };
    if (scratch_alloc((void **)&grad, sizeof(float) * ni, s) || scratch_alloc((void **)&tmp, sizeof(float) * ni, s) ||
        scratch_alloc((void **)&step, sizeof(float) * ni, s) ||
        scratch_alloc((void **)&taps, sizeof(float) * (kg.size() + kf.size()), s) ||
        scratch_alloc((void **)&scale, sizeof(float), s) ||
        scratch_alloc((void **)&terms, sizeof(float) * 12, s) || scratch_alloc((void **)&apart, sizeof(float) * ab, s) ||
        scratch_alloc((void **)&hits, sizeof(unsigned long long), s))
        return bail(fail(SVP_ENOMEM, "svp_pre_level: scratch"));
    if (cudaMemcpyAsync(taps, kg.data(), sizeof(float) * kg.size(), cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(taps + kg.size(), kf.data(), sizeof(float) * kf.size(), cudaMemcpyHostToDevice, s) ||
        cudaMemsetAsync(hits, 0, sizeof(unsigned long long), s) || cudaMemsetAsync(terms, 0, sizeof(float) * 12, s))
        return bail(fail(SVP_ECUDA, "svp_pre_level: setup copies"));
    const int dz = D - 2, dy = H - 2, dx = W - 2;
    auto smooth = [&](float *x, const float *k, int r) -> int {
        // z, then y, then x; x -> tmp -> x -> tmp -> ... ending in x
        SVP_LAUNCH_KEEP(gauss_axis_kernel<<<grid_for(ni), PT, 0, s>>>(x, tmp, dz, dy, dx, 0, k, r));
        SVP_LAUNCH_KEEP(gauss_axis_kernel<<<grid_for(ni), PT, 0, s>>>(tmp, step, dz, dy, dx, 1, k, r));
        SVP_LAUNCH_KEEP(gauss_axis_kernel<<<grid_for(ni), PT, 0, s>>>(step, x, dz, dy, dx, 2, k, r));
        return SVP_OK;
    };
    for (int it = 0; it < iterations; it++) {
        float *tdev = terms + (it == 0 ? 0 : 6);
        if ((rc = pre_gradient(fixed, moving, D, H, W, h, u_int, prm->mu, prm->alpha, prm->kappa, prm->j0, grad, tdev,
                               w, s)))
            return bail(rc);
        if (prm->sigma_grad > 0) smooth(grad, taps, rg);
        const int t = first_iteration + it + 1;
        // PyTorch divides by the float bias corrections as a multiplication by their float32 reciprocals
        const float rc1 = 1.f / (float)(1. - std::pow(prm->beta1, t));
        const float rc2 = 1.f / (float)(1. - std::pow(prm->beta2, t));
        { svp::KernelTimer _t("adam_kernel", s); SVP_LAUNCH_KEEP(adam_kernel<<<ab, PT, 0, s>>>(ni, grad, m, v, (float)prm->beta1, (float)(1. - prm->beta1), (float)prm->beta2, (float)(1. - prm->beta2), (float)prm->lr, rc1, rc2, (float)prm->eps, step, apart)); }
        SVP_LAUNCH_KEEP(cap_kernel<<<1, PT, 0, s>>>(apart, (int)ab, prm->cap, scale, hits));
        SVP_LAUNCH_KEEP(update_kernel<<<ab, PT, 0, s>>>(ni, step, scale, u_int));
        if (prm->sigma_field > 0) smooth(u_int, taps + kg.size(), rf);
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) return bail(cuda_fail(le, "pre-optimizer iteration"));
    }
    unsigned long long h_hits = 0;
    float th[12];
    if (cudaMemcpyAsync(th, terms, sizeof th, cudaMemcpyDeviceToHost, s) ||
        cudaMemcpyAsync(&h_hits, hits, sizeof h_hits, cudaMemcpyDeviceToHost, s))
        return bail(fail(SVP_ECUDA, "svp_pre_level: result copies"));
    rc = bail(SVP_OK);
    SVP_CUDA(cudaStreamSynchronize(s));
    if (terms_first) for (int k = 0; k < 6; k++) terms_first[k] = th[k];
    if (terms_last) for (int k = 0; k < 6; k++) terms_last[k] = iterations > 1 ? th[6 + k] : th[k];
    if (cap_hits) *cap_hits = (int64_t)h_hits;
    return rc;
}

extern "C" int svp_image_downsample(const double *src, int32_t nz, int32_t ny, int32_t nx, double *dst, int32_t mz,
                                    int32_t my, int32_t mx, void *stream) {
    SVP_REQUIRE(src && dst && nz >= 2 && ny >= 2 && nx >= 2 && mz >= 2 && my >= 2 && mx >= 2 && mz <= nz &&
                    my <= ny && mx <= nx, "svp_image_downsample: invalid sizes");
    cudaStream_t s = (cudaStream_t)stream;
    // nifti.py:128 downsample_array: Gaussian sigma = .5 sqrt(ratio^2 - 1) per axis (mode nearest, truncate 4), then
    // linear resampling at linspace(0, n - 1, m)
    const int n3[3] = {nz, ny, nx}, m3[3] = {mz, my, mx};
    const long long n = (long long)nz * ny * nx;
    double *a = nullptr, *b = nullptr, *kdev = nullptr, *wdev = nullptr;
    int *ldev = nullptr;
    auto bail = [&](int code) {
        for (void *p : {(void *)a, (void *)b, (void *)kdev, (void *)wdev, (void *)ldev}) if (p) scratch_free(p, s);
        return code;
    };
    std::vector<double> taps;
    std::vector<int> offs(4, 0), radius(3);
    for (int ax = 0; ax < 3; ax++) {
        const double ratio = (double)(n3[ax] - 1) / (double)(m3[ax] - 1);
        const double sd = .5 * std::sqrt(ratio * ratio - 1.);
        const int r = sd > 0 ? (int)(4. * sd + .5) : 0;
        radius[ax] = r;
        offs[ax] = (int)taps.size();
        std::vector<double> k(2 * r + 1);
        double sum = 0.;
        for (int j = -r; j <= r; j++) { k[j + r] = sd > 0 ? std::exp(-.5 / (sd * sd) * (double)j * j) : 1.; sum += k[j + r]; }
        for (double &v : k) taps.push_back(v / sum);
    }
    std::vector<int> left;
    std::vector<double> weight;
    for (int ax = 0; ax < 3; ax++) {
        for (int i = 0; i < m3[ax]; i++) {
            // np.linspace(0, n - 1, m): start + i * step, the last point exactly n - 1
            const double step = (double)(n3[ax] - 1) / (double)(m3[ax] - 1);
            double t = i == m3[ax] - 1 ? (double)(n3[ax] - 1) : i * step;
            int l = (int)std::floor(t);
            if (l > n3[ax] - 2) l = n3[ax] - 2;
            left.push_back(l);
            weight.push_back(t - l);
        }
    }
    if (scratch_alloc((void **)&a, sizeof(double) * n, s) || scratch_alloc((void **)&b, sizeof(double) * n, s) ||
        scratch_alloc((void **)&kdev, sizeof(double) * taps.size(), s) ||
        scratch_alloc((void **)&wdev, sizeof(double) * weight.size(), s) ||
        scratch_alloc((void **)&ldev, sizeof(int) * left.size(), s))
        return bail(fail(SVP_ENOMEM, "svp_image_downsample: scratch"));
    if (cudaMemcpyAsync(kdev, taps.data(), sizeof(double) * taps.size(), cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(wdev, weight.data(), sizeof(double) * weight.size(), cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(ldev, left.data(), sizeof(int) * left.size(), cudaMemcpyHostToDevice, s))
        return bail(fail(SVP_ECUDA, "svp_image_downsample: copies"));
    // scipy's gaussian_filter goes axis 0, 1, 2 (z, y, x)
    SVP_LAUNCH_KEEP(image_gauss_kernel<<<grid_for(n), PT, 0, s>>>(src, a, nz, ny, nx, 0, kdev + offs[0], radius[0]));
    SVP_LAUNCH_KEEP(image_gauss_kernel<<<grid_for(n), PT, 0, s>>>(a, b, nz, ny, nx, 1, kdev + offs[1], radius[1]));
    SVP_LAUNCH_KEEP(image_gauss_kernel<<<grid_for(n), PT, 0, s>>>(b, a, nz, ny, nx, 2, kdev + offs[2], radius[2]));
    SVP_LAUNCH_KEEP(resample_kernel<<<grid_for((long long)mz * my * mx), PT, 0, s>>>(a, nz, ny, nx, 1, dst, mz, my, mx,
                                                                          ldev, wdev, ldev + mz, wdev + mz,
                                                                          ldev + mz + my, wdev + mz + my));
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return bail(cuda_fail(le, "svp_image_downsample"));
    return bail(SVP_OK);
}

extern "C" int svp_field_prolong(const double *u, int32_t sz, int32_t sy, int32_t sx, double *out, int32_t tz,
                                 int32_t ty, int32_t tx, const int32_t *left_zyx, const double *weight_zyx,
                                 void *stream) {
    SVP_REQUIRE(u && out && left_zyx && weight_zyx && sz >= 2 && sy >= 2 && sx >= 2, "svp_field_prolong: arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const int nt = tz + ty + tx;
    for (int i = 0; i < nt; i++) {
        const int lim = i < tz ? sz : (i < tz + ty ? sy : sx);
        SVP_REQUIRE(left_zyx[i] >= 0 && left_zyx[i] <= lim - 2, "svp_field_prolong: left index out of range");
    }
    double *wdev = nullptr;
    int *ldev = nullptr;
    if (scratch_alloc((void **)&wdev, sizeof(double) * nt, s) || scratch_alloc((void **)&ldev, sizeof(int) * nt, s)) {
        if (wdev) scratch_free(wdev, s);
        return fail(SVP_ENOMEM, "svp_field_prolong: scratch");
    }
    int rc = SVP_OK;
    if (cudaMemcpyAsync(wdev, weight_zyx, sizeof(double) * nt, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(ldev, left_zyx, sizeof(int) * nt, cudaMemcpyHostToDevice, s))
        rc = fail(SVP_ECUDA, "svp_field_prolong: copies");
    if (!rc) {
        resample_kernel<<<grid_for((long long)tz * ty * tx), PT, 0, s>>>(u, sz, sy, sx, 3, out, tz, ty, tx, ldev, wdev,
                                                                        ldev + tz, wdev + tz, ldev + tz + ty,
                                                                        wdev + tz + ty);
        count_launch();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "resample_kernel");
    }
    scratch_free(wdev, s);
    scratch_free(ldev, s);
    if (!rc) SVP_CUDA(cudaStreamSynchronize(s));     // the host tables above must outlive the copies
    return rc;
}
