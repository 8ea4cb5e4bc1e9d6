// Shared device/host helpers of libsvp3d: error state, grid geometry, binary64 interval primitives.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/svp3d.h"

// ------------------------------------------------------------------------------------------------ error handling
namespace svp {
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t err, const char *what);
void count_launch();
// Stream-ordered scratch from the library's own memory pool on the current device (it keeps its memory between
// calls, so the small per-call reductions never map new pages): cudaMallocFromPoolAsync / cudaFreeAsync.
cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream);
cudaError_t scratch_free(void *ptr, cudaStream_t stream);

// Opt-in per-kernel CUDA-event timing (svp_timers_enable): a scope records an event pair on its stream around the
// launches inside it; svp_timer_read resolves and sums them.
class KernelTimer {
  public:
    KernelTimer(const char *name, cudaStream_t stream);
    ~KernelTimer();
  private:
    int slot_;
    cudaStream_t stream_;
};
}  // namespace svp

#define SVP_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess) return svp::cuda_fail(_e, #call);                             \
    } while (0)

#define SVP_LAUNCH_CHECK(what)                                                               \
    do {                                                                                     \
        cudaError_t _e = cudaGetLastError();                                                 \
        if (_e != cudaSuccess) return svp::cuda_fail(_e, what);                              \
    } while (0)

// Every kernel launch of the library goes through SVP_LAUNCH: it is counted (svp_counters) and its launch error
// returned as an SVP status.
#define SVP_LAUNCH(...)                                                                      \
    do {                                                                                     \
        __VA_ARGS__;                                                                         \
        svp::count_launch();                                                                 \
        cudaError_t _e = cudaGetLastError();                                                 \
        if (_e != cudaSuccess) return svp::cuda_fail(_e, #__VA_ARGS__);                      \
    } while (0)

// SVP_LAUNCH without the early return, for launches between a scratch allocation and its release: the caller reads
// cudaGetLastError() after releasing the scratch, so no error path leaks it.
#define SVP_LAUNCH_KEEP(...)                                                                 \
    do {                                                                                     \
        __VA_ARGS__;                                                                         \
        svp::count_launch();                                                                 \
    } while (0)

#define SVP_REQUIRE(cond, msg)                                                               \
    do {                                                                                     \
        if (!(cond)) return svp::fail(SVP_EINVAL, msg);                                      \
    } while (0)

namespace svp {

constexpr int kSMs = 148;  // B200: grid sizes are multiples of the SM count

// Flat index -> (x, y, z) over rows of nx entries and planes of ny rows.  In 32-bit unsigned arithmetic when the
// index and the plane size fit (a 64-bit integer division is a long instruction sequence on the GPU; every grid below
// 2^32 entries takes this path), in 64 bits otherwise.
__device__ __forceinline__ void unflatten3(long long i, long long nx, long long ny, long long &x, long long &y,
                                           long long &z) {
    if ((unsigned long long)i <= 0xFFFFFFFFull && (unsigned long long)(nx * ny) <= 0xFFFFFFFFull) {
        const unsigned u = (unsigned)i, a = (unsigned)nx, b = (unsigned)ny;
        const unsigned r = u / a;
        x = (long long)(u - r * a);
        y = (long long)(r % b);
        z = (long long)(r / b);
    } else {
        x = i % nx;
        y = (i / nx) % ny;
        z = i / (nx * ny);
    }
}

inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Grid launch helper: enough blocks to cover n items, capped at a multiple of the SM count (grid-stride kernels).
inline unsigned blocks_for(int64_t n, int threads, int per_sm = 16) {
    int64_t need = div_up(n, threads);
    int64_t cap = (int64_t)kSMs * per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

inline bool grid_ok(const svp_grid *g) {
    return g && g->nx >= 2 && g->ny >= 2 && g->nz >= 2 && g->hx > 0 && g->hy > 0 && g->hz > 0;
}
inline int64_t n_nodes(const svp_grid *g) { return g->nx * g->ny * g->nz; }
inline int64_t n_cells(const svp_grid *g) { return (g->nx - 1) * (g->ny - 1) * (g->nz - 1); }
inline int64_t n_free(const svp_grid *g) { return (g->nx - 2) * (g->ny - 2) * (g->nz - 2); }

// ------------------------------------------------------------------------------------------------ device numerics
// Every certificate operation is an explicit round-to-nearest intrinsic: none can be contracted into an FMA.
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ bool finite64(double x) {
    return (__double_as_longlong(x) & 0x7FF0000000000000LL) != 0x7FF0000000000000LL;
}

// nextafter(x, -inf) and nextafter(x, +inf) as integer steps on the IEEE-754 encoding: the adjacent representable
// value toward the direction (subnormals, signed zeros and infinities included); a NaN is returned with its quiet
// bit set.
__device__ __forceinline__ double step_down(double x) {
    long long b = __double_as_longlong(x);
    long long a = b & 0x7FFFFFFFFFFFFFFFLL;
    if (a > 0x7FF0000000000000LL) return __longlong_as_double(b | 0x0008000000000000LL);
    if (b == (long long)0xFFF0000000000000ULL) return x;                   // -inf
    if (a == 0) return __longlong_as_double((long long)0x8000000000000001ULL);  // +-0 -> -min subnormal
    return __longlong_as_double(b >= 0 ? b - 1 : b + 1);
}
__device__ __forceinline__ double step_up(double x) {
    long long b = __double_as_longlong(x);
    long long a = b & 0x7FFFFFFFFFFFFFFFLL;
    if (a > 0x7FF0000000000000LL) return __longlong_as_double(b | 0x0008000000000000LL);
    if (b == 0x7FF0000000000000LL) return x;                                // +inf
    if (a == 0) return __longlong_as_double(1LL);                           // +-0 -> +min subnormal
    return __longlong_as_double(b >= 0 ? b + 1 : b - 1);
}

// Numba's scalar np.minimum / np.maximum: the first operand when a <= b (a >= b) or when a is NaN, else the second.
__device__ __forceinline__ double nmin(double a, double b) { return (a <= b || a != a) ? a : b; }
__device__ __forceinline__ double nmax(double a, double b) { return (a >= b || a != a) ? a : b; }

// Outward step after a round-to-nearest operation; valid iff both ends finite and lo <= hi.
__device__ __forceinline__ bool iout(double lo, double hi, double &rl, double &rh) {
    rl = step_down(lo);
    rh = step_up(hi);
    return finite64(rl) && finite64(rh) && rl <= rh;
}
__device__ __forceinline__ bool iadd(double al, double ah, double bl, double bh, double &rl, double &rh) {
    return iout(radd(al, bl), radd(ah, bh), rl, rh);
}
__device__ __forceinline__ bool isub(double al, double ah, double bl, double bh, double &rl, double &rh) {
    return iout(rsub(al, bh), rsub(ah, bl), rl, rh);
}
__device__ __forceinline__ bool imul(double al, double ah, double bl, double bh, double &rl, double &rh) {
    double x = rmul(al, bl), y = rmul(al, bh), z = rmul(ah, bl), w = rmul(ah, bh);
    return iout(nmin(nmin(nmin(x, y), z), w), nmax(nmax(nmax(x, y), z), w), rl, rh);
}

// Left-associated cofactor expansion of an interval 3x3 matrix, every operation outward.
__device__ __forceinline__ bool idet(const double fl[3][3], const double fh[3][3], double &jl, double &jh) {
    double p1l, p1h, p2l, p2h, al, ah, bl, bh, cl, ch, t1l, t1h, t2l, t2h, sl, sh, t3l, t3h;
    bool ok = true;
    ok &= imul(fl[1][1], fh[1][1], fl[2][2], fh[2][2], p1l, p1h);
    ok &= imul(fl[1][2], fh[1][2], fl[2][1], fh[2][1], p2l, p2h);
    ok &= isub(p1l, p1h, p2l, p2h, al, ah);
    ok &= imul(fl[1][2], fh[1][2], fl[2][0], fh[2][0], p1l, p1h);
    ok &= imul(fl[1][0], fh[1][0], fl[2][2], fh[2][2], p2l, p2h);
    ok &= isub(p1l, p1h, p2l, p2h, bl, bh);
    ok &= imul(fl[1][0], fh[1][0], fl[2][1], fh[2][1], p1l, p1h);
    ok &= imul(fl[1][1], fh[1][1], fl[2][0], fh[2][0], p2l, p2h);
    ok &= isub(p1l, p1h, p2l, p2h, cl, ch);
    ok &= imul(fl[0][0], fh[0][0], al, ah, t1l, t1h);
    ok &= imul(fl[0][1], fh[0][1], bl, bh, t2l, t2h);
    ok &= iadd(t1l, t1h, t2l, t2h, sl, sh);
    ok &= imul(fl[0][2], fh[0][2], cl, ch, t3l, t3h);
    ok &= iadd(sl, sh, t3l, t3h, jl, jh);
    return ok;
}

// Order-preserving map of a double onto int64 (for atomicMin/atomicMax of finite values; -0 sorts below +0).
__device__ __forceinline__ long long order_key(double x) {
    long long b = __double_as_longlong(x);
    return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFFLL);
}
__host__ __device__ inline double key_value(long long k) {
    long long b = k ^ ((k >> 63) & 0x7FFFFFFFFFFFFFFFLL);
#ifdef __CUDA_ARCH__
    return __longlong_as_double(b);
#else
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
#endif
}
constexpr long long kKeyPosInf = 0x7FF0000000000000LL;  // order_key(+inf)

}  // namespace svp
