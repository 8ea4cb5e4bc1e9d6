// Library-wide C ABI pieces: per-thread error messages and the ABI version.
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "svp_common.cuh"

namespace svp {
namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
std::atomic<bool> g_timing{false};
std::mutex g_tmu;
struct TimerRec {
    std::string name;
    std::vector<cudaEvent_t> start, stop;  // recorded pairs not yet resolved
    std::vector<cudaEvent_t> pool;         // resolved events for reuse
    long long count = 0;
    double total_ms = 0.;
};
std::vector<TimerRec> g_timers;

int timer_slot(const char *name) {
    for (size_t k = 0; k < g_timers.size(); k++)
        if (g_timers[k].name == name) return (int)k;
    g_timers.push_back(TimerRec());
    g_timers.back().name = name;
    return (int)g_timers.size() - 1;
}
cudaEvent_t take_event(TimerRec &t) {
    if (!t.pool.empty()) {
        cudaEvent_t e = t.pool.back();
        t.pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
void resolve(TimerRec &t) {
    for (size_t k = 0; k < t.start.size(); k++) {
        float ms = 0.f;
        cudaEventSynchronize(t.stop[k]);
        if (cudaEventElapsedTime(&ms, t.start[k], t.stop[k]) == cudaSuccess) {
            t.total_ms += ms;
            t.count += 1;
        }
        t.pool.push_back(t.start[k]);
        t.pool.push_back(t.stop[k]);
    }
    t.start.clear();
    t.stop.clear();
}
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

KernelTimer::KernelTimer(const char *name, cudaStream_t stream) : slot_(-1), stream_(stream) {
    if (!g_timing.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lock(g_tmu);
    slot_ = timer_slot(name);
    TimerRec &t = g_timers[slot_];
    cudaEvent_t e = take_event(t);
    cudaEventRecord(e, stream_);
    t.start.push_back(e);
    if (t.start.size() > 8192) {  // bound the number of outstanding events
        t.stop.push_back(take_event(t));
        cudaEventRecord(t.stop.back(), stream_);
        t.start.pop_back(); t.stop.pop_back();
        resolve(t);
        t.start.push_back(take_event(t));
        cudaEventRecord(t.start.back(), stream_);
    }
}

KernelTimer::~KernelTimer() {
    if (slot_ < 0) return;
    std::lock_guard<std::mutex> lock(g_tmu);
    TimerRec &t = g_timers[slot_];
    cudaEvent_t e = take_event(t);
    cudaEventRecord(e, stream_);
    t.stop.push_back(e);
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (!g_pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t created;
            if ((e = cudaMemPoolCreate(&created, &props)) != cudaSuccess) return e;
            uint64_t keep = 64ull << 20;     // keep up to 64 MB mapped between calls
            cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
            g_pools[dev] = created;
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
}

cudaError_t scratch_free(void *ptr, cudaStream_t stream) { return cudaFreeAsync(ptr, stream); }

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t err, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
    return err == cudaErrorMemoryAllocation ? SVP_ENOMEM : SVP_ECUDA;
}
}  // namespace svp

extern "C" int svp_last_error(char *buf, size_t len) {
    const std::string &m = svp::g_last_error;
    if (buf && len) {
        size_t n = m.size() < len - 1 ? m.size() : len - 1;
        memcpy(buf, m.data(), n);
        buf[n] = 0;
    }
    return (int)m.size();
}

extern "C" int svp_version(void) { return 100; }

extern "C" int svp_counters(int64_t *launches) {
    if (launches) *launches = svp::g_launches.load();
    return SVP_OK;
}

extern "C" int svp_timers_enable(int on) {
    std::lock_guard<std::mutex> lock(svp::g_tmu);
    for (auto &t : svp::g_timers) {
        svp::resolve(t);
        t.count = 0;
        t.total_ms = 0.;
    }
    svp::g_timing.store(on != 0);
    return SVP_OK;
}

extern "C" int svp_timer_read(const char *name, int64_t *count, double *total_ms) {
    if (!name || !count || !total_ms) return svp::fail(SVP_EINVAL, "svp_timer_read: null argument");
    std::lock_guard<std::mutex> lock(svp::g_tmu);
    *count = 0;
    *total_ms = 0.;
    for (auto &t : svp::g_timers)
        if (t.name == name) {
            svp::resolve(t);
            *count = t.count;
            *total_ms = t.total_ms;
        }
    return SVP_OK;
}
