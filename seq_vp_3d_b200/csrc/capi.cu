// Library-wide C ABI pieces: per-thread error messages and the ABI version.
#include <cstring>
#include <string>

#include "svp_common.cuh"

namespace svp {
namespace {
thread_local std::string g_last_error;
}

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
