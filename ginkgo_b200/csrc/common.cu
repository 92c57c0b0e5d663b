// Error reporting and version query of libginkgo_b200.
#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "common.cuh"

namespace b2s {

namespace {
thread_local char g_error[512] = "";
}

void set_error(const char* fmt, ...)
{
    va_list args;
    va_start(args, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, args);
    va_end(args);
}

int num_sms()
{
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices];  // 0 = not looked up yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        (void)cudaGetLastError();
        return kMaxSMs;
    }
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                cudaSuccess ||
            n < 1) {
            (void)cudaGetLastError();
            n = kMaxSMs;
        }
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

}  // namespace b2s

extern "C" {

const char* b2s_last_error(void) { return b2s::g_error; }

int b2s_version(void) { return B2S_VERSION; }

}  // extern "C"
