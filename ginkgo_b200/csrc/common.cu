// Error reporting and version query of libginkgo_b200.
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

}  // namespace b2s

extern "C" {

const char* b2s_last_error(void) { return b2s::g_error; }

int b2s_version(void) { return B2S_VERSION; }

}  // extern "C"
