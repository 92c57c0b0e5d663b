// Shared device/host helpers of libginkgo_b200 (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/ginkgo_b200.h"

namespace b2s {

constexpr int kWarp = 32;
// Upper bound on the SM count for the grid bounds that size partial-sum
// buffers (B200: 148 SMs on two dies); launches use the device's own count
// from num_sms(), capped at this bound where a buffer is sized by it.
constexpr int kMaxSMs = 148;

// Multiprocessors of the current device (cudaDevAttrMultiProcessorCount),
// looked up once per device; kMaxSMs when the query fails.
int num_sms();

// The grid of a persistent (grid-stride) kernel launched with `threads`
// threads per block: `grid` cut to the blocks of `kernel` resident at once
// on all SMs (the occupancy query cached per kernel), so its last blocks do
// not run as a partial second wave: eight 256-thread blocks per SM are 1.6
// waves of a 48-register kernel, which holds five.
template <typename Kern>
int resident_grid(Kern kernel, int threads, int64_t grid)
{
    static std::mutex m;
    static std::vector<std::pair<const void*, int>> cache;
    const void* key = reinterpret_cast<const void*>(kernel);
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(m);
        for (const auto& e : cache) {
            if (e.first == key) per_sm = e.second;
        }
        if (per_sm == 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) !=
                    cudaSuccess ||
                per_sm < 1) {
                (void)cudaGetLastError();
                per_sm = 64;  // unknown: leave the grid as it is
            }
            cache.emplace_back(key, per_sm);
        }
    }
    const int64_t resident = int64_t(per_sm) * num_sms();
    return int(grid < 1 ? 1 : (grid < resident ? grid : resident));
}

// Thread-local last-error message, read through b2s_last_error().
void set_error(const char* fmt, ...);

#define B2S_CHECK_ARG(cond, ...)                  \
    do {                                          \
        if (!(cond)) {                            \
            ::b2s::set_error(__VA_ARGS__);        \
            return B2S_ERR_INVALID_ARG;           \
        }                                         \
    } while (0)

#define B2S_CUDA_TRY(expr)                                                  \
    do {                                                                    \
        cudaError_t err_ = (expr);                                          \
        if (err_ != cudaSuccess) {                                          \
            ::b2s::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,    \
                             cudaGetErrorString(err_));                     \
            return B2S_ERR_CUDA;                                            \
        }                                                                   \
    } while (0)

#define B2S_LAUNCH_CHECK() B2S_CUDA_TRY(cudaGetLastError())

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

__host__ __device__ inline int64_t ceildiv(int64_t a, int64_t b)
{
    return (a + b - 1) / b;
}

// ---- device helpers ----

template <typename T>
__device__ __forceinline__ T ldg(const T* p)
{
    return __ldg(p);
}

// Streaming (read-once) loads: evict-first so matrix data does not push the
// reused vectors out of L2.
__device__ __forceinline__ double ld_stream(const double* p)
{
    return __ldcs(p);
}
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }

template <int SW, typename T>
__device__ __forceinline__ T subwarp_sum(T v, unsigned mask = 0xffffffffu)
{
#pragma unroll
    for (int off = SW / 2; off > 0; off /= 2) {
        v += __shfl_xor_sync(mask, v, off, SW);
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
    return subwarp_sum<32>(v);
}

// Loads K consecutive values starting at p (K a power of two <= 16);
// VEC selects 16-byte vector loads (caller guarantees alignment).
template <typename T, int K, bool VEC>
struct RowLoad {
    __device__ __forceinline__ static void load(const T* p, T (&out)[K])
    {
#pragma unroll
        for (int j = 0; j < K; ++j) out[j] = __ldg(p + j);
    }
};

template <int K>
struct RowLoad<double, K, true> {
    __device__ __forceinline__ static void load(const double* p,
                                                double (&out)[K])
    {
#pragma unroll
        for (int j = 0; j < K; j += 2) {
            double2 t = __ldg(reinterpret_cast<const double2*>(p + j));
            out[j] = t.x;
            out[j + 1] = t.y;
        }
    }
};

template <int K>
struct RowLoad<float, K, true> {
    __device__ __forceinline__ static void load(const float* p, float (&out)[K])
    {
        if constexpr (K % 4 == 0) {
#pragma unroll
            for (int j = 0; j < K; j += 4) {
                float4 t = __ldg(reinterpret_cast<const float4*>(p + j));
                out[j] = t.x;
                out[j + 1] = t.y;
                out[j + 2] = t.z;
                out[j + 3] = t.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < K; j += 2) {
                float2 t = __ldg(reinterpret_cast<const float2*>(p + j));
                out[j] = t.x;
                out[j + 1] = t.y;
            }
        }
    }
};

// c = alpha * acc + beta * c, with Ginkgo's rule that beta == 0 ignores the
// old contents of c (NaN included); alpha == nullptr selects c = acc.
template <typename T>
__device__ __forceinline__ T combine(T acc, const T* alpha, const T* beta,
                                     const T* c_old)
{
    if (alpha == nullptr) return acc;
    T a = *alpha, b = *beta;
    return b == T(0) ? a * acc : a * acc + b * *c_old;
}

}  // namespace b2s
