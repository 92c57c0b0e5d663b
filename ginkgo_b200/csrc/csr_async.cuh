// The pipelined Csr SpMV kernel, shared by the SpMV entry points and the
// fused solvers (which pass a device flag that makes an idle launch return
// at once).
#pragma once

#include <mutex>
#include <utility>
#include <vector>

#include "common.cuh"

namespace b2s {


// ---------------------------------------------------------------------------
// Csr, persistent and pipelined: every warp walks groups of R = 32 / LPR
// consecutive rows with a stride of the grid's warp count.  The values and
// column indices of the next group are copied into shared memory with
// cp.async while the current group is reduced, and the row pointers of the
// group after that are loaded at the same time, so neither the matrix
// stream nor the next copy waits for a row-pointer load or an x gather.
// Each row is then summed from shared memory by LPR lanes (LPR = 1: each
// lane sums its own row in order, the reference's sequential row sum of
// reference/matrix/csr_kernels.cpp:65-74).  Groups with more than kAsyncCap
// entries are reduced row by row by the whole warp straight from global
// memory.
// ---------------------------------------------------------------------------
constexpr int kAsyncCap = 256;  // staged entries per group and stage
constexpr int kAsyncBlock = 256;

// Lanes per row: the fewest that keep a group of 32 / LPR rows of the
// longest length within one stage, at most 4 (groups of 8 rows): with
// longer rows the groups that overflow a stage take the row-by-row path,
// and the short rows of an irregular matrix still share warps.
inline int async_lanes_per_row(int64_t max_row_nnz)
{
    int lpr = 1;
    while (lpr < 4 && (32 / lpr) * max_row_nnz > kAsyncCap) lpr *= 2;
    return lpr;
}

// Blocks of kAsyncBlock threads of `kernel` that are resident at once on all
// SMs: the persistent grid (cached per kernel).
template <typename Kern>
int async_resident_blocks(Kern kernel)
{
    static std::mutex m;
    static std::vector<std::pair<const void*, int>> cache;
    std::lock_guard<std::mutex> lock(m);
    const void* key = reinterpret_cast<const void*>(kernel);
    for (const auto& e : cache) {
        if (e.first == key) return e.second * num_sms();
    }
    // four 48 KB blocks per SM leave the rest of the unified L1 (about a
    // fifth) for the x gathers; a larger shared-memory carveout measured
    // slower on the 7-point matrix
    (void)cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 80);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kAsyncBlock, 0) !=
            cudaSuccess ||
        per_sm < 1) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    cache.emplace_back(key, per_sm);
    return per_sm * num_sms();
}

// One element copy of 4 or 8 bytes (the element's own size and alignment).
template <typename E>
__device__ __forceinline__ void cp_async_elem(E* smem, const E* gmem)
{
    static_assert(sizeof(E) == 4 || sizeof(E) == 8, "4- or 8-byte elements");
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (sizeof(E) == 8) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
    }
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void cp_async_wait_one()
{
    asm volatile("cp.async.wait_group 1;\n" ::);
}

// A stage holds one group's values and column indices.
template <typename T>
struct __align__(16) AsyncStage {
    T vals[kAsyncCap];
    int32_t cols[kAsyncCap];
};

template <typename T, int K, bool VEC, int LPR = 1>
__global__ void __launch_bounds__(kAsyncBlock)
    csr_async_kernel(int64_t n, const int32_t* __restrict__ rp,
                     const int32_t* __restrict__ ci, const T* __restrict__ v,
                     const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
                     int64_t ldc, const T* __restrict__ alpha,
                     const T* __restrict__ beta,
                     const int* __restrict__ skip = nullptr)
{
    static_assert(LPR >= 1 && LPR <= 32 && (32 % LPR) == 0, "LPR divides 32");
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int R = kWarp / LPR;  // rows per group
    constexpr int kCap = kAsyncCap;  // staged entries
    __shared__ AsyncStage<T> stages[kAsyncBlock / kWarp][2];
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const int myrow = lane / LPR, sub = lane % LPR;
    const int64_t ngroups = (n + R - 1) / R;
    const int64_t nwarps = int64_t(gridDim.x) * (kAsyncBlock / kWarp);
    AsyncStage<T>* st = stages[wid];
    // row pointers of group g: lane l holds rp[row0 + l], pe = rp[row0 + R]
    // (clamped at n); loaded one group before they are needed
    auto load_ptrs = [&](int64_t g, int& p, int& pe) {
        const int64_t row0 = g * R;
        const int64_t pl = row0 + lane;
        p = __ldg(rp + (pl < n ? pl : n));
        pe = __ldg(rp + (row0 + R < n ? row0 + R : n));
    };
    // row span [rs, re) of this lane's row, group start and count
    auto desc = [&](int p, int pe, int& rs, int& re, int& start, int& cnt) {
        rs = __shfl_sync(kFull, p, myrow);
        const int nx = __shfl_sync(kFull, p, myrow + 1 < kWarp ? myrow + 1 : kWarp - 1);
        re = myrow + 1 < R ? nx : pe;
        start = __shfl_sync(kFull, p, 0);
        cnt = pe - start;
    };
    auto issue = [&](int s, int start, int cnt) {
        for (int i = lane; i < cnt; i += kWarp) {
            cp_async_elem(&st[s].vals[i], v + start + i);
            cp_async_elem(&st[s].cols[i], ci + start + i);
        }
    };
    if (skip != nullptr && *skip) return;  // whole grid (solver idle)
    int64_t g = blockIdx.x * int64_t(kAsyncBlock / kWarp) + wid;
    if (g >= ngroups) return;  // whole warp
    int rs, re, start, cnt, p, pe;
    load_ptrs(g, p, pe);
    desc(p, pe, rs, re, start, cnt);
    if (cnt <= kCap) issue(0, start, cnt);
    cp_async_commit();
    // pointers of the group after the next
    int pn = 0, pen = 0;
    if (g + nwarps < ngroups) load_ptrs(g + nwarps, pn, pen);
    int s = 0;
    for (; g < ngroups; g += nwarps) {
        const int64_t gn = g + nwarps;
        int nrs = 0, nre = 0, nstart = 0, ncnt = 0;
        if (gn < ngroups) {
            desc(pn, pen, nrs, nre, nstart, ncnt);
            if (ncnt <= kCap) issue(s ^ 1, nstart, ncnt);
            if (gn + nwarps < ngroups) load_ptrs(gn + nwarps, pn, pen);
        }
        cp_async_commit();
        cp_async_wait_one();
        __syncwarp();
        T acc[K];
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = T(0);
        const int64_t row = g * R + myrow;
        if (cnt <= kCap) {
            const AsyncStage<T>& cur = st[s];
            const T* cv = cur.vals;
            const int32_t* cc = cur.cols;
#pragma unroll 4
            for (int i = rs - start + sub; i < re - start; i += LPR) {
                T xr[K];
                RowLoad<T, K, VEC>::load(b + int64_t(cc[i]) * ldb, xr);
#pragma unroll
                for (int j = 0; j < K; ++j) acc[j] += cv[i] * xr[j];
            }
            if constexpr (LPR > 1) {
#pragma unroll
                for (int j = 0; j < K; ++j) acc[j] = subwarp_sum<LPR>(acc[j]);
            }
        } else {
            for (int l = 0; l < R; ++l) {
                const int s0 = __shfl_sync(kFull, rs, l * LPR);
                const int e0 = __shfl_sync(kFull, re, l * LPR);
                T a[K];
#pragma unroll
                for (int j = 0; j < K; ++j) a[j] = T(0);
                for (int ee = s0 + lane; ee < e0; ee += kWarp) {
                    const T val = ld_stream(v + ee);
                    T xr[K];
                    RowLoad<T, K, VEC>::load(b + int64_t(ld_stream(ci + ee)) * ldb, xr);
#pragma unroll
                    for (int j = 0; j < K; ++j) a[j] += val * xr[j];
                }
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    a[j] = warp_sum(a[j]);
                    if (myrow == l) acc[j] = a[j];
                }
            }
        }
        if (row < n) {
            T* dst = c + row * ldc;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (j % LPR == sub) dst[j] = combine(acc[j], alpha, beta, dst + j);
            }
        }
        __syncwarp();  // stage s is refilled two groups later
        s ^= 1;
        rs = nrs;
        re = nre;
        start = nstart;
        cnt = ncnt;
    }
}

// Calls f(csr_async_kernel<T, K, VEC, LPR>) for the runtime lanes-per-row
// value lpr (1, 2 or 4, from async_lanes_per_row).
template <typename T, int K, bool VEC, typename F>
void with_async_kernel(int lpr, F&& f)
{
    switch (lpr) {
    case 1: f(csr_async_kernel<T, K, VEC, 1>); break;
    case 2: f(csr_async_kernel<T, K, VEC, 2>); break;
    default: f(csr_async_kernel<T, K, VEC, 4>); break;
    }
}


}  // namespace b2s
