// SpMV with several right-hand sides in 16-byte aligned row-major blocks:
// the column-slice kernel shared by the SpMV entry points and the solvers.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace b2s {

constexpr int kLanesBlock = 256;

// ---------------------------------------------------------------------------
// Four or more right-hand sides: KL = K / VW lanes share one row and each
// owns VW consecutive columns (one 16-byte vector), so the lanes of a row
// read one contiguous stretch of b(col, :) and write one of c(row, :); the
// row's values and column indices are broadcast loads.  Used for Csr, Ell
// and Sellp; needs 16-byte aligned b/c rows.
// ---------------------------------------------------------------------------
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int width = 2;
};
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int width = 4;
};

template <typename T>
__device__ __forceinline__ void fma_vec(typename Vec16<T>::type& acc, T a,
                                        const T* p)
{
    const auto x = __ldg(reinterpret_cast<const typename Vec16<T>::type*>(p));
    if constexpr (Vec16<T>::width == 2) {
        acc.x += a * x.x;
        acc.y += a * x.y;
    } else {
        acc.x += a * x.x;
        acc.y += a * x.y;
        acc.z += a * x.z;
        acc.w += a * x.w;
    }
}

template <typename T>
__device__ __forceinline__ void store_vec(T* dst, const typename Vec16<T>::type& acc,
                                          const T* alpha, const T* beta)
{
    constexpr int W = Vec16<T>::width;
    const T* a = reinterpret_cast<const T*>(&acc);
    T out[W];
#pragma unroll
    for (int u = 0; u < W; ++u) out[u] = combine(a[u], alpha, beta, dst + u);
    *reinterpret_cast<typename Vec16<T>::type*>(dst) =
        *reinterpret_cast<const typename Vec16<T>::type*>(out);
}

// FMT 0: Csr, 1: Ell, 2: Sellp.  skip: when non-null and set, the whole
// grid returns (a solver whose columns have all stopped).
template <typename T, int K, int FMT>
__global__ void __launch_bounds__(kLanesBlock)
    rhs_lanes_kernel(int64_t n, const int32_t* __restrict__ rp,
                     int64_t width_or_slice, int64_t stride,
                     const uint64_t* __restrict__ slice_sets,
                     const uint64_t* __restrict__ slice_lengths,
                     const int32_t* __restrict__ ci, const T* __restrict__ v,
                     const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
                     int64_t ldc, const T* __restrict__ alpha,
                     const T* __restrict__ beta, const int* __restrict__ skip = nullptr)
{
    if (skip != nullptr && *skip) return;
    using V = typename Vec16<T>::type;
    constexpr int VW = Vec16<T>::width;
    constexpr int KL = K / VW;
    const int64_t g = blockIdx.x * int64_t(kLanesBlock) + threadIdx.x;
    const int64_t row = g / KL;
    if (row >= n) return;
    const int sub = int(g % KL);
    const T* bc = b + sub * VW;
    V acc;
    {
        T* a = reinterpret_cast<T*>(&acc);
#pragma unroll
        for (int u = 0; u < VW; ++u) a[u] = T(0);
    }
    int64_t first, step, len;
    if constexpr (FMT == 0) {
        first = rp[row];
        len = rp[row + 1] - first;
        step = 1;
    } else if constexpr (FMT == 1) {
        first = row;
        len = width_or_slice;
        step = stride;
    } else {
        const int64_t s = row / width_or_slice;
        first = int64_t(slice_sets[s]) * width_or_slice + (row - s * width_or_slice);
        len = int64_t(slice_lengths[s]);
        step = width_or_slice;
    }
    int64_t i = 0;
    for (; i + 4 <= len; i += 4) {
        int32_t col[4];
        T val[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            col[u] = __ldg(ci + first + (i + u) * step);
            val[u] = __ldg(v + first + (i + u) * step);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (FMT == 0 || col[u] != -1) fma_vec<T>(acc, val[u], bc + int64_t(col[u]) * ldb);
        }
    }
    for (; i < len; ++i) {
        const int32_t col = __ldg(ci + first + i * step);
        const T val = __ldg(v + first + i * step);
        if (FMT == 0 || col != -1) fma_vec<T>(acc, val, bc + int64_t(col) * ldb);
    }
    store_vec<T>(c + row * ldc + sub * VW, acc, alpha, beta);
}


// Ell (FMT 1) and Sellp (FMT 2) with two neighbouring rows per lane slot:
// the rows' column indices and values at each entry are one 8- or 16-byte
// vector load (the layouts are column-major, so rows r and r + 1 sit next
// to each other), and each slot gathers two 16-byte pieces of b per entry.
// Needs an even stride (Ell) or slice size (Sellp) and 16-byte aligned b
// and c rows; a row pair whose second row lies past the storage (odd n with
// stride n) falls back to single loads.
template <typename T, int K, int FMT>
__global__ void __launch_bounds__(kLanesBlock)
    rhs_lanes2_kernel(int64_t n, int64_t width_or_slice, int64_t stride,
                      const uint64_t* __restrict__ slice_sets,
                      const uint64_t* __restrict__ slice_lengths,
                      const int32_t* __restrict__ ci, const T* __restrict__ v,
                      const T* __restrict__ b, int64_t ldb, T* __restrict__ c, int64_t ldc,
                      const T* __restrict__ alpha, const T* __restrict__ beta)
{
    static_assert(FMT == 1 || FMT == 2, "Ell or Sellp");
    using V = typename Vec16<T>::type;
    using V2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    constexpr int VW = Vec16<T>::width;
    constexpr int KL = K / VW;
    const int64_t g = blockIdx.x * int64_t(kLanesBlock) + threadIdx.x;
    const int64_t r0 = 2 * (g / KL);
    if (r0 >= n) return;
    const int sub = int(g % KL);
    const T* bc = b + sub * VW;
    V acc0, acc1;
    {
        T* a0 = reinterpret_cast<T*>(&acc0);
        T* a1 = reinterpret_cast<T*>(&acc1);
#pragma unroll
        for (int u = 0; u < VW; ++u) a0[u] = a1[u] = T(0);
    }
    int64_t first, step, len;
    bool pair;
    if constexpr (FMT == 1) {
        first = r0;
        len = width_or_slice;
        step = stride;
        pair = r0 + 1 < stride;
    } else {
        const int64_t sl = r0 / width_or_slice;
        first = int64_t(slice_sets[sl]) * width_or_slice + (r0 - sl * width_or_slice);
        len = int64_t(slice_lengths[sl]);
        step = width_or_slice;
        pair = true;
    }
    const bool second = r0 + 1 < n;
    if (pair) {
        // four entries' index and value pairs in flight before their gathers
        // (padding-heavy slices are bound by these loads, not the gathers)
        int64_t i = 0;
        for (; i + 4 <= len; i += 4) {
            int2 cc[4];
            V2 vv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int64_t e = first + (i + u) * step;
                cc[u] = __ldg(reinterpret_cast<const int2*>(ci + e));
                vv[u] = __ldg(reinterpret_cast<const V2*>(v + e));
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (cc[u].x != -1) fma_vec<T>(acc0, vv[u].x, bc + int64_t(cc[u].x) * ldb);
                if (second && cc[u].y != -1) {
                    fma_vec<T>(acc1, vv[u].y, bc + int64_t(cc[u].y) * ldb);
                }
            }
        }
        for (; i < len; ++i) {
            const int64_t e = first + i * step;
            const int2 cc = __ldg(reinterpret_cast<const int2*>(ci + e));
            const V2 vv = __ldg(reinterpret_cast<const V2*>(v + e));
            if (cc.x != -1) fma_vec<T>(acc0, vv.x, bc + int64_t(cc.x) * ldb);
            if (second && cc.y != -1) fma_vec<T>(acc1, vv.y, bc + int64_t(cc.y) * ldb);
        }
    } else {
        for (int64_t i = 0; i < len; ++i) {
            const int64_t e = first + i * step;
            const int32_t col = __ldg(ci + e);
            if (col != -1) fma_vec<T>(acc0, __ldg(v + e), bc + int64_t(col) * ldb);
        }
    }
    store_vec<T>(c + r0 * ldc + sub * VW, acc0, alpha, beta);
    if (second) store_vec<T>(c + (r0 + 1) * ldc + sub * VW, acc1, alpha, beta);
}

// Launches rhs_lanes_kernel on Csr for K right-hand sides (K >= 4 and a
// multiple of the 16-byte vector width; b and c rows 16-byte aligned).
template <typename T, int K>
void launch_csr_lanes(int64_t n, const int32_t* rp, const int32_t* ci, const T* v, const T* b,
                      int64_t ldb, T* c, int64_t ldc, const T* alpha, const T* beta,
                      cudaStream_t st, const int* skip = nullptr)
{
    static_assert(K >= 4 && K % Vec16<T>::width == 0, "column slices of 16 bytes");
    constexpr int KL = K / Vec16<T>::width;
    rhs_lanes_kernel<T, K, 0><<<ceildiv(n * KL, kLanesBlock), kLanesBlock, 0, st>>>(
        n, rp, 0, 0, nullptr, nullptr, ci, v, b, ldb, c, ldc, alpha, beta, skip);
}

}  // namespace b2s
