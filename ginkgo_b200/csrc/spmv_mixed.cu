// Sparse matrix times dense block with mixed value types: the matrix, the
// input block and the output block each FP64 or FP32, the arithmetic in the
// most precise of the three (the reference's highest_precision,
// common/cuda_hip/matrix/csr_kernels.template.cpp:2109-2110; the kernels
// are instantiated for every mixed combination by
// GKO_INSTANTIATE_FOR_EACH_MIXED_VALUE_AND_INDEX_TYPE,
// core/matrix/csr_kernels.hpp:29-42, core/matrix/ell_kernels.hpp:21-26).
// Csr and Ell take mixed operands in the reference (mixed_precision_dispatch
// in core/matrix/csr.cpp:257-314, ell.cpp:125-160); Sellp converts its
// operands to the matrix type (precision_dispatch, sellp.cpp:150-180), which
// b2s_dense_convert provides here.
//
// Advanced form: c = alpha A b + beta c with alpha in the matrix type and
// beta in the output type, both converted to the arithmetic type; beta == 0
// ignores the old c.  Values and products are formed in the arithmetic type
// and the result rounded once to the output type.
//
// Kernels: Csr with one column, the pipelined kernel (csr_async_mixed_kernel);
// with several, one subwarp of SW lanes per row (SW from the longest row),
// KC columns per pass; Ell, one thread per row over the column-major slots.
// Uniform types are accepted too, but the tuned kernels of spmv.cu
// (b2s_csr_spmv_f64/_f32, b2s_ell_spmv_*) are the fast path for them.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "csr_async.cuh"

namespace b2s {
namespace {

constexpr int kMixBlock = 256;

template <typename A, typename B>
using wider_t = std::conditional_t<(sizeof(A) >= sizeof(B)), A, B>;

template <typename TM, typename TI, typename TO>
using arith_t = wider_t<wider_t<TM, TI>, TO>;

template <typename TA, typename TO, typename TM>
__device__ __forceinline__ TO finish(TA acc, const TM* alpha, const TO* beta,
                                     const TO* c_old)
{
    if (alpha == nullptr) return TO(acc);
    const TA a = TA(*alpha), b = TA(*beta);
    return b == TA(0) ? TO(a * acc) : TO(a * acc + b * TA(*c_old));
}

template <typename TM, typename TI, typename TO, int SW, int KC>
__global__ void __launch_bounds__(kMixBlock)
    csr_mixed_kernel(int64_t n, const int32_t* __restrict__ rp,
                     const int32_t* __restrict__ ci, const TM* __restrict__ v,
                     const TI* __restrict__ b, int64_t ldb, TO* __restrict__ c,
                     int64_t ldc, int k, int col0, const TM* __restrict__ alpha,
                     const TO* __restrict__ beta)
{
    using TA = arith_t<TM, TI, TO>;
    const int64_t row = (blockIdx.x * int64_t(kMixBlock) + threadIdx.x) / SW;
    const int lane = threadIdx.x % SW;
    // rows past n run with an empty range, so every lane of the subwarp
    // reaches the shuffles
    const bool valid = row < n;
    const int begin = valid ? __ldg(rp + row) : 0;
    const int end = valid ? __ldg(rp + row + 1) : 0;
    const int kc = min(KC, k - col0);
    TA acc[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) acc[j] = TA(0);
    for (int e = begin + lane; e < end; e += SW) {
        const TA val = TA(ld_stream(v + e));
        const TI* xr = b + int64_t(ld_stream(ci + e)) * ldb + col0;
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            if (j < kc) acc[j] += val * TA(__ldg(xr + j));
        }
    }
#pragma unroll
    for (int j = 0; j < KC; ++j) acc[j] = subwarp_sum<SW>(acc[j]);
    if (valid) {
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            if (j < kc && j % SW == lane) {
                TO* dst = c + row * ldc + col0 + j;
                *dst = finish<TA>(acc[j], alpha, beta, dst);
            }
        }
    }
}

template <typename TM, typename TI, typename TO, int KC>
__global__ void __launch_bounds__(kMixBlock)
    ell_mixed_kernel(int64_t n, int width, int64_t stride,
                     const int32_t* __restrict__ ci, const TM* __restrict__ v,
                     const TI* __restrict__ b, int64_t ldb, TO* __restrict__ c,
                     int64_t ldc, int k, int col0, const TM* __restrict__ alpha,
                     const TO* __restrict__ beta)
{
    using TA = arith_t<TM, TI, TO>;
    const int64_t row = blockIdx.x * int64_t(kMixBlock) + threadIdx.x;
    if (row >= n) return;
    const int kc = min(KC, k - col0);
    TA acc[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) acc[j] = TA(0);
    for (int s = 0; s < width; ++s) {
        const int64_t slot = row + int64_t(s) * stride;
        const int col = ld_stream(ci + slot);
        if (col < 0) continue;  // padding (invalid_index)
        const TA val = TA(ld_stream(v + slot));
        const TI* xr = b + int64_t(col) * ldb + col0;
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            if (j < kc) acc[j] += val * TA(__ldg(xr + j));
        }
    }
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        if (j < kc) {
            TO* dst = c + row * ldc + col0 + j;
            *dst = finish<TA>(acc[j], alpha, beta, dst);
        }
    }
}

template <typename TS, typename TD>
__global__ void dense_convert_kernel(int64_t n, int64_t k, const TS* __restrict__ src,
                                     int64_t lds, TD* __restrict__ dst, int64_t ldd)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i >= n * k) return;
    const int64_t r = i / k, j = i - r * k;
    dst[r * ldd + j] = TD(src[r * lds + j]);
}

// One column: the pipelined Csr kernel of csr_async.cuh with the matrix,
// input and output types apart (a warp stages the next group's values and
// column indices with cp.async while it sums the current group, LPR lanes
// per row; groups beyond the stage are summed by the whole warp from
// global memory).  Values and gathered inputs are widened to the
// arithmetic type, the sum rounded once to the output type.
template <typename TM, typename TI, typename TO, int LPR>
__global__ void __launch_bounds__(kAsyncBlock)
    csr_async_mixed_kernel(int64_t n, const int32_t* __restrict__ rp,
                           const int32_t* __restrict__ ci, const TM* __restrict__ v,
                           const TI* __restrict__ b, int64_t ldb, TO* __restrict__ c,
                           int64_t ldc, const TM* __restrict__ alpha,
                           const TO* __restrict__ beta)
{
    using TA = arith_t<TM, TI, TO>;
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int R = kWarp / LPR;  // rows per group
    constexpr int kCap = kAsyncCap;
    __shared__ AsyncStage<TM> stages[kAsyncBlock / kWarp][2];
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const int myrow = lane / LPR, sub = lane % LPR;
    const int64_t ngroups = (n + R - 1) / R;
    const int64_t nwarps = int64_t(gridDim.x) * (kAsyncBlock / kWarp);
    AsyncStage<TM>* st = stages[wid];
    auto load_ptrs = [&](int64_t g, int& p, int& pe) {
        const int64_t row0 = g * R;
        const int64_t pl = row0 + lane;
        p = __ldg(rp + (pl < n ? pl : n));
        pe = __ldg(rp + (row0 + R < n ? row0 + R : n));
    };
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
    int64_t g = blockIdx.x * int64_t(kAsyncBlock / kWarp) + wid;
    if (g >= ngroups) return;  // whole warp
    int rs, re, start, cnt, p, pe;
    load_ptrs(g, p, pe);
    desc(p, pe, rs, re, start, cnt);
    if (cnt <= kCap) issue(0, start, cnt);
    cp_async_commit();
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
        TA acc = TA(0);
        const int64_t row = g * R + myrow;
        if (cnt <= kCap) {
            const TM* cv = st[s].vals;
            const int32_t* cc = st[s].cols;
#pragma unroll 4
            for (int i = rs - start + sub; i < re - start; i += LPR) {
                acc += TA(cv[i]) * TA(__ldg(b + int64_t(cc[i]) * ldb));
            }
            if constexpr (LPR > 1) acc = subwarp_sum<LPR>(acc);
        } else {
            for (int l = 0; l < R; ++l) {
                const int s0 = __shfl_sync(kFull, rs, l * LPR);
                const int e0 = __shfl_sync(kFull, re, l * LPR);
                TA a = TA(0);
                for (int ee = s0 + lane; ee < e0; ee += kWarp) {
                    a += TA(ld_stream(v + ee)) * TA(__ldg(b + int64_t(ld_stream(ci + ee)) * ldb));
                }
                a = warp_sum(a);
                if (myrow == l) acc = a;
            }
        }
        if (row < n && sub == 0) {
            c[row * ldc] = finish<TA, TO, TM>(acc, alpha, beta, c + row * ldc);
        }
        __syncwarp();  // stage s is refilled two groups later
        s ^= 1;
        rs = nrs;
        re = nre;
        start = nstart;
        cnt = ncnt;
    }
}

// subwarp width for rows of up to max_row_nnz entries
inline int mixed_subwarp(int64_t max_row_nnz)
{
    return max_row_nnz <= 4 ? 2 : max_row_nnz <= 32 ? 8 : 32;
}

template <typename TM, typename TI, typename TO>
int csr_mixed(int64_t n, const int32_t* rp, const int32_t* ci, const void* v,
              int64_t max_row_nnz, const void* b, int64_t ldb, void* c, int64_t ldc,
              int64_t k, const void* alpha, const void* beta, cudaStream_t st)
{
    if (k == 1) {
        // one column: the pipelined kernel (persistent, one wave)
        const int lpr = async_lanes_per_row(max_row_nnz);
        auto launch = [&](auto kernel) {
            const int64_t need = ceildiv(ceildiv(n, kWarp / lpr), kAsyncBlock / kWarp);
            const int64_t grid = std::min<int64_t>(need, async_resident_blocks(kernel));
            kernel<<<grid, kAsyncBlock, 0, st>>>(
                n, rp, ci, static_cast<const TM*>(v), static_cast<const TI*>(b), ldb,
                static_cast<TO*>(c), ldc, static_cast<const TM*>(alpha),
                static_cast<const TO*>(beta));
        };
        switch (lpr) {
        case 1: launch(csr_async_mixed_kernel<TM, TI, TO, 1>); break;
        case 2: launch(csr_async_mixed_kernel<TM, TI, TO, 2>); break;
        default: launch(csr_async_mixed_kernel<TM, TI, TO, 4>); break;
        }
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    }
    const int sw = mixed_subwarp(max_row_nnz);
    for (int64_t c0 = 0; c0 < k; c0 += 16) {
        const int kc = int(std::min<int64_t>(16, k - c0));
        const int64_t grid = ceildiv(n * sw, kMixBlock);
        auto launch = [&](auto kernel) {
            kernel<<<grid, kMixBlock, 0, st>>>(
                n, rp, ci, static_cast<const TM*>(v), static_cast<const TI*>(b), ldb,
                static_cast<TO*>(c), ldc, int(k), int(c0), static_cast<const TM*>(alpha),
                static_cast<const TO*>(beta));
        };
#define B2S_MIX_SW(SWV)                                                           \
    if (sw == SWV) {                                                              \
        if (kc == 1) launch(csr_mixed_kernel<TM, TI, TO, SWV, 1>);                \
        else if (kc <= 4) launch(csr_mixed_kernel<TM, TI, TO, SWV, 4>);           \
        else launch(csr_mixed_kernel<TM, TI, TO, SWV, 16>);                       \
    }
        B2S_MIX_SW(2)
        B2S_MIX_SW(8)
        B2S_MIX_SW(32)
#undef B2S_MIX_SW
        B2S_LAUNCH_CHECK();
    }
    return B2S_OK;
}

template <typename TM, typename TI, typename TO>
int ell_mixed(int64_t n, int64_t width, int64_t stride, const int32_t* ci, const void* v,
              const void* b, int64_t ldb, void* c, int64_t ldc, int64_t k,
              const void* alpha, const void* beta, cudaStream_t st)
{
    for (int64_t c0 = 0; c0 < k; c0 += 16) {
        const int kc = int(std::min<int64_t>(16, k - c0));
        const int64_t grid = ceildiv(n, kMixBlock);
        auto launch = [&](auto kernel) {
            kernel<<<grid, kMixBlock, 0, st>>>(
                n, int(width), stride, ci, static_cast<const TM*>(v),
                static_cast<const TI*>(b), ldb, static_cast<TO*>(c), ldc, int(k), int(c0),
                static_cast<const TM*>(alpha), static_cast<const TO*>(beta));
        };
        if (kc == 1) launch(ell_mixed_kernel<TM, TI, TO, 1>);
        else if (kc <= 4) launch(ell_mixed_kernel<TM, TI, TO, 4>);
        else launch(ell_mixed_kernel<TM, TI, TO, 16>);
        B2S_LAUNCH_CHECK();
    }
    return B2S_OK;
}

// Calls fn(TM{}, TI{}, TO{}) for the three type codes (value tags).
template <typename F>
int dispatch_types(int tm, int ti, int to, F&& fn)
{
    auto pick_o = [&](auto m, auto i) -> int {
        if (to == B2S_VALUE_F64) return fn(m, i, double{});
        return fn(m, i, float{});
    };
    auto pick_i = [&](auto m) -> int {
        if (ti == B2S_VALUE_F64) return pick_o(m, double{});
        return pick_o(m, float{});
    };
    if (tm == B2S_VALUE_F64) return pick_i(double{});
    return pick_i(float{});
}

inline bool valid_type(int t) { return t == B2S_VALUE_F64 || t == B2S_VALUE_F32; }

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_csr_spmv_mixed(int matrix_type, int input_type, int output_type,
                       int64_t num_rows, int64_t num_cols, const int32_t* row_ptrs,
                       const int32_t* col_idxs, const void* values,
                       int64_t max_row_nnz, const void* b, int64_t ldb, void* c,
                       int64_t ldc, int64_t num_rhs, const void* alpha,
                       const void* beta, void* stream)
{
    B2S_CHECK_ARG(valid_type(matrix_type) && valid_type(input_type) &&
                      valid_type(output_type),
                  "value types must be B2S_VALUE_F64 or B2S_VALUE_F32");
    B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0 && num_rhs >= 0, "negative size");
    B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),
                  "alpha and beta must both be given or both be null");
    B2S_CHECK_ARG(num_rhs <= 1 || (ldb >= num_rhs && ldc >= num_rhs),
                  "leading dimension < num_rhs");
    B2S_CHECK_ARG(max_row_nnz >= 0, "negative max_row_nnz");
    if (num_rows == 0 || num_rhs == 0) return B2S_OK;
    B2S_CHECK_ARG(row_ptrs && b && c, "null pointer");
    cudaStream_t st = as_stream(stream);
    return dispatch_types(matrix_type, input_type, output_type, [&](auto m, auto i, auto o) {
        return csr_mixed<decltype(m), decltype(i), decltype(o)>(num_rows, row_ptrs, col_idxs, values, max_row_nnz, b,
                                     ldb, c, ldc, num_rhs, alpha, beta, st);
    });
}

int b2s_ell_spmv_mixed(int matrix_type, int input_type, int output_type,
                       int64_t num_rows, int64_t num_cols, int64_t width, int64_t stride,
                       const int32_t* col_idxs, const void* values, const void* b,
                       int64_t ldb, void* c, int64_t ldc, int64_t num_rhs,
                       const void* alpha, const void* beta, void* stream)
{
    B2S_CHECK_ARG(valid_type(matrix_type) && valid_type(input_type) &&
                      valid_type(output_type),
                  "value types must be B2S_VALUE_F64 or B2S_VALUE_F32");
    B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0 && num_rhs >= 0 && width >= 0,
                  "negative size");
    B2S_CHECK_ARG(stride >= num_rows, "Ell stride < num_rows");
    B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),
                  "alpha and beta must both be given or both be null");
    B2S_CHECK_ARG(num_rhs <= 1 || (ldb >= num_rhs && ldc >= num_rhs),
                  "leading dimension < num_rhs");
    if (num_rows == 0 || num_rhs == 0) return B2S_OK;
    B2S_CHECK_ARG(b && c && (width == 0 || (col_idxs && values)), "null pointer");
    cudaStream_t st = as_stream(stream);
    return dispatch_types(matrix_type, input_type, output_type, [&](auto m, auto i, auto o) {
        return ell_mixed<decltype(m), decltype(i), decltype(o)>(num_rows, width, stride, col_idxs, values, b, ldb, c,
                                     ldc, num_rhs, alpha, beta, st);
    });
}

int b2s_dense_convert(int src_type, int dst_type, int64_t num_rows, int64_t num_cols,
                      const void* src, int64_t lds, void* dst, int64_t ldd, void* stream)
{
    B2S_CHECK_ARG(valid_type(src_type) && valid_type(dst_type),
                  "value types must be B2S_VALUE_F64 or B2S_VALUE_F32");
    B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0, "negative size");
    B2S_CHECK_ARG(num_cols <= 1 || (lds >= num_cols && ldd >= num_cols),
                  "leading dimension < num_cols");
    const int64_t total = num_rows * num_cols;
    if (total == 0) return B2S_OK;
    B2S_CHECK_ARG(src && dst, "null pointer");
    cudaStream_t st = as_stream(stream);
    const int64_t grid = ceildiv(total, kMixBlock);
    auto run = [&](auto s, auto d) {
        using TS = decltype(s);
        using TD = decltype(d);
        dense_convert_kernel<TS, TD><<<grid, kMixBlock, 0, st>>>(
            num_rows, num_cols, static_cast<const TS*>(src), lds, static_cast<TD*>(dst),
            ldd);
    };
    if (src_type == B2S_VALUE_F64) {
        if (dst_type == B2S_VALUE_F64) run(double{}, double{});
        else run(double{}, float{});
    } else {
        if (dst_type == B2S_VALUE_F64) run(float{}, double{});
        else run(float{}, float{});
    }
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

}  // extern "C"
