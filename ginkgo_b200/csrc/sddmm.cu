// Sampled dense-dense product on a Csr pattern: out[e] = alpha * sum_k
// u(row_e, k) * w(col_e, k) for every stored entry e.  With u = lambda (the
// adjoint solution) and w = x (the forward solution), alpha = -1 this is the
// gradient dL/dA = -lambda x^T restricted to A's pattern, the backward of the
// differentiable solve.  u, w row-major n x k / m x k with leading
// dimensions.  Narrow blocks (k * sizeof(T) < 32 bytes): one subwarp per
// row, the row's u(row, :) in registers.  Wider blocks: one warp per row and
// L = k * sizeof(T) / 16 lanes per stored entry, each lane owning one
// 16-byte slice of the columns, so w(col, :) of an entry is one coalesced
// load of k * sizeof(T) bytes and the warp serves 32 / L entries at a time;
// the slices' partial dots are summed across the L lanes.
#include <algorithm>

#include "common.cuh"

namespace b2s {
namespace {

constexpr int kBlock = 256;

template <typename T, int SW, int K>
__global__ void __launch_bounds__(kBlock)
    sddmm_kernel(int64_t n, const int32_t* __restrict__ rp,
                 const int32_t* __restrict__ ci, const T* __restrict__ u,
                 int64_t ldu, const T* __restrict__ w, int64_t ldw, int k,
                 T alpha, T* __restrict__ out)
{
    const int64_t row = (blockIdx.x * int64_t(kBlock) + threadIdx.x) / SW;
    const int lane = threadIdx.x % SW;
    if (row >= n) return;
    T ur[K];
#pragma unroll
    for (int j = 0; j < K; ++j) ur[j] = j < k ? u[row * ldu + j] : T(0);
    const int end = rp[row + 1];
    for (int e = rp[row] + lane; e < end; e += SW) {
        const T* wr = w + int64_t(ci[e]) * ldw;
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j < k) acc += ur[j] * wr[j];
        }
        out[e] = alpha * acc;
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    sddmm_lanes_kernel(int64_t n, const int32_t* __restrict__ rp,
                       const int32_t* __restrict__ ci, const T* __restrict__ u,
                       int64_t ldu, const T* __restrict__ w, int64_t ldw, T alpha,
                       T* __restrict__ out)
{
    constexpr int VW = int(16 / sizeof(T));  // values per lane slice
    constexpr int L = K / VW;                // lanes per entry
    constexpr int EPW = kWarp / L;           // entries per warp step
    const int lane = threadIdx.x % kWarp;
    const int slot = lane / L, part = lane % L;
    const int64_t nwarps = int64_t(gridDim.x) * (kBlock / kWarp);
    for (int64_t row = (blockIdx.x * int64_t(kBlock) + threadIdx.x) / kWarp; row < n;
         row += nwarps) {
        T ur[VW];
        RowLoad<T, VW, true>::load(u + row * ldu + part * VW, ur);
        const int b = rp[row], e_end = rp[row + 1];
        // warp-uniform trip count: every lane reaches the shuffles
        for (int e0 = b; e0 < e_end; e0 += EPW) {
            const int e = e0 + slot;
            T acc = T(0);
            if (e < e_end) {
                T wr[VW];
                RowLoad<T, VW, true>::load(w + int64_t(ci[e]) * ldw + part * VW, wr);
#pragma unroll
                for (int q = 0; q < VW; ++q) acc += ur[q] * wr[q];
            }
            acc = subwarp_sum<L>(acc);
            if (part == 0 && e < e_end) out[e] = alpha * acc;
        }
    }
}

template <typename T>
int sddmm(int64_t n, const int32_t* rp, const int32_t* ci, int64_t max_row_nnz,
          const T* u, int64_t ldu, const T* w, int64_t ldw, int64_t k,
          double alpha, T* out, void* stream)
{
    B2S_CHECK_ARG(n >= 0 && k >= 1 && k <= 16, "num_rhs must be 1..16");
    B2S_CHECK_ARG(ldu >= k && ldw >= k, "leading dimension < num_rhs");
    if (n == 0) return B2S_OK;
    cudaStream_t st = as_stream(stream);
    // 16-byte slices when the block rows are whole multiples of 16 bytes and
    // aligned (k = 4 or 16 in FP64, 8 or 16 in FP32)
    constexpr int VW = int(16 / sizeof(T));
    const bool aligned = reinterpret_cast<uintptr_t>(u) % 16 == 0 &&
                         reinterpret_cast<uintptr_t>(w) % 16 == 0 && ldu % VW == 0 &&
                         ldw % VW == 0;
    if (aligned && (k == 16 || (k == 8 && sizeof(T) == 4) || (k == 4 && sizeof(T) == 8))) {
        const int64_t grid = std::min<int64_t>(ceildiv(n, kBlock / kWarp),
                                               int64_t(num_sms()) * 16);
        if (k == 16) {
            sddmm_lanes_kernel<T, 16><<<grid, kBlock, 0, st>>>(n, rp, ci, u, ldu, w, ldw,
                                                               T(alpha), out);
        } else {
            sddmm_lanes_kernel<T, 2 * VW><<<grid, kBlock, 0, st>>>(n, rp, ci, u, ldu, w,
                                                                   ldw, T(alpha), out);
        }
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    }
    int sw = 1;
    while (sw * 2 <= max_row_nnz && sw < 32) sw *= 2;
    const int64_t grid = ceildiv(n * sw, kBlock);
    const int kk = k <= 1 ? 1 : (k <= 4 ? 4 : 16);
#define B2S_SDDMM(SW_, K_)                                                    \
    sddmm_kernel<T, SW_, K_><<<grid, kBlock, 0, st>>>(n, rp, ci, u, ldu, w,   \
                                                      ldw, int(k), T(alpha),  \
                                                      out)
#define B2S_SDDMM_K(SW_)                      \
    if (kk == 1) B2S_SDDMM(SW_, 1);           \
    else if (kk == 4) B2S_SDDMM(SW_, 4);      \
    else B2S_SDDMM(SW_, 16);
    switch (sw) {
    case 32: B2S_SDDMM_K(32) break;
    case 16: B2S_SDDMM_K(16) break;
    case 8: B2S_SDDMM_K(8) break;
    case 4: B2S_SDDMM_K(4) break;
    case 2: B2S_SDDMM_K(2) break;
    default: B2S_SDDMM_K(1) break;
    }
#undef B2S_SDDMM_K
#undef B2S_SDDMM
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

extern "C" {

int b2s_csr_sddmm_f64(int64_t num_rows, const int32_t* row_ptrs,
                      const int32_t* col_idxs, int64_t max_row_nnz,
                      const double* u, int64_t ldu, const double* w,
                      int64_t ldw, int64_t num_rhs, double alpha, double* out,
                      void* stream)
{
    return b2s::sddmm<double>(num_rows, row_ptrs, col_idxs, max_row_nnz, u,
                              ldu, w, ldw, num_rhs, alpha, out, stream);
}

int b2s_csr_sddmm_f32(int64_t num_rows, const int32_t* row_ptrs,
                      const int32_t* col_idxs, int64_t max_row_nnz,
                      const float* u, int64_t ldu, const float* w,
                      int64_t ldw, int64_t num_rhs, double alpha, float* out,
                      void* stream)
{
    return b2s::sddmm<float>(num_rows, row_ptrs, col_idxs, max_row_nnz, u, ldu,
                             w, ldw, num_rhs, alpha, out, stream);
}

}  // extern "C"
