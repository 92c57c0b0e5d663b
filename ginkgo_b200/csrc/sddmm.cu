// Sampled dense-dense product on a Csr pattern: out[e] = alpha * sum_k
// u(row_e, k) * w(col_e, k) for every stored entry e.  With u = lambda (the
// adjoint solution) and w = x (the forward solution), alpha = -1 this is the
// gradient dL/dA = -lambda x^T restricted to A's pattern, the backward of the
// differentiable solve.  u, w row-major n x k / m x k with leading
// dimensions.  Narrow blocks (k * sizeof(T) < 32 bytes): one subwarp per
// row, the row's u(row, :) in registers.  Wider blocks: one warp per 32
// consecutive rows, walking their stored entries as one flat range in chunks
// of 32 (each lane loads one column index and finds its entry's row by a
// shuffle search over the rows' starts), L = k * sizeof(T) / 16 lanes per
// entry, each owning one 16-byte slice of the columns, so w(col, :) and
// u(row, :) of an entry are coalesced loads of k * sizeof(T) bytes; the loads
// of two (FP64) or four (FP32) steps of 32 / L entries are issued before any
// of their sums,
// the slices' partial dots are summed across the L lanes, and the chunk's 32
// results are stored as one coalesced write.
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
__global__ void __launch_bounds__(kBlock, sizeof(T) == 8 ? 5 : 1)
    sddmm_lanes_kernel(int64_t n, const int32_t* __restrict__ rp,
                       const int32_t* __restrict__ ci, const T* __restrict__ u,
                       int64_t ldu, const T* __restrict__ w, int64_t ldw, T alpha,
                       T* __restrict__ out)
{
    constexpr int VW = int(16 / sizeof(T));  // values per lane slice
    constexpr int L = K / VW;                // lanes per entry
    constexpr int EPW = kWarp / L;           // entries per warp step
    // steps whose loads are issued together: two in FP64, held to 48
    // registers for five blocks per SM (16 FP64 columns on the 7-point 128^3
    // pattern: 350 us, against 408 us for four steps at three blocks per
    // SM); four in FP32 (172 us, against 179 us for two)
    constexpr int UMAX = sizeof(T) == 8 ? 2 : 4;
    constexpr int U = L < UMAX ? L : UMAX;
    static_assert(L % U == 0, "a 32-entry chunk is L steps");
    constexpr unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x % kWarp;
    const int slot = lane / L, part = lane % L;
    const int64_t nwarps = int64_t(gridDim.x) * (kBlock / kWarp);
    const int64_t nblk = (n + kWarp - 1) / kWarp;
    for (int64_t rb = (blockIdx.x * int64_t(kBlock) + threadIdx.x) / kWarp; rb < nblk;
         rb += nwarps) {
        // the warp owns rows [r0, r0 + nr); lane j holds the start of row r0 + j
        const int64_t r0 = rb * kWarp;
        const int nr = int(n - r0 < kWarp ? n - r0 : kWarp);
        const int rs = rp[r0 + (lane < nr ? lane : nr)];
        const int e_end = rp[r0 + nr];
        const int e_beg = __shfl_sync(kFull, rs, 0);
        for (int c0 = e_beg; c0 < e_end; c0 += kWarp) {
            // lane l loads entry c0 + l's column and finds its row: the last
            // j < nr with rs_j <= c0 + l (rs is non-decreasing, rs_0 = e_beg)
            const int e = c0 + lane;
            const int cnt = e_end - c0 < kWarp ? e_end - c0 : kWarp;
            const int col = lane < cnt ? ci[e] : 0;
            int ro = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int v = __shfl_sync(kFull, rs, ro + step);
                if (ro + step < nr && v <= e) ro += step;
            }
            // steps of EPW entries, U of them with all their loads in flight;
            // entry c0 + l's dot ends in lane l, stored once per chunk
            const int nst = (cnt + EPW - 1) / EPW;
            T mine = T(0);
            for (int s0 = 0; s0 < nst; s0 += U) {
                T wr[U][VW], ur[U][VW];
#pragma unroll
                for (int q = 0; q < U; ++q) {
                    const int idx = (s0 + q) * EPW + slot;
                    const int c = __shfl_sync(kFull, col, idx);
                    const int r = __shfl_sync(kFull, ro, idx);
                    if (idx < cnt) {
                        RowLoad<T, VW, true>::load(w + int64_t(c) * ldw + part * VW, wr[q]);
                        RowLoad<T, VW, true>::load(u + (r0 + r) * ldu + part * VW, ur[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < U; ++q) {
                    const int idx = (s0 + q) * EPW + slot;
                    T acc = T(0);
                    if (idx < cnt) {
#pragma unroll
                        for (int p = 0; p < VW; ++p) acc += ur[q][p] * wr[q][p];
                    }
                    acc = subwarp_sum<L>(acc);
                    const T got = __shfl_sync(kFull, acc, (lane % EPW) * L);
                    if (lane / EPW == s0 + q) mine = got;
                }
            }
            if (lane < cnt) out[e] = alpha * mine;
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
        // one warp per 32 rows, one wave of resident blocks
        const int64_t want = ceildiv(ceildiv(n, int64_t(kWarp)), int64_t(kBlock / kWarp));
        if (k == 16) {
            const int grid = resident_grid(sddmm_lanes_kernel<T, 16>, kBlock, want);
            sddmm_lanes_kernel<T, 16><<<grid, kBlock, 0, st>>>(n, rp, ci, u, ldu, w, ldw,
                                                               T(alpha), out);
        } else {
            const int grid = resident_grid(sddmm_lanes_kernel<T, 2 * VW>, kBlock, want);
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
