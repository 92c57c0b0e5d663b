// Format conversions on the GPU: Csr -> Ell, Csr -> Sellp (slice sets and
// scatter), Csr transpose, plus the scalar Jacobi generate/apply.  Every
// output is bit-exact with the reference executor:
//   convert_to_ell     reference/matrix/csr_kernels.cpp:576-601
//   compute_slice_sets reference/matrix/sellp_kernels.cpp:109-131
//   convert_to_sellp   reference/matrix/csr_kernels.cpp:529-570
//   transpose          reference/matrix/csr_kernels.cpp:678-730
//   jacobi             common/unified/preconditioner/jacobi_kernels.cpp:24-101
#include <mutex>

#include "common.cuh"
#include "scan.cuh"

namespace b2s {
namespace {

constexpr int kBlock = 256;

// ---- max row length -------------------------------------------------------
__global__ void __launch_bounds__(kBlock)
    max_row_nnz_kernel(int64_t n, const int32_t* __restrict__ rp,
                       unsigned long long* __restrict__ out)
{
    int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    unsigned long long m = 0;
    for (; i < n; i += int64_t(gridDim.x) * kBlock) {
        m = max(m, (unsigned long long)(rp[i + 1] - rp[i]));
    }
    for (int off = 16; off > 0; off /= 2) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    }
    if (threadIdx.x % kWarp == 0 && m > 0) atomicMax(out, m);
}

// ---- Csr -> Ell -------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kBlock)
    csr_to_ell_kernel(int64_t n, const int32_t* __restrict__ rp,
                      const int32_t* __restrict__ ci, const T* __restrict__ v,
                      int64_t width, int64_t stride, int32_t* __restrict__ eci,
                      T* __restrict__ ev)
{
    const int64_t row = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (row >= n) return;
    const int64_t b = rp[row], len = rp[row + 1] - b;
    for (int64_t i = 0; i < width; ++i) {
        const bool in = i < len;
        eci[row + i * stride] = in ? ci[b + i] : -1;
        ev[row + i * stride] = in ? v[b + i] : T(0);
    }
}

// ---- Csr -> Sellp -------------------------------------------------------------
__global__ void __launch_bounds__(kBlock)
    slice_lengths_kernel(int64_t n, const int32_t* __restrict__ rp,
                         int64_t slice_size, int64_t stride_factor,
                         int64_t num_slices, uint64_t* __restrict__ lens)
{
    const int64_t s = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (s >= num_slices) return;
    uint64_t len = 0;
    for (int64_t l = 0; l < slice_size; ++l) {
        const int64_t row = s * slice_size + l;
        const int64_t rl = row < n ? rp[row + 1] - rp[row] : 0;
        const uint64_t padded =
            uint64_t(ceildiv(rl, stride_factor) * stride_factor);
        len = padded > len ? padded : len;
    }
    lens[s] = len;
}

template <typename T>
__global__ void __launch_bounds__(kBlock)
    csr_to_sellp_kernel(int64_t n, const int32_t* __restrict__ rp,
                        const int32_t* __restrict__ ci, const T* __restrict__ v,
                        int64_t slice_size,
                        const uint64_t* __restrict__ slice_sets,
                        const uint64_t* __restrict__ slice_lengths,
                        int32_t* __restrict__ sci, T* __restrict__ sv)
{
    const int64_t row = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (row >= n) return;
    const int64_t s = row / slice_size, local = row - s * slice_size;
    const int64_t b = rp[row], len = rp[row + 1] - b;
    const int64_t slen = int64_t(slice_lengths[s]);
    int64_t idx = int64_t(slice_sets[s]) * slice_size + local;
    for (int64_t i = 0; i < slen; ++i, idx += slice_size) {
        const bool in = i < len;
        sci[idx] = in ? ci[b + i] : -1;
        sv[idx] = in ? v[b + i] : T(0);
    }
}

// ---- transpose -------------------------------------------------------------
__global__ void __launch_bounds__(kBlock)
    count_cols_kernel(int64_t nnz, const int32_t* __restrict__ ci,
                      int32_t* __restrict__ counts)
{
    for (int64_t e = blockIdx.x * int64_t(kBlock) + threadIdx.x; e < nnz;
         e += int64_t(gridDim.x) * kBlock) {
        atomicAdd(counts + ci[e], 1);
    }
}

// Scatter (in any order) into per-column slots; one thread per source row.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    scatter_transpose_kernel(int64_t nrows, const int32_t* __restrict__ rp,
                             const int32_t* __restrict__ ci,
                             const T* __restrict__ v,
                             int32_t* __restrict__ fill,
                             int32_t* __restrict__ tmp_row,
                             T* __restrict__ tmp_val)
{
    const int64_t row = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (row >= nrows) return;
    for (int64_t e = rp[row]; e < rp[row + 1]; ++e) {
        const int32_t dst = atomicAdd(fill + ci[e], 1);
        tmp_row[dst] = int32_t(row);
        tmp_val[dst] = v[e];
    }
}

// One warp per transposed row: the source rows in one column are distinct,
// so the rank of each entry (number of smaller row indices) is its slot.
// This reproduces the increasing-row order of the sequential scatter.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    rank_transpose_kernel(int64_t ncols, const int32_t* __restrict__ trp,
                          const int32_t* __restrict__ tmp_row,
                          const T* __restrict__ tmp_val,
                          int32_t* __restrict__ tci, T* __restrict__ tv)
{
    const int64_t col = (blockIdx.x * int64_t(kBlock) + threadIdx.x) / kWarp;
    const int lane = threadIdx.x % kWarp;
    if (col >= ncols) return;
    const int32_t b = trp[col], len = trp[col + 1] - b;
    for (int32_t i = lane; i < len; i += kWarp) {
        const int32_t key = tmp_row[b + i];
        int32_t rank = 0;
        for (int32_t j = 0; j < len; ++j) rank += tmp_row[b + j] < key;
        tci[b + rank] = key;
        tv[b + rank] = tmp_val[b + i];
    }
}

// ---- scalar Jacobi ----------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kBlock)
    invert_diagonal_kernel(int64_t n, const int32_t* __restrict__ rp,
                           const int32_t* __restrict__ ci,
                           const T* __restrict__ v, T* __restrict__ inv, int l1)
{
    const int64_t row = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (row >= n) return;
    T d = T(0), off = T(0);
    for (int64_t e = rp[row]; e < rp[row + 1]; ++e) {
        if (ci[e] == row) {
            d = v[e];
        } else if (l1) {
            off += v[e] < T(0) ? -v[e] : v[e];
        }
    }
    // scalar_l1 (reference/preconditioner/jacobi_kernels.cpp:726-745): the
    // absolute sum of the off-diagonal entries, in storage order, added to
    // the diagonal before the inversion
    if (l1) d += off;
    inv[row] = d == T(0) ? T(1) : T(1) / d;
}

// x = diag^-1 b (simple_scalar_apply) or x = alpha diag^-1 b + beta x
// (scalar_apply); common/unified/preconditioner/jacobi_kernels.cpp:39-101.
template <typename T>
__global__ void __launch_bounds__(kBlock)
    jacobi_apply_kernel(int64_t n, int64_t k, const T* __restrict__ inv,
                        const T* __restrict__ b, int64_t ldb,
                        T* __restrict__ x, int64_t ldx,
                        const T* __restrict__ alpha, const T* __restrict__ beta)
{
    const int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (i >= n * k) return;
    const int64_t row = i / k, col = i - row * k;
    const T val = inv[row] * b[row * ldb + col];
    T* dst = x + row * ldx + col;
    *dst = combine(val, alpha, beta, dst);
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_csr_max_row_nnz(int64_t num_rows, const int32_t* row_ptrs,
                        int64_t* result, void* workspace, void* stream)
{
    B2S_CHECK_ARG(result != nullptr && workspace != nullptr, "null pointer");
    cudaStream_t st = as_stream(stream);
    auto* w = static_cast<unsigned long long*>(workspace);
    B2S_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(*w), st));
    if (num_rows > 0) {
        const int64_t grid = std::min<int64_t>(ceildiv(num_rows, kBlock), 4 * num_sms());
        max_row_nnz_kernel<<<grid, kBlock, 0, st>>>(num_rows, row_ptrs, w);
        B2S_LAUNCH_CHECK();
    }
    unsigned long long h = 0;
    B2S_CUDA_TRY(cudaMemcpyAsync(&h, w, sizeof(h), cudaMemcpyDeviceToHost, st));
    B2S_CUDA_TRY(cudaStreamSynchronize(st));
    *result = int64_t(h);
    return B2S_OK;
}

int64_t b2s_sellp_slice_sets_workspace_bytes(int64_t num_rows, int64_t slice_size)
{
    if (slice_size < 1) return -1;
    const int64_t ns = ceildiv(num_rows, slice_size);
    return scan_work_entries<unsigned long long>(ns) * 8;
}

int b2s_sellp_compute_slice_sets(int64_t num_rows, const int32_t* row_ptrs,
                                 int64_t slice_size, int64_t stride_factor,
                                 uint64_t* slice_sets, uint64_t* slice_lengths,
                                 void* workspace, int64_t workspace_bytes,
                                 void* stream)
{
    B2S_CHECK_ARG(num_rows >= 0 && slice_size >= 1 && stride_factor >= 1,
                  "bad Sellp parameters");
    B2S_CHECK_ARG(slice_sets != nullptr, "null slice_sets");
    B2S_CHECK_ARG(num_rows == 0 || (row_ptrs != nullptr && slice_lengths != nullptr),
                  "null row_ptrs or slice_lengths");
    const int64_t need = b2s_sellp_slice_sets_workspace_bytes(num_rows, slice_size);
    if (workspace_bytes < need) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)need);
        return B2S_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    const int64_t ns = ceildiv(num_rows, slice_size);
    if (ns > 0) {
        slice_lengths_kernel<<<ceildiv(ns, kBlock), kBlock, 0, st>>>(
            num_rows, row_ptrs, slice_size, stride_factor, ns, slice_lengths);
        B2S_LAUNCH_CHECK();
    }
    using U = unsigned long long;
    return exclusive_scan<U>(reinterpret_cast<const U*>(slice_lengths), ns,
                             reinterpret_cast<U*>(slice_sets),
                             static_cast<U*>(workspace), st);
}

int64_t b2s_csr_transpose_workspace_bytes(int64_t num_rows, int64_t num_cols,
                                          int64_t nnz, int value_bytes)
{
    // fill counters, scan work, tmp rows, tmp values
    return (num_cols + 1) * 4 + scan_work_entries<int32_t>(num_cols) * 4 +
           nnz * 4 + nnz * int64_t(value_bytes) + 64;
}

#define B2S_CONVERT_ENTRIES(T, S)                                              \
    int b2s_csr_convert_to_ell_##S(int64_t num_rows, const int32_t* row_ptrs,  \
                                   const int32_t* col_idxs, const T* values,   \
                                   int64_t width, int64_t stride,              \
                                   int32_t* ell_col_idxs, T* ell_values,       \
                                   void* stream)                               \
    {                                                                          \
        B2S_CHECK_ARG(stride >= num_rows && width >= 0, "bad Ell shape");      \
        if (num_rows == 0) return B2S_OK;                                      \
        csr_to_ell_kernel<T><<<ceildiv(num_rows, kBlock), kBlock, 0,           \
                               as_stream(stream)>>>(                           \
            num_rows, row_ptrs, col_idxs, values, width, stride,               \
            ell_col_idxs, ell_values);                                         \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    int b2s_csr_convert_to_sellp_##S(                                          \
        int64_t num_rows, const int32_t* row_ptrs, const int32_t* col_idxs,    \
        const T* values, int64_t slice_size, const uint64_t* slice_sets,       \
        const uint64_t* slice_lengths, int32_t* sellp_col_idxs,                \
        T* sellp_values, void* stream)                                         \
    {                                                                          \
        B2S_CHECK_ARG(slice_size >= 1, "slice_size must be >= 1");             \
        if (num_rows == 0) return B2S_OK;                                      \
        csr_to_sellp_kernel<T><<<ceildiv(num_rows, kBlock), kBlock, 0,         \
                                 as_stream(stream)>>>(                         \
            num_rows, row_ptrs, col_idxs, values, slice_size, slice_sets,      \
            slice_lengths, sellp_col_idxs, sellp_values);                      \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    int b2s_csr_transpose_##S(int64_t num_rows, int64_t num_cols, int64_t nnz, \
                              const int32_t* row_ptrs,                         \
                              const int32_t* col_idxs, const T* values,        \
                              int32_t* t_row_ptrs, int32_t* t_col_idxs,        \
                              T* t_values, void* workspace,                    \
                              int64_t workspace_bytes, void* stream)           \
    {                                                                          \
        B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0 && nnz >= 0,              \
                      "negative size");                                        \
        const int64_t need = b2s_csr_transpose_workspace_bytes(                \
            num_rows, num_cols, nnz, sizeof(T));                               \
        if (workspace_bytes < need) {                                          \
            set_error("workspace of %lld bytes < %lld",                        \
                      (long long)workspace_bytes, (long long)need);            \
            return B2S_ERR_WORKSPACE;                                          \
        }                                                                      \
        cudaStream_t st = as_stream(stream);                                   \
        char* w = static_cast<char*>(workspace);                               \
        int32_t* counts = reinterpret_cast<int32_t*>(w);                       \
        w += (num_cols + 1) * 4;                                               \
        int32_t* scan_work = reinterpret_cast<int32_t*>(w);                    \
        w += scan_work_entries<int32_t>(num_cols) * 4;                         \
        T* tmp_val = reinterpret_cast<T*>(                                     \
            (reinterpret_cast<uintptr_t>(w) + 15) & ~uintptr_t(15));           \
        int32_t* tmp_row = reinterpret_cast<int32_t*>(tmp_val + nnz);          \
        B2S_CUDA_TRY(cudaMemsetAsync(counts, 0, (num_cols + 1) * 4, st));      \
        if (nnz > 0) {                                                         \
            const int64_t grid =                                               \
                std::min<int64_t>(ceildiv(nnz, kBlock), 16 * num_sms());        \
            count_cols_kernel<<<grid, kBlock, 0, st>>>(nnz, col_idxs, counts); \
            B2S_LAUNCH_CHECK();                                                \
        }                                                                      \
        int rc = exclusive_scan<int32_t>(counts, num_cols, t_row_ptrs,         \
                                         scan_work, st);                       \
        if (rc != B2S_OK) return rc;                                           \
        if (nnz == 0) return B2S_OK;                                           \
        B2S_CUDA_TRY(cudaMemcpyAsync(counts, t_row_ptrs, num_cols * 4,         \
                                     cudaMemcpyDeviceToDevice, st));           \
        scatter_transpose_kernel<T><<<ceildiv(num_rows, kBlock), kBlock, 0,    \
                                      st>>>(num_rows, row_ptrs, col_idxs,      \
                                            values, counts, tmp_row, tmp_val); \
        B2S_LAUNCH_CHECK();                                                    \
        rank_transpose_kernel<T><<<ceildiv(num_cols * kWarp, kBlock), kBlock,  \
                                   0, st>>>(num_cols, t_row_ptrs, tmp_row,     \
                                            tmp_val, t_col_idxs, t_values);    \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    int b2s_jacobi_invert_diagonal_##S(int64_t num_rows,                       \
                                       const int32_t* row_ptrs,                \
                                       const int32_t* col_idxs,                \
                                       const T* values, T* inv_diag,           \
                                       int aggregate_l1, void* stream)         \
    {                                                                          \
        if (num_rows == 0) return B2S_OK;                                      \
        invert_diagonal_kernel<T><<<ceildiv(num_rows, kBlock), kBlock, 0,      \
                                    as_stream(stream)>>>(                      \
            num_rows, row_ptrs, col_idxs, values, inv_diag, aggregate_l1);     \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    int b2s_jacobi_apply_##S(int64_t num_rows, int64_t num_rhs,                \
                             const T* inv_diag, const T* b, int64_t ldb, T* x, \
                             int64_t ldx, const T* alpha, const T* beta,       \
                             void* stream)                                     \
    {                                                                          \
        B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),                 \
                      "alpha and beta must both be given or both be null");    \
        const int64_t total = num_rows * num_rhs;                              \
        if (total == 0) return B2S_OK;                                         \
        jacobi_apply_kernel<T><<<ceildiv(total, kBlock), kBlock, 0,            \
                                 as_stream(stream)>>>(                         \
            num_rows, num_rhs, inv_diag, b, ldb, x, ldx, alpha, beta);         \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }

B2S_CONVERT_ENTRIES(double, f64)
B2S_CONVERT_ENTRIES(float, f32)

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free Sellp slice sets.
//
// Some callers cannot allocate device memory when they build a Sellp matrix:
// hosts that hand the library one fixed device arena and forbid any further
// allocation, and latency-sensitive loops that must not call cudaMalloc
// (it can synchronise the whole device).  For them the scan scratch of the
// slice-set computation lives in this file-scope device array instead of a
// caller workspace.  Limit: 4096 scratch entries, i.e. at most
// 4095 * 2048 = 8,386,560 slices per call.  Every GPU that loads the library
// holds these 32 KiB until the process exits.  All calls share the array:
// calls that overlap on the GPU (different streams or threads at the same
// time) race on it and give wrong results.
// ---------------------------------------------------------------------------
namespace {
constexpr int64_t kNoAllocScanEntries = 4096;
constexpr int64_t kNoAllocMaxSlices = (kNoAllocScanEntries - 1) * b2s::kScanTile;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned long long
    g_slice_scan_scratch[kNoAllocScanEntries];

namespace {
std::mutex g_noalloc_mutex;
void* g_noalloc_scratch[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the name is only a host-side stand-in for the device symbol).
// The cached address is not refreshed after a device reset; the header says
// so to callers.
int noalloc_scratch(void** out)
{
    int dev = -1;
    B2S_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        b2s::set_error("device %d out of range for the static scratch", dev);
        return B2S_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_scratch[dev] == nullptr) {
        void* p = nullptr;
        B2S_CUDA_TRY(cudaGetSymbolAddress(&p, g_slice_scan_scratch));
        g_noalloc_scratch[dev] = p;
    }
    *out = g_noalloc_scratch[dev];
    return B2S_OK;
}
}  // namespace

extern "C" int b2s_sellp_compute_slice_sets_noalloc(
    int64_t num_rows, const int32_t* row_ptrs, int64_t slice_size,
    int64_t stride_factor, uint64_t* slice_sets, uint64_t* slice_lengths,
    void* stream)
{
    B2S_CHECK_ARG(num_rows >= 0 && slice_size >= 1 && stride_factor >= 1,
                  "bad Sellp parameters");
    const int64_t ns = b2s::ceildiv(num_rows, slice_size);
    if (ns > kNoAllocMaxSlices) {
        b2s::set_error(
            "%lld slices exceed the static scratch of the allocation-free "
            "entry point (at most %lld slices); use "
            "b2s_sellp_compute_slice_sets with a workspace",
            (long long)ns, (long long)kNoAllocMaxSlices);
        return B2S_ERR_INVALID_ARG;
    }
    B2S_CHECK_ARG(slice_sets != nullptr, "null slice_sets");
    B2S_CHECK_ARG(num_rows == 0 || (row_ptrs != nullptr && slice_lengths != nullptr),
                  "null row_ptrs or slice_lengths");
    void* scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc != B2S_OK) return rc;
    cudaStream_t st = b2s::as_stream(stream);
    if (ns > 0) {
        b2s::slice_lengths_kernel<<<b2s::ceildiv(ns, b2s::kBlock), b2s::kBlock,
                                    0, st>>>(num_rows, row_ptrs, slice_size,
                                             stride_factor, ns, slice_lengths);
        B2S_LAUNCH_CHECK();
    }
    // exclusive_scan rewrites every scratch entry it reads and clears the
    // one it accumulates into, so no state leaks between calls
    using U = unsigned long long;
    return b2s::exclusive_scan<U>(reinterpret_cast<const U*>(slice_lengths), ns,
                                  reinterpret_cast<U*>(slice_sets),
                                  static_cast<U*>(scratch), st);
}
