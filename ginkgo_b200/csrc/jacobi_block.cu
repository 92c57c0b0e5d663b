// Block Jacobi: inversion of the diagonal blocks (at most 32 rows) and their
// application, one warp per block.  Lane r owns row r of its block in shared
// memory; Gauss-Jordan with partial pivoting follows the reference's
// invert_block (reference/preconditioner/jacobi_kernels.cpp:128-240) step
// for step, with the pivot search as a warp arg-max.
#include "common.cuh"

namespace b2s {
namespace {

constexpr int kJacobiWarps = 4;  // warps (blocks of the matrix) per CTA
constexpr int kMaxBs = 32;

// Valid extent of block `blk`: 0 <= s <= e <= n and e - s <= max_bs.
__device__ __forceinline__ bool block_extent(const int32_t* ptrs, int64_t blk, int64_t n,
                                             int max_bs, int& s, int& bs)
{
    const int64_t s64 = ptrs[blk], e64 = ptrs[blk + 1];
    if (s64 < 0 || e64 > n || e64 < s64 || e64 - s64 > max_bs) return false;
    s = int(s64);
    bs = int(e64 - s64);
    return true;
}

template <typename T>
__device__ __forceinline__ T magnitude(T v)
{
    return v < T(0) ? -v : v;
}

template <typename T>
__global__ void __launch_bounds__(kJacobiWarps * kWarp)
    jacobi_block_generate_kernel(int64_t n, const int32_t* __restrict__ rp,
                                 const int32_t* __restrict__ ci, const T* __restrict__ v,
                                 int64_t num_blocks, const int32_t* __restrict__ ptrs,
                                 int max_bs, T* __restrict__ blocks)
{
    __shared__ T tile[kJacobiWarps][kMaxBs][kMaxBs + 1];
    __shared__ int perm_sh[kJacobiWarps][kMaxBs];
    const int lane = threadIdx.x % kWarp, w = threadIdx.x / kWarp;
    const int64_t blk = int64_t(blockIdx.x) * kJacobiWarps + w;
    if (blk >= num_blocks) return;
    int s, bs;
    if (!block_extent(ptrs, blk, n, max_bs, s, bs)) return;
    T(*A)[kMaxBs + 1] = tile[w];
    int* perm = perm_sh[w];
    // extract_block: row `lane` of the block, zeros outside the pattern
    for (int j = 0; j < kMaxBs; ++j) A[lane][j] = T(0);
    perm[lane] = lane;
    if (lane < bs) {
        const int row = s + lane;
        for (int k = rp[row]; k < rp[row + 1]; ++k) {
            const int c = ci[k] - s;
            if (0 <= c && c < bs) A[lane][c] = v[k];
        }
    }
    __syncwarp();
    for (int k = 0; k < bs; ++k) {
        // choose_pivot: the first row (from k) of largest |A(i, k)|
        T best = lane >= k && lane < bs ? magnitude(A[lane][k]) : T(-1);
        int idx = lane >= k && lane < bs ? lane : kMaxBs;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const T ob = __shfl_xor_sync(0xffffffffu, best, off);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, off);
            if (ob > best || (ob == best && oi < idx)) {
                best = ob;
                idx = oi;
            }
        }
        // every lane takes lane 0's result (the combine is not associative
        // for NaN magnitudes, so lanes could otherwise disagree)
        idx = __shfl_sync(0xffffffffu, idx, 0);
        const int cp = idx >= k && idx < bs ? idx : k;
        // swap_rows(k, cp): lane j swaps column j
        if (cp != k && lane < bs) {
            const T t = A[k][lane];
            A[k][lane] = A[cp][lane];
            A[cp][lane] = t;
        }
        if (lane == 0 && cp != k) {
            const int t = perm[k];
            perm[k] = perm[cp];
            perm[cp] = t;
        }
        __syncwarp();
        const T d = A[k][k];
        if (d == T(0)) break;  // singular: the block stays as far as it got
        // apply_gauss_jordan_transform(k, k): column k scaled by -1/d ...
        if (lane < bs) A[lane][k] = A[lane][k] / -d;
        __syncwarp();
        if (lane == 0) A[k][k] = T(0);
        __syncwarp();
        // ... the rank-one update of every row but k (row k gains 0 there) ...
        if (lane < bs && lane != k) {
            const T aik = A[lane][k];
            for (int j = 0; j < bs; ++j) A[lane][j] += aik * A[k][j];
        }
        __syncwarp();
        // ... and row k divided by d, its diagonal 1/d
        if (lane < bs) A[k][lane] = A[k][lane] / d;
        __syncwarp();
        if (lane == 0) A[k][k] = T(1) / d;
        __syncwarp();
    }
    // permute_and_transpose_block: inverse(i, perm[j]) = A(i, j), stored
    // column-major with stride max_bs
    T* out = blocks + blk * int64_t(max_bs) * max_bs;
    if (lane < bs) {
        for (int j = 0; j < bs; ++j) out[lane + int64_t(perm[j]) * max_bs] = A[lane][j];
    }
}

// Apply: floor(32 / max_bs) blocks per warp, lane = (block in warp, row),
// so small blocks keep the whole warp busy.  Every lane runs the same
// max_bs broadcast steps (full-mask shuffles); lanes outside a valid row
// only pass values along.
template <typename T>
__global__ void __launch_bounds__(kJacobiWarps * kWarp)
    jacobi_block_apply_kernel(int64_t n, int64_t num_blocks, const int32_t* __restrict__ ptrs,
                              int max_bs, const T* __restrict__ blocks,
                              const T* __restrict__ b, int64_t ldb, T* __restrict__ x,
                              int64_t ldx, int64_t k, const T* __restrict__ alpha,
                              const T* __restrict__ beta)
{
    const int lane = threadIdx.x % kWarp, w = threadIdx.x / kWarp;
    const int per_warp = kWarp / max_bs;
    const int sub = lane / max_bs, r = lane % max_bs;
    const int64_t warp = int64_t(blockIdx.x) * kJacobiWarps + w;
    const int64_t blk = warp * per_warp + sub;
    if (warp * per_warp >= num_blocks) return;  // the whole warp: uniform
    int s = 0, bs = 0;
    const bool in_block = sub < per_warp && blk < num_blocks &&
                          block_extent(ptrs, blk, n, max_bs, s, bs);
    const bool active = in_block && r < bs;
    const T* inv = blocks + (in_block ? blk : 0) * int64_t(max_bs) * max_bs;
    const T a = alpha ? *alpha : T(1);
    const T be = beta ? *beta : T(0);
    const int base = sub * max_bs;  // first lane of this lane's block
    for (int64_t col = 0; col < k; ++col) {
        const T bv = active ? b[(s + r) * ldb + col] : T(0);
        T acc = T(0);
        if (active && be != T(0)) acc = x[(s + r) * ldx + col] * be;
        // apply_block: x(row) += alpha * inv(row, inner) * b(inner), inner in order
        for (int inner = 0; inner < max_bs; ++inner) {
            const T bi = __shfl_sync(0xffffffffu, bv, (base + inner) % kWarp);
            if (active && inner < bs) acc += a * inv[r + int64_t(inner) * max_bs] * bi;
        }
        if (active) x[(s + r) * ldx + col] = acc;
    }
}

template <typename T>
int block_generate(int64_t n, const int32_t* rp, const int32_t* ci, const T* v,
                   int64_t num_blocks, const int32_t* ptrs, int max_bs, T* blocks,
                   void* stream)
{
    B2S_CHECK_ARG(n >= 0 && num_blocks >= 0, "negative size");
    B2S_CHECK_ARG(max_bs >= 1 && max_bs <= kMaxBs, "max_block_size must be 1..32");
    if (num_blocks == 0) return B2S_OK;
    jacobi_block_generate_kernel<T><<<ceildiv(num_blocks, kJacobiWarps),
                                      kJacobiWarps * kWarp, 0, as_stream(stream)>>>(
        n, rp, ci, v, num_blocks, ptrs, max_bs, blocks);
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

template <typename T>
int block_apply(int64_t n, int64_t num_blocks, const int32_t* ptrs, int max_bs,
                const T* blocks, const T* b, int64_t ldb, T* x, int64_t ldx, int64_t k,
                const T* alpha, const T* beta, void* stream)
{
    B2S_CHECK_ARG(n >= 0 && num_blocks >= 0 && k >= 0, "negative size");
    B2S_CHECK_ARG(max_bs >= 1 && max_bs <= kMaxBs, "max_block_size must be 1..32");
    B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),
                  "alpha and beta must both be given or both be null");
    B2S_CHECK_ARG(k == 0 || (ldb >= k && ldx >= k), "leading dimension < num_rhs");
    if (num_blocks == 0 || k == 0) return B2S_OK;
    const int64_t warps = ceildiv(num_blocks, kWarp / max_bs);
    jacobi_block_apply_kernel<T><<<ceildiv(warps, kJacobiWarps), kJacobiWarps * kWarp,
                                   0, as_stream(stream)>>>(n, num_blocks, ptrs, max_bs,
                                                           blocks, b, ldb, x, ldx, k,
                                                           alpha, beta);
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_jacobi_block_generate_f64(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const double* values,
                                  int64_t num_blocks, const int32_t* block_ptrs,
                                  int max_block_size, double* blocks, void* stream)
{
    return block_generate(num_rows, row_ptrs, col_idxs, values, num_blocks, block_ptrs,
                          max_block_size, blocks, stream);
}

int b2s_jacobi_block_generate_f32(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const float* values,
                                  int64_t num_blocks, const int32_t* block_ptrs,
                                  int max_block_size, float* blocks, void* stream)
{
    return block_generate(num_rows, row_ptrs, col_idxs, values, num_blocks, block_ptrs,
                          max_block_size, blocks, stream);
}

int b2s_jacobi_block_apply_f64(int64_t num_rows, int64_t num_blocks,
                               const int32_t* block_ptrs, int max_block_size,
                               const double* blocks, const double* b, int64_t ldb,
                               double* x, int64_t ldx, int64_t num_rhs,
                               const double* alpha, const double* beta, void* stream)
{
    return block_apply(num_rows, num_blocks, block_ptrs, max_block_size, blocks, b, ldb,
                       x, ldx, num_rhs, alpha, beta, stream);
}

int b2s_jacobi_block_apply_f32(int64_t num_rows, int64_t num_blocks,
                               const int32_t* block_ptrs, int max_block_size,
                               const float* blocks, const float* b, int64_t ldb,
                               float* x, int64_t ldx, int64_t num_rhs,
                               const float* alpha, const float* beta, void* stream)
{
    return block_apply(num_rows, num_blocks, block_ptrs, max_block_size, blocks, b, ldb,
                       x, ldx, num_rhs, alpha, beta, stream);
}

}  // extern "C"
