// Block Jacobi: inversion of the diagonal blocks (at most 32 rows) and their
// application.  Generation runs one warp per block: lane r owns row r of its
// block in shared memory; Gauss-Jordan with partial pivoting follows the
// reference's invert_block (reference/preconditioner/jacobi_kernels.cpp:
// 128-240) step for step, with the pivot search as a warp arg-max.
//
// The inverses are stored in the reference's block-interleaved layout
// (block_interleaved_storage_scheme, include/ginkgo/core/preconditioner/
// jacobi.hpp:37-140, with the CUDA executor's block stride of 32,
// jacobi.hpp:589-621): blocks form groups of gs = 32 / pow2ceil(max_bs);
// element (row, col) of block b sits at
//   (b / gs) * group_offset + (b % gs) * max_bs + row + col * stride,
// stride = gs * max_bs, group_offset = max_bs * stride.  Column col of the
// gs blocks of a group is one contiguous run of gs * max_bs values, so the
// apply reads it with one coalesced warp load.
#include "jacobi_scheme.cuh"

namespace b2s {
namespace {

constexpr int kJacobiWarps = 4;  // warps per CTA

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
                                 int max_bs, T* __restrict__ blocks, int l1)
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
        T off = T(0);
        for (int k = rp[row]; k < rp[row + 1]; ++k) {
            const int c = ci[k] - s;
            if (0 <= c && c < bs) {
                A[lane][c] = v[k];
            } else if (l1) {
                off += magnitude(v[k]);
            }
        }
        // block_l1 (reference/preconditioner/jacobi_kernels.cpp:751-779): the
        // absolute sum of the row's entries outside its block, in storage
        // order, added to the row's diagonal (a missing diagonal counts as 0)
        if (l1) A[lane][lane] += off;
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
    // permute_and_transpose_block: inverse(i, perm[j]) = A(i, j), in the
    // interleaved layout
    const BlockScheme sc = block_scheme(max_bs);
    T* out = blocks + (blk >> sc.power) * sc.group + (blk & (sc.gs - 1)) * max_bs;
    if (lane < bs) {
        for (int j = 0; j < bs; ++j) out[lane + int64_t(perm[j]) * sc.stride] = A[lane][j];
    }
}

// Apply: one warp per group of gs blocks, lane = (block in the group, row),
// so column `inner` of the whole group is one coalesced load; all max_bs
// columns of the lane's row are loaded before the sums (MB2 = pow2ceil of
// max_bs, a compile-time bound).  Every lane runs the same broadcast steps
// (full-mask shuffles); lanes outside a valid row only pass values along.
// x(row) = beta x(row) (or 0), then += (alpha inv(row, inner)) b(inner) for
// inner in order, as apply_block (jacobi_kernels.cpp:419-445); KC columns of
// b at a time reuse the loaded block.
template <typename T, int MB2, int KC>
__global__ void __launch_bounds__(kJacobiWarps * kWarp)
    jacobi_block_apply_kernel(int64_t n, int64_t num_blocks, const int32_t* __restrict__ ptrs,
                              int max_bs, const T* __restrict__ blocks,
                              const T* __restrict__ b, int64_t ldb, T* __restrict__ x,
                              int64_t ldx, int64_t k, const T* __restrict__ alpha,
                              const T* __restrict__ beta)
{
    const BlockScheme sc = block_scheme(max_bs);
    const int lane = threadIdx.x % kWarp, w = threadIdx.x / kWarp;
    const int sub = lane / max_bs, r = lane % max_bs;
    const int64_t grp = int64_t(blockIdx.x) * kJacobiWarps + w;
    if (grp * sc.gs >= num_blocks) return;  // the whole warp: uniform
    const int64_t blk = grp * sc.gs + sub;
    int s = 0, bs = 0;
    const bool in_block = sub < sc.gs && blk < num_blocks &&
                          block_extent(ptrs, blk, n, max_bs, s, bs);
    const bool active = in_block && r < bs;
    // the lane's row of the inverse, one coalesced load per column
    const T* g = blocks + grp * sc.group + lane;
    const bool in_group = lane < sc.gs * max_bs;
    T inv[MB2];
#pragma unroll
    for (int inner = 0; inner < MB2; ++inner) {
        inv[inner] = in_group && inner < max_bs ? __ldg(g + inner * sc.stride) : T(0);
    }
    const T a = alpha ? *alpha : T(1);
    const T be = beta ? *beta : T(0);
    const int base = sub * max_bs;  // first lane of this lane's block
    for (int64_t c0 = 0; c0 < k; c0 += KC) {
        T bv[KC], acc[KC];
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            const bool col_ok = c0 + c < k;
            bv[c] = active && col_ok ? b[(s + r) * ldb + c0 + c] : T(0);
            acc[c] = active && col_ok && be != T(0) ? x[(s + r) * ldx + c0 + c] * be : T(0);
        }
#pragma unroll
        for (int inner = 0; inner < MB2; ++inner) {
            if (inner < max_bs) {
                const T ai = a * inv[inner];
                const bool use = active && inner < bs;
#pragma unroll
                for (int c = 0; c < KC; ++c) {
                    const T bi = __shfl_sync(0xffffffffu, bv[c], (base + inner) % kWarp);
                    if (use) acc[c] += ai * bi;
                }
            }
        }
        if (active) {
#pragma unroll
            for (int c = 0; c < KC; ++c) {
                if (c0 + c < k) x[(s + r) * ldx + c0 + c] = acc[c];
            }
        }
    }
}

template <typename T>
int block_generate(int64_t n, const int32_t* rp, const int32_t* ci, const T* v,
                   int64_t num_blocks, const int32_t* ptrs, int max_bs, T* blocks,
                   int aggregate_l1, void* stream)
{
    B2S_CHECK_ARG(n >= 0 && num_blocks >= 0, "negative size");
    B2S_CHECK_ARG(max_bs >= 1 && max_bs <= kMaxBs, "max_block_size must be 1..32");
    if (num_blocks == 0) return B2S_OK;
    jacobi_block_generate_kernel<T><<<ceildiv(num_blocks, kJacobiWarps),
                                      kJacobiWarps * kWarp, 0, as_stream(stream)>>>(
        n, rp, ci, v, num_blocks, ptrs, max_bs, blocks, aggregate_l1);
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
    const BlockScheme sc = block_scheme(max_bs);
    const int64_t grid = ceildiv(ceildiv(num_blocks, sc.gs), kJacobiWarps);
    cudaStream_t st = as_stream(stream);
    auto launch = [&](auto kernel) {
        kernel<<<grid, kJacobiWarps * kWarp, 0, st>>>(n, num_blocks, ptrs, max_bs, blocks, b,
                                                      ldb, x, ldx, k, alpha, beta);
    };
    const int mb2 = kMaxBs / sc.gs;
#define B2S_JAC_APPLY(MB)                                                    \
    if (mb2 == MB) {                                                         \
        if (k == 1) launch(jacobi_block_apply_kernel<T, MB, 1>);             \
        else if (k == 2) launch(jacobi_block_apply_kernel<T, MB, 2>);        \
        else launch(jacobi_block_apply_kernel<T, MB, 4>);                    \
    }
    B2S_JAC_APPLY(1)
    B2S_JAC_APPLY(2)
    B2S_JAC_APPLY(4)
    B2S_JAC_APPLY(8)
    B2S_JAC_APPLY(16)
    B2S_JAC_APPLY(32)
#undef B2S_JAC_APPLY
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_jacobi_storage_scheme(int max_block_size, int64_t num_blocks, int64_t* block_offset,
                              int64_t* group_offset, int32_t* group_power,
                              int64_t* storage_space)
{
    B2S_CHECK_ARG(max_block_size >= 1 && max_block_size <= kMaxBs,
                  "max_block_size must be 1..32");
    B2S_CHECK_ARG(num_blocks >= 0, "negative number of blocks");
    const BlockScheme sc = block_scheme(max_block_size);
    if (block_offset) *block_offset = max_block_size;
    if (group_offset) *group_offset = sc.group;
    if (group_power) *group_power = sc.power;
    if (storage_space) *storage_space = ceildiv(num_blocks, sc.gs) * sc.group;
    return B2S_OK;
}

int b2s_jacobi_block_generate_f64(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const double* values,
                                  int64_t num_blocks, const int32_t* block_ptrs,
                                  int max_block_size, double* blocks, int aggregate_l1,
                                  void* stream)
{
    return block_generate(num_rows, row_ptrs, col_idxs, values, num_blocks, block_ptrs,
                          max_block_size, blocks, aggregate_l1, stream);
}

int b2s_jacobi_block_generate_f32(int64_t num_rows, const int32_t* row_ptrs,
                                  const int32_t* col_idxs, const float* values,
                                  int64_t num_blocks, const int32_t* block_ptrs,
                                  int max_block_size, float* blocks, int aggregate_l1,
                                  void* stream)
{
    return block_generate(num_rows, row_ptrs, col_idxs, values, num_blocks, block_ptrs,
                          max_block_size, blocks, aggregate_l1, stream);
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
