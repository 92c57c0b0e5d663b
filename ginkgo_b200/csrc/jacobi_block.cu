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

// Separately rounded product and sum (no fused multiply-add), so the
// elimination rounds as the reference's host code does.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// In-place Gauss-Jordan elimination with partial pivoting of the bs x bs
// block in A (lane r owns row r), perm recording the row swaps: the steps of
// the reference's invert_block (reference/preconditioner/jacobi_kernels.cpp:
// 128-240).  False when a zero pivot ended the elimination (the block then
// stays as far as it got, as the reference's generate keeps it).
template <typename T>
__device__ bool warp_gauss_jordan(T (*A)[kMaxBs + 1], int* perm, int bs, int lane)
{
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
        if (d == T(0)) return false;  // singular: the block stays as far as it got
        // apply_gauss_jordan_transform(k, k): column k scaled by -1/d ...
        if (lane < bs) A[lane][k] = A[lane][k] / -d;
        __syncwarp();
        if (lane == 0) A[k][k] = T(0);
        __syncwarp();
        // ... the rank-one update of every row but k (row k gains 0 there) ...
        if (lane < bs && lane != k) {
            const T aik = A[lane][k];
            for (int j = 0; j < bs; ++j) A[lane][j] = add_rn(A[lane][j], mul_rn(aik, A[k][j]));
        }
        __syncwarp();
        // ... and row k divided by d, its diagonal 1/d
        if (lane < bs) A[k][lane] = A[k][lane] / d;
        __syncwarp();
        if (lane == 0) A[k][k] = T(1) / d;
        __syncwarp();
    }
    return true;
}

// extract_block: row `lane` of the block starting at row s into A, zeros
// outside the pattern, perm the identity.  With l1, block_l1
// (reference/preconditioner/jacobi_kernels.cpp:751-779): the absolute sum of
// the row's entries outside its block, in storage order, added to the row's
// diagonal (a missing diagonal counts as 0).
template <typename T>
__device__ void warp_extract_block(const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ ci, const T* __restrict__ v,
                                   int s, int bs, int l1, T (*A)[kMaxBs + 1], int* perm,
                                   int lane)
{
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
        if (l1) A[lane][lane] += off;
    }
    __syncwarp();
}

// permute_and_transpose_block: inverse(i, perm[j]) = A(i, j), written at full
// precision to block blk of the interleaved layout.
template <typename T>
__device__ void store_inverse(const T (*A)[kMaxBs + 1], const int* perm, int bs, int64_t blk,
                              int max_bs, T* __restrict__ blocks, int lane)
{
    const BlockScheme sc = block_scheme(max_bs);
    T* out = blocks + (blk >> sc.power) * sc.group + (blk & (sc.gs - 1)) * max_bs;
    if (lane < bs) {
        for (int j = 0; j < bs; ++j) out[lane + int64_t(perm[j]) * sc.stride] = A[lane][j];
    }
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
    warp_extract_block(rp, ci, v, s, bs, l1, A, perm, lane);
    warp_gauss_jordan(A, perm, bs, lane);
    store_inverse(A, perm, bs, blk, max_bs, blocks, lane);
}

// compute_inf_norm (reference/preconditioner/jacobi_kernels.cpp:248-262): the
// largest absolute row sum of the bs x bs block, every lane getting it; a NaN
// row sum never wins (the reference's running max keeps the earlier value).
template <typename T>
__device__ T warp_inf_norm(const T (*A)[kMaxBs + 1], int bs, int lane)
{
    T sum = T(0);
    if (lane < bs) {
        for (int j = 0; j < bs; ++j) sum += magnitude(A[lane][j]);
    }
    if (!(sum == sum)) sum = T(0);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const T o = __shfl_xor_sync(0xffffffffu, sum, off);
        sum = sum < o ? o : sum;
    }
    return sum;
}

// float_traits<T>::eps, half of the machine epsilon.
template <typename T>
__device__ __forceinline__ T unit_roundoff()
{
    return sizeof(T) == 8 ? T(1.1102230246251565e-16) : T(5.9604644775390625e-08);
}

// validate_precision_reduction_feasibility (reference/preconditioner/
// jacobi_kernels.cpp:280-306): the eliminated block E rounded to storage
// kind K and back, in scratch tile B, stays invertible and well conditioned
// (cond >= 1 and cond * eps(T) < 1e-3).
template <int K, typename T>
__device__ bool warp_feasible(const T (*E)[kMaxBs + 1], T (*B)[kMaxBs + 1], int* perm, int bs,
                              int lane)
{
    for (int j = 0; j < kMaxBs; ++j) B[lane][j] = lane < bs && j < bs ? roundtrip<K>(E[lane][j]) : T(0);
    perm[lane] = lane;
    __syncwarp();
    T cond = warp_inf_norm(B, bs, lane);
    if (!warp_gauss_jordan(B, perm, bs, lane)) return false;
    cond = cond * warp_inf_norm(B, bs, lane);
    return cond >= T(1) && cond * unit_roundoff<T>() < T(1e-3);
}

// get_supported_storage_reductions (core/preconditioner/jacobi_utils.hpp):
// the descriptor bits of the storage reductions whose precision keeps
// cond * eps below the accuracy; the non-preserving ones only after the
// feasibility check (the one-step check at most once).  eps per storage:
// truncate<truncate<T>>, truncate<reduce<T>>, reduce<reduce<T>>,
// truncate<T>, reduce<T>.
template <typename T>
__device__ uint32_t warp_supported_reductions(T accuracy, T cond, const T (*E)[kMaxBs + 1],
                                              T (*B)[kMaxBs + 1], int* perm, int bs, int lane)
{
    const bool f64 = sizeof(T) == 8;
    const T e_t2t = f64 ? T(0.0625) : T(0.0078125);
    const T e_tr = f64 ? T(0.0078125) : T(0.00048828125);
    const T e_rr = T(0.00048828125);
    const T e_t = f64 ? T(9.5367431640625e-07) : T(0.0078125);
    const T e_r = f64 ? T(5.9604644775390625e-08) : T(0.00048828125);
    constexpr int R1 = sizeof(T) == 8 ? kF32 : kF16;  // reduce<T>
    auto accurate = [&](T e) { return T(cond * e) < accuracy; };
    int verified1 = 2;  // 2: not checked yet
    uint32_t sup = 0;
    if (accurate(e_t2t)) sup |= kD20;
    if (accurate(e_tr)) {
        verified1 = warp_feasible<R1>(E, B, perm, bs, lane) ? 1 : 0;
        if (verified1) sup |= kD11;
    }
    if (accurate(e_rr) && verified1 != 0 && warp_feasible<kF16>(E, B, perm, bs, lane)) {
        sup |= kD02;
    }
    if (accurate(e_t)) sup |= kD10;
    if (accurate(e_r)) {
        if (verified1 == 2) verified1 = warp_feasible<R1>(E, B, perm, bs, lane) ? 1 : 0;
        if (verified1 == 1) sup |= kD01;
    }
    return sup;
}

// precision_reduction_descriptor::singleton.
__device__ __forceinline__ uint32_t singleton_descriptor(uint8_t p)
{
    switch (p) {
    case kP02: return kD02;
    case kP11: return kD11;
    case kP20: return kD20;
    case kP01: return kD01;
    case kP10: return kD10;
    default: return 0;
    }
}

// get_optimal_storage_reduction: the most reduced of the supported storages.
__device__ __forceinline__ uint8_t optimal_reduction(uint32_t sup)
{
    if (sup & kD02) return kP02;
    if (sup & kD11) return kP11;
    if (sup & kD20) return kP20;
    if (sup & kD01) return kP01;
    if (sup & kD10) return kP10;
    return kP00;
}

constexpr int kAdaptiveWarps = 2;  // warps per CTA (two tiles each)

// Adaptive generation, step one (reference/preconditioner/jacobi_kernels.cpp:
// 309-370), one warp per block: the block's conditioning
// ||B||_inf ||B^-1||_inf, its inverse at full precision in the interleaved
// layout, and the descriptor of the storages it supports (the requested
// precision's singleton unless autodetection is asked for).
template <typename T>
__global__ void __launch_bounds__(kAdaptiveWarps * kWarp)
    jacobi_adaptive_generate_kernel(int64_t n, const int32_t* __restrict__ rp,
                                    const int32_t* __restrict__ ci, const T* __restrict__ v,
                                    int64_t num_blocks, const int32_t* __restrict__ ptrs,
                                    int max_bs, T accuracy,
                                    const uint8_t* __restrict__ requested,
                                    T* __restrict__ conditioning,
                                    uint32_t* __restrict__ descriptors, T* __restrict__ blocks,
                                    int l1)
{
    __shared__ T tile[kAdaptiveWarps][2][kMaxBs][kMaxBs + 1];
    __shared__ int perm_sh[kAdaptiveWarps][2][kMaxBs];
    const int lane = threadIdx.x % kWarp, w = threadIdx.x / kWarp;
    const int64_t blk = int64_t(blockIdx.x) * kAdaptiveWarps + w;
    if (blk >= num_blocks) return;
    int s, bs;
    if (!block_extent(ptrs, blk, n, max_bs, s, bs)) {
        if (lane == 0) descriptors[blk] = ~0u;  // leaves the group's choice alone
        return;
    }
    T(*A)[kMaxBs + 1] = tile[w][0];
    int* perm = perm_sh[w][0];
    warp_extract_block(rp, ci, v, s, bs, l1, A, perm, lane);
    T cond = warp_inf_norm(A, bs, lane);
    warp_gauss_jordan(A, perm, bs, lane);
    cond = cond * warp_inf_norm(A, bs, lane);
    const uint8_t req = requested[blk];
    const uint32_t desc =
        req == kAutodetect
            ? warp_supported_reductions(accuracy, cond, A, tile[w][1], perm_sh[w][1], bs, lane)
            : singleton_descriptor(req);
    if (lane == 0) {
        conditioning[blk] = cond;
        descriptors[blk] = desc;
    }
    store_inverse(A, perm, bs, blk, max_bs, blocks, lane);
}

constexpr int kGroupThreads = 128;
constexpr int kGroupValues = kMaxBs * kMaxBs / kGroupThreads;  // values per thread

// Adaptive generation, step two, and the storage conversions, one CTA per
// group.  With descriptors: the group's precision is the optimal reduction
// of the AND of its blocks' descriptors, written to every block of the group
// (jacobi_kernels.cpp:372-381); without, it is the group's recorded one.
// TO_REDUCED converts the group's full-precision slot of src to that storage
// in dst; otherwise the reduced storage of src is widened to full precision
// in dst.  All values are read before any is written, so dst may be src.
template <typename T, bool TO_REDUCED>
__global__ void __launch_bounds__(kGroupThreads)
    jacobi_group_storage_kernel(int64_t num_blocks, int max_bs,
                                const uint32_t* __restrict__ descriptors, uint8_t* precisions,
                                const T* src, T* dst)
{
    const BlockScheme sc = block_scheme(max_bs);
    const int64_t grp = blockIdx.x;
    const int t = threadIdx.x;
    __shared__ uint8_t group_prec;
    if (t < kWarp) {
        const int64_t b = grp * sc.gs + t;
        const bool valid = t < sc.gs && b < num_blocks;
        uint8_t p;
        if (descriptors) {
            uint32_t d = valid ? descriptors[b] : ~0u;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) d &= __shfl_xor_sync(0xffffffffu, d, off);
            p = optimal_reduction(d);
            if (valid) precisions[b] = p;
        } else {
            p = precisions[grp * sc.gs];
        }
        if (t == 0) group_prec = p;
    }
    __syncthreads();
    const int kind = storage_kind<T>(group_prec);
    const int64_t base = grp * sc.group;
    if (kind == kFull) {
        if (src != dst) {
            for (int64_t i = t; i < sc.group; i += kGroupThreads) dst[base + i] = src[base + i];
        }
        return;
    }
    T vals[kGroupValues];
    with_storage_kind(kind, [&](auto kc) {
        constexpr int K = decltype(kc)::value;
#pragma unroll
        for (int i = 0; i < kGroupValues; ++i) {
            const int64_t idx = t + int64_t(i) * kGroupThreads;
            if (idx < sc.group) {
                vals[i] = TO_REDUCED ? src[base + idx] : load_reduced<K, T>(src + base, idx);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kGroupValues; ++i) {
            const int64_t idx = t + int64_t(i) * kGroupThreads;
            if (idx < sc.group) {
                if (TO_REDUCED) {
                    store_reduced<K, T>(dst + base, idx, vals[i]);
                } else {
                    dst[base + idx] = vals[i];
                }
            }
        }
    });
}

// Apply: one warp per group of gs blocks, lane = (block in the group, row),
// so column `inner` of the whole group is one coalesced load; all max_bs
// columns of the lane's row are loaded before the sums (MB2 = pow2ceil of
// max_bs, a compile-time bound).  Every lane runs the same broadcast steps
// (full-mask shuffles); lanes outside a valid row only pass values along.
// x(row) = beta x(row) (or 0), then += (alpha inv(row, inner)) b(inner) for
// inner in order, as apply_block (jacobi_kernels.cpp:419-445); KC columns of
// b at a time reuse the loaded block.
//
// With precisions (adaptive storage), the group's values are read from its
// storage type and widened to T before the same arithmetic (apply_block's
// converter, jacobi_kernels.cpp:417-447).
template <typename T, int MB2, int KC, bool AP>
__global__ void __launch_bounds__(kJacobiWarps * kWarp)
    jacobi_block_apply_kernel(int64_t n, int64_t num_blocks, const int32_t* __restrict__ ptrs,
                              int max_bs, const uint8_t* __restrict__ precisions,
                              const T* __restrict__ blocks, const T* __restrict__ b,
                              int64_t ldb, T* __restrict__ x, int64_t ldx, int64_t k,
                              const T* __restrict__ alpha, const T* __restrict__ beta)
{
    const BlockScheme sc = block_scheme(max_bs);
    const int lane = threadIdx.x % kWarp, w = threadIdx.x / kWarp;
    const int sub = lane / max_bs, r = lane % max_bs;
    const int64_t nwarps = int64_t(gridDim.x) * kJacobiWarps;
    // persistent: a warp walks the groups with a grid stride (uniform per warp)
    for (int64_t grp = int64_t(blockIdx.x) * kJacobiWarps + w; grp * sc.gs < num_blocks;
         grp += nwarps) {
    const int64_t blk = grp * sc.gs + sub;
    int s = 0, bs = 0;
    const bool in_block = sub < sc.gs && blk < num_blocks &&
                          block_extent(ptrs, blk, n, max_bs, s, bs);
    const bool active = in_block && r < bs;
    // the lane's row of the inverse, one coalesced load per column
    const bool in_group = lane < sc.gs * max_bs;
    T inv[MB2];
    auto load = [&](auto kc) {
        constexpr int K = decltype(kc)::value;
        load_widened<K, MB2>(blocks + grp * sc.group, lane, sc.stride, in_group, max_bs, inv);
    };
    if constexpr (AP) {
        with_storage_kind(storage_kind<T>(precisions[grp * sc.gs]), load);
    } else {
        load(std::integral_constant<int, kFull>{});
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
                const uint8_t* precisions, const T* blocks, const T* b, int64_t ldb, T* x,
                int64_t ldx, int64_t k, const T* alpha, const T* beta, void* stream)
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
        kernel<<<resident_grid(kernel, kJacobiWarps * kWarp, grid), kJacobiWarps * kWarp, 0,
                 st>>>(n, num_blocks, ptrs, max_bs, precisions, blocks, b, ldb, x, ldx, k,
                       alpha, beta);
    };
    const int mb2 = kMaxBs / sc.gs;
#define B2S_JAC_APPLY_AP(MB, AP)                                             \
    if (k == 1) launch(jacobi_block_apply_kernel<T, MB, 1, AP>);             \
    else if (k == 2) launch(jacobi_block_apply_kernel<T, MB, 2, AP>);        \
    else launch(jacobi_block_apply_kernel<T, MB, 4, AP>);
#define B2S_JAC_APPLY(MB)                                                    \
    if (mb2 == MB) {                                                         \
        if (precisions) {                                                    \
            B2S_JAC_APPLY_AP(MB, true)                                       \
        } else {                                                             \
            B2S_JAC_APPLY_AP(MB, false)                                      \
        }                                                                    \
    }
    B2S_JAC_APPLY(1)
    B2S_JAC_APPLY(2)
    B2S_JAC_APPLY(4)
    B2S_JAC_APPLY(8)
    B2S_JAC_APPLY(16)
    B2S_JAC_APPLY(32)
#undef B2S_JAC_APPLY
#undef B2S_JAC_APPLY_AP
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

template <typename T>
int adaptive_generate(int64_t n, const int32_t* rp, const int32_t* ci, const T* v,
                      int64_t num_blocks, const int32_t* ptrs, int max_bs, T accuracy,
                      T* conditioning, uint8_t* precisions, T* blocks, int aggregate_l1,
                      void* workspace, void* stream)
{
    B2S_CHECK_ARG(n >= 0 && num_blocks >= 0, "negative size");
    B2S_CHECK_ARG(max_bs >= 1 && max_bs <= kMaxBs, "max_block_size must be 1..32");
    if (num_blocks == 0) return B2S_OK;
    B2S_CHECK_ARG(conditioning && precisions && blocks && workspace,
                  "conditioning, block_precisions, blocks and workspace are required");
    cudaStream_t st = as_stream(stream);
    auto* desc = static_cast<uint32_t*>(workspace);
    jacobi_adaptive_generate_kernel<T><<<ceildiv(num_blocks, kAdaptiveWarps),
                                         kAdaptiveWarps * kWarp, 0, st>>>(
        n, rp, ci, v, num_blocks, ptrs, max_bs, accuracy, precisions, conditioning, desc,
        blocks, aggregate_l1);
    B2S_LAUNCH_CHECK();
    const BlockScheme sc = block_scheme(max_bs);
    jacobi_group_storage_kernel<T, true><<<ceildiv(num_blocks, sc.gs), kGroupThreads, 0, st>>>(
        num_blocks, max_bs, desc, precisions, blocks, blocks);
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

template <typename T>
int group_storage(int64_t num_blocks, int max_bs, const uint8_t* precisions, const T* src,
                  T* dst, bool to_reduced, void* stream)
{
    B2S_CHECK_ARG(num_blocks >= 0, "negative size");
    B2S_CHECK_ARG(max_bs >= 1 && max_bs <= kMaxBs, "max_block_size must be 1..32");
    if (num_blocks == 0) return B2S_OK;
    B2S_CHECK_ARG(precisions && src && dst, "block_precisions and blocks are required");
    const BlockScheme sc = block_scheme(max_bs);
    const int64_t grid = ceildiv(num_blocks, sc.gs);
    cudaStream_t st = as_stream(stream);
    auto* prec = const_cast<uint8_t*>(precisions);  // only read without descriptors
    if (to_reduced) {
        jacobi_group_storage_kernel<T, true><<<grid, kGroupThreads, 0, st>>>(
            num_blocks, max_bs, nullptr, prec, src, dst);
    } else {
        jacobi_group_storage_kernel<T, false><<<grid, kGroupThreads, 0, st>>>(
            num_blocks, max_bs, nullptr, prec, src, dst);
    }
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
    return block_apply(num_rows, num_blocks, block_ptrs, max_block_size,
                       static_cast<const uint8_t*>(nullptr), blocks, b, ldb, x, ldx, num_rhs,
                       alpha, beta, stream);
}

int b2s_jacobi_block_apply_f32(int64_t num_rows, int64_t num_blocks,
                               const int32_t* block_ptrs, int max_block_size,
                               const float* blocks, const float* b, int64_t ldb,
                               float* x, int64_t ldx, int64_t num_rhs,
                               const float* alpha, const float* beta, void* stream)
{
    return block_apply(num_rows, num_blocks, block_ptrs, max_block_size,
                       static_cast<const uint8_t*>(nullptr), blocks, b, ldb, x, ldx, num_rhs,
                       alpha, beta, stream);
}

int b2s_jacobi_adaptive_workspace_bytes(int64_t num_blocks, int64_t* bytes)
{
    B2S_CHECK_ARG(num_blocks >= 0 && bytes, "negative number of blocks or null output");
    *bytes = num_blocks * int64_t(sizeof(uint32_t));
    return B2S_OK;
}

int b2s_jacobi_block_generate_adaptive_f64(int64_t num_rows, const int32_t* row_ptrs,
                                           const int32_t* col_idxs, const double* values,
                                           int64_t num_blocks, const int32_t* block_ptrs,
                                           int max_block_size, double accuracy,
                                           double* conditioning, uint8_t* block_precisions,
                                           double* blocks, int aggregate_l1, void* workspace,
                                           void* stream)
{
    return adaptive_generate(num_rows, row_ptrs, col_idxs, values, num_blocks, block_ptrs,
                             max_block_size, accuracy, conditioning, block_precisions, blocks,
                             aggregate_l1, workspace, stream);
}

int b2s_jacobi_block_apply_adaptive_f64(int64_t num_rows, int64_t num_blocks,
                                        const int32_t* block_ptrs, int max_block_size,
                                        const uint8_t* block_precisions, const double* blocks,
                                        const double* b, int64_t ldb, double* x, int64_t ldx,
                                        int64_t num_rhs, const double* alpha, const double* beta,
                                        void* stream)
{
    B2S_CHECK_ARG(block_precisions || num_blocks == 0, "block_precisions is required");
    return block_apply(num_rows, num_blocks, block_ptrs, max_block_size, block_precisions,
                       blocks, b, ldb, x, ldx, num_rhs, alpha, beta, stream);
}

int b2s_jacobi_block_expand_f64(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const double* blocks,
                                double* full_blocks, void* stream)
{
    return group_storage(num_blocks, max_block_size, block_precisions, blocks, full_blocks,
                         false, stream);
}

int b2s_jacobi_block_reduce_f64(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const double* full_blocks,
                                double* blocks, void* stream)
{
    return group_storage(num_blocks, max_block_size, block_precisions, full_blocks, blocks,
                         true, stream);
}

int b2s_jacobi_block_generate_adaptive_f32(int64_t num_rows, const int32_t* row_ptrs,
                                           const int32_t* col_idxs, const float* values,
                                           int64_t num_blocks, const int32_t* block_ptrs,
                                           int max_block_size, float accuracy,
                                           float* conditioning, uint8_t* block_precisions,
                                           float* blocks, int aggregate_l1, void* workspace,
                                           void* stream)
{
    return adaptive_generate(num_rows, row_ptrs, col_idxs, values, num_blocks, block_ptrs,
                             max_block_size, accuracy, conditioning, block_precisions, blocks,
                             aggregate_l1, workspace, stream);
}

int b2s_jacobi_block_apply_adaptive_f32(int64_t num_rows, int64_t num_blocks,
                                        const int32_t* block_ptrs, int max_block_size,
                                        const uint8_t* block_precisions, const float* blocks,
                                        const float* b, int64_t ldb, float* x, int64_t ldx,
                                        int64_t num_rhs, const float* alpha, const float* beta,
                                        void* stream)
{
    B2S_CHECK_ARG(block_precisions || num_blocks == 0, "block_precisions is required");
    return block_apply(num_rows, num_blocks, block_ptrs, max_block_size, block_precisions,
                       blocks, b, ldb, x, ldx, num_rhs, alpha, beta, stream);
}

int b2s_jacobi_block_expand_f32(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const float* blocks,
                                float* full_blocks, void* stream)
{
    return group_storage(num_blocks, max_block_size, block_precisions, blocks, full_blocks,
                         false, stream);
}

int b2s_jacobi_block_reduce_f32(int64_t num_blocks, int max_block_size,
                                const uint8_t* block_precisions, const float* full_blocks,
                                float* blocks, void* stream)
{
    return group_storage(num_blocks, max_block_size, block_precisions, full_blocks, blocks,
                         true, stream);
}

}  // extern "C"
