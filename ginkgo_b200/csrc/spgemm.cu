// Sparse products and sums on Csr, and the Hybrid (Ell + Coo) format.
//
//   spgemm           C = A B                 reference/matrix/csr_kernels.cpp:199-245
//   advanced_spgemm  C = alpha A B + beta D  reference/matrix/csr_kernels.cpp:247-300
//   spgeam           C = alpha A + beta B    reference/matrix/csr_kernels.cpp:424-470
//                                            (abstract_spgeam, reference/components/
//                                            csr_spgeam.hpp)
//   convert_to_hybrid, hybrid spmv and Hybrid -> Csr
//                                            (include/ginkgo/core/matrix/hybrid.hpp)
//
// Results are bit-exact with the reference executor: C's rows hold the
// union of the contributing columns in ascending order, and every entry is
// accumulated in the reference's order with the reference's roundings
// (no fused multiply-add): for a product row, D's contribution beta * d
// first, then for each entry a of A's row in storage order, + (alpha * a) * b
// for the entries b of the B row it selects.  B's rows must not repeat a
// column (the Csr invariant), so the contributions of one A entry land on
// distinct C entries and are added in parallel.
//
// SpGEMM runs in two calls, as the caller owns C's arrays: symbolic (C's row
// pointers and entry count) and numeric (C's columns and values).  Rows are
// binned by their product bound (the number of candidate entries):
//   <= 512    one warp per row: candidates sorted in shared memory (bitonic),
//             duplicates dropped, values accumulated in shared memory at the
//             positions found by binary search;
//   <= 8192   the same with one block of 256 threads per row;
//   larger    one block per row with a bitmap of B's columns in the
//             workspace: positions from per-word prefix counts, values
//             accumulated in C's own value array.
#include <algorithm>

#include "common.cuh"
#include "scan.cuh"

namespace b2s {
namespace {

constexpr int kGemmBlock = 256;
constexpr int kWarpCap = 512;    // candidates per row in the warp bin
constexpr int kBlockCap = 8192;  // candidates per row in the block bin
constexpr int kBitmapBlocks = 64;  // blocks sharing the bitmap scratch
constexpr int kBins = 3;
constexpr int32_t kNoCol = 0x7fffffff;

template <typename T>
__device__ __forceinline__ T mul_rn(T a, T b);
template <>
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <>
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ T add_rn(T a, T b);
template <>
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <>
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

struct GemmArgs {
    int64_t n;                    // rows of A (and C)
    int64_t m;                    // columns of B (and C)
    const int32_t* a_rp;
    const int32_t* a_ci;
    const int32_t* b_rp;
    const int32_t* b_ci;
    const int32_t* d_rp;          // D (advanced form) or null
    const int32_t* d_ci;
};

// Product bound of every row of A (and its bin): warp per row.
__global__ void __launch_bounds__(kGemmBlock)
    gemm_bound_kernel(GemmArgs g, int64_t* __restrict__ bound,
                      int32_t* __restrict__ bin_rows, int32_t* __restrict__ bin_count)
{
    const int64_t row = (blockIdx.x * int64_t(kGemmBlock) + threadIdx.x) / kWarp;
    const int lane = threadIdx.x % kWarp;
    if (row >= g.n) return;  // whole warps leave together
    int64_t ub = 0;
    for (int e = g.a_rp[row] + lane; e < g.a_rp[row + 1]; e += kWarp) {
        const int k = g.a_ci[e];
        ub += g.b_rp[k + 1] - g.b_rp[k];
    }
#pragma unroll
    for (int off = 16; off > 0; off /= 2) ub += __shfl_xor_sync(0xffffffffu, ub, off);
    if (g.d_rp) ub += g.d_rp[row + 1] - g.d_rp[row];
    if (lane == 0) {
        bound[row] = ub;
        const int bin = ub <= kWarpCap ? 0 : ub <= kBlockCap ? 1 : 2;
        const int slot = atomicAdd(bin_count + bin, 1);
        bin_rows[int64_t(bin) * g.n + slot] = int32_t(row);
    }
}

// Group-wide barrier of a warp (G = 32) or of the whole block.
template <int G>
__device__ __forceinline__ void group_barrier()
{
    if constexpr (G == kWarp) {
        __syncwarp();
    } else {
        __syncthreads();
    }
}

// Exclusive scan of one int per thread over the group; total to *total.
template <int G>
__device__ __forceinline__ int group_exclusive_scan(int v, int* sh, int* total)
{
    const int lane = threadIdx.x % kWarp;
    int x = v;
#pragma unroll
    for (int off = 1; off < kWarp; off *= 2) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if constexpr (G == kWarp) {
        *total = __shfl_sync(0xffffffffu, x, kWarp - 1);
        return x - v;
    } else {
        const int wid = threadIdx.x / kWarp;
        constexpr int W = G / kWarp;
        __syncthreads();
        if (lane == kWarp - 1) sh[wid] = x;
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < W; ++w) {
            const int s = sh[w];
            if (w < wid) off += s;
            tot += s;
        }
        *total = tot;
        return off + x - v;
    }
}

// Bitonic sort of cols[0..len) (len a power of two) by a group of G threads.
template <int G>
__device__ void group_sort(int32_t* cols, int len, int tid)
{
    for (int k = 2; k <= len; k *= 2) {
        for (int j = k / 2; j > 0; j /= 2) {
            for (int i = tid; i < len; i += G) {
                const int p = i ^ j;
                if (p > i) {
                    const int32_t a = cols[i], b = cols[p];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        cols[i] = b;
                        cols[p] = a;
                    }
                }
            }
            group_barrier<G>();
        }
    }
}

// Index of col in the ascending list cols[0..len) (present by construction).
__device__ __forceinline__ int find_col(const int32_t* cols, int len, int32_t col)
{
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (cols[mid] < col) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// One row of the shared-memory bins by a group of G threads (tid its
// thread): gather the candidate columns, sort them, drop duplicates.  In the
// symbolic pass the count goes to counts[row]; in the numeric pass the
// columns are written to C and the values accumulated in shared memory.
template <typename T, int G, int CAP, bool NUMERIC>
__device__ void gemm_row_smem(const GemmArgs& g, int64_t row, int tid, int32_t* cols,
                              T* vals, int* sh, int32_t* __restrict__ counts,
                              const T* __restrict__ a_v, const T* __restrict__ b_v,
                              const T* __restrict__ d_v, const T* alpha, const T* beta,
                              const int32_t* __restrict__ c_rp, int32_t* __restrict__ c_ci,
                              T* __restrict__ c_v)
{
    // gather: D's columns, then every B row that A's row selects
    int fill = 0;
    if (g.d_rp) {
        const int d0 = g.d_rp[row], d1 = g.d_rp[row + 1];
        for (int e = d0 + tid; e < d1; e += G) cols[e - d0] = g.d_ci[e];
        fill = d1 - d0;
    }
    const int a0 = g.a_rp[row], a1 = g.a_rp[row + 1];
    for (int e = a0; e < a1; ++e) {
        const int k = g.a_ci[e];
        const int b0 = g.b_rp[k], b1 = g.b_rp[k + 1];
        for (int q = b0 + tid; q < b1; q += G) cols[fill + q - b0] = g.b_ci[q];
        fill += b1 - b0;
    }
    int len = 32;
    while (len < fill) len *= 2;
    for (int i = fill + tid; i < len; i += G) cols[i] = kNoCol;
    group_barrier<G>();
    group_sort<G>(cols, len, tid);
    // drop duplicates: thread tid owns the run [tid * per, (tid + 1) * per)
    // and reads it (with the entry before it) into registers; flags[q] marks
    // the first entry of every distinct column
    const int per = len >= G ? len / G : 1;
    const int i0 = tid * per;
    int32_t mine[CAP / G > 0 ? CAP / G : 1];
    unsigned flags = 0;  // per <= 32
    int keep = 0;
    if (i0 < len) {
        int32_t prev = i0 > 0 ? cols[i0 - 1] : kNoCol;
        for (int q = 0; q < per; ++q) {
            const int32_t c = cols[i0 + q];
            mine[q] = c;
            if (c != kNoCol && (i0 + q == 0 || prev != c)) {
                flags |= 1u << q;
                ++keep;
            }
            prev = c;
        }
    }
    int total = 0;
    const int pos0 = group_exclusive_scan<G>(keep, sh, &total);
    if constexpr (!NUMERIC) {
        if (tid == 0) counts[row] = total;
        group_barrier<G>();
        return;
    } else {
        group_barrier<G>();  // every run is in registers: compact in place
        if (i0 < len) {
            int pos = pos0;
            for (int q = 0; q < per; ++q) {
                if (flags & (1u << q)) cols[pos++] = mine[q];
            }
        }
        group_barrier<G>();
        const int base = c_rp[row];
        for (int i = tid; i < total; i += G) {
            c_ci[base + i] = cols[i];
            vals[i] = T(0);
        }
        group_barrier<G>();
        if (g.d_rp) {
            const T bt = *beta;
            for (int e = g.d_rp[row] + tid; e < g.d_rp[row + 1]; e += G) {
                const int p = find_col(cols, total, g.d_ci[e]);
                vals[p] = add_rn(vals[p], mul_rn(bt, d_v[e]));
            }
            group_barrier<G>();
        }
        const T at = alpha ? *alpha : T(1);
        for (int e = a0; e < a1; ++e) {
            const int k = g.a_ci[e];
            const T sa = mul_rn(at, a_v[e]);
            for (int q = g.b_rp[k] + tid; q < g.b_rp[k + 1]; q += G) {
                const int p = find_col(cols, total, g.b_ci[q]);
                vals[p] = add_rn(vals[p], mul_rn(sa, b_v[q]));
            }
            group_barrier<G>();
        }
        for (int i = tid; i < total; i += G) c_v[base + i] = vals[i];
        group_barrier<G>();
    }
}

template <typename T, bool NUMERIC>
__global__ void __launch_bounds__(kGemmBlock)
    gemm_warp_rows_kernel(GemmArgs g, const int32_t* __restrict__ rows, int count,
                          int32_t* __restrict__ counts, const T* __restrict__ a_v,
                          const T* __restrict__ b_v, const T* __restrict__ d_v,
                          const T* alpha, const T* beta, const int32_t* __restrict__ c_rp,
                          int32_t* __restrict__ c_ci, T* __restrict__ c_v)
{
    constexpr int W = kGemmBlock / kWarp;
    __shared__ int32_t cols_sm[W][kWarpCap];
    __shared__ T vals_sm[NUMERIC ? W : 1][NUMERIC ? kWarpCap : 1];
    const int wid = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const int64_t q = blockIdx.x * int64_t(W) + wid;
    if (q >= count) return;  // whole warps leave together
    gemm_row_smem<T, kWarp, kWarpCap, NUMERIC>(
        g, rows[q], lane, cols_sm[wid], NUMERIC ? vals_sm[wid] : nullptr, nullptr, counts,
        a_v, b_v, d_v, alpha, beta, c_rp, c_ci, c_v);
}

template <typename T, bool NUMERIC>
__global__ void __launch_bounds__(kGemmBlock)
    gemm_block_rows_kernel(GemmArgs g, const int32_t* __restrict__ rows, int count,
                           int32_t* __restrict__ counts, const T* __restrict__ a_v,
                           const T* __restrict__ b_v, const T* __restrict__ d_v,
                           const T* alpha, const T* beta, const int32_t* __restrict__ c_rp,
                           int32_t* __restrict__ c_ci, T* __restrict__ c_v)
{
    extern __shared__ __align__(16) unsigned char gemm_smem[];
    T* vals = reinterpret_cast<T*>(gemm_smem);
    int32_t* cols = reinterpret_cast<int32_t*>(gemm_smem + (NUMERIC ? kBlockCap * sizeof(T) : 0));
    __shared__ int sh[kGemmBlock / kWarp];
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x) {
        gemm_row_smem<T, kGemmBlock, kBlockCap, NUMERIC>(
            g, rows[q], threadIdx.x, cols, vals, sh, counts, a_v, b_v, d_v, alpha, beta,
            c_rp, c_ci, c_v);
        __syncthreads();
    }
}

// Rows above the block bin: one block per row with a bitmap of B's columns
// (words, then their exclusive prefix counts) in the workspace.
template <typename T, bool NUMERIC>
__global__ void __launch_bounds__(kGemmBlock)
    gemm_bitmap_rows_kernel(GemmArgs g, const int32_t* __restrict__ rows, int count,
                            int32_t* __restrict__ counts, const T* __restrict__ a_v,
                            const T* __restrict__ b_v, const T* __restrict__ d_v,
                            const T* alpha, const T* beta, const int32_t* __restrict__ c_rp,
                            int32_t* __restrict__ c_ci, T* __restrict__ c_v,
                            unsigned* __restrict__ scratch)
{
    __shared__ int sh[kGemmBlock / kWarp];
    const int64_t words = ceildiv(g.m, 32);
    unsigned* bits = scratch + blockIdx.x * 2 * words;
    unsigned* prefix = bits + words;  // exclusive prefix popcounts (numeric)
    const int tid = threadIdx.x;
    for (int64_t q = blockIdx.x; q < count; q += gridDim.x) {
        const int64_t row = rows[q];
        // mark the candidate columns (the bitmap is all zero on entry)
        if (g.d_rp) {
            for (int e = g.d_rp[row] + tid; e < g.d_rp[row + 1]; e += kGemmBlock) {
                const int c = g.d_ci[e];
                atomicOr(bits + (c >> 5), 1u << (c & 31));
            }
        }
        const int a0 = g.a_rp[row], a1 = g.a_rp[row + 1];
        for (int e = a0; e < a1; ++e) {
            const int k = g.a_ci[e];
            for (int p = g.b_rp[k] + tid; p < g.b_rp[k + 1]; p += kGemmBlock) {
                const int c = g.b_ci[p];
                atomicOr(bits + (c >> 5), 1u << (c & 31));
            }
        }
        __syncthreads();
        // prefix counts over the words, in tiles of 256 words
        int carry = 0;
        for (int64_t w0 = 0; w0 < words; w0 += kGemmBlock) {
            const int64_t w = w0 + tid;
            const unsigned word = w < words ? __ldcg(bits + w) : 0u;
            const int cnt = __popc(word);
            int tile = 0;
            const int ex = group_exclusive_scan<kGemmBlock>(cnt, sh, &tile) + carry;
            if (NUMERIC && w < words) {
                prefix[w] = unsigned(ex);
                // the row's columns in ascending order
                unsigned rest = word;
                int pos = ex;
                while (rest) {
                    const int bit = __ffs(rest) - 1;
                    rest &= rest - 1;
                    c_ci[c_rp[row] + pos] = int32_t(w * 32 + bit);
                    ++pos;
                }
            }
            if (!NUMERIC && w < words) bits[w] = 0u;  // count-and-clear
            carry += tile;
        }
        if constexpr (!NUMERIC) {
            if (tid == 0) counts[row] = carry;
            __syncthreads();
            continue;
        } else {
            const int64_t base = c_rp[row];
            for (int i = tid; i < carry; i += kGemmBlock) __stcg(c_v + base + i, T(0));
            __syncthreads();
            auto slot = [&](int c) {
                const unsigned word = __ldcg(bits + (c >> 5));
                return int(__ldcg(prefix + (c >> 5))) +
                       __popc(word & ((1u << (c & 31)) - 1u));
            };
            if (g.d_rp) {
                const T bt = *beta;
                for (int e = g.d_rp[row] + tid; e < g.d_rp[row + 1]; e += kGemmBlock) {
                    T* dst = c_v + base + slot(g.d_ci[e]);
                    __stcg(dst, add_rn(__ldcg(dst), mul_rn(bt, d_v[e])));
                }
                __syncthreads();
            }
            const T at = alpha ? *alpha : T(1);
            for (int e = a0; e < a1; ++e) {
                const int k = g.a_ci[e];
                const T sa = mul_rn(at, a_v[e]);
                for (int p = g.b_rp[k] + tid; p < g.b_rp[k + 1]; p += kGemmBlock) {
                    T* dst = c_v + base + slot(g.b_ci[p]);
                    __stcg(dst, add_rn(__ldcg(dst), mul_rn(sa, b_v[p])));
                }
                __syncthreads();
            }
            // clear the bitmap for the next row
            for (int64_t w = tid; w < words; w += kGemmBlock) bits[w] = 0u;
            __syncthreads();
        }
    }
}

// counts (int32, n) -> row pointers (int32, n + 1) through an int64 scan;
// the total goes to *total (host) and must fit the int32 index type.
__global__ void widen_kernel(int64_t n, const int32_t* __restrict__ in,
                             int64_t* __restrict__ out)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = in[i];
}
__global__ void narrow_kernel(int64_t n, const int64_t* __restrict__ in,
                              int32_t* __restrict__ out)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i <= n) out[i] = int32_t(in[i]);
}

struct GemmWork {
    int64_t* bound;
    int32_t* bin_rows;   // [kBins][n]
    int32_t* bin_count;  // [kBins]
    int64_t* wide;       // n + 1 (scan of the counts)
    int64_t* scan_work;
    unsigned* bitmap;    // kBitmapBlocks x 2 x ceil(m / 32)
    int64_t bytes;
};

GemmWork gemm_work(void* base, int64_t n, int64_t m)
{
    GemmWork w{};
    char* p = static_cast<char*>(base);
    int64_t off = 0;
    auto take = [&](int64_t bytes) {
        char* r = p ? p + off : nullptr;
        off += (bytes + 255) / 256 * 256;
        return r;
    };
    w.bound = reinterpret_cast<int64_t*>(take(n * 8));
    w.bin_rows = reinterpret_cast<int32_t*>(take(int64_t(kBins) * n * 4));
    w.bin_count = reinterpret_cast<int32_t*>(take(kBins * 4));
    w.wide = reinterpret_cast<int64_t*>(take((n + 1) * 8));
    w.scan_work = reinterpret_cast<int64_t*>(take(scan_work_entries<int64_t>(n) * 8));
    w.bitmap = reinterpret_cast<unsigned*>(take(int64_t(kBitmapBlocks) * 2 * ceildiv(m, 32) * 4));
    w.bytes = off;
    return w;
}

// Bins the rows; returns the bin sizes on the host.
int gemm_bins(const GemmArgs& g, const GemmWork& w, int (&sizes)[kBins], cudaStream_t st)
{
    B2S_CUDA_TRY(cudaMemsetAsync(w.bin_count, 0, kBins * 4, st));
    if (g.n > 0) {
        gemm_bound_kernel<<<ceildiv(g.n * kWarp, kGemmBlock), kGemmBlock, 0, st>>>(
            g, w.bound, w.bin_rows, w.bin_count);
        B2S_LAUNCH_CHECK();
    }
    B2S_CUDA_TRY(cudaMemcpyAsync(sizes, w.bin_count, sizeof(sizes), cudaMemcpyDeviceToHost, st));
    B2S_CUDA_TRY(cudaStreamSynchronize(st));
    return B2S_OK;
}

template <typename T, bool NUMERIC>
int gemm_rows(const GemmArgs& g, const GemmWork& w, const int (&sizes)[kBins],
              int32_t* counts, const T* a_v, const T* b_v, const T* d_v, const T* alpha,
              const T* beta, const int32_t* c_rp, int32_t* c_ci, T* c_v, cudaStream_t st)
{
    if (sizes[0] > 0) {
        constexpr int W = kGemmBlock / kWarp;
        gemm_warp_rows_kernel<T, NUMERIC><<<ceildiv(sizes[0], W), kGemmBlock, 0, st>>>(
            g, w.bin_rows, sizes[0], counts, a_v, b_v, d_v, alpha, beta, c_rp, c_ci, c_v);
        B2S_LAUNCH_CHECK();
    }
    if (sizes[1] > 0) {
        auto k = gemm_block_rows_kernel<T, NUMERIC>;
        const size_t sm = size_t(kBlockCap) * (4 + (NUMERIC ? sizeof(T) : 0));
        B2S_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(sm)));
        const int grid = int(std::min<int64_t>(sizes[1], int64_t(num_sms()) * 2));
        k<<<grid, kGemmBlock, sm, st>>>(g, w.bin_rows + g.n, sizes[1], counts, a_v, b_v,
                                         d_v, alpha, beta, c_rp, c_ci, c_v);
        B2S_LAUNCH_CHECK();
    }
    if (sizes[2] > 0) {
        const int grid = std::min(sizes[2], kBitmapBlocks);
        // the bitmaps start empty; every row leaves its block's bitmap empty
        B2S_CUDA_TRY(cudaMemsetAsync(w.bitmap, 0, int64_t(grid) * 2 * ceildiv(g.m, 32) * 4,
                                     st));
        gemm_bitmap_rows_kernel<T, NUMERIC><<<grid, kGemmBlock, 0, st>>>(
            g, w.bin_rows + 2 * g.n, sizes[2], counts, a_v, b_v, d_v, alpha, beta, c_rp,
            c_ci, c_v, w.bitmap);
        B2S_LAUNCH_CHECK();
    }
    return B2S_OK;
}

// ---------------------------------------------------------------- SpGEAM --

// Merge of two ascending rows (abstract_spgeam): the count, or the entries
// alpha * a + beta * b with a missing side read as zero.
template <typename T, bool NUMERIC>
__global__ void __launch_bounds__(kGemmBlock)
    geam_kernel(int64_t n, const int32_t* __restrict__ a_rp, const int32_t* __restrict__ a_ci,
                const T* __restrict__ a_v, const int32_t* __restrict__ b_rp,
                const int32_t* __restrict__ b_ci, const T* __restrict__ b_v, const T* alpha,
                const T* beta, int32_t* __restrict__ counts, const int32_t* __restrict__ c_rp,
                int32_t* __restrict__ c_ci, T* __restrict__ c_v)
{
    const int64_t row = blockIdx.x * int64_t(kGemmBlock) + threadIdx.x;
    if (row >= n) return;
    int i = a_rp[row];
    const int ie = a_rp[row + 1];
    int j = b_rp[row];
    const int je = b_rp[row + 1];
    T al = T(0), be = T(0);
    if constexpr (NUMERIC) {
        al = *alpha;
        be = *beta;
    }
    int out = NUMERIC ? c_rp[row] : 0;
    while (i < ie || j < je) {
        const int32_t ca = i < ie ? a_ci[i] : kNoCol;
        const int32_t cb = j < je ? b_ci[j] : kNoCol;
        const int32_t c = min(ca, cb);
        if constexpr (NUMERIC) {
            const T av = ca == c ? a_v[i] : T(0);
            const T bv = cb == c ? b_v[j] : T(0);
            c_ci[out] = c;
            c_v[out] = add_rn(mul_rn(al, av), mul_rn(be, bv));
        }
        ++out;
        i += ca <= cb;
        j += cb <= ca;
    }
    if constexpr (!NUMERIC) counts[row] = out;
}

// ---------------------------------------------------------------- Hybrid --

// Coo entries of every row: max(len - width, 0).
__global__ void hybrid_coo_count_kernel(int64_t n, const int32_t* __restrict__ rp,
                                        int64_t width, int64_t* __restrict__ counts)
{
    const int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (row >= n) return;
    const int64_t len = rp[row + 1] - rp[row];
    counts[row] = len > width ? len - width : 0;
}

// The first `width` entries of each row into the Ell part (column-major,
// padding -1 / 0), the rest into Coo at the row's offset
// (csr::convert_to_hybrid).
template <typename T>
__global__ void hybrid_fill_kernel(int64_t n, const int32_t* __restrict__ rp,
                                   const int32_t* __restrict__ ci, const T* __restrict__ v,
                                   int64_t width, int64_t stride,
                                   const int64_t* __restrict__ coo_off,
                                   int32_t* __restrict__ ell_ci, T* __restrict__ ell_v,
                                   int32_t* __restrict__ coo_r, int32_t* __restrict__ coo_c,
                                   T* __restrict__ coo_v)
{
    const int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (row >= n) return;
    const int64_t b0 = rp[row], len = rp[row + 1] - b0;
    for (int64_t s = 0; s < width; ++s) {
        const int64_t slot = row + s * stride;
        if (s < len) {
            ell_ci[slot] = ci[b0 + s];
            ell_v[slot] = v[b0 + s];
        } else {
            ell_ci[slot] = -1;
            ell_v[slot] = T(0);
        }
    }
    int64_t o = coo_off[row];
    for (int64_t s = width; s < len; ++s, ++o) {
        coo_r[o] = int32_t(row);
        coo_c[o] = ci[b0 + s];
        coo_v[o] = v[b0 + s];
    }
}

// First Coo entry of row `row` (the Coo part is sorted by row).
__device__ __forceinline__ int64_t coo_lower(const int32_t* __restrict__ r, int64_t nnz,
                                             int64_t row)
{
    int64_t lo = 0, hi = nnz;
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (__ldg(r + mid) < row) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// y = A x (or alpha A x + beta y) for Hybrid: per row, the Ell slots in
// order, then the row's Coo entries in order (found by binary search in the
// row-sorted Coo part); K columns per pass.
template <typename T, int K>
__global__ void __launch_bounds__(kGemmBlock)
    hybrid_spmv_kernel(int64_t n, int64_t width, int64_t stride,
                       const int32_t* __restrict__ ell_ci, const T* __restrict__ ell_v,
                       int64_t coo_nnz, const int32_t* __restrict__ coo_r,
                       const int32_t* __restrict__ coo_c, const T* __restrict__ coo_v,
                       const T* __restrict__ b, int64_t ldb, T* __restrict__ c, int64_t ldc,
                       int k, int col0, const T* alpha, const T* beta)
{
    const int64_t row = blockIdx.x * int64_t(kGemmBlock) + threadIdx.x;
    if (row >= n) return;
    const int kc = min(K, k - col0);
    T acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    for (int64_t s = 0; s < width; ++s) {
        const int col = ld_stream(ell_ci + row + s * stride);
        if (col < 0) continue;
        const T val = ld_stream(ell_v + row + s * stride);
        const T* xr = b + int64_t(col) * ldb + col0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j < kc) acc[j] = add_rn(acc[j], mul_rn(val, __ldg(xr + j)));
        }
    }
    if (coo_nnz > 0) {
        for (int64_t e = coo_lower(coo_r, coo_nnz, row); e < coo_nnz && coo_r[e] == row; ++e) {
            const T val = coo_v[e];
            const T* xr = b + int64_t(coo_c[e]) * ldb + col0;
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (j < kc) acc[j] = add_rn(acc[j], mul_rn(val, __ldg(xr + j)));
            }
        }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
        if (j < kc) {
            T* dst = c + row * ldc + col0 + j;
            *dst = combine(acc[j], alpha, beta, dst);
        }
    }
}

// Entries per row of the Csr form of a Hybrid matrix.
__global__ void hybrid_row_count_kernel(int64_t n, int64_t width, int64_t stride,
                                        const int32_t* __restrict__ ell_ci, int64_t coo_nnz,
                                        const int32_t* __restrict__ coo_r,
                                        int32_t* __restrict__ counts)
{
    const int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (row >= n) return;
    int cnt = 0;
    for (int64_t s = 0; s < width; ++s) cnt += ell_ci[row + s * stride] >= 0;
    if (coo_nnz > 0) {
        for (int64_t e = coo_lower(coo_r, coo_nnz, row); e < coo_nnz && coo_r[e] == row; ++e)
            ++cnt;
    }
    counts[row] = cnt;
}

// Hybrid -> Csr: the row's Ell entries then its Coo entries, then a stable
// insertion sort by column (rows are short).
template <typename T>
__global__ void hybrid_to_csr_kernel(int64_t n, int64_t width, int64_t stride,
                                     const int32_t* __restrict__ ell_ci,
                                     const T* __restrict__ ell_v, int64_t coo_nnz,
                                     const int32_t* __restrict__ coo_r,
                                     const int32_t* __restrict__ coo_c,
                                     const T* __restrict__ coo_v,
                                     const int32_t* __restrict__ rp, int32_t* __restrict__ ci,
                                     T* __restrict__ v)
{
    const int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (row >= n) return;
    const int64_t b0 = rp[row];
    int64_t o = b0;
    for (int64_t s = 0; s < width; ++s) {
        const int col = ell_ci[row + s * stride];
        if (col >= 0) {
            ci[o] = col;
            v[o] = ell_v[row + s * stride];
            ++o;
        }
    }
    if (coo_nnz > 0) {
        for (int64_t e = coo_lower(coo_r, coo_nnz, row); e < coo_nnz && coo_r[e] == row; ++e) {
            ci[o] = coo_c[e];
            v[o] = coo_v[e];
            ++o;
        }
    }
    for (int64_t i = b0 + 1; i < o; ++i) {
        const int32_t c = ci[i];
        const T x = v[i];
        int64_t j = i - 1;
        while (j >= b0 && ci[j] > c) {
            ci[j + 1] = ci[j];
            v[j + 1] = v[j];
            --j;
        }
        ci[j + 1] = c;
        v[j + 1] = x;
    }
}

// counts (int32) -> int32 row pointers and the host total, through int64.
int counts_to_row_ptrs(int64_t n, const int32_t* counts, int32_t* row_ptrs, int64_t* wide,
                       int64_t* scan_work, int64_t* total, cudaStream_t st)
{
    if (n > 0) {
        widen_kernel<<<ceildiv(n, 256), 256, 0, st>>>(n, counts, wide);
        B2S_LAUNCH_CHECK();
    }
    const int rc = exclusive_scan<int64_t>(wide, n, wide, scan_work, st);
    if (rc != B2S_OK) return rc;
    int64_t tot = 0;
    B2S_CUDA_TRY(cudaMemcpyAsync(&tot, wide + n, 8, cudaMemcpyDeviceToHost, st));
    B2S_CUDA_TRY(cudaStreamSynchronize(st));
    if (tot > int64_t(INT32_MAX)) {
        set_error("result has %lld entries, more than the int32 index type holds",
                  (long long)tot);
        return B2S_ERR_UNSUPPORTED;
    }
    narrow_kernel<<<ceildiv(n + 1, 256), 256, 0, st>>>(n, wide, row_ptrs);
    B2S_LAUNCH_CHECK();
    *total = tot;
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int64_t b2s_csr_spgemm_workspace_bytes(int64_t num_rows, int64_t num_cols)
{
    if (num_rows < 0 || num_cols < 0) return -1;
    return gemm_work(nullptr, num_rows, num_cols).bytes;
}

int b2s_csr_spgemm_symbolic(int64_t num_rows, int64_t num_cols, const int32_t* a_row_ptrs,
                            const int32_t* a_col_idxs, const int32_t* b_row_ptrs,
                            const int32_t* b_col_idxs, const int32_t* d_row_ptrs,
                            const int32_t* d_col_idxs, int32_t* c_row_ptrs, int64_t* c_nnz,
                            void* workspace, int64_t workspace_bytes, void* stream)
{
    B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0, "negative size");
    B2S_CHECK_ARG(c_row_ptrs && c_nnz, "null output");
    B2S_CHECK_ARG((d_row_ptrs == nullptr) == (d_col_idxs == nullptr),
                  "D's row pointers and columns must both be given or both be null");
    const GemmWork w = gemm_work(workspace, num_rows, num_cols);
    if (workspace_bytes < w.bytes) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)w.bytes);
        return B2S_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    GemmArgs g{num_rows, num_cols, a_row_ptrs, a_col_idxs, b_row_ptrs, b_col_idxs,
               d_row_ptrs, d_col_idxs};
    int sizes[kBins];
    int rc = gemm_bins(g, w, sizes, st);
    if (rc != B2S_OK) return rc;
    // the counts go to the first n entries of C's row pointers
    rc = gemm_rows<double, false>(g, w, sizes, c_row_ptrs, nullptr, nullptr, nullptr, nullptr,
                                  nullptr, nullptr, nullptr, nullptr, st);
    if (rc != B2S_OK) return rc;
    return counts_to_row_ptrs(num_rows, c_row_ptrs, c_row_ptrs, w.wide, w.scan_work, c_nnz,
                              st);
}

#define B2S_GEMM_ENTRIES(T, S)                                                      \
    int b2s_csr_spgemm_numeric_##S(                                                 \
        int64_t num_rows, int64_t num_cols, const T* alpha, const int32_t* a_row_ptrs, \
        const int32_t* a_col_idxs, const T* a_values, const int32_t* b_row_ptrs,      \
        const int32_t* b_col_idxs, const T* b_values, const T* beta,                  \
        const int32_t* d_row_ptrs, const int32_t* d_col_idxs, const T* d_values,      \
        const int32_t* c_row_ptrs, int32_t* c_col_idxs, T* c_values, void* workspace, \
        int64_t workspace_bytes, void* stream)                                        \
    {                                                                                 \
        B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0, "negative size");              \
        B2S_CHECK_ARG((d_row_ptrs == nullptr) == (beta == nullptr) &&                 \
                          (d_row_ptrs == nullptr) == (d_col_idxs == nullptr),         \
                      "D and beta must all be given or all be null");                 \
        const GemmWork w = gemm_work(workspace, num_rows, num_cols);                  \
        if (workspace_bytes < w.bytes) {                                              \
            set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,   \
                      (long long)w.bytes);                                            \
            return B2S_ERR_WORKSPACE;                                                 \
        }                                                                             \
        cudaStream_t st = as_stream(stream);                                          \
        GemmArgs g{num_rows, num_cols, a_row_ptrs, a_col_idxs, b_row_ptrs,            \
                   b_col_idxs, d_row_ptrs, d_col_idxs};                               \
        int sizes[kBins];                                                             \
        int rc = gemm_bins(g, w, sizes, st);                                          \
        if (rc != B2S_OK) return rc;                                                  \
        return gemm_rows<T, true>(g, w, sizes, nullptr, a_values, b_values,           \
                                  d_values, alpha, beta, c_row_ptrs, c_col_idxs,      \
                                  c_values, st);                                      \
    }                                                                                 \
    int b2s_csr_spgeam_numeric_##S(                                                   \
        int64_t num_rows, const T* alpha, const int32_t* a_row_ptrs,                  \
        const int32_t* a_col_idxs, const T* a_values, const T* beta,                  \
        const int32_t* b_row_ptrs, const int32_t* b_col_idxs, const T* b_values,      \
        const int32_t* c_row_ptrs, int32_t* c_col_idxs, T* c_values, void* stream)    \
    {                                                                                 \
        B2S_CHECK_ARG(num_rows >= 0, "negative size");                                \
        B2S_CHECK_ARG(alpha && beta, "alpha and beta are required");                  \
        if (num_rows == 0) return B2S_OK;                                             \
        geam_kernel<T, true><<<ceildiv(num_rows, kGemmBlock), kGemmBlock, 0,          \
                               as_stream(stream)>>>(                                  \
            num_rows, a_row_ptrs, a_col_idxs, a_values, b_row_ptrs, b_col_idxs,       \
            b_values, alpha, beta, nullptr, c_row_ptrs, c_col_idxs, c_values);        \
        B2S_LAUNCH_CHECK();                                                           \
        return B2S_OK;                                                                \
    }                                                                                 \
    int b2s_csr_convert_to_hybrid_##S(                                                \
        int64_t num_rows, const int32_t* row_ptrs, const int32_t* col_idxs,           \
        const T* values, int64_t ell_width, int64_t ell_stride, int32_t* ell_col_idxs, \
        T* ell_values, int64_t coo_nnz, int32_t* coo_row_idxs, int32_t* coo_col_idxs, \
        T* coo_values, void* workspace, int64_t workspace_bytes, void* stream)        \
    {                                                                                 \
        B2S_CHECK_ARG(num_rows >= 0 && ell_width >= 0 && coo_nnz >= 0,               \
                      "negative size");                                               \
        B2S_CHECK_ARG(ell_stride >= num_rows, "Ell stride < num_rows");               \
        const int64_t need = b2s_hybrid_convert_workspace_bytes(num_rows);            \
        if (workspace_bytes < need) {                                                 \
            set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,   \
                      (long long)need);                                               \
            return B2S_ERR_WORKSPACE;                                                 \
        }                                                                             \
        if (num_rows == 0) return B2S_OK;                                             \
        cudaStream_t st = as_stream(stream);                                          \
        int64_t* off = static_cast<int64_t*>(workspace);                              \
        int64_t* sw = off + num_rows + 1;                                             \
        hybrid_coo_count_kernel<<<ceildiv(num_rows, 256), 256, 0, st>>>(              \
            num_rows, row_ptrs, ell_width, off);                                      \
        B2S_LAUNCH_CHECK();                                                           \
        int rc = exclusive_scan<int64_t>(off, num_rows, off, sw, st);                 \
        if (rc != B2S_OK) return rc;                                                  \
        int64_t total = 0;                                                            \
        B2S_CUDA_TRY(cudaMemcpyAsync(&total, off + num_rows, 8,                      \
                                     cudaMemcpyDeviceToHost, st));                    \
        B2S_CUDA_TRY(cudaStreamSynchronize(st));                                      \
        if (total != coo_nnz) {                                                       \
            set_error("the matrix has %lld entries past the Ell width, not %lld",     \
                      (long long)total, (long long)coo_nnz);                          \
            return B2S_ERR_INVALID_ARG;                                               \
        }                                                                             \
        hybrid_fill_kernel<T><<<ceildiv(num_rows, 256), 256, 0, st>>>(                \
            num_rows, row_ptrs, col_idxs, values, ell_width, ell_stride, off,         \
            ell_col_idxs, ell_values, coo_row_idxs, coo_col_idxs, coo_values);        \
        B2S_LAUNCH_CHECK();                                                           \
        return B2S_OK;                                                                \
    }                                                                                 \
    int b2s_hybrid_spmv_##S(int64_t num_rows, int64_t num_cols, int64_t ell_width,    \
                            int64_t ell_stride, const int32_t* ell_col_idxs,          \
                            const T* ell_values, int64_t coo_nnz,                     \
                            const int32_t* coo_row_idxs, const int32_t* coo_col_idxs, \
                            const T* coo_values, const T* b, int64_t ldb, T* c,       \
                            int64_t ldc, int64_t num_rhs, const T* alpha,             \
                            const T* beta, void* stream)                              \
    {                                                                                 \
        B2S_CHECK_ARG(num_rows >= 0 && num_cols >= 0 && num_rhs >= 0 &&              \
                          ell_width >= 0 && coo_nnz >= 0,                             \
                      "negative size");                                               \
        B2S_CHECK_ARG(ell_stride >= num_rows, "Ell stride < num_rows");               \
        B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),                        \
                      "alpha and beta must both be given or both be null");           \
        B2S_CHECK_ARG(num_rhs <= 1 || (ldb >= num_rhs && ldc >= num_rhs),             \
                      "leading dimension < num_rhs");                                 \
        if (num_rows == 0 || num_rhs == 0) return B2S_OK;                             \
        cudaStream_t st = as_stream(stream);                                          \
        const int64_t grid = ceildiv(num_rows, kGemmBlock);                           \
        for (int64_t c0 = 0; c0 < num_rhs; c0 += 4) {                                 \
            const int kc = int(std::min<int64_t>(4, num_rhs - c0));                   \
            if (kc == 1) {                                                            \
                hybrid_spmv_kernel<T, 1><<<grid, kGemmBlock, 0, st>>>(                \
                    num_rows, ell_width, ell_stride, ell_col_idxs, ell_values,        \
                    coo_nnz, coo_row_idxs, coo_col_idxs, coo_values, b, ldb, c, ldc,  \
                    int(num_rhs), int(c0), alpha, beta);                              \
            } else {                                                                  \
                hybrid_spmv_kernel<T, 4><<<grid, kGemmBlock, 0, st>>>(                \
                    num_rows, ell_width, ell_stride, ell_col_idxs, ell_values,        \
                    coo_nnz, coo_row_idxs, coo_col_idxs, coo_values, b, ldb, c, ldc,  \
                    int(num_rhs), int(c0), alpha, beta);                              \
            }                                                                         \
            B2S_LAUNCH_CHECK();                                                       \
        }                                                                             \
        return B2S_OK;                                                                \
    }                                                                                 \
    int b2s_hybrid_convert_to_csr_##S(                                                \
        int64_t num_rows, int64_t ell_width, int64_t ell_stride,                      \
        const int32_t* ell_col_idxs, const T* ell_values, int64_t coo_nnz,            \
        const int32_t* coo_row_idxs, const int32_t* coo_col_idxs, const T* coo_values, \
        const int32_t* row_ptrs, int32_t* col_idxs, T* values, void* stream)          \
    {                                                                                 \
        B2S_CHECK_ARG(num_rows >= 0 && ell_width >= 0 && coo_nnz >= 0,               \
                      "negative size");                                               \
        if (num_rows == 0) return B2S_OK;                                             \
        hybrid_to_csr_kernel<T><<<ceildiv(num_rows, 256), 256, 0, as_stream(stream)>>>( \
            num_rows, ell_width, ell_stride, ell_col_idxs, ell_values, coo_nnz,       \
            coo_row_idxs, coo_col_idxs, coo_values, row_ptrs, col_idxs, values);      \
        B2S_LAUNCH_CHECK();                                                           \
        return B2S_OK;                                                                \
    }

int b2s_csr_spgeam_symbolic(int64_t num_rows, const int32_t* a_row_ptrs,
                            const int32_t* a_col_idxs, const int32_t* b_row_ptrs,
                            const int32_t* b_col_idxs, int32_t* c_row_ptrs, int64_t* c_nnz,
                            void* workspace, int64_t workspace_bytes, void* stream)
{
    B2S_CHECK_ARG(num_rows >= 0, "negative size");
    B2S_CHECK_ARG(c_row_ptrs && c_nnz, "null output");
    const int64_t need = b2s_csr_spgeam_workspace_bytes(num_rows);
    if (workspace_bytes < need) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)need);
        return B2S_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    int64_t* wide = static_cast<int64_t*>(workspace);
    int64_t* sw = wide + num_rows + 1;
    if (num_rows > 0) {
        geam_kernel<double, false><<<ceildiv(num_rows, kGemmBlock), kGemmBlock, 0, st>>>(
            num_rows, a_row_ptrs, a_col_idxs, nullptr, b_row_ptrs, b_col_idxs, nullptr,
            nullptr, nullptr, c_row_ptrs, nullptr, nullptr, nullptr);
        B2S_LAUNCH_CHECK();
    }
    return counts_to_row_ptrs(num_rows, c_row_ptrs, c_row_ptrs, wide, sw, c_nnz, st);
}

int64_t b2s_csr_spgeam_workspace_bytes(int64_t num_rows)
{
    if (num_rows < 0) return -1;
    return (num_rows + 1) * 8 + scan_work_entries<int64_t>(num_rows) * 8;
}

int64_t b2s_hybrid_convert_workspace_bytes(int64_t num_rows)
{
    if (num_rows < 0) return -1;
    return (num_rows + 1) * 8 + scan_work_entries<int64_t>(num_rows) * 8;
}

int b2s_hybrid_csr_row_ptrs(int64_t num_rows, int64_t ell_width, int64_t ell_stride,
                            const int32_t* ell_col_idxs, int64_t coo_nnz,
                            const int32_t* coo_row_idxs, int32_t* row_ptrs, int64_t* nnz,
                            void* workspace, int64_t workspace_bytes, void* stream)
{
    B2S_CHECK_ARG(num_rows >= 0 && ell_width >= 0 && coo_nnz >= 0, "negative size");
    B2S_CHECK_ARG(ell_stride >= num_rows, "Ell stride < num_rows");
    B2S_CHECK_ARG(row_ptrs && nnz, "null output");
    const int64_t need = b2s_hybrid_convert_workspace_bytes(num_rows);
    if (workspace_bytes < need) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)need);
        return B2S_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    int64_t* wide = static_cast<int64_t*>(workspace);
    int64_t* sw = wide + num_rows + 1;
    if (num_rows > 0) {
        hybrid_row_count_kernel<<<ceildiv(num_rows, 256), 256, 0, st>>>(
            num_rows, ell_width, ell_stride, ell_col_idxs, coo_nnz, coo_row_idxs, row_ptrs);
        B2S_LAUNCH_CHECK();
    }
    return counts_to_row_ptrs(num_rows, row_ptrs, row_ptrs, wide, sw, nnz, st);
}

B2S_GEMM_ENTRIES(double, f64)
B2S_GEMM_ENTRIES(float, f32)

}  // extern "C"
