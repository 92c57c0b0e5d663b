// Sparse matrix times dense block: Csr (classical, load_balance), Ell, Sellp.
//
// Semantics follow the reference executor (reference/matrix/csr_kernels.cpp:
// 48-110, ell_kernels.cpp:29-130, sellp_kernels.cpp:27-105): c = A b, or
// c = alpha A b + beta c with beta == 0 ignoring c.  Dense blocks are
// row-major n x k with a leading dimension, so the k right-hand-side values
// of one row are contiguous and every kernel serves all k columns from ONE
// pass over the matrix (the reference's CUDA kernels re-read A per column).
#include <algorithm>

#include "common.cuh"
#include "csr_async.cuh"
#include "ell_rows.cuh"

namespace b2s {
namespace {

constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// Csr classical: one subwarp of SW lanes per row, lanes stride over the row's
// entries (coalesced across the subwarp), K right-hand sides per pass held
// in registers, xor-shuffle reduction inside the subwarp.
// ---------------------------------------------------------------------------
template <typename T, int SW, int K, bool VEC>
__global__ void __launch_bounds__(kBlock)
    csr_classical_kernel(int64_t n, const int32_t* __restrict__ rp,
                         const int32_t* __restrict__ ci,
                         const T* __restrict__ v, const T* __restrict__ b,
                         int64_t ldb, T* __restrict__ c, int64_t ldc,
                         const T* __restrict__ alpha,
                         const T* __restrict__ beta)
{
    const int64_t row = (blockIdx.x * int64_t(kBlock) + threadIdx.x) / SW;
    const int lane = threadIdx.x % SW;
    const bool valid = row < n;
    const int begin = valid ? __ldg(rp + row) : 0;
    const int end = valid ? __ldg(rp + row + 1) : 0;
    T acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    for (int e = begin + lane; e < end; e += SW) {
        const T val = ld_stream(v + e);
        const int64_t col = ld_stream(ci + e);
        T xr[K];
        RowLoad<T, K, VEC>::load(b + col * ldb, xr);
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] += val * xr[j];
    }
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = subwarp_sum<SW>(acc[j]);
    if (valid) {
        // lane l writes columns l, l + SW, ... (coalesced for K >= SW)
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (j % SW == lane) {
                T* dst = c + row * ldc + j;
                *dst = combine(acc[j], alpha, beta, dst);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Csr load_balance: the rows are binned into tiles of kTileItems merge-path
// items (one item per row plus one per stored entry; row r goes to tile
// floor((r + rp[r]) / kTileItems)), built once on the GPU by
// csr_tile_rows_kernel.  A block stages its tile's products val * b(col, :)
// through shared memory with coalesced loads, in chunks of kChunk entries,
// and a block-wide segmented scan (heads at row starts) sums every row.  A
// row longer than a chunk is carried from chunk to chunk inside the block,
// so no row is split across blocks: no atomics, no fix-up pass, and the
// result does not depend on scheduling.
// ---------------------------------------------------------------------------
constexpr int kTileItems = 2048;

__global__ void csr_tile_rows_kernel(int64_t n, const int32_t* __restrict__ rp,
                                     int64_t num_tiles,
                                     int32_t* __restrict__ tile_rows)
{
    const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (t > num_tiles) return;
    // first row r with r + rp[r] >= t * kTileItems (n when none)
    const int64_t target = t * kTileItems;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (mid + int64_t(__ldg(rp + mid)) >= target) {
            hi = mid;
        } else {
            lo = mid + 1;
        }
    }
    tile_rows[t] = int32_t(t == num_tiles ? n : lo);
}

// One pad word per 16: thread t scans the 8-byte words [8t, 8t + 8), which
// would otherwise fall into the same banks every other thread.
__device__ __forceinline__ int lb_pad(int w) { return w + (w >> 4); }

template <typename T, int K>
struct LbSmem {
    static constexpr int kIpt = K >= 8 ? 1 : 8 / K;  // entries per thread
    static constexpr int kChunk = kBlock * kIpt;
    T prod[kChunk * K + kChunk * K / 16 + 1];
    unsigned char head[kChunk];
    int32_t rows[kTileItems + 1];  // rp[r0 .. r1]
    T carry[K];
    T warp_sum[kBlock / kWarp][K];
    int warp_flag[kBlock / kWarp];
};

template <typename T, int K, bool VEC>
__global__ void __launch_bounds__(kBlock)
    csr_lb_kernel(const int32_t* __restrict__ tile_rows,
                  const int32_t* __restrict__ rp,
                  const int32_t* __restrict__ ci, const T* __restrict__ v,
                  const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
                  int64_t ldc, const T* __restrict__ alpha,
                  const T* __restrict__ beta)
{
    using Smem = LbSmem<T, K>;
    constexpr int kIpt = Smem::kIpt;
    constexpr int kChunk = Smem::kChunk;
    __shared__ Smem sm;
    const int tid = threadIdx.x;
    const int32_t r0 = tile_rows[blockIdx.x];
    const int32_t r1 = tile_rows[blockIdx.x + 1];
    if (r0 >= r1) return;
    const int nrows = r1 - r0;  // <= kTileItems by construction
    for (int i = tid; i <= nrows; i += kBlock) sm.rows[i] = __ldg(rp + r0 + i);
    if (tid < K) sm.carry[tid] = T(0);
    __syncthreads();
    const int e_begin = sm.rows[0];
    const int e_end = sm.rows[nrows];
    // empty rows produce 0 (alpha A b is 0 there)
    for (int i = tid; i < nrows; i += kBlock) {
        if (sm.rows[i] == sm.rows[i + 1]) {
            T* dst = c + int64_t(r0 + i) * ldc;
#pragma unroll
            for (int j = 0; j < K; ++j) dst[j] = combine(T(0), alpha, beta, dst + j);
        }
    }
    for (int cs = e_begin; cs < e_end; cs += kChunk) {
        const int ce = min(cs + kChunk, e_end);
        const int cnt = ce - cs;
        // 1. stage products and clear head flags
        for (int i = tid; i < kChunk; i += kBlock) {
            sm.head[i] = 0;
            if (i < cnt) {
                const T val = ld_stream(v + cs + i);
                const int64_t col = ld_stream(ci + cs + i);
                T xr[K];
                RowLoad<T, K, VEC>::load(b + col * ldb, xr);
#pragma unroll
                for (int j = 0; j < K; ++j) sm.prod[lb_pad(i * K + j)] = val * xr[j];
            }
        }
        __syncthreads();
        // 2. mark row starts inside the chunk (rows sorted by start)
        for (int i = tid; i < nrows; i += kBlock) {
            const int s = sm.rows[i];
            if (s > cs && s < ce && sm.rows[i + 1] > s) sm.head[s - cs] = 1;
        }
        if (tid == 0) sm.head[0] = 1;  // chunk start: carry added below
        __syncthreads();
        // 3. segmented inclusive scan: per-thread run, then warp/block
        T run[K];
        int any_head = 0;
        const int base = tid * kIpt;
#pragma unroll
        for (int j = 0; j < K; ++j) run[j] = T(0);
#pragma unroll
        for (int q = 0; q < kIpt; ++q) {
            const int i = base + q;
            if (i < cnt) {
                if (sm.head[i]) {
                    any_head = 1;
#pragma unroll
                    for (int j = 0; j < K; ++j) run[j] = T(0);
                }
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    run[j] += sm.prod[lb_pad(i * K + j)];
                    sm.prod[lb_pad(i * K + j)] = run[j];
                }
            }
        }
        // exclusive segmented prefix of thread aggregates (flag, run)
        const int lane = tid % kWarp, wid = tid / kWarp;
        T pre[K];
        int pflag = any_head;
#pragma unroll
        for (int j = 0; j < K; ++j) pre[j] = run[j];
#pragma unroll
        for (int off = 1; off < kWarp; off *= 2) {
            const int of = __shfl_up_sync(0xffffffffu, pflag, off);
            T ov[K];
#pragma unroll
            for (int j = 0; j < K; ++j) ov[j] = __shfl_up_sync(0xffffffffu, pre[j], off);
            if (lane >= off) {
                if (!pflag) {
#pragma unroll
                    for (int j = 0; j < K; ++j) pre[j] += ov[j];
                }
                pflag |= of;
            }
        }
        // pre/pflag: inclusive over lanes 0..lane
        if (lane == kWarp - 1) {
            sm.warp_flag[wid] = pflag;
#pragma unroll
            for (int j = 0; j < K; ++j) sm.warp_sum[wid][j] = pre[j];
        }
        __syncthreads();
        // exclusive prefix for this thread = inclusive of lane-1 combined
        // with the preceding warps' aggregates
        T ex[K];
        {
            int f = __shfl_up_sync(0xffffffffu, pflag, 1);
            T t[K];
#pragma unroll
            for (int j = 0; j < K; ++j) t[j] = __shfl_up_sync(0xffffffffu, pre[j], 1);
            if (lane == 0) {
                f = 0;
#pragma unroll
                for (int j = 0; j < K; ++j) t[j] = T(0);
            }
            if (!f) {
                // walk back over previous warps until one has a head
                for (int w = wid - 1; w >= 0; --w) {
#pragma unroll
                    for (int j = 0; j < K; ++j) t[j] += sm.warp_sum[w][j];
                    if (sm.warp_flag[w]) {
                        f = 1;
                        break;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < K; ++j) ex[j] = t[j];
        }
        // add the exclusive prefix to this thread's entries up to its first
        // head (those continue the previous segment)
#pragma unroll
        for (int q = 0; q < kIpt; ++q) {
            const int i = base + q;
            if (i < cnt) {
                if (sm.head[i]) break;
#pragma unroll
                for (int j = 0; j < K; ++j) sm.prod[lb_pad(i * K + j)] += ex[j];
            }
        }
        __syncthreads();
        // 4. rows ending in this chunk write their sums; the first of them
        //    adds the carry when it started in an earlier chunk
        for (int i = tid; i < nrows; i += kBlock) {
            const int s = sm.rows[i], e = sm.rows[i + 1];
            if (e > s && e > cs && e <= ce) {
                T* dst = c + int64_t(r0 + i) * ldc;
#pragma unroll
                for (int j = 0; j < K; ++j) {
                    T val = sm.prod[lb_pad((e - 1 - cs) * K + j)];
                    if (s < cs) val += sm.carry[j];
                    dst[j] = combine(val, alpha, beta, dst + j);
                }
            }
        }
        __syncthreads();
        // 5. carry of the row still open at the chunk end: the row holding
        //    entry ce - 1 is the last i with rows[i] <= ce - 1; its partial
        //    is prod[cnt - 1], plus the old carry if it began before cs
        if (tid < K && ce < e_end) {
            int lo = 0, hi = nrows;  // rows[lo] <= ce - 1 < rows[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) / 2;
                if (sm.rows[mid] <= ce - 1) {
                    lo = mid;
                } else {
                    hi = mid;
                }
            }
            const T part = sm.prod[lb_pad((cnt - 1) * K + tid)];
            sm.carry[tid] = sm.rows[lo] < cs ? sm.carry[tid] + part : part;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Ell (column-major, stride >= n, padding column -1) and Sellp (slices of
// slice_size rows, column-major inside a slice).  One thread per row; for a
// fixed entry index the threads of a warp read consecutive addresses.
// ---------------------------------------------------------------------------
template <typename T, int K, bool VEC>
__global__ void __launch_bounds__(kBlock)
    ell_kernel(int64_t n, int64_t width, int64_t stride,
               const int32_t* __restrict__ ci, const T* __restrict__ v,
               const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
               int64_t ldc, const T* __restrict__ alpha,
               const T* __restrict__ beta)
{
    const int64_t row = blockIdx.x * int64_t(kBlock) + threadIdx.x;
    if (row >= n) return;
    T acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    int64_t idx = row;
#pragma unroll 4
    for (int64_t i = 0; i < width; ++i, idx += stride) {
        const int32_t col = ld_stream(ci + idx);
        const T val = ld_stream(v + idx);
        if (col != -1) {
            T xr[K];
            RowLoad<T, K, VEC>::load(b + int64_t(col) * ldb, xr);
#pragma unroll
            for (int j = 0; j < K; ++j) acc[j] += val * xr[j];
        }
    }
    T* dst = c + row * ldc;
#pragma unroll
    for (int j = 0; j < K; ++j) dst[j] = combine(acc[j], alpha, beta, dst + j);
}

// Row count fits in int32 (the index type); slice arithmetic in 32 bits.
template <typename T, int K, bool VEC>
__global__ void __launch_bounds__(kBlock)
    sellp_kernel(int n, int slice_size,
                 const uint64_t* __restrict__ slice_sets,
                 const uint64_t* __restrict__ slice_lengths,
                 const int32_t* __restrict__ ci, const T* __restrict__ v,
                 const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
                 int64_t ldc, const T* __restrict__ alpha,
                 const T* __restrict__ beta)
{
    const int row = blockIdx.x * kBlock + threadIdx.x;
    if (row >= n) return;
    const unsigned slice = unsigned(row) / unsigned(slice_size);
    const unsigned local = unsigned(row) - slice * unsigned(slice_size);
    const int len = int(__ldg(slice_lengths + slice));
    const T* vp = v + int64_t(__ldg(slice_sets + slice)) * slice_size + local;
    const int32_t* cp = ci + (vp - v);
    T acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    int i = 0;
    for (; i + 4 <= len; i += 4) {
        int32_t col[4];
        T val[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            col[u] = ld_stream(cp + (i + u) * slice_size);
            val[u] = ld_stream(vp + (i + u) * slice_size);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (col[u] != -1) {
                T xr[K];
                RowLoad<T, K, VEC>::load(b + int64_t(col[u]) * ldb, xr);
#pragma unroll
                for (int j = 0; j < K; ++j) acc[j] += val[u] * xr[j];
            }
        }
    }
    for (; i < len; ++i) {
        const int32_t col = ld_stream(cp + i * slice_size);
        const T val = ld_stream(vp + i * slice_size);
        if (col != -1) {
            T xr[K];
            RowLoad<T, K, VEC>::load(b + int64_t(col) * ldb, xr);
#pragma unroll
            for (int j = 0; j < K; ++j) acc[j] += val * xr[j];
        }
    }
    T* dst = c + int64_t(row) * ldc;
#pragma unroll
    for (int j = 0; j < K; ++j) dst[j] = combine(acc[j], alpha, beta, dst + j);
}

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

// FMT 0: Csr, 1: Ell, 2: Sellp
template <typename T, int K, int FMT>
__global__ void __launch_bounds__(kBlock)
    rhs_lanes_kernel(int64_t n, const int32_t* __restrict__ rp,
                     int64_t width_or_slice, int64_t stride,
                     const uint64_t* __restrict__ slice_sets,
                     const uint64_t* __restrict__ slice_lengths,
                     const int32_t* __restrict__ ci, const T* __restrict__ v,
                     const T* __restrict__ b, int64_t ldb, T* __restrict__ c,
                     int64_t ldc, const T* __restrict__ alpha,
                     const T* __restrict__ beta)
{
    using V = typename Vec16<T>::type;
    constexpr int VW = Vec16<T>::width;
    constexpr int KL = K / VW;
    const int64_t g = blockIdx.x * int64_t(kBlock) + threadIdx.x;
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

// ---------------------------------------------------------------------------
// host-side dispatch
// ---------------------------------------------------------------------------

// Largest chunk of right-hand sides handled per pass: 16, 8, 4, 2 or 1.
inline int rhs_chunk(int64_t remaining)
{
    for (int kk : {16, 8, 4, 2}) {
        if (remaining >= kk) return kk;
    }
    return 1;
}

template <typename T>
bool vec_ok(const T* b, int64_t ldb, int64_t col0, int kk)
{
    if (kk < 2) return false;
    const size_t bytes = sizeof(T);
    return (reinterpret_cast<uintptr_t>(b + col0) % 16 == 0) &&
           ((ldb * bytes) % 16 == 0);
}

// 16-byte vector path for >= 4 right-hand sides: both b and c rows aligned
template <typename T>
bool lanes_ok(const T* b, int64_t ldb, const T* c, int64_t ldc, int64_t col0,
              int kk)
{
    return kk >= 4 && kk % Vec16<T>::width == 0 && vec_ok(b, ldb, col0, kk) &&
           vec_ok(static_cast<const T*>(c), ldc, col0, kk);
}

template <typename T, int K, int FMT>
void launch_lanes(int64_t n, const int32_t* rp, int64_t w_or_s, int64_t stride,
                  const uint64_t* sets, const uint64_t* lens, const int32_t* ci,
                  const T* v, const T* b, int64_t ldb, T* c, int64_t ldc,
                  const T* alpha, const T* beta, cudaStream_t st)
{
    if constexpr (K >= 4 && K % Vec16<T>::width == 0) {
        constexpr int KL = K / Vec16<T>::width;
        rhs_lanes_kernel<T, K, FMT><<<ceildiv(n * KL, kBlock), kBlock, 0, st>>>(
            n, rp, w_or_s, stride, sets, lens, ci, v, b, ldb, c, ldc, alpha,
            beta);
    }
}

#define B2S_DISPATCH_K(kk, VEC, ...)                   \
    switch (kk) {                                      \
    case 16: { constexpr int K = 16; __VA_ARGS__; break; } \
    case 8: { constexpr int K = 8; __VA_ARGS__; break; }   \
    case 4: { constexpr int K = 4; __VA_ARGS__; break; }   \
    case 2: { constexpr int K = 2; __VA_ARGS__; break; }   \
    default: { constexpr int K = 1; __VA_ARGS__; break; }  \
    }

template <typename T, int K, bool VEC>
void launch_classical(int sw, int64_t n, const int32_t* rp, const int32_t* ci,
                      const T* v, const T* b, int64_t ldb, T* c, int64_t ldc,
                      const T* alpha, const T* beta, cudaStream_t st)
{
    const int64_t grid = ceildiv(n * sw, kBlock);
#define B2S_CL(SW)                                                          \
    csr_classical_kernel<T, SW, K, VEC><<<grid, kBlock, 0, st>>>(           \
        n, rp, ci, v, b, ldb, c, ldc, alpha, beta)
    switch (sw) {
    case 32: B2S_CL(32); break;
    case 16: B2S_CL(16); break;
    case 8: B2S_CL(8); break;
    case 4: B2S_CL(4); break;
    case 2: B2S_CL(2); break;
    default: B2S_CL(1); break;
    }
#undef B2S_CL
}

// Subwarp size: the largest power of two <= the longest row, capped at 32
// (the rule of common/cuda_hip/matrix/csr_kernels.template.cpp:2398-2419).
inline int classical_subwarp(int64_t max_row_nnz)
{
    int sw = 1;
    while (sw * 2 <= max_row_nnz && sw < 32) sw *= 2;
    return sw;
}

template <typename T>
int csr_spmv(int strategy, int64_t n, int64_t num_cols, const int32_t* rp,
             const int32_t* ci, const T* v, int64_t max_row_nnz,
             const int32_t* tile_rows, int64_t num_tiles, const T* b,
             int64_t ldb, T* c, int64_t ldc, int64_t k, const T* alpha,
             const T* beta, void* stream)
{
    B2S_CHECK_ARG(n >= 0 && num_cols >= 0 && k >= 0, "negative size");
    B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),
                  "alpha and beta must both be given or both be null");
    B2S_CHECK_ARG(k == 0 || (ldb >= k && ldc >= k), "leading dimension < k");
    if (n == 0 || k == 0) return B2S_OK;
    B2S_CHECK_ARG(rp && b && c, "null pointer");
    cudaStream_t st = as_stream(stream);
    if (strategy == B2S_CSR_LOAD_BALANCE) {
        B2S_CHECK_ARG(tile_rows != nullptr && num_tiles >= 1,
                      "load_balance needs the tile partition");
    } else {
        B2S_CHECK_ARG(strategy == B2S_CSR_CLASSICAL, "unknown strategy %d",
                      strategy);
    }
    const int sw = classical_subwarp(max_row_nnz);
    for (int64_t col0 = 0; col0 < k;) {
        const int kk = rhs_chunk(k - col0);
        const bool vec = vec_ok(b, ldb, col0, kk);
        const T* bb = b + col0;
        T* cc = c + col0;
        if (strategy == B2S_CSR_LOAD_BALANCE) {
            B2S_DISPATCH_K(kk, VEC, {
                if (vec) {
                    csr_lb_kernel<T, K, true><<<num_tiles, kBlock, 0, st>>>(
                        tile_rows, rp, ci, v, bb, ldb, cc, ldc, alpha, beta);
                } else {
                    csr_lb_kernel<T, K, false><<<num_tiles, kBlock, 0, st>>>(
                        tile_rows, rp, ci, v, bb, ldb, cc, ldc, alpha, beta);
                }
            });
        } else if (lanes_ok(b, ldb, c, ldc, col0, kk)) {
            B2S_DISPATCH_K(kk, VEC, {
                launch_lanes<T, K, 0>(n, rp, 0, 0, nullptr, nullptr, ci, v, bb,
                                      ldb, cc, ldc, alpha, beta, st);
            });
        } else if (kk <= 2) {
            // persistent: as many blocks as fit on the SMs at once; rows of
            // the longest length share a stage 32 / lpr at a time
            const int lpr = async_lanes_per_row(max_row_nnz);
            const int64_t need = ceildiv(ceildiv(n, kWarp / lpr), kAsyncBlock / kWarp);
            auto launch = [&](auto kernel) {
                const int64_t grid = std::min<int64_t>(need, async_resident_blocks(kernel));
                kernel<<<grid, kAsyncBlock, 0, st>>>(n, rp, ci, v, bb, ldb, cc, ldc,
                                                     alpha, beta, nullptr);
            };
            if (kk == 2 && vec) {
                with_async_kernel<T, 2, true>(lpr, launch);
            } else if (kk == 2) {
                with_async_kernel<T, 2, false>(lpr, launch);
            } else {
                with_async_kernel<T, 1, false>(lpr, launch);
            }
        } else {
            B2S_DISPATCH_K(kk, VEC, {
                if (vec) {
                    launch_classical<T, K, true>(sw, n, rp, ci, v, bb, ldb, cc,
                                                 ldc, alpha, beta, st);
                } else {
                    launch_classical<T, K, false>(sw, n, rp, ci, v, bb, ldb,
                                                  cc, ldc, alpha, beta, st);
                }
            });
        }
        B2S_LAUNCH_CHECK();
        col0 += kk;
    }
    return B2S_OK;
}

template <typename T>
int ell_spmv(int64_t n, int64_t num_cols, int64_t width, int64_t stride,
             const int32_t* ci, const T* v, const T* b, int64_t ldb, T* c,
             int64_t ldc, int64_t k, const T* alpha, const T* beta,
             void* stream)
{
    B2S_CHECK_ARG(n >= 0 && k >= 0 && width >= 0, "negative size");
    B2S_CHECK_ARG(stride >= n, "Ell stride %lld < rows %lld", (long long)stride,
                  (long long)n);
    B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),
                  "alpha and beta must both be given or both be null");
    B2S_CHECK_ARG(k == 0 || (ldb >= k && ldc >= k), "leading dimension < k");
    if (n == 0 || k == 0) return B2S_OK;
    cudaStream_t st = as_stream(stream);
    const int64_t grid = ceildiv(n, kBlock);
    constexpr int RV = int(16 / sizeof(T));
    const int R = ell_rows_per_thread<T>(width);
    if (k == 1 && R == RV && stride % R == 0 && reinterpret_cast<uintptr_t>(ci) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(v) % 16 == 0 && width <= INT32_MAX) {
        // one right-hand side: R rows per thread, 16-byte loads of values
        // (wide FP64 rows stay on the row-per-thread kernel below, which
        // measured faster there)
        const int64_t g = std::min<int64_t>(ceildiv(ceildiv(n, R), kBlock),
                                            int64_t(num_sms()) * 16);
        ell_rows_kernel_for<T, RV>()<<<g, kBlock, 0, st>>>(
            n, int(width), stride, ci, v, b, ldb, c, ldc, alpha, beta, nullptr);
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    }
    for (int64_t col0 = 0; col0 < k;) {
        const int kk = rhs_chunk(k - col0);
        const bool vec = vec_ok(b, ldb, col0, kk);
        if (lanes_ok(b, ldb, c, ldc, col0, kk)) {
            B2S_DISPATCH_K(kk, VEC, {
                launch_lanes<T, K, 1>(n, nullptr, width, stride, nullptr,
                                      nullptr, ci, v, b + col0, ldb, c + col0,
                                      ldc, alpha, beta, st);
            });
            B2S_LAUNCH_CHECK();
            col0 += kk;
            continue;
        }
        B2S_DISPATCH_K(kk, VEC, {
            if (vec) {
                ell_kernel<T, K, true><<<grid, kBlock, 0, st>>>(
                    n, width, stride, ci, v, b + col0, ldb, c + col0, ldc,
                    alpha, beta);
            } else {
                ell_kernel<T, K, false><<<grid, kBlock, 0, st>>>(
                    n, width, stride, ci, v, b + col0, ldb, c + col0, ldc,
                    alpha, beta);
            }
        });
        B2S_LAUNCH_CHECK();
        col0 += kk;
    }
    return B2S_OK;
}

template <typename T>
int sellp_spmv(int64_t n, int64_t num_cols, int64_t slice_size,
               const uint64_t* slice_sets, const uint64_t* slice_lengths,
               const int32_t* ci, const T* v, const T* b, int64_t ldb, T* c,
               int64_t ldc, int64_t k, const T* alpha, const T* beta,
               void* stream)
{
    B2S_CHECK_ARG(n >= 0 && k >= 0, "negative size");
    B2S_CHECK_ARG(slice_size >= 1 && slice_size <= (1 << 20),
                  "slice_size must be in 1..2^20");
    B2S_CHECK_ARG(n < (int64_t(1) << 31), "row count exceeds int32");
    B2S_CHECK_ARG((alpha == nullptr) == (beta == nullptr),
                  "alpha and beta must both be given or both be null");
    B2S_CHECK_ARG(k == 0 || (ldb >= k && ldc >= k), "leading dimension < k");
    if (n == 0 || k == 0) return B2S_OK;
    cudaStream_t st = as_stream(stream);
    const int64_t grid = ceildiv(n, kBlock);
    constexpr int R = int(16 / sizeof(T));
    if (k == 1 && slice_size % R == 0 && reinterpret_cast<uintptr_t>(ci) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(v) % 16 == 0) {
        // one right-hand side: R rows of a slice per thread, 16-byte loads
        int shift = -1;
        if ((slice_size & (slice_size - 1)) == 0) {
            shift = 0;
            while ((int64_t(1) << shift) < slice_size) ++shift;
        }
        // FP64 (2-row groups): a persistent grid, so most slice lookups
        // are prefetched; FP32 (4-row groups): one group per thread (each
        // measured faster on the 7-point matrix)
        const int64_t groups_blocks = ceildiv(ceildiv(n, R), kBlock);
        if constexpr (sizeof(T) == 8) {
            const int64_t g = std::min<int64_t>(groups_blocks, int64_t(num_sms()) * 16);
            if (alpha == nullptr && ldb == 1 && ldc == 1) {
                sellp_rows_kernel<T, R, true, true><<<g, kBlock, 0, st>>>(
                    int(n), int(slice_size), shift, slice_sets, slice_lengths, ci, v, b, ldb,
                    c, ldc, alpha, beta);
            } else {
                sellp_rows_kernel<T, R, true><<<g, kBlock, 0, st>>>(
                    int(n), int(slice_size), shift, slice_sets, slice_lengths, ci, v, b, ldb,
                    c, ldc, alpha, beta);
            }
        } else {
            sellp_rows_kernel<T, R, false><<<groups_blocks, kBlock, 0, st>>>(
                int(n), int(slice_size), shift, slice_sets, slice_lengths, ci, v, b, ldb, c,
                ldc, alpha, beta);
        }
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    }
    for (int64_t col0 = 0; col0 < k;) {
        const int kk = rhs_chunk(k - col0);
        const bool vec = vec_ok(b, ldb, col0, kk);
        if (lanes_ok(b, ldb, c, ldc, col0, kk)) {
            B2S_DISPATCH_K(kk, VEC, {
                launch_lanes<T, K, 2>(n, nullptr, slice_size, 0, slice_sets,
                                      slice_lengths, ci, v, b + col0, ldb,
                                      c + col0, ldc, alpha, beta, st);
            });
            B2S_LAUNCH_CHECK();
            col0 += kk;
            continue;
        }
        B2S_DISPATCH_K(kk, VEC, {
            if (vec) {
                sellp_kernel<T, K, true><<<grid, kBlock, 0, st>>>(
                    int(n), int(slice_size), slice_sets, slice_lengths, ci, v, b + col0,
                    ldb, c + col0, ldc, alpha, beta);
            } else {
                sellp_kernel<T, K, false><<<grid, kBlock, 0, st>>>(
                    int(n), int(slice_size), slice_sets, slice_lengths, ci, v, b + col0,
                    ldb, c + col0, ldc, alpha, beta);
            }
        });
        B2S_LAUNCH_CHECK();
        col0 += kk;
    }
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int64_t b2s_csr_load_balance_num_tiles(int64_t num_rows, int64_t nnz)
{
    if (num_rows <= 0) return 1;
    return ceildiv(num_rows + nnz, kTileItems);
}

int b2s_csr_load_balance_setup(int64_t num_rows, int64_t nnz,
                               const int32_t* row_ptrs, int64_t num_tiles,
                               int32_t* tile_rows, void* stream)
{
    B2S_CHECK_ARG(num_tiles == b2s_csr_load_balance_num_tiles(num_rows, nnz),
                  "num_tiles must come from b2s_csr_load_balance_num_tiles");
    B2S_CHECK_ARG(tile_rows != nullptr, "null tile_rows");
    if (num_rows <= 0) {
        B2S_CUDA_TRY(cudaMemsetAsync(tile_rows, 0, 2 * sizeof(int32_t),
                                     as_stream(stream)));
        return B2S_OK;
    }
    const int64_t threads = num_tiles + 1;
    csr_tile_rows_kernel<<<ceildiv(threads, 256), 256, 0, as_stream(stream)>>>(
        num_rows, row_ptrs, num_tiles, tile_rows);
    B2S_LAUNCH_CHECK();
    return B2S_OK;
}

#define B2S_SPMV_ENTRIES(T, S)                                                 \
    int b2s_csr_spmv_##S(int strategy, int64_t num_rows, int64_t num_cols,     \
                         const int32_t* row_ptrs, const int32_t* col_idxs,     \
                         const T* values, int64_t max_row_nnz,                 \
                         const int32_t* tile_rows, int64_t num_tiles,          \
                         const T* b, int64_t ldb, T* c, int64_t ldc,           \
                         int64_t num_rhs, const T* alpha, const T* beta,       \
                         void* stream)                                         \
    {                                                                          \
        return csr_spmv<T>(strategy, num_rows, num_cols, row_ptrs, col_idxs,   \
                           values, max_row_nnz, tile_rows, num_tiles, b, ldb,  \
                           c, ldc, num_rhs, alpha, beta, stream);              \
    }                                                                          \
    int b2s_ell_spmv_##S(int64_t num_rows, int64_t num_cols, int64_t width,    \
                         int64_t stride, const int32_t* col_idxs,              \
                         const T* values, const T* b, int64_t ldb, T* c,       \
                         int64_t ldc, int64_t num_rhs, const T* alpha,         \
                         const T* beta, void* stream)                          \
    {                                                                          \
        return ell_spmv<T>(num_rows, num_cols, width, stride, col_idxs,        \
                           values, b, ldb, c, ldc, num_rhs, alpha, beta,       \
                           stream);                                            \
    }                                                                          \
    int b2s_sellp_spmv_##S(int64_t num_rows, int64_t num_cols,                 \
                           int64_t slice_size, const uint64_t* slice_sets,     \
                           const uint64_t* slice_lengths,                      \
                           const int32_t* col_idxs, const T* values,           \
                           const T* b, int64_t ldb, T* c, int64_t ldc,         \
                           int64_t num_rhs, const T* alpha, const T* beta,     \
                           void* stream)                                       \
    {                                                                          \
        return sellp_spmv<T>(num_rows, num_cols, slice_size, slice_sets,       \
                             slice_lengths, col_idxs, values, b, ldb, c, ldc,  \
                             num_rhs, alpha, beta, stream);                    \
    }

B2S_SPMV_ENTRIES(double, f64)
B2S_SPMV_ENTRIES(float, f32)

}  // extern "C"
