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
#include "rhs_lanes.cuh"
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
// Csr load_balance: the stored entries are cut into chunks of kLbChunk
// consecutive entries (nnz-balanced, whatever the row lengths), one warp per
// chunk, persistent over the chunks.  A warp stages its chunk's values and
// column indices in shared memory with coalesced loads and sums the rows it
// owns, the rows whose last entry lies in the chunk (an empty row belongs to
// the chunk holding its position): a lane per row for short segments, the
// whole warp for a segment of more than 32 entries.  The part of a row that
// lies in earlier chunks arrives through those chunks' tail partials: a
// chunk whose last entry's row continues past it sums that row's entries in
// the chunk into its partial slot, and a fix-up pass adds every run of
// partials to its row (alpha times their sum, in chunk order).  No atomics;
// the result does not depend on scheduling.
//
// The partition buffer (built once per matrix on the GPU, the role of
// srow): own_first[nc + 1] (the first row each chunk owns), tail_row[nc],
// and nc slots of 16 partial sums (the scratch of the fix-up, rewritten by
// every SpMV: SpMVs of one matrix that overlap on the GPU race on it).
// ---------------------------------------------------------------------------
constexpr int kLbChunk = 256;  // entries per chunk
constexpr int kLbSlot = 16;    // partial sums per chunk (right-hand sides)

inline int64_t lb_chunks(int64_t nnz) { return std::max<int64_t>(1, ceildiv(nnz, kLbChunk)); }
// int32 words of the partition buffer of nc chunks: own_first, tail_row, an
// 8-byte aligned block of nc * 16 doubles
inline int64_t lb_words(int64_t nc) { return 34 * nc + 4; }
inline int64_t lb_chunks_of_words(int64_t words) { return (words - 4) / 34; }
inline int64_t lb_partials_offset(int64_t nc) { return (2 * nc + 1 + 1) / 2 * 2; }

// The chunk that owns row r: that of its last entry, or (empty row) that of
// its position, clamped to the last chunk.
__device__ __forceinline__ int64_t lb_owner(const int32_t* __restrict__ rp, int64_t r,
                                            int64_t nc)
{
    const int64_t s = __ldg(rp + r), e = __ldg(rp + r + 1);
    const int64_t q = e > s ? e - 1 : min(s, nc * kLbChunk - 1);
    return q / kLbChunk;
}

// own_first[c]: the first row whose owner is c or later (n for c = nc).
__global__ void csr_lb_setup_kernel(int64_t n, const int32_t* __restrict__ rp, int64_t nc,
                                    int32_t* __restrict__ own_first)
{
    const int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (c > nc) return;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (lb_owner(rp, mid, nc) >= c) {
            hi = mid;
        } else {
            lo = mid + 1;
        }
    }
    own_first[c] = int32_t(c == nc ? n : lo);
}

// K sums of the staged chunk entries [s, e) (offsets into the chunk's stage
// sv/sc), taking every step-th entry from s + first.
template <typename T, int K, bool VEC>
__device__ __forceinline__ void lb_row_sum(const T* sv, const int32_t* sc, int s, int e,
                                           int step, int first, const T* __restrict__ b,
                                           int64_t ldb, T (&acc)[K])
{
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    // unrolled so that several gathers of b are in flight per lane
#pragma unroll 4
    for (int i = s + first; i < e; i += step) {
        const T val = sv[i];
        T xr[K];
        RowLoad<T, K, VEC>::load(b + int64_t(sc[i]) * ldb, xr);
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] += val * xr[j];
    }
}

// lane j < K receives the warp total of acc[j]
template <typename T, int K>
__device__ __forceinline__ T lb_warp_totals(T (&acc)[K], int lane)
{
    T a = T(0);
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const T t = warp_sum(acc[j]);
        if (lane == j) a = t;
    }
    return a;
}

// A row of more than 32 entries in the chunk, summed by the whole warp.  Kept
// out of line: rows this long are rare, and inlined the loop costs the
// lane-per-row path registers.
template <typename T, int K, bool VEC>
__device__ __noinline__ void lb_long_row(const T* sv, const int32_t* sc, int s, int e, int lane,
                                         const T* __restrict__ b, int64_t ldb, T* dst,
                                         const T* __restrict__ alpha, const T* __restrict__ beta)
{
    T acc[K];
    lb_row_sum<T, K, VEC>(sv, sc, s, e, kWarp, lane, b, ldb, acc);
    const T a = lb_warp_totals<T, K>(acc, lane);
    if (lane < K) dst[lane] = combine(a, alpha, beta, dst + lane);
}

// (holding one right-hand side to six blocks per SM, 40 registers, measured
// 4 % slower on the 7-point 128^3 matrix and 22 % slower on the power-law
// matrix than the unconstrained 48 registers and five blocks)
template <typename T, int K, bool VEC>
__global__ void __launch_bounds__(kBlock)
    csr_lb_kernel(int64_t n, int64_t nc, const int32_t* __restrict__ own_first,
                  int32_t* __restrict__ tail_row, T* __restrict__ partials,
                  const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                  const T* __restrict__ v, const T* __restrict__ b, int64_t ldb,
                  T* __restrict__ c, int64_t ldc, const T* __restrict__ alpha,
                  const T* __restrict__ beta)
{
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ T sv_all[kBlock / kWarp][kLbChunk];
    __shared__ int32_t sc_all[kBlock / kWarp][kLbChunk];
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    T* sv = sv_all[wid];
    int32_t* sc = sc_all[wid];
    const int64_t nwarps = int64_t(gridDim.x) * (kBlock / kWarp);
    const int64_t nnz = __ldg(rp + n);
    for (int64_t ch = blockIdx.x * int64_t(kBlock / kWarp) + wid; ch < nc; ch += nwarps) {
        const int64_t e0 = ch * kLbChunk;
        const int len = int(min(int64_t(kLbChunk), nnz - e0));  // entries in the chunk
        for (int i = lane; i < len; i += kWarp) {
            sv[i] = ld_stream(v + e0 + i);
            sc[i] = ld_stream(ci + e0 + i);
        }
        __syncwarp();
        const int r0 = own_first[ch], r1 = own_first[ch + 1];
        // owned rows, 32 at a time (warp-uniform trip count); entry offsets
        // are relative to the chunk: an owned row ends inside it and may
        // start before it
        for (int rb = r0; rb < r1; rb += kWarp) {
            const int r = rb + lane;
            const bool valid = r < r1;
            const int s = valid ? int(max(int64_t(__ldg(rp + r)) - e0, int64_t(0))) : 0;
            const int e = valid ? int(int64_t(__ldg(rp + r + 1)) - e0) : 0;
            const bool longseg = e - s > kWarp;
            if (valid && !longseg) {
                T acc[K];
                lb_row_sum<T, K, VEC>(sv, sc, s, e, 1, 0, b, ldb, acc);
                T* dst = c + int64_t(r) * ldc;
#pragma unroll
                for (int j = 0; j < K; ++j) dst[j] = combine(acc[j], alpha, beta, dst + j);
            }
            unsigned mask = __ballot_sync(kFull, longseg);
            while (mask) {
                const int bit = __ffs(mask) - 1;
                mask &= mask - 1;
                const int rl = __shfl_sync(kFull, r, bit);
                const int sl = __shfl_sync(kFull, s, bit);
                const int el = __shfl_sync(kFull, e, bit);
                lb_long_row<T, K, VEC>(sv, sc, sl, el, lane, b, ldb, c + int64_t(rl) * ldc,
                                       alpha, beta);
            }
        }
        // the row that continues past the chunk: its part here, as a partial
        const int rt = r1;
        const int64_t st = rt < n ? int64_t(__ldg(rp + rt)) : nnz;
        const bool tail = st < e0 + len;
        if (tail) {
            T acc[K];
            lb_row_sum<T, K, VEC>(sv, sc, int(max(st - e0, int64_t(0))), len, kWarp, lane, b,
                                  ldb, acc);
            const T a = lb_warp_totals<T, K>(acc, lane);
            if (lane < K) partials[ch * kLbSlot + lane] = a;
        }
        if (lane == 0) tail_row[ch] = tail ? rt : -1;
        __syncwarp();  // the stage is refilled for the next chunk
    }
}

// load_balance with one right-hand side, products first: each lane loads
// entries lane, lane + 32, ... of the chunk and gathers b at their columns,
// so all of the chunk's gathers are in flight at once (a lane-per-row loop
// over rows of ~20 entries waits for one gather round per four entries);
// the products go to shared memory and the owned rows are summed from there
// (a lane per row in entry order, which rounds as the reference executor's
// row loop; the whole warp for a row of more than 32 entries in the chunk),
// with the same ownership, tail partials and fix-up as csr_lb_kernel.
constexpr int kLbPerLane = kLbChunk / kWarp;

template <typename T>
__global__ void __launch_bounds__(kBlock, 5)
    csr_lb1_kernel(int64_t n, int64_t nc, const int32_t* __restrict__ own_first,
                   int32_t* __restrict__ tail_row, T* __restrict__ partials,
                   const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                   const T* __restrict__ v, const T* __restrict__ b, int64_t ldb,
                   T* __restrict__ c, int64_t ldc, const T* __restrict__ alpha,
                   const T* __restrict__ beta)
{
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ T sp_all[kBlock / kWarp][kLbChunk];
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    T* sp = sp_all[wid];
    const int64_t nwarps = int64_t(gridDim.x) * (kBlock / kWarp);
    const int64_t nnz = __ldg(rp + n);
    for (int64_t ch = blockIdx.x * int64_t(kBlock / kWarp) + wid; ch < nc; ch += nwarps) {
        const int64_t e0 = ch * kLbChunk;
        const int len = int(min(int64_t(kLbChunk), nnz - e0));  // entries in the chunk
        // the owned rows and the first 32 rows' extents are loaded alongside
        // the entries and the gathers, not after them
        const int r0 = __ldg(own_first + ch), r1 = __ldg(own_first + ch + 1);
        T pv[kLbPerLane];
        int32_t pc[kLbPerLane];
#pragma unroll
        for (int j = 0; j < kLbPerLane; ++j) {
            const int i = lane + j * kWarp;
            pc[j] = i < len ? ld_stream(ci + e0 + i) : 0;
            pv[j] = i < len ? ld_stream(v + e0 + i) : T(0);
        }
        const int rf = r0 + lane;
        const int64_t rs0 = rf < r1 ? int64_t(__ldg(rp + rf)) : 0;
        const int64_t re0 = rf < r1 ? int64_t(__ldg(rp + rf + 1)) : 0;
        const int64_t st = r1 < n ? int64_t(__ldg(rp + r1)) : nnz;
#pragma unroll
        for (int j = 0; j < kLbPerLane; ++j) {
            if (lane + j * kWarp < len) pv[j] = pv[j] * __ldg(b + int64_t(pc[j]) * ldb);
        }
#pragma unroll
        for (int j = 0; j < kLbPerLane; ++j) sp[lane + j * kWarp] = pv[j];
        __syncwarp();
        for (int rb = r0; rb < r1; rb += kWarp) {
            const int r = rb + lane;
            const bool valid = r < r1;
            int64_t rs = rs0, re = re0;
            if (rb != r0) {
                rs = valid ? int64_t(__ldg(rp + r)) : 0;
                re = valid ? int64_t(__ldg(rp + r + 1)) : 0;
            }
            const int s = valid ? int(max(rs - e0, int64_t(0))) : 0;
            const int e = valid ? int(re - e0) : 0;
            const bool longseg = e - s > kWarp;
            if (valid && !longseg) {
                T acc = T(0);
                for (int i = s; i < e; ++i) acc += sp[i];
                T* dst = c + int64_t(r) * ldc;
                *dst = combine(acc, alpha, beta, dst);
            }
            unsigned mask = __ballot_sync(kFull, longseg);
            while (mask) {
                const int bit = __ffs(mask) - 1;
                mask &= mask - 1;
                const int rl = __shfl_sync(kFull, r, bit);
                const int sl = __shfl_sync(kFull, s, bit);
                const int el = __shfl_sync(kFull, e, bit);
                T acc = T(0);
                for (int i = sl + lane; i < el; i += kWarp) acc += sp[i];
                acc = warp_sum(acc);
                if (lane == 0) {
                    T* dst = c + int64_t(rl) * ldc;
                    *dst = combine(acc, alpha, beta, dst);
                }
            }
        }
        // the row that continues past the chunk: its part here, as a partial
        const int rt = r1;
        const bool tail = st < e0 + len;
        if (tail) {
            T acc = T(0);
            for (int i = int(max(st - e0, int64_t(0))) + lane; i < len; i += kWarp) acc += sp[i];
            acc = warp_sum(acc);
            if (lane == 0) partials[ch * kLbSlot] = acc;
        }
        if (lane == 0) tail_row[ch] = tail ? rt : -1;
        __syncwarp();  // the products are rewritten for the next chunk
    }
}

// Adds each run of tail partials to its row: c(r, :) += alpha * sum.
template <typename T, int K>
__global__ void csr_lb_fixup_kernel(int64_t nc, const int32_t* __restrict__ tail_row,
                                    const T* __restrict__ partials, T* __restrict__ c,
                                    int64_t ldc, const T* __restrict__ alpha)
{
    const int64_t ch = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (ch >= nc) return;
    const int32_t r = tail_row[ch];
    if (r < 0 || (ch > 0 && tail_row[ch - 1] == r)) return;  // not a run start
    T acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    for (int64_t q = ch; q < nc && tail_row[q] == r; ++q) {
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] += partials[q * kLbSlot + j];
    }
    const T a = alpha ? *alpha : T(1);
    T* dst = c + int64_t(r) * ldc;
#pragma unroll
    for (int j = 0; j < K; ++j) dst[j] += a * acc[j];
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
// Csr load_balance with K >= 4 right-hand sides in 16-byte aligned rows: the
// chunk partition and partial sums of csr_lb_kernel, with KL = K / VW lanes
// per row each owning one 16-byte column slice (as rhs_lanes_kernel), so
// 32 / KL rows of a chunk run at a time.  A row with more than 2 * 32 / KL
// entries in the chunk, and the row that continues past it, are summed by
// all 32 / KL row slots together (entries strided by the slot count, then
// a shuffle reduction over the slots).
// ---------------------------------------------------------------------------
template <typename T, int K>
__device__ __forceinline__ void lb_slice_sum(const T* sv, const int32_t* sc, int s, int e,
                                             int step, int first, const T* __restrict__ bc,
                                             int64_t ldb, typename Vec16<T>::type& acc)
{
#pragma unroll 4
    for (int i = s + first; i < e; i += step) fma_vec<T>(acc, sv[i], bc + int64_t(sc[i]) * ldb);
}

template <typename T, int KL>
__device__ __forceinline__ void lb_slot_reduce(typename Vec16<T>::type& acc)
{
    T* a = reinterpret_cast<T*>(&acc);
#pragma unroll
    for (int off = KL; off < kWarp; off *= 2) {
#pragma unroll
        for (int u = 0; u < Vec16<T>::width; ++u) {
            a[u] += __shfl_xor_sync(0xffffffffu, a[u], off);
        }
    }
}

template <typename T>
__device__ __forceinline__ void vec_zero(typename Vec16<T>::type& acc)
{
    T* a = reinterpret_cast<T*>(&acc);
#pragma unroll
    for (int u = 0; u < Vec16<T>::width; ++u) a[u] = T(0);
}

template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    csr_lb_lanes_kernel(int64_t n, int64_t nc, const int32_t* __restrict__ own_first,
                        int32_t* __restrict__ tail_row, T* __restrict__ partials,
                        const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                        const T* __restrict__ v, const T* __restrict__ b, int64_t ldb,
                        T* __restrict__ c, int64_t ldc, const T* __restrict__ alpha,
                        const T* __restrict__ beta)
{
    using V = typename Vec16<T>::type;
    constexpr int VW = Vec16<T>::width;
    constexpr int KL = K / VW;     // lanes per row
    constexpr int R = kWarp / KL;  // rows at a time
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ T sv_all[kBlock / kWarp][kLbChunk];
    __shared__ int32_t sc_all[kBlock / kWarp][kLbChunk];
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const int part = lane % KL, slot = lane / KL;
    T* sv = sv_all[wid];
    int32_t* sc = sc_all[wid];
    const T* bc = b + part * VW;
    const int64_t nwarps = int64_t(gridDim.x) * (kBlock / kWarp);
    const int64_t nnz = __ldg(rp + n);
    for (int64_t ch = blockIdx.x * int64_t(kBlock / kWarp) + wid; ch < nc; ch += nwarps) {
        const int64_t e0 = ch * kLbChunk;
        const int len = int(min(int64_t(kLbChunk), nnz - e0));
        for (int i = lane; i < len; i += kWarp) {
            sv[i] = ld_stream(v + e0 + i);
            sc[i] = ld_stream(ci + e0 + i);
        }
        __syncwarp();
        const int r0 = own_first[ch], r1 = own_first[ch + 1];
        for (int rb = r0; rb < r1; rb += R) {  // warp-uniform trip count
            const int r = rb + slot;
            const bool valid = r < r1;
            const int s = valid ? int(max(int64_t(__ldg(rp + r)) - e0, int64_t(0))) : 0;
            const int e = valid ? int(int64_t(__ldg(rp + r + 1)) - e0) : 0;
            const bool longseg = e - s > 2 * R;
            if (valid && !longseg) {
                V acc;
                vec_zero<T>(acc);
                lb_slice_sum<T, K>(sv, sc, s, e, 1, 0, bc, ldb, acc);
                store_vec<T>(c + int64_t(r) * ldc + part * VW, acc, alpha, beta);
            }
            unsigned mask = __ballot_sync(kFull, longseg && part == 0);
            while (mask) {
                const int bit = __ffs(mask) - 1;
                mask &= mask - 1;
                const int rl = __shfl_sync(kFull, r, bit);
                const int sl = __shfl_sync(kFull, s, bit);
                const int el = __shfl_sync(kFull, e, bit);
                V acc;
                vec_zero<T>(acc);
                lb_slice_sum<T, K>(sv, sc, sl, el, R, slot, bc, ldb, acc);
                lb_slot_reduce<T, KL>(acc);
                if (slot == 0) store_vec<T>(c + int64_t(rl) * ldc + part * VW, acc, alpha, beta);
            }
        }
        // the row that continues past the chunk: its part here, as a partial
        const int rt = r1;
        const int64_t st = rt < n ? int64_t(__ldg(rp + rt)) : nnz;
        const bool tail = st < e0 + len;
        if (tail) {
            V acc;
            vec_zero<T>(acc);
            lb_slice_sum<T, K>(sv, sc, int(max(st - e0, int64_t(0))), len, R, slot, bc, ldb, acc);
            lb_slot_reduce<T, KL>(acc);
            if (slot == 0) {
                const T* a = reinterpret_cast<const T*>(&acc);
#pragma unroll
                for (int u = 0; u < VW; ++u) partials[ch * kLbSlot + part * VW + u] = a[u];
            }
        }
        if (lane == 0) tail_row[ch] = tail ? rt : -1;
        __syncwarp();  // the stage is refilled for the next chunk
    }
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

// Longest Sellp slice (entries per row) for which rows are paired per lane
// slot with four or more right-hand sides.
constexpr int64_t kPairMaxSlice = 64;

template <typename T, int K, int FMT>
void launch_lanes(int64_t n, const int32_t* rp, int64_t w_or_s, int64_t stride,
                  const uint64_t* sets, const uint64_t* lens, const int32_t* ci,
                  const T* v, const T* b, int64_t ldb, T* c, int64_t ldc,
                  const T* alpha, const T* beta, cudaStream_t st,
                  int64_t max_slice_len = 0)
{
    if constexpr (K >= 4 && K % Vec16<T>::width == 0) {
        constexpr int KL = K / Vec16<T>::width;
        // Ell: row pairs per lane slot when the column-major layout keeps
        // rows r, r + 1 adjacent at 8-byte alignment (0.84-0.90 of the
        // single-row time at 4 and 16 columns on the 7-point 128^3 matrix).
        // Sellp pairs its rows only when the caller gives the longest slice
        // and it is short: on the power-law matrix its longest slices (1,805
        // entries) doubled the per-thread chain and took 1.3 to 2.4 times as
        // long with pairs.
        const bool aligned = reinterpret_cast<uintptr_t>(ci) % 8 == 0 &&
                             reinterpret_cast<uintptr_t>(v) % (2 * sizeof(T)) == 0;
        // (Sellp FP32 with four columns measured 9 % slower with pairs, so
        // FP32 pairs need eight or more)
        const bool pairs = aligned && ((FMT == 1 && stride % 2 == 0) ||
                                       (FMT == 2 && w_or_s % 2 == 0 && max_slice_len > 0 &&
                                        max_slice_len <= kPairMaxSlice &&
                                        (sizeof(T) == 8 || K >= 8)));
        if (FMT != 0 && pairs) {
            if constexpr (FMT != 0) {
                rhs_lanes2_kernel<T, K, FMT><<<ceildiv(ceildiv(n, 2) * KL, kBlock), kBlock, 0,
                                               st>>>(n, w_or_s, stride, sets, lens, ci, v, b,
                                                     ldb, c, ldc, alpha, beta);
            }
            return;
        }
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
        B2S_CHECK_ARG(tile_rows != nullptr && num_tiles >= 37 && (num_tiles - 3) % 34 == 0,
                      "load_balance needs the partition from b2s_csr_load_balance_setup");
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
            const int64_t nc = lb_chunks_of_words(num_tiles + 1);
            int32_t* own_first = const_cast<int32_t*>(tile_rows);
            int32_t* tail_row = own_first + nc + 1;
            T* partials = reinterpret_cast<T*>(own_first + lb_partials_offset(nc));
            const int64_t grid = std::min<int64_t>(ceildiv(nc, kBlock / kWarp),
                                                   int64_t(num_sms()) * 8);
            const bool lanes = lanes_ok(b, ldb, c, ldc, col0, kk);
            // lanes_ok implies K >= 4 and K a multiple of the vector width
            B2S_DISPATCH_K(kk, VEC, {
                bool launched = false;
                if constexpr (K >= 4 && K % Vec16<T>::width == 0) {
                    if (lanes) {
                        auto kernel = csr_lb_lanes_kernel<T, K>;
                        kernel<<<resident_grid(kernel, kBlock, grid), kBlock, 0, st>>>(
                            n, nc, own_first, tail_row, partials, rp, ci, v, bb, ldb, cc, ldc,
                            alpha, beta);
                        launched = true;
                    }
                }
                if constexpr (K == 1) {
                    auto kernel = csr_lb1_kernel<T>;
                    kernel<<<resident_grid(kernel, kBlock, grid), kBlock, 0, st>>>(
                        n, nc, own_first, tail_row, partials, rp, ci, v, bb, ldb, cc, ldc,
                        alpha, beta);
                    launched = true;
                }
                if (launched) {
                    // the column-slice or one-column form above
                } else if (vec) {
                    auto kernel = csr_lb_kernel<T, K, true>;
                    kernel<<<resident_grid(kernel, kBlock, grid), kBlock, 0, st>>>(
                        n, nc, own_first, tail_row, partials, rp, ci, v, bb, ldb, cc, ldc,
                        alpha, beta);
                } else {
                    auto kernel = csr_lb_kernel<T, K, false>;
                    kernel<<<resident_grid(kernel, kBlock, grid), kBlock, 0, st>>>(
                        n, nc, own_first, tail_row, partials, rp, ci, v, bb, ldb, cc, ldc,
                        alpha, beta);
                }
                B2S_LAUNCH_CHECK();
                csr_lb_fixup_kernel<T, K><<<ceildiv(nc, 256), 256, 0, st>>>(
                    nc, tail_row, partials, cc, ldc, alpha);
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
               void* stream, int64_t max_slice_len = 0)
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
                                      c + col0, ldc, alpha, beta, st, max_slice_len);
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
    if (num_rows < 0 || nnz < 0) return -1;
    return lb_words(lb_chunks(nnz)) - 1;
}

int b2s_csr_load_balance_setup(int64_t num_rows, int64_t nnz,
                               const int32_t* row_ptrs, int64_t num_tiles,
                               int32_t* tile_rows, void* stream)
{
    B2S_CHECK_ARG(num_rows >= 0 && nnz >= 0, "negative size");
    B2S_CHECK_ARG(num_tiles == b2s_csr_load_balance_num_tiles(num_rows, nnz),
                  "num_tiles must come from b2s_csr_load_balance_num_tiles");
    B2S_CHECK_ARG(tile_rows != nullptr && (num_rows == 0 || row_ptrs != nullptr),
                  "null pointer");
    const int64_t nc = lb_chunks(nnz);
    csr_lb_setup_kernel<<<ceildiv(nc + 1, 256), 256, 0, as_stream(stream)>>>(
        num_rows, row_ptrs, nc, tile_rows);
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
    }                                                                          \
    int b2s_sellp_spmv_hinted_##S(int64_t num_rows, int64_t num_cols,          \
                                  int64_t slice_size, const uint64_t* slice_sets, \
                                  const uint64_t* slice_lengths,               \
                                  const int32_t* col_idxs, const T* values,    \
                                  const T* b, int64_t ldb, T* c, int64_t ldc,  \
                                  int64_t num_rhs, const T* alpha,             \
                                  const T* beta, int64_t max_slice_length,     \
                                  void* stream)                                \
    {                                                                          \
        B2S_CHECK_ARG(max_slice_length >= 0, "negative max_slice_length");     \
        return sellp_spmv<T>(num_rows, num_cols, slice_size, slice_sets,       \
                             slice_lengths, col_idxs, values, b, ldb, c, ldc,  \
                             num_rhs, alpha, beta, stream, max_slice_length);  \
    }

B2S_SPMV_ENTRIES(double, f64)
B2S_SPMV_ENTRIES(float, f32)

}  // extern "C"
