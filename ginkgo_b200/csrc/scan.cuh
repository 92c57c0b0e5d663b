// Device-wide exclusive scan of integer arrays in three deterministic
// phases (tile sums, one-block scan of the tile sums, apply), used by the
// format conversions and the sparse products.
#pragma once

#include "common.cuh"

namespace b2s {
namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;                   // per thread
constexpr int kScanTile = kScanBlock * kScanItems;  // per block

template <typename I>
__device__ I block_exclusive_scan(I v, I* sh, I* total)
{
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    I x = v;
#pragma unroll
    for (int off = 1; off < kWarp; off *= 2) {
        I y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == kWarp - 1) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        I w = lane < kScanBlock / kWarp ? sh[lane] : I(0);
#pragma unroll
        for (int off = 1; off < kWarp; off *= 2) {
            I y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        if (lane < kScanBlock / kWarp) sh[lane] = w;
    }
    __syncthreads();
    const I warp_off = wid > 0 ? sh[wid - 1] : I(0);
    if (total) *total = sh[kScanBlock / kWarp - 1];
    __syncthreads();
    return warp_off + x - v;
}

template <typename I>
__global__ void __launch_bounds__(kScanBlock)
    scan_tile_sums(const I* __restrict__ in, int64_t n, I* __restrict__ sums)
{
    __shared__ I sh[kScanBlock / kWarp];
    const int64_t base = blockIdx.x * int64_t(kScanTile) + threadIdx.x * kScanItems;
    I acc = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < n) acc += in[base + q];
    }
    I total;
    block_exclusive_scan(acc, sh, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename I>
__global__ void __launch_bounds__(kScanBlock)
    scan_single_block(I* __restrict__ data, int64_t n)
{
    // in-place exclusive scan of up to any n, one block, sequential tiles
    __shared__ I sh[kScanBlock / kWarp];
    I carry = 0;
    for (int64_t t0 = 0; t0 < n; t0 += kScanTile) {
        const int64_t base = t0 + threadIdx.x * kScanItems;
        I vals[kScanItems];
        I acc = 0;
#pragma unroll
        for (int q = 0; q < kScanItems; ++q) {
            vals[q] = base + q < n ? data[base + q] : I(0);
            acc += vals[q];
        }
        I total;
        I ex = block_exclusive_scan(acc, sh, &total) + carry;
#pragma unroll
        for (int q = 0; q < kScanItems; ++q) {
            if (base + q < n) data[base + q] = ex;
            ex += vals[q];
        }
        carry += total;
    }
}

template <typename I>
__global__ void __launch_bounds__(kScanBlock)
    scan_apply(const I* __restrict__ in, int64_t n, const I* __restrict__ sums,
               I* __restrict__ out)
{
    __shared__ I sh[kScanBlock / kWarp];
    const int64_t base = blockIdx.x * int64_t(kScanTile) + threadIdx.x * kScanItems;
    I vals[kScanItems];
    I acc = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        vals[q] = base + q < n ? in[base + q] : I(0);
        acc += vals[q];
    }
    I ex = block_exclusive_scan(acc, sh, (I*)nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < n) out[base + q] = ex;
        ex += vals[q];
    }
}

// out[i] = sum(in[0..i)) for i in [0, n]; out may alias in only if it has
// n + 1 entries and in[n] is ignored.  Workspace: ceil(n / kScanTile) + 1
// entries of I.
template <typename I>
int exclusive_scan(const I* in, int64_t n, I* out, I* work, cudaStream_t st)
{
    const int64_t tiles = ceildiv(n, kScanTile);
    if (n > 0) {
        scan_tile_sums<I><<<tiles, kScanBlock, 0, st>>>(in, n, work);
        B2S_LAUNCH_CHECK();
    }
    // work[tiles] collects the grand total through the one-block scan
    B2S_CUDA_TRY(cudaMemsetAsync(work + tiles, 0, sizeof(I), st));
    scan_single_block<I><<<1, kScanBlock, 0, st>>>(work, tiles + 1);
    B2S_LAUNCH_CHECK();
    if (n > 0) {
        scan_apply<I><<<tiles, kScanBlock, 0, st>>>(in, n, work, out);
        B2S_LAUNCH_CHECK();
    }
    B2S_CUDA_TRY(cudaMemcpyAsync(out + n, work + tiles, sizeof(I),
                                 cudaMemcpyDeviceToDevice, st));
    return B2S_OK;
}

template <typename I>
int64_t scan_work_entries(int64_t n)
{
    return ceildiv(n, kScanTile) + 1;
}

}  // namespace
}  // namespace b2s
