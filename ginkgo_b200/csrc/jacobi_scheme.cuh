// The block-interleaved storage of block Jacobi inverses (the reference's
// block_interleaved_storage_scheme, include/ginkgo/core/preconditioner/
// jacobi.hpp:37-140, with the CUDA executor's block stride of 32): blocks
// form groups of gs = 32 / pow2ceil(max_bs); element (row, col) of block b
// sits at (b / gs) * group + (b % gs) * max_bs + row + col * stride, with
// stride = gs * max_bs and group = max_bs * stride.  Shared by the block
// Jacobi kernels and the solvers that apply the blocks inside their passes.
#pragma once

#include "common.cuh"

namespace b2s {

constexpr int kMaxBs = 32;

struct BlockScheme {
    int gs;          // blocks per group (a power of two)
    int power;       // log2(gs)
    int64_t stride;  // between the columns of a block
    int64_t group;   // between groups
};

inline __host__ __device__ BlockScheme block_scheme(int max_bs)
{
    int p2 = 1;
    while (p2 < max_bs) p2 *= 2;
    BlockScheme sc;
    sc.gs = kMaxBs / p2;
    sc.power = 0;
    while ((1 << sc.power) < sc.gs) ++sc.power;
    sc.stride = int64_t(sc.gs) * max_bs;
    sc.group = int64_t(max_bs) * sc.stride;
    return sc;
}

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

// A block Jacobi preconditioner as the solvers take it: num_blocks blocks
// delimited by ptrs (num_blocks + 1 entries), inverses in the interleaved
// storage above.
template <typename T>
struct BlockPrec {
    int64_t num_blocks = 0;
    const int32_t* ptrs = nullptr;
    int max_bs = 0;
    const T* blocks = nullptr;
};

}  // namespace b2s
