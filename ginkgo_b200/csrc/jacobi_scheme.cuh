// The block-interleaved storage of block Jacobi inverses (the reference's
// block_interleaved_storage_scheme, include/ginkgo/core/preconditioner/
// jacobi.hpp:37-140, with the CUDA executor's block stride of 32): blocks
// form groups of gs = 32 / pow2ceil(max_bs); element (row, col) of block b
// sits at (b / gs) * group + (b % gs) * max_bs + row + col * stride, with
// stride = gs * max_bs and group = max_bs * stride.  Shared by the block
// Jacobi kernels and the solvers that apply the blocks inside their passes.
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

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
    const uint8_t* prec = nullptr;  // per-block storage precisions, or null: full
    int kind = -1;  // with prec: the storage kind all groups share, or -1 (mixed)
};

// Adaptive precision.  A block's storage precision is precision_reduction's
// byte (preserving << 4) | non-preserving (include/ginkgo/core/base/types.hpp,
// precision_reduction), 0xff asking for autodetection.  The blocks of one
// group share a precision; a reduced group holds its values as an array of
// the storage type with the same interleaved indexing, from the start of the
// group's slot (the reference's reinterpret_cast<resolved_precision*>(blocks
// + group_offset) + block_offset, reference/preconditioner/
// jacobi_kernels.cpp:380-395).
constexpr uint8_t kP00 = 0x00, kP01 = 0x01, kP02 = 0x02, kP10 = 0x10, kP11 = 0x11,
                  kP20 = 0x20, kAutodetect = 0xff;
// precision_reduction_descriptor bits (core/preconditioner/jacobi_utils.hpp)
constexpr uint32_t kD02 = 0x01, kD11 = 0x02, kD20 = 0x04, kD01 = 0x08, kD10 = 0x10;

// Storage types: the value type, FP32, FP16 (gko::half), and the top 32 or
// 16 bits of an FP64 value or the top 16 bits of an FP32 value
// (truncated<T, N>).
enum StorageKind { kFull, kF32, kF16, kHi32, kHi16F32, kHi16F64 };

// GKO_PRECONDITIONER_JACOBI_RESOLVE_PRECISION (core/preconditioner/
// jacobi_utils.hpp): reduce_precision<double> = float, of float = half, of
// half = half; truncate_type<double> = truncated<double, 2>, of float =
// truncated<float, 2>.  Encodings outside the six store at full precision.
template <typename T>
__host__ __device__ inline int storage_kind(uint8_t p)
{
    if (sizeof(T) == 8) {
        switch (p) {
        case kP01: return kF32;
        case kP02: return kF16;
        case kP10: return kHi32;
        case kP11: return kHi16F32;
        case kP20: return kHi16F64;
        default: return kFull;
        }
    }
    switch (p) {
    case kP01:
    case kP02:
    case kP11: return kF16;
    case kP10:
    case kP20: return kHi16F32;
    default: return kFull;
    }
}

// FP32 to gko::half: round to nearest even, magnitudes below the smallest
// normal half (2^-14) flushed to a zero of the same sign.
__device__ __forceinline__ uint16_t half_bits(float f)
{
    if (fabsf(f) < 6.103515625e-05f) return (__float_as_uint(f) >> 16) & 0x8000u;
    return __half_as_ushort(__float2half_rn(f));
}

// Element idx of a storage array of kind K starting at base.
template <int K, typename T>
__device__ __forceinline__ void store_reduced(void* base, int64_t idx, T v)
{
    if constexpr (K == kFull) {
        static_cast<T*>(base)[idx] = v;
    } else if constexpr (K == kF32) {
        static_cast<float*>(base)[idx] = float(v);
    } else if constexpr (K == kF16) {
        static_cast<uint16_t*>(base)[idx] = half_bits(float(v));
    } else if constexpr (K == kHi32) {
        static_cast<uint32_t*>(base)[idx] =
            uint32_t(uint64_t(__double_as_longlong(double(v))) >> 32);
    } else if constexpr (K == kHi16F32) {
        static_cast<uint16_t*>(base)[idx] = uint16_t(__float_as_uint(float(v)) >> 16);
    } else {
        static_cast<uint16_t*>(base)[idx] =
            uint16_t(uint64_t(__double_as_longlong(double(v))) >> 48);
    }
}

// The word one stored value of kind K occupies, and its value widened to T.
template <int K, typename T>
struct StorageWord {
    using type = T;
};
template <typename T>
struct StorageWord<kF32, T> {
    using type = float;
};
template <typename T>
struct StorageWord<kF16, T> {
    using type = uint16_t;
};
template <typename T>
struct StorageWord<kHi32, T> {
    using type = uint32_t;
};
template <typename T>
struct StorageWord<kHi16F32, T> {
    using type = uint16_t;
};
template <typename T>
struct StorageWord<kHi16F64, T> {
    using type = uint16_t;
};

template <int K, typename T>
__device__ __forceinline__ T widen(typename StorageWord<K, T>::type w)
{
    if constexpr (K == kFull) {
        return w;
    } else if constexpr (K == kF32) {
        return T(w);
    } else if constexpr (K == kF16) {
        return T(__half2float(__ushort_as_half(w)));
    } else if constexpr (K == kHi32) {
        return T(__longlong_as_double((long long)(uint64_t(w) << 32)));
    } else if constexpr (K == kHi16F32) {
        return T(__uint_as_float(uint32_t(w) << 16));
    } else {
        return T(__longlong_as_double((long long)(uint64_t(w) << 48)));
    }
}

template <int K, typename T>
__device__ __forceinline__ T load_reduced(const void* base, int64_t idx)
{
    using W = typename StorageWord<K, T>::type;
    return widen<K, T>(__ldg(static_cast<const W*>(base) + idx));
}

// A value rounded to storage kind K and read back.
template <int K, typename T>
__device__ __forceinline__ T roundtrip(T v)
{
    if constexpr (K == kFull) {
        return v;
    } else if constexpr (K == kF32) {
        return T(float(v));
    } else if constexpr (K == kF16) {
        return T(__half2float(__ushort_as_half(half_bits(float(v)))));
    } else if constexpr (K == kHi32) {
        return T(__longlong_as_double(__double_as_longlong(double(v)) &
                                      (long long)0xffffffff00000000ull));
    } else if constexpr (K == kHi16F32) {
        return T(__uint_as_float(__float_as_uint(float(v)) & 0xffff0000u));
    } else {
        return T(__longlong_as_double(__double_as_longlong(double(v)) &
                                      (long long)0xffff000000000000ull));
    }
}

// Runs f(std::integral_constant<int, K>{}) for the storage kind k.
template <typename F>
__device__ __forceinline__ void with_storage_kind(int k, F&& f)
{
    switch (k) {
    case kF32: f(std::integral_constant<int, kF32>{}); break;
    case kF16: f(std::integral_constant<int, kF16>{}); break;
    case kHi32: f(std::integral_constant<int, kHi32>{}); break;
    case kHi16F32: f(std::integral_constant<int, kHi16F32>{}); break;
    case kHi16F64: f(std::integral_constant<int, kHi16F64>{}); break;
    default: f(std::integral_constant<int, kFull>{}); break;
    }
}

// inv[c] = element lane + c * stride of the storage array of kind K at base,
// widened to T (zero past max_bs or outside the group): every word is loaded
// before the first is widened, so the loads are in flight together.
template <int K, int MB2, typename T>
__device__ __forceinline__ void load_widened(const void* base, int lane, int64_t stride,
                                             bool in_group, int max_bs, T (&inv)[MB2])
{
    using W = typename StorageWord<K, T>::type;
    const W* g = static_cast<const W*>(base) + lane;
    W w[MB2];
#pragma unroll
    for (int c = 0; c < MB2; ++c) w[c] = in_group && c < max_bs ? __ldg(g + c * stride) : W(0);
#pragma unroll
    for (int c = 0; c < MB2; ++c) inv[c] = widen<K, T>(w[c]);
}

// How a block pass reads the blocks (a template parameter of the passes, so
// the full-precision instances keep their register counts): kSkFull without
// precisions, kSkMixed with a switch on each group's storage, or one
// StorageKind every group shares.
constexpr int kSkFull = -2, kSkMixed = -1;

// inv[c] = column c (< max_bs) of the row this lane holds in group grp of
// bp's blocks, widened to T; zero for lanes outside the group and columns
// past max_bs.
template <int SK, int MB2, typename T>
__device__ __forceinline__ void load_block_columns(const BlockPrec<T>& bp,
                                                   const BlockScheme& bsc, int64_t grp,
                                                   int lane, bool in_group, T (&inv)[MB2])
{
    const T* gb = bp.blocks + grp * bsc.group;
    auto load = [&](auto kc) {
        constexpr int K = decltype(kc)::value;
#pragma unroll
        for (int c = 0; c < MB2; ++c) {
            inv[c] = in_group && c < bp.max_bs ? load_reduced<K, T>(gb, lane + c * bsc.stride)
                                               : T(0);
        }
    };
    if constexpr (SK == kSkMixed) {
        with_storage_kind(storage_kind<T>(bp.prec[grp * bsc.gs]), load);
    } else if constexpr (SK == kSkFull) {
        load(std::integral_constant<int, kFull>{});
    } else {
        load(std::integral_constant<int, SK>{});
    }
}

// The row of a block group that one lane holds (as load_block_columns), kept
// as stored words for a fixed storage kind and widened where each column is
// used, so that all of the row's loads are in flight before the first
// conversion waits for one.
template <int SK, int MB2, typename T>
struct BlockRow {
    using Word = typename StorageWord<(SK >= 0 ? SK : int(kFull)), T>::type;
    Word w[MB2];

    __device__ __forceinline__ void load(const BlockPrec<T>& bp, const BlockScheme& bsc,
                                         int64_t grp, int lane, bool in_group)
    {
        if constexpr (SK >= 0) {
            const Word* g = reinterpret_cast<const Word*>(bp.blocks + grp * bsc.group) + lane;
#pragma unroll
            for (int c = 0; c < MB2; ++c) {
                w[c] = in_group && c < bp.max_bs ? __ldg(g + c * bsc.stride) : Word(0);
            }
        } else {
            load_block_columns<SK>(bp, bsc, grp, lane, in_group, w);
        }
    }

    __device__ __forceinline__ T operator[](int c) const
    {
        if constexpr (SK >= 0) {
            return widen<SK, T>(w[c]);
        } else {
            return w[c];
        }
    }
};

namespace {  // a copy per translation unit

// *out = the storage kind every group of the precisions shares, or
// kSkMixed.  One block.
template <typename T>
__global__ void storage_summary_kernel(int64_t num_groups, int gs,
                                       const uint8_t* __restrict__ prec, int* out)
{
    const int first = storage_kind<T>(prec[0]);
    int differ = 0;
    for (int64_t g = threadIdx.x; g < num_groups; g += blockDim.x) {
        differ |= storage_kind<T>(prec[g * gs]) != first;
    }
    differ = __syncthreads_or(differ);
    if (threadIdx.x == 0) *out = differ ? kSkMixed : first;
}

}  // namespace

// bp.kind from bp.prec; scratch is one int of device memory.  Waits for the
// stream.
template <typename T>
inline cudaError_t resolve_storage_kind(BlockPrec<T>& bp, int* scratch, cudaStream_t st)
{
    bp.kind = kSkMixed;
    if (bp.prec == nullptr || bp.num_blocks <= 0) return cudaSuccess;
    const BlockScheme bsc = block_scheme(bp.max_bs);
    storage_summary_kernel<T><<<1, 1024, 0, st>>>((bp.num_blocks + bsc.gs - 1) / bsc.gs, bsc.gs,
                                                 bp.prec, scratch);
    int kind = kSkMixed;
    cudaError_t e = cudaMemcpyAsync(&kind, scratch, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    bp.kind = kind;
    return e;
}

// The pass instance for bp: fixed storage kinds for the single right-hand
// side (K1), where the pass is bandwidth-bound; the per-group switch
// otherwise.  Calls f(std::integral_constant<int, SK>).
template <typename T, bool K1, typename F>
inline void with_pass_kind(const BlockPrec<T>& bp, F&& f)
{
    if (bp.prec == nullptr) {
        f(std::integral_constant<int, kSkFull>{});
        return;
    }
    if constexpr (K1) {
        if (bp.kind == kF16) {
            f(std::integral_constant<int, kF16>{});
            return;
        }
        if (sizeof(T) == 8 && bp.kind == kF32) {
            f(std::integral_constant<int, kF32>{});
            return;
        }
    }
    f(std::integral_constant<int, kSkMixed>{});
}

}  // namespace b2s
