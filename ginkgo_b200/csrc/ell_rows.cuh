// Column-major (Ell-layout) SpMV with R consecutive rows per thread: the
// values and column indices of entry k of rows r0 .. r0 + R - 1 are one
// vector load each (16 bytes of values), so a warp moves 32 R entries per
// instruction and the gathers of x for neighbouring rows stay coalesced for
// banded matrices.  Used for Ell and Sellp SpMV with one right-hand side
// and by the GMRES engine on its column-major copy of A.
#pragma once

#include <cstring>

#include "common.cuh"

namespace b2s {

// R consecutive elements of 2, 4, 8, 16 or 32 bytes in total, evict-first.
template <typename T, int R>
__device__ __forceinline__ void load_stream_rows(const T* p, T (&o)[R])
{
    constexpr int kBytes = int(R * sizeof(T));
    static_assert(kBytes == 2 || kBytes == 4 || kBytes == 8 || kBytes % 16 == 0,
                  "vector width");
    if constexpr (kBytes == 2) {
        const unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
        memcpy(o, &u, 2);
    } else if constexpr (kBytes == 4) {
        const unsigned u = __ldcs(reinterpret_cast<const unsigned*>(p));
        memcpy(o, &u, 4);
    } else if constexpr (kBytes == 8) {
        const uint2 u = __ldcs(reinterpret_cast<const uint2*>(p));
        memcpy(o, &u, 8);
    } else {
        uint4 u[kBytes / 16];
#pragma unroll
        for (int k = 0; k < kBytes / 16; ++k) u[k] = __ldcs(reinterpret_cast<const uint4*>(p) + k);
        memcpy(o, u, kBytes);
    }
}

// Padding marker of the 16-bit offset layout (offsets lie in -32767..32767).
constexpr int16_t kEllPad16 = INT16_MIN;

// y = A x (or alpha A x + beta y) over an Ell layout: entry k of row r at
// k * ld + r (ld a multiple of R, every row group 16-byte aligned), padding
// entries with column -1; the slots of rows n .. ld - 1 are never gathered
// through.  x and y are strided by ldx and ldy.  Entries are
// summed in stored order.  PLAIN: unit strides and y = A x (no alpha/beta).
// A launch whose *skip is non-zero returns at once.  Launched through
// ell_rows_kernel_for (below), which picks the register-bounded form for
// FP64 two-row groups.
template <typename T, int R, bool PLAIN, typename IT>
__device__ __forceinline__ void ell_rows_body(int64_t n, int width, int64_t ld,
                                              const IT* __restrict__ cols,
                                              const T* __restrict__ vals,
                                              const T* __restrict__ x, int64_t ldx,
                                              T* __restrict__ y, int64_t ldy,
                                              const T* __restrict__ alpha,
                                              const T* __restrict__ beta,
                                              const int* __restrict__ skip)
{
    if (skip != nullptr && *skip) return;
    const int64_t groups = (n + R - 1) / R;
    for (int64_t grp = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; grp < groups;
         grp += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r0 = grp * R;
        // slots of rows n .. ld - 1 may hold anything: they are loaded with
        // the group but never used as gather indices
        const int valid = n - r0 < R ? int(n - r0) : R;
        T acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = T(0);
        const IT* cp = cols + r0;
        const T* vp = vals + r0;
#pragma unroll(sizeof(T) == 4 ? 8 : 4)
        for (int k = 0; k < width; ++k) {
            IT c[R];
            T v[R];
            load_stream_rows<IT, R>(cp + int64_t(k) * ld, c);
            load_stream_rows<T, R>(vp + int64_t(k) * ld, v);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                // 16-bit entries are offsets from the row, kEllPad16 padding
                int64_t col;
                bool used;
                if constexpr (sizeof(IT) == 2) {
                    col = r0 + r + c[r];
                    used = c[r] != kEllPad16;
                } else {
                    col = c[r];
                    used = c[r] >= 0;
                }
                const int64_t xo = PLAIN ? col : col * ldx;
                const T xv = r < valid && used ? __ldg(x + xo) : T(0);
                acc[r] += v[r] * xv;
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (r < valid) {
                if constexpr (PLAIN) {
                    y[r0 + r] = acc[r];
                } else {
                    T* dst = y + (r0 + r) * ldy;
                    *dst = combine(acc[r], alpha, beta, dst);
                }
            }
        }
    }
}

#define B2S_ELL_ROWS_PARAMS                                                          \
    int64_t n, int width, int64_t ld, const IT *__restrict__ cols,                   \
        const T *__restrict__ vals, const T *__restrict__ x, int64_t ldx,            \
        T *__restrict__ y, int64_t ldy, const T *__restrict__ alpha,                 \
        const T *__restrict__ beta, const int *__restrict__ skip

template <typename T, int R, bool PLAIN = false, typename IT = int32_t>
__global__ void __launch_bounds__(256) ell_rows_kernel(B2S_ELL_ROWS_PARAMS)
{
    ell_rows_body<T, R, PLAIN, IT>(n, width, ld, cols, vals, x, ldx, y, ldy, alpha, beta,
                                   skip);
}

// The same kernel held to 32 registers, eight blocks per SM.  FP64 two-row
// groups gain from it (7-point 128^3 Ell: 33 us instead of 35.6 us); FP32
// forms spill under the bound, and any explicit bound changes their code.
template <typename T, int R, bool PLAIN = false, typename IT = int32_t>
__global__ void __launch_bounds__(256, 8) ell_rows_kernel_b8(B2S_ELL_ROWS_PARAMS)
{
    ell_rows_body<T, R, PLAIN, IT>(n, width, ld, cols, vals, x, ldx, y, ldy, alpha, beta,
                                   skip);
}

#undef B2S_ELL_ROWS_PARAMS

// The Ell row kernel to launch for T and R (a pointer to a __global__
// function, launched with <<<...>>>).
template <typename T, int R, bool PLAIN = false, typename IT = int32_t>
constexpr auto ell_rows_kernel_for()
{
    if constexpr (sizeof(T) == 8 && R == 2) {
        return &ell_rows_kernel_b8<T, R, PLAIN, IT>;
    } else {
        return &ell_rows_kernel<T, R, PLAIN, IT>;
    }
}

// Sellp with R consecutive rows of one slice per thread (slice_size a
// multiple of R): entry k of local rows l .. l + R - 1 of slice s sits at
// (slice_sets[s] + k) * slice_size + l, one vector load of values and one
// of column indices.  Padding entries (column -1) and rows past n are not
// gathered through.  PLAIN: unit strides and y = A x; the FP64 persistent
// plain form is held to 32 registers so that eight blocks fit on an SM (measured
// 38-39 us instead of 41-42 us on the 7-point 128^3 matrix in slices of 32).
template <typename T, int R, bool PREFETCH, bool PLAIN = false>
__global__ void __launch_bounds__(256, sizeof(T) == 8 && PREFETCH ? (PLAIN ? 8 : 6) : 5)
    sellp_rows_kernel(int n, int slice_size, int slice_shift,
                      const uint64_t* __restrict__ slice_sets,
                      const uint64_t* __restrict__ slice_lengths,
                      const int32_t* __restrict__ cols, const T* __restrict__ vals,
                      const T* __restrict__ x, int64_t ldx, T* __restrict__ y,
                      int64_t ldy, const T* __restrict__ alpha,
                      const T* __restrict__ beta)
{
    // PREFETCH: grid-stride over row groups, the slice length and start of
    // the next group loaded while the current one is summed; else one group
    // per thread (the grid covers every group).  32-bit slice
    // arithmetic (n < 2^31), a shift when the slice size is a power of two
    // (slice_shift >= 0).
    const unsigned groups = unsigned((int64_t(n) + R - 1) / R);
    const unsigned stride = gridDim.x * blockDim.x;
    unsigned grp = blockIdx.x * blockDim.x + threadIdx.x;
    if (grp >= groups) return;
    auto lookup = [&](unsigned g, int& len, int64_t& base) {
        const unsigned r0 = g * unsigned(R);
        const unsigned slice = slice_shift >= 0 ? r0 >> slice_shift : r0 / unsigned(slice_size);
        const unsigned local = r0 - slice * unsigned(slice_size);
        len = int(__ldg(slice_lengths + slice));
        base = int64_t(__ldg(slice_sets + slice)) * slice_size + local;
    };
    int len;
    int64_t base;
    lookup(grp, len, base);
    for (; grp < groups; grp += stride) {
        int len_n = 0;
        int64_t base_n = 0;
        if (PREFETCH && grp + stride < groups) lookup(grp + stride, len_n, base_n);
        const unsigned r0 = grp * unsigned(R);
        const int valid = n - int(r0) < R ? n - int(r0) : R;
        T acc[R];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = T(0);
        if constexpr (R <= 2) {
#pragma unroll 4
            for (int k = 0; k < len; ++k) {
                int32_t c[R];
                T v[R];
                load_stream_rows<int32_t, R>(cols + base + int64_t(k) * slice_size, c);
                load_stream_rows<T, R>(vals + base + int64_t(k) * slice_size, v);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int64_t xo = PLAIN ? int64_t(c[r]) : int64_t(c[r]) * ldx;
                    const T xv = r < valid && c[r] >= 0 ? __ldg(x + xo) : T(0);
                    acc[r] += v[r] * xv;
                }
            }
        } else {
            // 4-row groups (FP32): chunks of CH entries with predicated loads,
            // so a short slice issues all its loads at once instead of
            // finishing in a serial remainder loop (measured faster; in FP64
            // the extra registers cost more than they gain)
            constexpr int CH = 4;
            for (int k0 = 0; k0 < len; k0 += CH) {
                int32_t c[CH][R];
                T v[CH][R];
#pragma unroll
                for (int u = 0; u < CH; ++u) {
                    if (k0 + u < len) {
                        load_stream_rows<int32_t, R>(cols + base + int64_t(k0 + u) * slice_size, c[u]);
                        load_stream_rows<T, R>(vals + base + int64_t(k0 + u) * slice_size, v[u]);
                    } else {
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            c[u][r] = -1;
                            v[u][r] = T(0);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < CH; ++u) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int64_t xo = PLAIN ? int64_t(c[u][r]) : int64_t(c[u][r]) * ldx;
                        const T xv = r < valid && c[u][r] >= 0 ? __ldg(x + xo) : T(0);
                        acc[r] += v[u][r] * xv;
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (r < valid) {
                if constexpr (PLAIN) {
                    y[int64_t(r0) + r] = acc[r];
                } else {
                    T* dst = y + (int64_t(r0) + r) * ldy;
                    *dst = combine(acc[r], alpha, beta, dst);
                }
            }
        }
        if (!PREFETCH) break;  // one group per thread: the grid covers all
        len = len_n;
        base = base_n;
    }
}

// Rows per thread: 16 bytes of values, except one FP64 row per thread for
// rows wider than 16 entries (measured faster on the 27-point matrix).
template <typename T>
inline int ell_rows_per_thread(int64_t width)
{
    return sizeof(T) == 8 && width > 16 ? 1 : int(16 / sizeof(T));
}

// Fills the Ell-layout copy (ld >= n rows, width entries per row) from Csr,
// converting the values to T; rows n .. ld - 1 and the tail of shorter rows
// are padding.  A row longer than width sets *too_long.
template <typename T>
__global__ void ell_fill_kernel(int64_t n, int64_t ld, int width,
                                const int32_t* __restrict__ rp,
                                const int32_t* __restrict__ ci,
                                const double* __restrict__ v,
                                int32_t* __restrict__ cols, T* __restrict__ vals,
                                int* too_long)
{
    const int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (row >= ld) return;
    const int rs = row < n ? rp[row] : 0;
    const int len = row < n ? rp[row + 1] - rs : 0;
    if (len > width) *too_long = 1;
    for (int k = 0; k < width; ++k) {
        const int64_t idx = int64_t(k) * ld + row;
        if (k < len) {
            cols[idx] = ci[rs + k];
            vals[idx] = T(v[rs + k]);
        } else {
            cols[idx] = -1;
            vals[idx] = T(0);
        }
    }
}

// The same copy with 16-bit column offsets col - row (a quarter less
// traffic for FP32 values); an offset outside -32767..32767 sets
// *too_far and the caller falls back to ell_fill_kernel.
template <typename T>
__global__ void ell_fill16_kernel(int64_t n, int64_t ld, int width,
                                  const int32_t* __restrict__ rp,
                                  const int32_t* __restrict__ ci,
                                  const double* __restrict__ v,
                                  int16_t* __restrict__ cols, T* __restrict__ vals,
                                  int* too_long, int* too_far)
{
    const int64_t row = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (row >= ld) return;
    const int rs = row < n ? rp[row] : 0;
    const int len = row < n ? rp[row + 1] - rs : 0;
    if (len > width) *too_long = 1;
    for (int k = 0; k < width; ++k) {
        const int64_t idx = int64_t(k) * ld + row;
        if (k < len) {
            const int64_t d = int64_t(ci[rs + k]) - row;
            if (d < -32767 || d > 32767) *too_far = 1;
            cols[idx] = int16_t(d < -32767 || d > 32767 ? 0 : d);
            vals[idx] = T(v[rs + k]);
        } else {
            cols[idx] = kEllPad16;
            vals[idx] = T(0);
        }
    }
}

}  // namespace b2s
