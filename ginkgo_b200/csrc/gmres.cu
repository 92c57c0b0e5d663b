// Restarted GMRES(d) with right scalar-Jacobi preconditioning and an FP64
// restart residual, in three precisions behind one engine:
//
//   B2S_GMRES_F64         Arnoldi in FP64, FP64 basis
//   B2S_GMRES_MIXED_F32   mixed precision: every restart (an outer step of
//   B2S_GMRES_MIXED_BF16  iterative refinement) computes r = b - A x and
//                         ||r|| in FP64; the Arnoldi cycle runs on an FP32
//                         copy of A with FP32 vectors and an FP32 or BF16
//                         basis; x += M V y is accumulated in FP64.
//
// Reference behaviour: core/solver/gmres.cpp:325-640 (restart, Arnoldi,
// Givens QR, solve_krylov, multi_axpy), core/solver/ir.cpp:191-257 with
// update_residual.hpp:20-60 (outer residual and check),
// reference/solver/common_gmres_kernels.cpp:29-180 (Givens formulas).
// Differences, all on the device: orthogonalisation is classical
// Gram-Schmidt with the re-orthogonalisation of CGS2 (the reference's
// ortho_method::cgs2) taken from the Gram matrix G = V^T V of the stored
// basis instead of a second pass over it: with h1 = V^T w, CGS2's second
// projection is V^T (w - V h1) = h1 - G h1, so h = (2I - G) h1 and
// w'' = w - V h in a single pass.  G gains one column per step from the
// same pass that forms h1.  The Hessenberg matrix, Givens rotations, G and
// the triangular solve are FP64 in every variant; a cycle ends early when
// the Givens residual estimate reaches the goal, and convergence is declared
// only on the explicit FP64 residual.
//
// The basis is stored unnormalised: V_i = round_basis(w''_{i-1}) (V_0 =
// round_basis(r)) with v_i = sigma_i V_i, sigma_i = 1 / ||w''_{i-1}||, and
// the sigmas are folded into the projection coefficients, so the vector
// that enters step j + 1 is written by step j's update pass itself.
//
// Kernels per Arnoldi step j (one CUDA graph per restart cycle):
//   spmv    w = A y on a column-major (Ell) copy of A in the Arnoldi type
//           with 16-bit column offsets (32-bit columns when an offset does
//           not fit), when its padding stays within a quarter of nnz; else
//           the pipelined Csr kernel on A
//   dots    h1 = V_{0..j}^T w and G(:, j) = V_{0..j}^T v_j in one pass over
//           the basis (all sums of a thread in registers); last block:
//           h = (2I - G) h1
//   update  w'' = sigma_j w - V (sigma h) and ||w''||, V_{j+1} and the next
//           SpMV input y = D^-1 V_{j+1} in the same pass; last block:
//           Hessenberg column, Givens update, residual estimate, early end
//           of the cycle, back substitution
// per cycle: x += D^-1 V (sigma y) (FP64 accumulate) with r = b, then
// r -= A x with the pipelined kernel in FP64, then ||r||, ||b||, V_0, the
// first SpMV input and the restart check.
// The serial parts (Givens chain, back substitution, (2I - G) h1) run in
// the last block on shared-memory copies of the small arrays.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "csr_async.cuh"
#include "ell_rows.cuh"
#include "jacobi_scheme.cuh"
#include "solver_common.cuh"

namespace b2s {
namespace {

constexpr int kMaxKrylov = 128;
constexpr int kLd = kMaxKrylov + 1;
constexpr int kDotsMaxGrid = kMaxSMs * 4;  // resident at 4 blocks per SM
constexpr int kDotsGroup = 32;  // blocks folded by one group's last block
constexpr int kSmallGram = 32;  // steps j < 32: the Gram matrix staged in shared memory
constexpr int kDotsMaxGroups = (kDotsMaxGrid + kDotsGroup - 1) / kDotsGroup;

// The Hessenberg matrix (column j at H[j * ld], ld = krylov_dim + 1) and
// the Gram matrix G of the stored basis (G(i, k) at G[i * ld + k]) live in
// the workspace beside this state.
struct GmresState {
    int done, cycle_done, j, final_iter;
    int total_iter, max_iters, outer_iter, converged;
    int krylov_dim, ld;
    int ortho;     // B2S_ORTHO_*: CGS (h = h1) or CGS2 (h = (2I - G) h1)
    int baseline;  // B2S_BASELINE_* of the residual goal
    int idle;  // done || cycle_done: the Arnoldi kernels have nothing to do
    unsigned ticket;
    int too_long;  // a row is longer than the Ell copy's width
    int too_far;   // a column offset does not fit 16 bits
    unsigned gticket[kDotsMaxGroups + 1];  // dots: per group of 32 blocks
    double bnorm, rnorm, reduction, inner_reduction, inner_thresh;
    double base;  // ||b||, ||r_0|| or 1, by the baseline, set at the first restart
    double qscale;  // scaled bases: factor from the formed vector to its storage
    double sigma[kLd];  // stored basis vector i is v_i / sigma[i] (unnormalised)
    double minus_one, one;       // alpha, beta of r = b - A x
    double h[kLd];               // combined projection coefficients of step j
    double g[kLd], cs[kMaxKrylov], sn[kMaxKrylov], y[kMaxKrylov];
};

// Bases stored scaled (CB-GMRES reduce2 and the scaled-integer formats of
// core/solver/cb_gmres.cpp:100-157): the next vector is formed in the
// arithmetic type first and written by a second pass once its norm and
// largest entry are known.  Half stores the normalised vector; an integer
// type stores trunc(v / s) with s = (max|v| / ||v||) * 2 / INT_MAX, one
// scale per vector (core/solver/cb_gmres_accessor.hpp), so that the stored
// vector read as a number times sigma is the normalised one.
template <typename TB>
struct BasisKind {
    static constexpr bool kScaled = false;
    static constexpr double kIntMax = 0.0;
};
template <>
struct BasisKind<__half> {
    static constexpr bool kScaled = true;
    static constexpr double kIntMax = 0.0;
};
template <>
struct BasisKind<int64_t> {
    static constexpr bool kScaled = true;
    static constexpr double kIntMax = 9223372036854775807.0;
};
template <>
struct BasisKind<int32_t> {
    static constexpr bool kScaled = true;
    static constexpr double kIntMax = 2147483647.0;
};
template <>
struct BasisKind<int16_t> {
    static constexpr bool kScaled = true;
    static constexpr double kIntMax = 32767.0;
};

// Storage scale and sigma of a scaled basis vector of norm nrm and largest
// entry mx: stored = formed * qscale, normalised = stored * sigma.
template <typename TB>
__device__ __forceinline__ void basis_scales(double nrm, double mx, double* qscale,
                                             double* sigma)
{
    constexpr double kMax = BasisKind<TB>::kIntMax;
    if constexpr (kMax == 0.0) {
        *qscale = nrm > 0.0 ? 1.0 / nrm : 0.0;
        *sigma = 1.0;
    } else {
        *qscale = mx > 0.0 ? kMax / (2.0 * mx) : 0.0;
        *sigma = nrm > 0.0 ? 2.0 * mx / (nrm * kMax) : 0.0;
    }
}

template <typename TB, typename TA>
__device__ __forceinline__ TB to_basis(TA v)
{
    return TB(v);
}
template <>
__device__ __forceinline__ __half to_basis<__half, double>(double v)
{
    return __double2half(v);
}
template <>
__device__ __forceinline__ int64_t to_basis<int64_t, double>(double v)
{
    return __double2ll_rz(v);
}
template <>
__device__ __forceinline__ int32_t to_basis<int32_t, double>(double v)
{
    return __double2int_rz(v);
}
template <>
__device__ __forceinline__ int16_t to_basis<int16_t, double>(double v)
{
    return int16_t(__double2int_rz(v));
}
template <>
__device__ __forceinline__ __nv_bfloat16 to_basis<__nv_bfloat16, float>(float v)
{
    return __float2bfloat16_rn(v);
}
template <typename TA, typename TB>
__device__ __forceinline__ TA from_basis(TB v)
{
    return TA(v);
}
template <>
__device__ __forceinline__ double from_basis<double, __half>(__half v)
{
    return double(__half2float(v));
}
template <>
__device__ __forceinline__ float from_basis<float, __nv_bfloat16>(__nv_bfloat16 v)
{
    return __bfloat162float(v);
}

// Row groups: every streamed vector (basis, w, y) has a leading dimension
// that is a multiple of 64 rows, so the R = 16 / sizeof(TB) rows of a group
// start on a 16-byte boundary and move as 16-byte vector loads.  The group
// that holds row n - 1 may be partial and is read element by element.
template <typename T, int R>
__device__ __forceinline__ void load_rows(const T* p, T (&o)[R])
{
    static_assert((R * sizeof(T)) % 16 == 0, "whole 16-byte vectors");
    constexpr int NV = int(R * sizeof(T) / 16);
    uint4 buf[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) buf[k] = reinterpret_cast<const uint4*>(p)[k];
    const T* q = reinterpret_cast<const T*>(buf);
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = q[r];
}
template <typename T, int R>
__device__ __forceinline__ void store_rows(T* p, const T (&v)[R])
{
    constexpr int NV = int(R * sizeof(T) / 16);
    uint4 buf[NV];
    T* q = reinterpret_cast<T*>(buf);
#pragma unroll
    for (int r = 0; r < R; ++r) q[r] = v[r];
#pragma unroll
    for (int k = 0; k < NV; ++k) reinterpret_cast<uint4*>(p)[k] = buf[k];
}
// rows r < valid of the group, zero past the end
template <typename T, int R>
__device__ __forceinline__ void load_rows(const T* p, T (&o)[R], int valid)
{
    if (valid >= R) {
        load_rows<T, R>(p, o);
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) o[r] = r < valid ? p[r] : T(0);
    }
}
template <typename T, int R>
__device__ __forceinline__ void store_rows(T* p, const T (&v)[R], int valid)
{
    if (valid >= R) {
        store_rows<T, R>(p, v);
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (r < valid) p[r] = v[r];
        }
    }
}
// basis rows converted to the arithmetic type
template <typename TA, typename TB, int R>
__device__ __forceinline__ void load_basis(const TB* p, TA (&o)[R], int valid)
{
    TB b[R];
    load_rows<TB, R>(p, b, valid);
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = from_basis<TA>(b[r]);
}

template <typename TB>
__host__ __device__ constexpr int rows_per_group()
{
    return int(16 / sizeof(TB));
}

// Sums each of the N values v[0..N) (N = 8, 16 or 32 P) over the warp:
// every level of the butterfly hands half of the values a lane carries to
// its partner.  On return lane l holds the total of value l * P + k in v[k]
// (N = 32 P), or of value l / (32 / N) in v[0] (N = 8, 16).
template <typename T, int N>
__device__ __forceinline__ void warp_multi_sum(T (&v)[N], int lane)
{
    static_assert(N == 8 || N == 16 || N % 32 == 0, "8, 16 or 32 P values");
    constexpr unsigned kFull = 0xffffffffu;
#pragma unroll
    for (int lvl = 0; lvl < 5; ++lvl) {
        const int m = 16 >> lvl;
        const int half = N >> (lvl + 1);
        if (half == 0) {
            v[0] += __shfl_xor_sync(kFull, v[0], m);
        } else {
            const bool up = lane & m;
#pragma unroll
            for (int i = 0; i < half; ++i) {
                const T send = up ? v[i] : v[i + half];
                const T keep = up ? v[i + half] : v[i];
                v[i] = keep + __shfl_xor_sync(kFull, send, m);
            }
        }
    }
}

// One pass of the dots kernel over C basis vectors i0 .. i0 + C - 1 (C a
// compile-time count, so the C 16-byte loads of a row group are issued
// back to back without predicates): acc[u] += V_{i0+u}^T w and
// acc[4 + u] += V_{i0+u}^T v_j over this thread's row groups.  Full groups
// take the unconditional vector loads; the one partial group at the end is
// read element by element by the thread it falls to.
template <typename TA, typename TB, int C>
__device__ __forceinline__ void dots_pass(int64_t n, int64_t ldv,
                                          const TB* __restrict__ V,
                                          const TA* __restrict__ w,
                                          const TB* __restrict__ vj, int i0,
                                          TA (&acc)[8])
{
    constexpr int R = rows_per_group<TB>();
    auto group = [&](int64_t r0, int valid) {
        TA wr[R], vr[R];
        load_rows<TA, R>(w + r0, wr, valid);
        load_basis<TA, TB, R>(vj + r0, vr, valid);
        TA x[C][R];
#pragma unroll
        for (int u = 0; u < C; ++u) load_basis<TA, TB, R>(V + int64_t(i0 + u) * ldv + r0, x[u], valid);
#pragma unroll
        for (int u = 0; u < C; ++u) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                acc[u] += x[u][r] * wr[r];
                acc[4 + u] += x[u][r] * vr[r];
            }
        }
    };
    const int64_t full = n / R;
    int64_t grp = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    for (; grp < full; grp += int64_t(gridDim.x) * blockDim.x) group(grp * R, R);
    if (grp == full && n % R != 0) group(full * R, int(n % R));
}

// compact value index c < 2 nvec -> partial row e (h1 at e < kLd, G after)
__device__ __forceinline__ int dots_row(int c, int nvec)
{
    return c < nvec ? c : kLd + c - nvec;
}

// Ticket of `count` arrivals; true in the last one to arrive (the caller's
// writes are fenced first), which resets the ticket.
__device__ __forceinline__ bool last_of(unsigned* ticket, unsigned count, int* flag_sm)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        *flag_sm = (t == count - 1);
        if (t == count - 1) *ticket = 0;
    }
    __syncthreads();
    const bool last = *flag_sm;
    if (last) __threadfence();
    return last;
}

// In one block: for the 2 nvec values c, the sum over the L partials
// src[dots_row(c) * ld + base + k], k < L <= 32, one warp load per value
// (warp w takes c = w, w + 8, ...; all loads issued before the sums).
__device__ __noinline__ void fold32(const double* src, int64_t ld, int base, int L,
                                       int nvec, double* dst, int64_t dst_ld, int dst_col)
{
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    // values per warp and round, their loads in flight together: one round
    // covers 2 nvec <= 64 (Krylov dimensions up to 32)
    constexpr int K = 8;
    for (int c0 = 0; c0 < 2 * nvec; c0 += 8 * K) {
        double v[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int c = c0 + wid + 8 * k;
            v[k] = c < 2 * nvec && lane < L
                       ? __ldcg(src + dots_row(c, nvec) * ld + base + lane)
                       : 0.0;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int c = c0 + wid + 8 * k;
            const double s = warp_sum(v[k]);
            if (lane == 0 && c < 2 * nvec) dst[dots_row(c, nvec) * dst_ld + dst_col] = s;
        }
    }
}

// Step j, part 3: h1 = V_{0..j}^T w and G(:, j) = V_{0..j}^T v_j: passes of
// up to 4 basis vectors, a thread taking one row group per iteration with
// the 8 sums of the pass in registers (4 blocks per SM).  Per pass
// one multi-value warp reduction and one block reduction into value-major
// partials (partials[e * gridDim.x + block]).  The last block of every 32
// blocks folds its group's partials; the last group to finish folds the
// groups, completes G's row and column j and forms h = (2I - G) h1 (CGS2),
// or h = h1 (CGS).  The summation order is fixed: the result does not
// depend on scheduling.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock, 4)
    gmres_dots_kernel(int64_t n, int64_t ldv, const TB* __restrict__ V,
                      const TA* __restrict__ w, GmresState* st,
                      double* __restrict__ partials, double* __restrict__ gpart,
                      double* __restrict__ Gm)
{
    constexpr int CMAX = 4;
    constexpr int W = kSolverBlock / kWarp;
    __shared__ double redv[W][8];
    __shared__ double tot[2 * kLd];
    __shared__ double Gs[kSmallGram * kSmallGram];
    __shared__ int last;
    if (st->idle) return;
    const int j = st->j;
    const int nvec = j + 1;
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const TB* vj = V + int64_t(j) * ldv;
    const int B = gridDim.x;
    for (int i0 = 0; i0 < nvec; i0 += CMAX) {
        const int c = nvec - i0 < CMAX ? nvec - i0 : CMAX;
        TA acc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = TA(0);
        switch (c) {
        case 1: dots_pass<TA, TB, 1>(n, ldv, V, w, vj, i0, acc); break;
        case 2: dots_pass<TA, TB, 2>(n, ldv, V, w, vj, i0, acc); break;
        case 3: dots_pass<TA, TB, 3>(n, ldv, V, w, vj, i0, acc); break;
        default: dots_pass<TA, TB, 4>(n, ldv, V, w, vj, i0, acc); break;
        }
        warp_multi_sum<TA, 8>(acc, lane);
        // lane l holds value l / 4: the h1 sum of vector i0 + l / 4 for
        // l < 16, the G sum of vector i0 + l / 4 - 4 after
        if ((lane & 3) == 0) redv[wid][lane / 4] = double(acc[0]);
        __syncthreads();
        if (threadIdx.x < 8) {
            const int u = threadIdx.x % 4;
            if (u < c) {
                double s = 0.0;
                for (int k = 0; k < W; ++k) s += redv[k][threadIdx.x];
                const int e = (threadIdx.x < 4 ? 0 : kLd) + i0 + u;
                partials[int64_t(e) * B + blockIdx.x] = s;
            }
        }
        __syncthreads();
    }
    const int g = blockIdx.x / kDotsGroup;
    const int ngroups = (B + kDotsGroup - 1) / kDotsGroup;
    const int gsize = B - g * kDotsGroup < kDotsGroup ? B - g * kDotsGroup : kDotsGroup;
    if (!last_of(&st->gticket[g], unsigned(gsize), &last)) return;
    fold32(partials, B, g * kDotsGroup, gsize, nvec, gpart, kDotsMaxGroups, g);
    if (!last_of(&st->ticket, unsigned(ngroups), &last)) return;
    // tot[0..nvec): h1, tot[kLd + i]: G(i, j), of the stored (unnormalised)
    // vectors; scaled to the normalised basis by sigma_i sigma_j
    fold32(gpart, kDotsMaxGroups, 0, ngroups, nvec, tot, 1, 0);
    __syncthreads();
    if (threadIdx.x <= j) {
        const double sc = st->sigma[threadIdx.x] * st->sigma[j];
        tot[threadIdx.x] *= sc;
        tot[kLd + threadIdx.x] *= sc;
    }
    __syncthreads();
    if (st->ortho == B2S_ORTHO_CGS) {
        // one projection: h = h1
        if (threadIdx.x <= j) st->h[threadIdx.x] = tot[threadIdx.x];
        return;
    }
    // row and column j of G; rows 0..j-1 hold the earlier steps of this
    // cycle (G is symmetric, so row i of G(0..j, 0..j) is complete)
    const int ld = st->ld;
    if (j < kSmallGram) {
        // the whole G(0..j, 0..j) in shared memory (one parallel pass of
        // loads), then one thread per row: the short serial tail of every
        // Arnoldi step of the usual Krylov dimensions
        for (int e = threadIdx.x; e < j * j; e += kSolverBlock) {
            const int i = e / j, k = e - i * j;  // G(i, k), i, k < j: earlier steps
            Gs[i * kSmallGram + k] = __ldcg(Gm + int64_t(i) * ld + k);
        }
        if (threadIdx.x <= j) {  // row and column j: this step
            const int i = threadIdx.x;
            const double gij = tot[kLd + i];
            Gs[i * kSmallGram + j] = gij;
            Gs[j * kSmallGram + i] = gij;
            Gm[int64_t(i) * ld + j] = gij;
            Gm[int64_t(j) * ld + i] = gij;
        }
        __syncthreads();
        if (threadIdx.x <= j) {
            const int i = threadIdx.x;
            double gh = 0.0;
            for (int k = 0; k <= j; ++k) gh += Gs[i * kSmallGram + k] * tot[k];
            st->h[i] = 2.0 * tot[i] - gh;
        }
        return;
    }
    if (threadIdx.x <= j) {
        const int i = threadIdx.x;
        const double gij = tot[kLd + i];
        Gm[int64_t(i) * ld + j] = gij;
        Gm[int64_t(j) * ld + i] = gij;
    }
    __syncthreads();  // the block's own writes of G are visible to it
    // h = (2I - G) h1: CGS2's second projection from G, one warp per row i
    // (row i of G is contiguous, so the lanes' loads coalesce)
    for (int i = wid; i <= j; i += W) {
        double gh = 0.0;
        for (int k = lane; k <= j; k += kWarp) gh += __ldcg(Gm + int64_t(i) * ld + k) * tot[k];
        gh = warp_sum(gh);
        if (lane == 0) st->h[i] = 2.0 * tot[i] - gh;
    }
}

// The end of Arnoldi step j, run by the whole last block of the update
// kernel: Givens update of column j, residual estimate, cycle bookkeeping
// and, when the cycle ends, the back substitution y = H \ g.  The small
// arrays are staged in shared memory, so the serial chain runs at
// shared-memory latency.
__device__ __noinline__ void close_step(GmresState* st, double hnorm, double* __restrict__ Hm)
{
    __shared__ double hc[kLd], gS[kLd], csS[kMaxKrylov], snS[kMaxKrylov];
    __shared__ double ts[kMaxKrylov];
    __shared__ int fin;
    const int j = st->j;
    const int ld = st->ld;
    for (int i = threadIdx.x; i <= j; i += kSolverBlock) {
        hc[i] = st->h[i];
        gS[i] = st->g[i];
    }
    for (int i = threadIdx.x; i < j; i += kSolverBlock) {
        csS[i] = st->cs[i];
        snS[i] = st->sn[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        st->ticket = 0;
        hc[j + 1] = hnorm;
        for (int i = 0; i < j; ++i) {
            const double t = csS[i] * hc[i] + snS[i] * hc[i + 1];
            hc[i + 1] = -snS[i] * hc[i] + csS[i] * hc[i + 1];
            hc[i] = t;
        }
        const double th = hc[j], nh = hc[j + 1];
        double c, s;
        if (th == 0.0) {
            c = 0.0;
            s = 1.0;
        } else {
            const double scale = fabs(th) + fabs(nh);
            const double a = fabs(th / scale), b = fabs(nh / scale);
            const double hyp = scale * sqrt(a * a + b * b);
            c = th / hyp;
            s = nh / hyp;
        }
        hc[j] = c * th + s * nh;
        hc[j + 1] = 0.0;
        gS[j + 1] = -s * gS[j];
        gS[j] = c * gS[j];
        st->cs[j] = c;
        st->sn[j] = s;
        st->g[j] = gS[j];
        st->g[j + 1] = gS[j + 1];
        const double est = fabs(gS[j + 1]);
        const int total = st->total_iter + 1;
        st->final_iter = j + 1;
        st->total_iter = total;
        st->sigma[j + 1] = hnorm > 0.0 ? 1.0 / hnorm : 0.0;
        st->j = j + 1;
        fin = est <= st->inner_thresh || j + 1 >= st->krylov_dim ||
              total >= st->max_iters || !(hnorm > 0.0);
        if (fin) {
            st->cycle_done = 1;
            st->idle = 1;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= j + 1; i += kSolverBlock) Hm[int64_t(j) * ld + i] = hc[i];
    if (!fin) return;
    // y = H \ g over the m = j + 1 finished columns: one warp, column by
    // column from the last (t -= H(:, k) y_k after each y_k).  Column k is
    // read from the workspace (this block wrote column j above); its loads
    // do not depend on y_k, so they are issued before the division.
    const int m = j + 1;
    for (int i = threadIdx.x; i <= j; i += kSolverBlock) ts[i] = gS[i];
    __syncthreads();
    if (threadIdx.x < kWarp) {
        const int lane = threadIdx.x;
        constexpr int KC = (kMaxKrylov + kWarp - 1) / kWarp;
        for (int k = m - 1; k >= 0; --k) {
            const double* col = Hm + int64_t(k) * ld;
            double hcol[KC];
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                const int i = lane + q * kWarp;
                hcol[q] = i < k ? __ldcg(col + i) : 0.0;
            }
            const double yk = ts[k] / __ldcg(col + k);
            if (lane == 0) st->y[k] = yk;
#pragma unroll
            for (int q = 0; q < KC; ++q) {
                const int i = lane + q * kWarp;
                if (i < k) ts[i] -= hcol[q] * yk;
            }
            __syncwarp();
        }
    }
}

// w'' = sigma_j w - sum_i (h_i sigma_i) V_i (the stored vectors are
// unnormalised), ||w''||, one row group per thread and iteration (16-byte
// basis loads, subtracted in order i = 0..j).  The same pass stores the
// next basis vector V_{j+1} = round_basis(w'') and the next SpMV input
// y = D^-1 V_{j+1}; its scale sigma_{j+1} = 1 / ||w''|| is set by the last
// block, which closes the Arnoldi step.
// Blocks per SM the update pass is held to: its registers decide how many
// row groups are in flight (measured: FP64 at 40 registers, six blocks per
// SM, runs 30 us per step on the 27-point 96^3 operator, 39 us at 48
// registers); the scaled bases, with up to eight rows per group, four.
template <typename TA, typename TB>
constexpr int update_min_blocks()
{
    return BasisKind<TB>::kScaled ? 4 : (sizeof(TA) == 8 && sizeof(TB) == 8 ? 6 : 5);
}

template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock, (update_min_blocks<TA, TB>()))
    gmres_update_kernel(int64_t n, int64_t ldv, TB* __restrict__ V,
                        const TA* __restrict__ w, const TA* __restrict__ dinv,
                        TA* __restrict__ y, GmresState* st,
                        double* __restrict__ partials, double* __restrict__ Hm,
                        TA* __restrict__ wq)
{
    constexpr int R = rows_per_group<TB>();
    constexpr bool kQ = BasisKind<TB>::kScaled;
    __shared__ double red[kSolverBlock / kWarp];
    __shared__ double tot[1];
    __shared__ TA hs[kLd];
    __shared__ int last;
    if (st->idle) return;
    const int j = st->j;
    for (int i = threadIdx.x; i <= j; i += kSolverBlock) hs[i] = TA(st->h[i] * st->sigma[i]);
    const TA sj = TA(st->sigma[j]);
    __syncthreads();
    TB* vnext = V + int64_t(j + 1) * ldv;
    double nrm = 0.0, mx = 0.0;
    auto group = [&](int64_t r0, int valid) {
        TA wr[R];
        load_rows<TA, R>(w + r0, wr, valid);
#pragma unroll
        for (int r = 0; r < R; ++r) wr[r] *= sj;
        // more loads in flight for the 4- and 8-row groups (fewer groups)
#pragma unroll(R == 2 ? 8 : 16)
        for (int i = 0; i <= j; ++i) {
            TA x[R];
            load_basis<TA, TB, R>(V + int64_t(i) * ldv + r0, x, valid);
            const TA hi = hs[i];
#pragma unroll
            for (int r = 0; r < R; ++r) wr[r] -= hi * x[r];
        }
        if constexpr (kQ) {
            // formed here, stored scaled by gmres_quantize_kernel
#pragma unroll
            for (int r = 0; r < R; ++r) {
                nrm += double(wr[r]) * double(wr[r]);
                mx = fmax(mx, fabs(double(wr[r])));
            }
            store_rows<TA, R>(wq + r0, wr, valid);
        } else {
            TB vb[R];
            TA yv[R];
            TA d[R];
            if (dinv) load_rows<TA, R>(dinv + r0, d, valid);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                vb[r] = to_basis<TB>(wr[r]);
                const TA va = from_basis<TA>(vb[r]);
                yv[r] = dinv ? d[r] * va : va;
                nrm += double(wr[r]) * double(wr[r]);
            }
            store_rows<TB, R>(vnext + r0, vb, valid);
            store_rows<TA, R>(y + r0, yv, valid);
        }
    };
    // full row groups on the vector path; the partial one by its thread
    const int64_t full = n / R;
    int64_t grp = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x;
    for (; grp < full; grp += int64_t(gridDim.x) * kSolverBlock) group(grp * R, R);
    if (grp == full && n % R != 0) group(full * R, int(n % R));
    if constexpr (kQ) {
        // the block's largest entry beside its partial sum
        double m = mx;
#pragma unroll
        for (int off = 16; off > 0; off /= 2) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
        __shared__ double mred[kSolverBlock / kWarp];
        if (threadIdx.x % kWarp == 0) mred[threadIdx.x / kWarp] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 1; k < kSolverBlock / kWarp; ++k) m = fmax(m, mred[k]);
            partials[kSolverGrid + blockIdx.x] = m;
        }
    }
    double a[1] = {nrm};
    block_partials<double, 1>(a, partials, red);
    if (last_block_done(&st->ticket, &last)) {
        sum_partials<double, 1>(partials, gridDim.x, tot, red);
        const double hnorm = sqrt(tot[0]);
        close_step(st, hnorm, Hm);
        if constexpr (kQ) {
            if (threadIdx.x == 0) {
                double m = 0.0;
                for (int b = 0; b < int(gridDim.x); ++b)
                    m = fmax(m, __ldcg(partials + kSolverGrid + b));
                basis_scales<TB>(hnorm, m, &st->qscale, &st->sigma[j + 1]);
            }
        }
    }
}

// Scaled bases: stored = round_basis(formed * qscale) and the SpMV input
// y = D^-1 stored, for the vector that the previous kernel formed (the next
// Arnoldi vector, index st->j, after gmres_update_kernel; V_0 after the
// restart).  Skipped when the cycle (restart: the solve) is over.
template <typename TA, typename TB, typename TS>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_quantize_kernel(int64_t n, int64_t ldv, const TS* __restrict__ src,
                          TB* __restrict__ V, const TA* __restrict__ dinv,
                          TA* __restrict__ y, const GmresState* st, int after_restart)
{
    if (after_restart ? st->done : st->idle) return;
    TB* dst = V + (after_restart ? 0 : int64_t(st->j) * ldv);
    const TA c = TA(st->qscale);
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        const TB vb = to_basis<TB>(TA(src[row]) * c);
        dst[row] = vb;
        const TA va = from_basis<TA>(vb);
        y[row] = dinv ? dinv[row] * va : va;
    }
}

// x += D^-1 (V y) over the m finished columns, accumulated into FP64 x, and
// r = b (the start of r = b - A x); one row group per thread and iteration.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_xupdate_kernel(int64_t n, int64_t ldv, const TB* __restrict__ V,
                         const TA* __restrict__ dinv, double* __restrict__ x,
                         const double* __restrict__ b, double* __restrict__ r,
                         GmresState* st)
{
    constexpr int R = rows_per_group<TB>();
    __shared__ TA ys[kMaxKrylov];
    if (st->done) return;
    const int m = st->final_iter;
    for (int i = threadIdx.x; i < m; i += kSolverBlock) ys[i] = TA(st->y[i] * st->sigma[i]);
    __syncthreads();
    const int64_t groups = ceildiv(n, R);
    for (int64_t grp = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; grp < groups;
         grp += int64_t(gridDim.x) * kSolverBlock) {
        const int64_t r0 = grp * R;
        const int valid = n - r0 < R ? int(n - r0) : R;
        if (m > 0) {
            TA u[R];
#pragma unroll
            for (int k = 0; k < R; ++k) u[k] = TA(0);
#pragma unroll 4
            for (int i = 0; i < m; ++i) {
                TA xv[R];
                load_basis<TA, TB, R>(V + int64_t(i) * ldv + r0, xv, valid);
                const TA yi = ys[i];
#pragma unroll
                for (int k = 0; k < R; ++k) u[k] += yi * xv[k];
            }
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (k < valid) {
                    const TA d = dinv ? dinv[r0 + k] : TA(1);
                    x[r0 + k] += double(d * u[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k < valid) r[r0 + k] = b[r0 + k];
        }
    }
}

// ||r||, ||b|| of r = b - A x, and V_0 = round_basis(r), y = D^-1 V_0 for
// the next cycle; the last block checks convergence and sets up the next
// cycle (the reference's restart step).
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_restart_kernel(int64_t n, const double* __restrict__ r,
                         const double* __restrict__ b, TB* __restrict__ V0,
                         const TA* __restrict__ dinv, TA* __restrict__ y,
                         GmresState* st, double* __restrict__ partials)
{
    constexpr bool kQ = BasisKind<TB>::kScaled;
    __shared__ double red[kSolverBlock / kWarp * 2];
    __shared__ double tot[2];
    __shared__ int last;
    if (st->done) return;
    double acc2[2] = {0.0, 0.0};
    double mx = 0.0;
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        const double rr = r[row], bb = b[row];
        acc2[0] += rr * rr;
        acc2[1] += bb * bb;
        if constexpr (kQ) {
            mx = fmax(mx, fabs(rr));  // V_0 is written by gmres_quantize_kernel
        } else {
            // the first basis vector of the next cycle, unnormalised
            // (sigma_0 = 1 / ||r||), and the first SpMV input
            const TB vb = to_basis<TB>(TA(rr));
            V0[row] = vb;
            const TA va = from_basis<TA>(vb);
            y[row] = dinv ? dinv[row] * va : va;
        }
    }
    if constexpr (kQ) {
#pragma unroll
        for (int off = 16; off > 0; off /= 2) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        __shared__ double mred[kSolverBlock / kWarp];
        if (threadIdx.x % kWarp == 0) mred[threadIdx.x / kWarp] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 1; k < kSolverBlock / kWarp; ++k) mx = fmax(mx, mred[k]);
            partials[2 * kSolverGrid + blockIdx.x] = mx;
        }
    }
    block_partials<double, 2>(acc2, partials, red);
    if (last_block_done(&st->ticket, &last)) {
        sum_partials<double, 2>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            st->ticket = 0;
            const double rn = sqrt(tot[0]);
            st->rnorm = rn;
            st->bnorm = sqrt(tot[1]);
            st->final_iter = 0;
            if (st->outer_iter == 0) {
                // the residual goal's baseline, fixed by the first residual
                // (stop::ResidualNorm, core/stop/residual_norm.cpp:95-150)
                st->base = st->baseline == B2S_BASELINE_INITIAL_RESNORM ? rn
                           : st->baseline == B2S_BASELINE_ABSOLUTE      ? 1.0
                                                                        : st->bnorm;
            }
            if (rn <= st->reduction * st->base) {
                st->converged = 1;
                st->done = 1;
                st->idle = 1;
            } else if (st->total_iter >= st->max_iters) {
                st->done = 1;
                st->idle = 1;
            } else {
                st->outer_iter += 1;
                st->j = 0;
                st->cycle_done = 0;
                st->idle = 0;
                st->g[0] = rn;
                for (int i = 1; i <= kMaxKrylov; ++i) st->g[i] = 0.0;
                st->sigma[0] = 1.0 / rn;
                if constexpr (kQ) {
                    double m = 0.0;
                    for (int b = 0; b < int(gridDim.x); ++b)
                        m = fmax(m, __ldcg(partials + 2 * kSolverGrid + b));
                    basis_scales<TB>(rn, m, &st->qscale, &st->sigma[0]);
                }
                st->inner_thresh = fmax(st->inner_reduction * rn,
                                        st->reduction * st->base);
            }
        }
    }
}

__global__ void float_copy_kernel(int64_t n, const double* __restrict__ src,
                                  float* __restrict__ dst)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i < n) dst[i] = float(src[i]);
}

// Leading dimension of the streamed vectors: a multiple of 64 rows.
inline int64_t gmres_ld(int64_t n) { return ceildiv(n, 64) * 64; }

// Width of the column-major (Ell) copy of A that the Arnoldi SpMV runs on,
// or 0 when its padding would exceed a quarter of nnz (then the Csr kernel
// runs on A itself).
inline int gmres_ell_width(int64_t n, int64_t nnz, int64_t max_row_nnz)
{
    if (max_row_nnz < 1 || max_row_nnz > (int64_t(1) << 20)) return 0;
    const int64_t padded = max_row_nnz * gmres_ld(n);
    return padded <= nnz + nnz / 4 ? int(max_row_nnz) : 0;
}

struct GmresLayout {
    int64_t bytes, off_st, off_r, off_w, off_y, off_v, off_partials,
        off_a32, off_d32, off_ell_c, off_ell_v, off_gpart, off_H, off_G,
        off_bcol, off_xcol, off_wq;
    int ell_width;
};

// cols: contiguous FP64 copies of one column of b and x, for strided or
// several right-hand sides (solved one column at a time)
template <typename TA, typename TB>
GmresLayout gmres_layout(int64_t n, int64_t nnz, int64_t max_row_nnz, int d, bool mixed,
                         bool cols)
{
    Carver c{nullptr};
    GmresLayout l;
    l.off_st = c.take<GmresState>(1);
    l.off_H = c.take<double>(int64_t(d) * (d + 1));
    l.off_G = c.take<double>(int64_t(d + 1) * (d + 1));
    l.off_bcol = cols ? c.take<double>(n) : 0;
    l.off_xcol = cols ? c.take<double>(n) : 0;
    l.off_r = c.take<double>(n);
    const int64_t ldv = gmres_ld(n);
    l.off_w = c.take<TA>(ldv);
    l.off_y = c.take<TA>(ldv);
    l.off_wq = BasisKind<TB>::kScaled ? c.take<TA>(ldv) : 0;
    l.off_v = c.take<TB>((int64_t(d) + 1) * ldv);
    l.off_partials = c.take<double>(int64_t(kSolverGrid) * 2 * kLd);
    l.off_gpart = c.take<double>(int64_t(kDotsMaxGroups) * 2 * kLd);
    l.ell_width = gmres_ell_width(n, nnz, max_row_nnz);
    l.off_a32 = mixed && l.ell_width == 0 ? c.take<float>(nnz) : 0;
    l.off_d32 = mixed ? c.take<float>(n) : 0;
    l.off_ell_c = l.ell_width ? c.take<int32_t>(int64_t(l.ell_width) * ldv) : 0;
    l.off_ell_v = l.ell_width ? c.take<TA>(int64_t(l.ell_width) * ldv) : 0;
    l.bytes = c.used;
    return l;
}

// One right-hand side (b, x contiguous FP64 vectors); the layout was
// checked against the workspace by the caller.
// ---------------------------------------------------------------------------
// Block Jacobi (right preconditioning by the block-diagonal inverse M): the
// SpMV input y = M V_{j+1} is no longer a row-wise scale, so the update,
// restart and quantize passes write y = V_{j+1} unscaled and
// gmres_block_apply_kernel applies M to it in place, one warp per group of
// the block-interleaved storage (every lane loads its row before the
// block's shuffles, so the in-place write is safe).  The cycle's solution
// update x += M V (sigma y) runs as gmres_xupdate_block_kernel, warp per
// group: the lanes form u = V (sigma y) for the group's rows, then M u by
// shuffles.  The blocks are FP64 in every variant; an FP32 Arnoldi cycle
// rounds M y to FP32.
// ---------------------------------------------------------------------------
// z = sum over c of M(i, c) v_c for the lane's row i of its block in group
// grp, v distributed one value per lane (column c of the block at lane
// base + c), the blocks read as load_block_columns reads them for SK.  Every
// lane takes part in the shuffles.
template <int SK, int MB2>
__device__ double block_times(const BlockPrec<double>& bp, const BlockScheme& bsc,
                              int64_t grp, int lane, bool in_group, int base, bool act, int bs,
                              double v)
{
    double z = 0.0;
    const double* gb = bp.blocks + grp * bsc.group;
    auto run = [&](auto kc) {
        constexpr int K = decltype(kc)::value;
#pragma unroll
        for (int c = 0; c < MB2; ++c) {
            if (c < bp.max_bs) {
                const double inv =
                    in_group ? load_reduced<K, double>(gb, lane + c * bsc.stride) : 0.0;
                const double vc = __shfl_sync(0xffffffffu, v, (base + c) % kWarp);
                if (act && c < bs) z += inv * vc;
            }
        }
    };
    if constexpr (SK == kSkMixed) {
        with_storage_kind(storage_kind<double>(bp.prec[grp * bsc.gs]), run);
    } else if constexpr (SK == kSkFull) {
        run(std::integral_constant<int, kFull>{});
    } else {
        run(std::integral_constant<int, SK>{});
    }
    return z;
}

template <typename TA, int MB2, int SK>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_block_apply_kernel(int64_t n, BlockPrec<double> bp, TA* __restrict__ y,
                             const int* __restrict__ skip)
{
    if (*skip) return;
    const BlockScheme bsc = block_scheme(bp.max_bs);
    const int lane = threadIdx.x % kWarp;
    const int sub = lane / bp.max_bs, i = lane % bp.max_bs;
    const bool in_group = lane < bsc.gs * bp.max_bs;
    const int base = sub * bp.max_bs;
    const int64_t ngroups = (bp.num_blocks + bsc.gs - 1) / bsc.gs;
    const int64_t nwarps = int64_t(gridDim.x) * (kSolverBlock / kWarp);
    for (int64_t grp = blockIdx.x * int64_t(kSolverBlock / kWarp) + threadIdx.x / kWarp;
         grp < ngroups; grp += nwarps) {
        const int64_t blk = grp * bsc.gs + sub;
        int s = 0, bs = 0;
        const bool in_block = in_group && blk < bp.num_blocks &&
                              block_extent(bp.ptrs, blk, n, bp.max_bs, s, bs);
        const bool act = in_block && i < bs;
        const double yv = act ? double(y[s + i]) : 0.0;
        const double z = block_times<SK, MB2>(bp, bsc, grp, lane, in_group, base, act, bs, yv);
        if (act) y[s + i] = TA(z);
    }
}

template <typename TA, typename TB, int MB2, int SK>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_xupdate_block_kernel(int64_t n, int64_t ldv, const TB* __restrict__ V,
                               BlockPrec<double> bp, double* __restrict__ x,
                               const double* __restrict__ b, double* __restrict__ r,
                               GmresState* st)
{
    __shared__ TA ys[kMaxKrylov];
    if (st->done) return;
    const int m = st->final_iter;
    for (int q = threadIdx.x; q < m; q += kSolverBlock) ys[q] = TA(st->y[q] * st->sigma[q]);
    __syncthreads();
    const BlockScheme bsc = block_scheme(bp.max_bs);
    const int lane = threadIdx.x % kWarp;
    const int sub = lane / bp.max_bs, i = lane % bp.max_bs;
    const bool in_group = lane < bsc.gs * bp.max_bs;
    const int base = sub * bp.max_bs;
    const int64_t ngroups = (bp.num_blocks + bsc.gs - 1) / bsc.gs;
    const int64_t nwarps = int64_t(gridDim.x) * (kSolverBlock / kWarp);
    for (int64_t grp = blockIdx.x * int64_t(kSolverBlock / kWarp) + threadIdx.x / kWarp;
         grp < ngroups; grp += nwarps) {
        const int64_t blk = grp * bsc.gs + sub;
        int s = 0, bs = 0;
        const bool in_block = in_group && blk < bp.num_blocks &&
                              block_extent(bp.ptrs, blk, n, bp.max_bs, s, bs);
        const bool act = in_block && i < bs;
        const int64_t row = s + i;
        TA u = TA(0);
        if (act) {
#pragma unroll 4
            for (int q = 0; q < m; ++q) u += ys[q] * from_basis<TA>(V[int64_t(q) * ldv + row]);
        }
        const double z =
            block_times<SK, MB2>(bp, bsc, grp, lane, in_group, base, act, bs, double(u));
        if (act) {
            if (m > 0) x[row] += z;
            r[row] = b[row];
        }
    }
}

// grid of the warp-per-group block kernels
inline int block_grid(const BlockPrec<double>& bp)
{
    const BlockScheme bsc = block_scheme(bp.max_bs);
    const int64_t ngroups = ceildiv(bp.num_blocks, bsc.gs);
    return int(std::min<int64_t>(std::max<int64_t>(1, ceildiv(ngroups, kSolverBlock / kWarp)),
                                 solver_grid()));
}

// Calls f(std::integral_constant<int, MB2>, std::integral_constant<int, SK>)
// for the block size class of bp and the way its blocks are read.
template <typename F>
void with_block_class(const BlockPrec<double>& bp, F&& f)
{
    with_pass_kind<double, true>(bp, [&](auto ap) {
        switch (kMaxBs / block_scheme(bp.max_bs).gs) {
        case 1: f(std::integral_constant<int, 1>{}, ap); break;
        case 2: f(std::integral_constant<int, 2>{}, ap); break;
        case 4: f(std::integral_constant<int, 4>{}, ap); break;
        case 8: f(std::integral_constant<int, 8>{}, ap); break;
        case 16: f(std::integral_constant<int, 16>{}, ap); break;
        default: f(std::integral_constant<int, 32>{}, ap); break;
        }
    });
}

template <typename TA, typename TB>
int gmres_engine(const GmresLayout& lay, int64_t n, int64_t nnz, const int32_t* rp,
                 const int32_t* ci, const double* v64, int64_t max_row_nnz,
                 const double* dinv64, const BlockPrec<double>* bp, const double* b,
                 double* x, int krylov_dim,
                 int ortho, int64_t max_iters, double reduction, int baseline,
                 double inner_reduction, void* workspace, int64_t* iterations,
                 int64_t* restarts, double* res_norm, uint8_t* status, cudaStream_t st)
{
    constexpr bool kMixed = !std::is_same<TA, double>::value;
    const int64_t ldv = gmres_ld(n);
    char* w = static_cast<char*>(workspace);
    auto* gs = reinterpret_cast<GmresState*>(w + lay.off_st);
    double* Hm = reinterpret_cast<double*>(w + lay.off_H);
    double* Gm = reinterpret_cast<double*>(w + lay.off_G);
    double* r = reinterpret_cast<double*>(w + lay.off_r);
    TA* wbuf = reinterpret_cast<TA*>(w + lay.off_w);
    TA* y = reinterpret_cast<TA*>(w + lay.off_y);
    TB* V = reinterpret_cast<TB*>(w + lay.off_v);
    constexpr bool kScaled = BasisKind<TB>::kScaled;
    TA* wq = kScaled ? reinterpret_cast<TA*>(w + lay.off_wq) : nullptr;
    double* partials = reinterpret_cast<double*>(w + lay.off_partials);
    double* gpart = reinterpret_cast<double*>(w + lay.off_gpart);
    const TA* va;
    const TA* da;
    if constexpr (kMixed) {
        float* a32 = reinterpret_cast<float*>(w + lay.off_a32);
        float* d32 = reinterpret_cast<float*>(w + lay.off_d32);
        if (nnz > 0 && lay.ell_width == 0) {
            float_copy_kernel<<<ceildiv(nnz, 256), 256, 0, st>>>(nnz, v64, a32);
            B2S_LAUNCH_CHECK();
        }
        if (dinv64) {
            float_copy_kernel<<<ceildiv(n, 256), 256, 0, st>>>(n, dinv64, d32);
            B2S_LAUNCH_CHECK();
        }
        va = a32;
        da = dinv64 ? d32 : nullptr;
    } else {
        va = v64;
        da = dinv64;
    }
    GmresState h{};
    h.max_iters = int(max_iters);
    h.krylov_dim = krylov_dim;
    h.ld = krylov_dim + 1;
    // modified Gram-Schmidt runs as CGS2: one pass over the basis per step
    // instead of j + 1, with orthogonality at least as good
    h.ortho = ortho == B2S_ORTHO_CGS ? B2S_ORTHO_CGS : B2S_ORTHO_CGS2;
    h.baseline = baseline;
    h.reduction = reduction;
    h.inner_reduction = inner_reduction;
    h.cycle_done = 1;
    h.idle = 1;
    h.minus_one = -1.0;
    h.one = 1.0;
    B2S_CUDA_TRY(cudaMemcpyAsync(gs, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    const int ell_w = lay.ell_width;
    int32_t* ell_c = reinterpret_cast<int32_t*>(w + lay.off_ell_c);
    TA* ell_v = reinterpret_cast<TA*>(w + lay.off_ell_v);
    // 16-bit column offsets when every |col - row| fits, else 32-bit columns
    bool ell16 = false;
    if (ell_w > 0) {
        ell_fill16_kernel<TA><<<ceildiv(ldv, 256), 256, 0, st>>>(
            n, ldv, ell_w, rp, ci, v64, reinterpret_cast<int16_t*>(ell_c), ell_v,
            &gs->too_long, &gs->too_far);
        B2S_LAUNCH_CHECK();
        int flags[2] = {0, 0};  // too_long, too_far
        B2S_CUDA_TRY(cudaMemcpyAsync(flags, &gs->too_long, sizeof(flags),
                                     cudaMemcpyDeviceToHost, st));
        B2S_CUDA_TRY(cudaStreamSynchronize(st));
        B2S_CHECK_ARG(!flags[0], "max_row_nnz (%lld) is smaller than the longest row",
                      (long long)max_row_nnz);
        ell16 = !flags[1];
        if (!ell16) {
            ell_fill_kernel<TA><<<ceildiv(ldv, 256), 256, 0, st>>>(
                n, ldv, ell_w, rp, ci, v64, ell_c, ell_v, &gs->too_long);
            B2S_LAUNCH_CHECK();
        }
    }
    constexpr int kEllRows = int(16 / sizeof(TA));
    const int ell_r = ell_rows_per_thread<TA>(ell_w);
    const int grid_ell = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(ceildiv(n, ell_r), 256)), int64_t(num_sms()) * 8));

    const int grid_vec = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n, kSolverBlock)), solver_grid()));
    // the update pass: one wave of resident blocks (it walks the row groups
    // with a grid stride), instead of a second, partial wave
    const int grid_upd = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(ceildiv(n, rows_per_group<TB>()), kSolverBlock)),
        std::min<int64_t>(solver_grid(), int64_t(update_min_blocks<TA, TB>()) * num_sms())));
    const int grid_dots = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(ceildiv(n, rows_per_group<TB>()), kSolverBlock)),
        std::min(kDotsMaxGrid, num_sms() * 4)));
    // pipelined SpMV: persistent grid, as many blocks as fit at once
    const int lpr = async_lanes_per_row(max_row_nnz);
    const int64_t async_need = ceildiv(ceildiv(n, kWarp / lpr), kAsyncBlock / kWarp);
    // x += D^-1 V y and r = b; r -= A x (FP64); ||r||, ||b|| and the check
    // block Jacobi: M applied to the SpMV input in place (skipped when the
    // cycle is over)
    auto block_apply = [&](cudaStream_t cs) {
        if (!bp) return;
        with_block_class(*bp, [&](auto mb, auto ap) {
            auto kernel = gmres_block_apply_kernel<TA, decltype(mb)::value, decltype(ap)::value>;
            kernel<<<pgrid(kernel, block_grid(*bp)), kSolverBlock, 0, cs>>>(n, *bp, y, &gs->idle);
        });
    };
    auto restart = [&](cudaStream_t cs) {
        if (bp) {
            with_block_class(*bp, [&](auto mb, auto ap) {
                auto kernel =
                    gmres_xupdate_block_kernel<TA, TB, decltype(mb)::value, decltype(ap)::value>;
                kernel<<<pgrid(kernel, block_grid(*bp)), kSolverBlock, 0, cs>>>(n, ldv, V, *bp,
                                                                                 x, b, r, gs);
            });
        } else {
            gmres_xupdate_kernel<TA, TB><<<pgrid(gmres_xupdate_kernel<TA, TB>, grid_vec), kSolverBlock, 0, cs>>>(n, ldv, V, da, x,
                                                                            b, r, gs);
        }
        with_async_kernel<double, 1, false>(lpr, [&](auto kernel) {
            const int64_t grid = std::min<int64_t>(async_need, async_resident_blocks(kernel));
            kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, v64, x, 1, r, 1,
                                                 &gs->minus_one, &gs->one, &gs->done);
        });
        gmres_restart_kernel<TA, TB><<<pgrid(gmres_restart_kernel<TA, TB>, grid_vec), kSolverBlock, 0, cs>>>(n, r, b, V, da, y,
                                                                        gs, partials);
        if constexpr (kScaled) {
            gmres_quantize_kernel<TA, TB, double><<<pgrid(gmres_quantize_kernel<TA, TB, double>, grid_vec), kSolverBlock, 0, cs>>>(
                n, ldv, r, V, da, y, gs, 1);
        }
        block_apply(cs);
    };
    // first residual outside the graph (final_iter = 0: x is not touched)
    restart(st);
    B2S_LAUNCH_CHECK();
    auto capture = [&](cudaStream_t cs) -> int {
        for (int j = 0; j < krylov_dim; ++j) {
            // y (the SpMV input) was written by the restart kernel (j = 0)
            // or by the previous step's update
            TA* dst = wbuf;
            if (ell_w > 0) {
                const int16_t* c16 = reinterpret_cast<const int16_t*>(ell_c);
                if (ell_r == kEllRows && ell16) {
                    ell_rows_kernel_for<TA, kEllRows, true, int16_t>()<<<grid_ell, 256, 0, cs>>>(
                        n, ell_w, ldv, c16, ell_v, y, 1, dst, 1, nullptr, nullptr, &gs->idle);
                } else if (ell_r == kEllRows) {
                    ell_rows_kernel_for<TA, kEllRows, true>()<<<grid_ell, 256, 0, cs>>>(
                        n, ell_w, ldv, ell_c, ell_v, y, 1, dst, 1, nullptr, nullptr,
                        &gs->idle);
                } else if (ell16) {
                    ell_rows_kernel_for<TA, 1, true, int16_t>()<<<grid_ell, 256, 0, cs>>>(
                        n, ell_w, ldv, c16, ell_v, y, 1, dst, 1, nullptr, nullptr, &gs->idle);
                } else {
                    ell_rows_kernel_for<TA, 1, true>()<<<grid_ell, 256, 0, cs>>>(
                        n, ell_w, ldv, ell_c, ell_v, y, 1, dst, 1, nullptr, nullptr,
                        &gs->idle);
                }
            } else {
                with_async_kernel<TA, 1, false>(lpr, [&](auto kernel) {
                    const int64_t grid = std::min<int64_t>(async_need,
                                                           async_resident_blocks(kernel));
                    kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, va, y, 1, dst, 1,
                                                         nullptr, nullptr, &gs->idle);
                });
            }
            gmres_dots_kernel<TA, TB><<<pgrid(gmres_dots_kernel<TA, TB>, grid_dots), kSolverBlock, 0, cs>>>(
                n, ldv, V, dst, gs, partials, gpart, Gm);
            gmres_update_kernel<TA, TB><<<pgrid(gmres_update_kernel<TA, TB>, grid_upd), kSolverBlock, 0, cs>>>(
                n, ldv, V, dst, da, y, gs, partials, Hm, wq);
            if constexpr (kScaled) {
                gmres_quantize_kernel<TA, TB, TA><<<pgrid(gmres_quantize_kernel<TA, TB, TA>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, ldv, wq, V, da, y, gs, 0);
            }
            block_apply(cs);
            B2S_LAUNCH_CHECK();
        }
        restart(cs);
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    };
    // every step: y -> spmv -> w -> dots, update -> V_{j+1}, y
    cudaStream_t cap;
    B2S_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = B2S_OK;
    do {
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { set_error("capture: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
        rc = capture(cap);
        e = cudaStreamEndCapture(cap, &graph);
        if (rc != B2S_OK) break;
        if (e != cudaSuccess) { set_error("capture: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) { set_error("instantiate: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
        // each cycle either finishes or advances >= 1 iteration
        const int64_t max_cycles = max_iters + 2;
        int done = 0;
        for (int64_t cyc = 0; cyc < max_cycles; ++cyc) {
            e = cudaMemcpyAsync(&done, &gs->done, sizeof(int),
                                cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) { set_error("replay: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
            if (done) break;
            e = cudaGraphLaunch(exec, st);
            if (e != cudaSuccess) { set_error("replay: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
        }
    } while (false);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    if (rc != B2S_OK) return rc;
    GmresState hs;
    B2S_CUDA_TRY(cudaMemcpyAsync(&hs, gs, sizeof(hs), cudaMemcpyDeviceToHost, st));
    B2S_CUDA_TRY(cudaStreamSynchronize(st));
    if (iterations) *iterations = hs.total_iter;
    if (restarts) *restarts = hs.outer_iter;
    if (res_norm) *res_norm = hs.rnorm;
    if (status) {
        uint8_t s = 0;
        if (hs.converged) {
            converge_status(s, kResidualId, true);
        } else {
            stop_status(s, kIterationId, true);
        }
        *status = s;
    }
    return B2S_OK;
}

// Validates the arguments, then solves the right-hand sides one column at a
// time (GMRES treats the columns independently: each has its own Krylov
// basis, Hessenberg matrix and stop status).  A column that is not a
// contiguous vector goes through FP64 copies in the workspace.
template <typename TA, typename TB>
int gmres_solve_columns(int64_t n, const int32_t* rp, const int32_t* ci,
                        const double* v64, int64_t max_row_nnz, const double* dinv64,
                        const BlockPrec<double>* bp,
                        const double* b, int64_t ldb, double* x, int64_t ldx,
                        int64_t k, int64_t krylov_dim, int ortho, int64_t max_iters,
                        double reduction, int baseline, double inner_reduction,
                        void* workspace, int64_t workspace_bytes, int64_t* iterations,
                        int64_t* restarts, double* res_norms, uint8_t* status,
                        void* stream)
{
    constexpr bool kMixed = !std::is_same<TA, double>::value;
    B2S_CHECK_ARG(n >= 1, "GMRES needs at least one row");
    B2S_CHECK_ARG(k >= 0, "negative number of right-hand sides");
    B2S_CHECK_ARG(krylov_dim >= 1 && krylov_dim <= kMaxKrylov,
                  "krylov_dim %lld is not supported: 1..%d", (long long)krylov_dim,
                  kMaxKrylov);
    B2S_CHECK_ARG(ortho == B2S_ORTHO_MGS || ortho == B2S_ORTHO_CGS || ortho == B2S_ORTHO_CGS2,
                  "unknown orthogonalisation method %d", ortho);
    B2S_CHECK_ARG(baseline == B2S_BASELINE_RHS_NORM ||
                      baseline == B2S_BASELINE_INITIAL_RESNORM ||
                      baseline == B2S_BASELINE_ABSOLUTE,
                  "unknown residual baseline %d", baseline);
    B2S_CHECK_ARG(max_iters >= 0 && max_iters < (int64_t(1) << 30),
                  "max_iters out of range");
    B2S_CHECK_ARG(k <= 1 || (ldb >= k && ldx >= k), "leading dimensions below num_rhs");
    if (bp) {
        B2S_CHECK_ARG(bp->max_bs >= 1 && bp->max_bs <= kMaxBs,
                      "max_block_size must be 1..32");
        B2S_CHECK_ARG(bp->num_blocks >= 1 && bp->ptrs && bp->blocks,
                      "block preconditioner without blocks");
        B2S_CHECK_ARG(dinv64 == nullptr, "scalar and block Jacobi together");
    }
    if (k == 0) return B2S_OK;
    B2S_CHECK_ARG(b != nullptr && x != nullptr && rp != nullptr, "null pointer");
    cudaStream_t st = as_stream(stream);
    int64_t nnz = 0;
    {
        int32_t h_nnz = 0;
        B2S_CUDA_TRY(cudaMemcpyAsync(&h_nnz, rp + n, sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, st));
        B2S_CUDA_TRY(cudaStreamSynchronize(st));
        nnz = h_nnz;
    }
    const bool cols = k > 1 || ldb != 1 || ldx != 1;
    const GmresLayout lay =
        gmres_layout<TA, TB>(n, nnz, max_row_nnz, int(krylov_dim), kMixed, cols);
    if (workspace_bytes < lay.bytes) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)lay.bytes);
        return B2S_ERR_WORKSPACE;
    }
    B2S_CHECK_ARG(reinterpret_cast<uintptr_t>(workspace) % 256 == 0,
                  "GMRES workspace must be 256-byte aligned");
    char* w = static_cast<char*>(workspace);
    double* bcol = cols ? reinterpret_cast<double*>(w + lay.off_bcol) : nullptr;
    double* xcol = cols ? reinterpret_cast<double*>(w + lay.off_xcol) : nullptr;
    for (int64_t c = 0; c < k; ++c) {
        const double* bc = b + c;
        double* xc = x + c;
        if (cols) {
            B2S_CUDA_TRY(cudaMemcpy2DAsync(bcol, sizeof(double), b + c, ldb * sizeof(double),
                                           sizeof(double), n, cudaMemcpyDeviceToDevice, st));
            B2S_CUDA_TRY(cudaMemcpy2DAsync(xcol, sizeof(double), x + c, ldx * sizeof(double),
                                           sizeof(double), n, cudaMemcpyDeviceToDevice, st));
            bc = bcol;
            xc = xcol;
        }
        const int rc = gmres_engine<TA, TB>(
            lay, n, nnz, rp, ci, v64, max_row_nnz, dinv64, bp, bc, xc, int(krylov_dim), ortho,
            max_iters, reduction, baseline, inner_reduction, workspace,
            iterations ? iterations + c : nullptr, restarts ? restarts + c : nullptr,
            res_norms ? res_norms + c : nullptr, status ? status + c : nullptr, st);
        if (rc != B2S_OK) return rc;
        if (cols) {
            B2S_CUDA_TRY(cudaMemcpy2DAsync(x + c, ldx * sizeof(double), xcol, sizeof(double),
                                           sizeof(double), n, cudaMemcpyDeviceToDevice, st));
        }
    }
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int64_t b2s_gmres_workspace_bytes(int64_t num_rows, int64_t nnz,
                                  int64_t max_row_nnz, int64_t num_rhs,
                                  int64_t krylov_dim, int variant)
{
    if (num_rows < 1 || num_rhs < 0 || krylov_dim < 1 || krylov_dim > kMaxKrylov) return -1;
    // strided or several columns go through contiguous copies; the solve
    // decides by the leading dimensions, so a single column reserves them too
    const bool cols = true;
    const int d = int(krylov_dim);
    switch (variant) {
    case B2S_GMRES_F64:
        return gmres_layout<double, double>(num_rows, nnz, max_row_nnz, d, false, cols).bytes;
    case B2S_GMRES_MIXED_F32:
        return gmres_layout<float, float>(num_rows, nnz, max_row_nnz, d, true, cols).bytes;
    case B2S_GMRES_MIXED_BF16:
        return gmres_layout<float, __nv_bfloat16>(num_rows, nnz, max_row_nnz, d, true, cols)
            .bytes;
    case B2S_GMRES_CB_F32:
        return gmres_layout<double, float>(num_rows, nnz, max_row_nnz, d, false, cols).bytes;
    case B2S_GMRES_CB_F16:
        return gmres_layout<double, __half>(num_rows, nnz, max_row_nnz, d, false, cols).bytes;
    case B2S_GMRES_CB_I64:
        return gmres_layout<double, int64_t>(num_rows, nnz, max_row_nnz, d, false, cols).bytes;
    case B2S_GMRES_CB_I32:
        return gmres_layout<double, int32_t>(num_rows, nnz, max_row_nnz, d, false, cols).bytes;
    case B2S_GMRES_CB_I16:
        return gmres_layout<double, int16_t>(num_rows, nnz, max_row_nnz, d, false, cols).bytes;
    default:
        return -1;
    }
}

}  // extern "C"

namespace b2s {
namespace {

int gmres_dispatch(int variant, int ortho_method, int64_t num_rows, const int32_t* row_ptrs,
                   const int32_t* col_idxs, const double* values, int64_t max_row_nnz,
                   const double* inv_diag, const BlockPrec<double>* bp, const double* b,
                   int64_t ldb, double* x, int64_t ldx, int64_t num_rhs, int64_t krylov_dim,
                   int64_t max_iters, double reduction_factor, int baseline,
                   double inner_reduction, void* workspace, int64_t workspace_bytes,
                   int64_t* iterations, int64_t* restarts, double* residual_norms,
                   uint8_t* status, void* stream)
{
#define B2S_GMRES_ARGS(INNER)                                                          \
    num_rows, row_ptrs, col_idxs, values, max_row_nnz, inv_diag, bp, b, ldb, x, ldx,  \
        num_rhs, krylov_dim, ortho_method, max_iters, reduction_factor, baseline,     \
        INNER, workspace, workspace_bytes, iterations, restarts, residual_norms,      \
        status, stream
    switch (variant) {
    case B2S_GMRES_F64:
        return gmres_solve_columns<double, double>(B2S_GMRES_ARGS(0.0));
    case B2S_GMRES_MIXED_F32:
        return gmres_solve_columns<float, float>(B2S_GMRES_ARGS(inner_reduction));
    case B2S_GMRES_MIXED_BF16:
        return gmres_solve_columns<float, __nv_bfloat16>(B2S_GMRES_ARGS(inner_reduction));
    case B2S_GMRES_CB_F32:
        // FP64 arithmetic over an FP32 basis: the plain (non-refinement)
        // engine; its row groups follow the basis type (4 rows, 16 bytes
        // of basis and 32 of FP64 vectors per load)
        return gmres_solve_columns<double, float>(B2S_GMRES_ARGS(0.0));
    // the other CB-GMRES storage formats: FP64 arithmetic over a basis
    // stored scaled (half: normalised; integers: per-vector scale)
    case B2S_GMRES_CB_F16:
        return gmres_solve_columns<double, __half>(B2S_GMRES_ARGS(0.0));
    case B2S_GMRES_CB_I64:
        return gmres_solve_columns<double, int64_t>(B2S_GMRES_ARGS(0.0));
    case B2S_GMRES_CB_I32:
        return gmres_solve_columns<double, int32_t>(B2S_GMRES_ARGS(0.0));
    case B2S_GMRES_CB_I16:
        return gmres_solve_columns<double, int16_t>(B2S_GMRES_ARGS(0.0));
    default:
        set_error("unknown GMRES variant %d", variant);
        return B2S_ERR_INVALID_ARG;
    }
#undef B2S_GMRES_ARGS
}

}  // namespace
}  // namespace b2s

extern "C" {

int b2s_gmres_solve(int variant, int ortho_method, int64_t num_rows,
                    const int32_t* row_ptrs, const int32_t* col_idxs,
                    const double* values, int64_t max_row_nnz,
                    const double* inv_diag, const double* b, int64_t ldb,
                    double* x, int64_t ldx, int64_t num_rhs,
                    int64_t krylov_dim, int64_t max_iters,
                    double reduction_factor, int baseline,
                    double inner_reduction, void* workspace,
                    int64_t workspace_bytes, int64_t* iterations,
                    int64_t* restarts, double* residual_norms,
                    uint8_t* status, void* stream)
{
    return gmres_dispatch(variant, ortho_method, num_rows, row_ptrs, col_idxs, values,
                          max_row_nnz, inv_diag, nullptr, b, ldb, x, ldx, num_rhs,
                          krylov_dim, max_iters, reduction_factor, baseline, inner_reduction,
                          workspace, workspace_bytes, iterations, restarts, residual_norms,
                          status, stream);
}

int b2s_gmres_block_solve(int variant, int ortho_method, int64_t num_rows,
                          const int32_t* row_ptrs, const int32_t* col_idxs,
                          const double* values, int64_t max_row_nnz, int64_t num_blocks,
                          const int32_t* block_ptrs, int max_block_size,
                          const uint8_t* block_precisions, const double* blocks,
                          const double* b, int64_t ldb, double* x,
                          int64_t ldx, int64_t num_rhs, int64_t krylov_dim,
                          int64_t max_iters, double reduction_factor, int baseline,
                          double inner_reduction, void* workspace,
                          int64_t workspace_bytes, int64_t* iterations,
                          int64_t* restarts, double* residual_norms, uint8_t* status,
                          void* stream)
{
    BlockPrec<double> bp;
    bp.num_blocks = num_blocks;
    bp.ptrs = block_ptrs;
    bp.max_bs = max_block_size;
    bp.blocks = blocks;
    bp.prec = block_precisions;
    if (bp.prec && workspace && workspace_bytes >= int64_t(sizeof(int))) {
        // the workspace's first word as scratch, before the solve
        B2S_CUDA_TRY(resolve_storage_kind(bp, static_cast<int*>(workspace), as_stream(stream)));
    }
    return gmres_dispatch(variant, ortho_method, num_rows, row_ptrs, col_idxs, values,
                          max_row_nnz, nullptr, &bp, b, ldb, x, ldx, num_rhs, krylov_dim,
                          max_iters, reduction_factor, baseline, inner_reduction, workspace,
                          workspace_bytes, iterations, restarts, residual_norms, status,
                          stream);
}

}  // extern "C"
