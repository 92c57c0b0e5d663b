// Fused preconditioned CG (scalar Jacobi, block Jacobi or identity), the loop of
// core/solver/cg.cpp:91-189 with the kernels of
// common/unified/solver/cg_kernels.cpp:23-107 regrouped into two passes per
// iteration and no host synchronisation inside the loop:
//
//   spmv pass   p' = z + (rho / prev_rho) p  with z = D^-1 r, formed on the
//               fly for every column index the SpMV touches (p is double
//               buffered, so every row reads the old p); q = A p';
//               dot(p', q) reduced in-kernel; the last block sets
//               alpha = rho / dot(p', q)  (step_1 + SpMV + dot)
//   update pass x += alpha p', r -= alpha q; rho' = dot(r, D^-1 r) and
//               ||r||^2 reduced in-kernel; the last block advances the
//               iteration, swaps rho, and applies the Iteration and
//               ResidualNorm(rhs_norm) checks  (step_2 + precond + 2 dots +
//               residual_norm check)
//
// With four or more right-hand sides (FP64; eight or more in FP32) the same
// two passes run with lanes owning 16-byte column slices of each row; with
// one right-hand side on a system of 2^19 rows or more the SpMV pass is
// split so that the matrix streams through the pipelined Csr kernel.
//
// With scalar Jacobi z is never stored.  A block Jacobi preconditioner
// stores z = M^-1 r, formed in the update pass (see cg_block_kernel), and
// the SpMV passes read it in place of D^-1 r.  Per-column stopping status
// uses the reference's bit
// layout; stopped columns are frozen as in the reference.  The host replays
// a CUDA graph of `check_every` iterations and reads the stop flag once per
// replay.
#include <cstring>

#include "csr_async.cuh"
#include "jacobi_scheme.cuh"
#include "solver_common.cuh"

namespace b2s {
namespace {

template <typename T>
struct CgScalars {
    T rho[kMaxRhs], prev_rho[kMaxRhs], alpha[kMaxRhs], tau[kMaxRhs],
        start[kMaxRhs];
};

template <typename T>
__device__ __forceinline__ T cg_p(T d, T r, T beta, T p, bool from_z)
{
    const T z = mul_rn(d, r);
    return from_z ? z : add_rn(z, mul_rn(beta, p));
}

// The last block's part of the initial pass (thread 0): tot holds ||b||^2,
// rho = dot(r, z) and ||r||^2 of every column (K each); sets the starting
// norms, rho and the initial stopping status.
template <typename T, int K>
__device__ void cg_init_finish(const T* tot, int k, SolveCtl* ctl, CgScalars<T>* sc)
{
    ctl->ticket = 0;
    ctl->iter = 0;
    int all = 1;
    for (int j = 0; j < K; ++j) {
        uint8_t s = 0;
        if (j >= k) {
            stop_status(s, kIterationId, true);  // padding column
        }
        sc->start[j] = start_norm(ctl, T(sqrt(tot[j])), T(sqrt(tot[2 * K + j])));
        sc->rho[j] = tot[K + j];
        sc->prev_rho[j] = T(1);
        sc->alpha[j] = T(0);
        sc->tau[j] = sqrt(tot[2 * K + j]);
        if (ctl->max_iters <= 0) stop_status(s, kIterationId, true);
        if (residual_met(ctl, sc->tau[j], sc->rho[j], sc->start[j])) {
            converge_status(s, kResidualId, true);
        }
        ctl->status[j] = s;
        all &= has_stopped(s);
    }
    ctl->all_stopped = all;
}

// The last block's part of the update pass (thread 0): tot holds the new
// rho = dot(r, z) and ||r||^2 per column; advances the iteration, swaps rho
// and applies the Iteration and residual checks.
template <typename T, int K>
__device__ void cg_update_finish(const T* tot, SolveCtl* ctl, CgScalars<T>* sc)
{
    ctl->ticket = 0;
    const int iter = ctl->iter + 1;
    ctl->iter = iter;
    int all = 1;
    for (int j = 0; j < K; ++j) {
        uint8_t s = ctl->status[j];
        if (!has_stopped(s)) {
            sc->prev_rho[j] = sc->rho[j];
            sc->rho[j] = tot[j];
            sc->tau[j] = sqrt(tot[K + j]);
            if (residual_met(ctl, sc->tau[j], sc->rho[j], sc->start[j])) {
                converge_status(s, kResidualId, true);
            }
            if (iter >= ctl->max_iters) stop_status(s, kIterationId, true);
            ctl->status[j] = s;
        }
        all &= has_stopped(s);
    }
    ctl->all_stopped = all;
}

template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    cg_init_kernel(int64_t n, const T* __restrict__ dinv,
                   const T* __restrict__ b, int64_t ldb, int k,
                   const T* __restrict__ r, T* __restrict__ p_old,
                   SolveCtl* ctl, CgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * 3 * K];
    __shared__ T tot[3 * K];
    __shared__ int last;
    T acc[3 * K];
#pragma unroll
    for (int j = 0; j < 3 * K; ++j) acc[j] = T(0);
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T d = dinv ? dinv[i] : T(1);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const T rr = r[i * K + j];
            const T bb = j < k ? b[i * ldb + j] : T(0);
            p_old[i * K + j] = T(0);
            acc[j] += bb * bb;
            acc[K + j] += rr * mul_rn(d, rr);
            acc[2 * K + j] += rr * rr;
        }
    }
    block_partials<T, 3 * K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 3 * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) cg_init_finish<T, K>(tot, k, ctl, sc);
    }
}

template <typename T, int SW, int K>
__global__ void __launch_bounds__(kSolverBlock)
    cg_spmv_kernel(int64_t n, const int32_t* __restrict__ rp,
                   const int32_t* __restrict__ ci, const T* __restrict__ v,
                   const T* __restrict__ dinv, const T* __restrict__ r,
                   const T* __restrict__ p_old, T* __restrict__ p_new,
                   T* __restrict__ q, SolveCtl* ctl, CgScalars<T>* sc,
                   T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * K];
    __shared__ T tot[K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    bool active[K], from_z[K];
    T beta[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = !has_stopped(ctl->status[j]);
        const T pr = sc->prev_rho[j];
        from_z[j] = pr == T(0);
        beta[j] = from_z[j] ? T(0) : sc->rho[j] / pr;
    }
    T dot[K];
#pragma unroll
    for (int j = 0; j < K; ++j) dot[j] = T(0);
    const int lane = threadIdx.x % SW;
    const int64_t nsub = int64_t(gridDim.x) * kSolverBlock / SW;
    // warp-uniform trip count: all lanes of a warp run every iteration, so
    // the subwarp shuffles below always see the whole warp
    for (int64_t wbase = (blockIdx.x * int64_t(kSolverBlock) + threadIdx.x) /
                         kWarp * (kWarp / SW);
         wbase < n; wbase += nsub) {
        const int64_t row = wbase + (threadIdx.x % kWarp) / SW;
        const bool valid = row < n;
        T acc[K];
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = T(0);
        const int end = valid ? rp[row + 1] : 0;
        for (int e = (valid ? rp[row] : end) + lane; e < end; e += SW) {
            const T a = v[e];
            const int64_t c = ci[e];
            const T d = dinv ? dinv[c] : T(1);
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (active[j]) {
                    acc[j] += a * cg_p(d, r[c * K + j], beta[j], p_old[c * K + j],
                                       from_z[j]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = subwarp_sum<SW>(acc[j]);
        if (valid && lane == 0) {
            const T d = dinv ? dinv[row] : T(1);
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (active[j]) {
                    const T pn = cg_p(d, r[row * K + j], beta[j],
                                      p_old[row * K + j], from_z[j]);
                    p_new[row * K + j] = pn;
                    q[row * K + j] = acc[j];
                    dot[j] += pn * acc[j];
                }
            }
        }
    }
    block_partials<T, K>(dot, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, K>(partials, gridDim.x, tot, red);
        if (threadIdx.x < K) {
            const T pq = tot[threadIdx.x];
            // step_2 skips the update when dot(p, q) == 0
            sc->alpha[threadIdx.x] = pq != T(0) ? sc->rho[threadIdx.x] / pq : T(0);
        }
        if (threadIdx.x == 0) ctl->ticket = 0;
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    cg_update_kernel(int64_t n, const T* __restrict__ dinv, T* __restrict__ x,
                     int64_t ldx, T* __restrict__ r, const T* __restrict__ p,
                     const T* __restrict__ q, SolveCtl* ctl, CgScalars<T>* sc,
                     T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * 2 * K];
    __shared__ T tot[2 * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    bool active[K];
    T alpha[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = !has_stopped(ctl->status[j]);
        alpha[j] = sc->alpha[j];
    }
    T acc[2 * K];
#pragma unroll
    for (int j = 0; j < 2 * K; ++j) acc[j] = T(0);
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T d = dinv ? dinv[i] : T(1);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (active[j]) {
                x[i * ldx + j] += alpha[j] * p[i * K + j];
                const T rr = r[i * K + j] - alpha[j] * q[i * K + j];
                r[i * K + j] = rr;
                acc[j] += rr * mul_rn(d, rr);
                acc[K + j] += rr * rr;
            }
        }
    }
    block_partials<T, 2 * K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 2 * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) cg_update_finish<T, K>(tot, ctl, sc);
    }
}

// ---------------------------------------------------------------------------
// Four or more right-hand sides: lanes own columns.  A row's KL = K / VW
// lanes each hold VW = 16 / sizeof(T) consecutive columns (one 16-byte
// vector of the row-major n x K blocks), so the gathers of r(c, :) and
// p(c, :) are contiguous 16-byte loads across the row's lanes and no
// shuffle reduction runs per row.  Stopped columns are computed along
// (their results are never used: the update pass freezes them).
// ---------------------------------------------------------------------------

template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    cg_spmv_lanes_kernel(int64_t n, const int32_t* __restrict__ rp,
                         const int32_t* __restrict__ ci, const T* __restrict__ v,
                         const T* __restrict__ dinv, const T* __restrict__ r,
                         const T* __restrict__ p_old, T* __restrict__ p_new,
                         T* __restrict__ q, SolveCtl* ctl, CgScalars<T>* sc,
                         T* __restrict__ partials)
{
    constexpr int VW = int(16 / sizeof(T));
    constexpr int KL = K / VW;         // lanes per row
    constexpr int RPW = kWarp / KL;    // rows per warp
    constexpr int W = kSolverBlock / kWarp;
    __shared__ T red[W][K];
    __shared__ T tot[K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const int col0 = (lane % KL) * VW;
    bool from_z[VW];
    T beta[VW];
#pragma unroll
    for (int u = 0; u < VW; ++u) {
        const T pr = sc->prev_rho[col0 + u];
        from_z[u] = pr == T(0);
        beta[u] = from_z[u] ? T(0) : sc->rho[col0 + u] / pr;
    }
    T dot[VW];
#pragma unroll
    for (int u = 0; u < VW; ++u) dot[u] = T(0);
    const int64_t nwarps = int64_t(gridDim.x) * W;
    for (int64_t g = blockIdx.x * int64_t(W) + wid; g * RPW < n; g += nwarps) {
        const int64_t row = g * RPW + lane / KL;
        if (row < n) {
            T acc[VW];
#pragma unroll
            for (int u = 0; u < VW; ++u) acc[u] = T(0);
            const int end = rp[row + 1];
            for (int e = rp[row]; e < end; ++e) {
                const T a = v[e];
                const int64_t c = ci[e];
                const T d = dinv ? dinv[c] : T(1);
                T rr[VW], pp[VW];
                ld_vec<T, VW>(r + c * K + col0, rr);
                ld_vec<T, VW>(p_old + c * K + col0, pp);
#pragma unroll
                for (int u = 0; u < VW; ++u) acc[u] += a * cg_p(d, rr[u], beta[u], pp[u], from_z[u]);
            }
            const T d = dinv ? dinv[row] : T(1);
            T rr[VW], pp[VW], pn[VW];
            ld_vec<T, VW>(r + row * K + col0, rr);
            ld_vec<T, VW>(p_old + row * K + col0, pp);
#pragma unroll
            for (int u = 0; u < VW; ++u) {
                pn[u] = cg_p(d, rr[u], beta[u], pp[u], from_z[u]);
                dot[u] += pn[u] * acc[u];
            }
            st_vec<T, VW>(p_new + row * K + col0, pn);
            st_vec<T, VW>(q + row * K + col0, acc);
        }
    }
    // lanes with the same columns: xor over the row bits of the lane index
#pragma unroll
    for (int off = KL; off < kWarp; off *= 2) {
#pragma unroll
        for (int u = 0; u < VW; ++u) dot[u] += __shfl_xor_sync(0xffffffffu, dot[u], off);
    }
    if (lane < KL) {
#pragma unroll
        for (int u = 0; u < VW; ++u) red[wid][col0 + u] = dot[u];
    }
    __syncthreads();
    if (threadIdx.x < K) {
        T s = T(0);
        for (int k = 0; k < W; ++k) s += red[k][threadIdx.x];
        partials[blockIdx.x * K + threadIdx.x] = s;
    }
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, K>(partials, gridDim.x, tot, reinterpret_cast<T*>(red));
        if (threadIdx.x < K) {
            const T pq = tot[threadIdx.x];
            sc->alpha[threadIdx.x] = pq != T(0) ? sc->rho[threadIdx.x] / pq : T(0);
        }
        if (threadIdx.x == 0) ctl->ticket = 0;
    }
}

// x += alpha p, r -= alpha q over the row-major n x K blocks as one flat
// array of 16-byte vectors (a thread keeps the same VW columns: the grid
// stride is a multiple of K); rho' = dot(r, D^-1 r) and ||r||^2 per column.
template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    cg_update_lanes_kernel(int64_t n, const T* __restrict__ dinv, T* __restrict__ x,
                           int64_t ldx, T* __restrict__ r, const T* __restrict__ p,
                           const T* __restrict__ q, SolveCtl* ctl, CgScalars<T>* sc,
                           T* __restrict__ partials)
{
    constexpr int VW = int(16 / sizeof(T));
    constexpr int KL = K / VW;
    constexpr int W = kSolverBlock / kWarp;
    __shared__ T red[W][2 * K];
    __shared__ T tot[2 * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const int64_t t0 = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x;
    const int col0 = int((t0 * VW) % K);
    bool active[VW];
    T alpha[VW];
#pragma unroll
    for (int u = 0; u < VW; ++u) {
        active[u] = !has_stopped(ctl->status[col0 + u]);
        alpha[u] = sc->alpha[col0 + u];
    }
    T acc[2 * VW];
#pragma unroll
    for (int u = 0; u < 2 * VW; ++u) acc[u] = T(0);
    const int64_t nvec = n * K / VW;
    for (int64_t t = t0; t < nvec; t += int64_t(gridDim.x) * kSolverBlock) {
        const int64_t i = t * VW / K;
        const T d = dinv ? dinv[i] : T(1);
        T pv[VW], qv[VW], rv[VW];
        ld_vec<T, VW>(p + t * VW, pv);
        ld_vec<T, VW>(q + t * VW, qv);
        ld_vec<T, VW>(r + t * VW, rv);
#pragma unroll
        for (int u = 0; u < VW; ++u) {
            if (active[u]) {
                x[i * ldx + col0 + u] += alpha[u] * pv[u];
                const T rr = rv[u] - alpha[u] * qv[u];
                rv[u] = rr;
                acc[u] += rr * mul_rn(d, rr);
                acc[VW + u] += rr * rr;
            }
        }
        st_vec<T, VW>(r + t * VW, rv);
    }
#pragma unroll
    for (int off = KL; off < kWarp; off *= 2) {
#pragma unroll
        for (int u = 0; u < 2 * VW; ++u) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], off);
    }
    if (lane < KL) {
#pragma unroll
        for (int u = 0; u < VW; ++u) {
            red[wid][col0 + u] = acc[u];
            red[wid][K + col0 + u] = acc[VW + u];
        }
    }
    __syncthreads();
    // partials: rho parts [block][K], then ||r||^2 parts [block][K] (two
    // K-wide sums keep the last block's register use low)
    if (threadIdx.x < 2 * K) {
        T s = T(0);
        for (int k = 0; k < W; ++k) s += red[k][threadIdx.x];
        const int j = threadIdx.x % K;
        partials[(threadIdx.x < K ? 0 : int64_t(gridDim.x) * K) + blockIdx.x * K + j] = s;
    }
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, K>(partials, gridDim.x, tot, reinterpret_cast<T*>(red));
        sum_partials<T, K>(partials + int64_t(gridDim.x) * K, gridDim.x, tot + K,
                           reinterpret_cast<T*>(red));
        if (threadIdx.x == 0) cg_update_finish<T, K>(tot, ctl, sc);
    }
}

// ---------------------------------------------------------------------------
// One right-hand side on a large system: the SpMV pass is split in three so
// the matrix streams through the pipelined Csr kernel (one x gather per
// stored entry instead of forming p' = D^-1 r + beta p at every gathered
// column, which triples the gathers once the vectors no longer sit in L2):
//   cg_pupdate_kernel  p' = cg_p(...)   (the same rounding as the fused pass)
//   csr_async_kernel   q = A p'
//   cg_pq_kernel       dot(p', q); the last block sets alpha
// ---------------------------------------------------------------------------
constexpr int64_t kCgSplitRows = int64_t(1) << 19;

template <typename T>
__global__ void __launch_bounds__(kSolverBlock)
    cg_pupdate_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r,
                      const T* __restrict__ p_old, T* __restrict__ p_new,
                      SolveCtl* ctl, CgScalars<T>* sc)
{
    if (ctl->all_stopped) return;
    const T pr = sc->prev_rho[0];
    const bool from_z = pr == T(0);
    const T beta = from_z ? T(0) : sc->rho[0] / pr;
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T d = dinv ? dinv[i] : T(1);
        p_new[i] = cg_p(d, r[i], beta, p_old[i], from_z);
    }
}

template <typename T>
__global__ void __launch_bounds__(kSolverBlock)
    cg_pq_kernel(int64_t n, const T* __restrict__ p, const T* __restrict__ q,
                 SolveCtl* ctl, CgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp];
    __shared__ T tot[1];
    __shared__ int last;
    if (ctl->all_stopped) return;
    T acc[1] = {T(0)};
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        acc[0] += p[i] * q[i];
    }
    block_partials<T, 1>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 1>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            const T pq = tot[0];
            // step_2 skips the update when dot(p, q) == 0
            sc->alpha[0] = pq != T(0) ? sc->rho[0] / pq : T(0);
            ctl->ticket = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Block Jacobi: z = M^-1 r is no longer a row-wise scale, so it is stored.
// The SpMV passes above run with z in place of r and no diagonal
// (p' = z + beta p); the update pass below (and the initial one, INIT)
// runs one warp per group of the block-interleaved storage, lane (sub, i)
// owning row i of block sub of the group: r -= alpha q and x += alpha p'
// for the lane's row, then z of the row from the block's new residual,
// which the block's lanes pass along by shuffles (inverse columns in the
// order of apply_block, reference/preconditioner/jacobi_kernels.cpp:
// 419-445), and dot(r, z), ||r||^2.  INIT additionally zeroes p and sums
// ||b||^2 (cg::initialize and the first z = M r, core/solver/cg.cpp:
// 122-149).
// ---------------------------------------------------------------------------
// A fixed storage kind widens its loads in registers; holding those
// instances to five blocks per SM keeps them at the full-precision pass's 48
// registers (64 otherwise); a minimum of 0 leaves the others unconstrained.
template <typename T, int MB2, int K, bool INIT, int SK>
__global__ void __launch_bounds__(kSolverBlock, (MB2 > 8 ? 0 : SK == kF16 ? 6 : SK >= 0 ? 5 : 0))
    cg_block_kernel(int64_t n, BlockPrec<T> bp, const T* __restrict__ b, int64_t ldb, int k,
                    T* __restrict__ x, int64_t ldx, T* __restrict__ r, T* __restrict__ z,
                    T* __restrict__ p, const T* __restrict__ q, SolveCtl* ctl,
                    CgScalars<T>* sc, T* __restrict__ partials)
{
    constexpr int NS = INIT ? 3 : 2;  // sums per column
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ T red[kSolverBlock / kWarp * NS * K];
    __shared__ T tot[NS * K];
    __shared__ int last;
    if (!INIT && ctl->all_stopped) return;
    bool active[K];
    T alpha[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = INIT || !has_stopped(ctl->status[j]);
        alpha[j] = INIT ? T(0) : sc->alpha[j];
    }
    T acc[NS * K];
#pragma unroll
    for (int j = 0; j < NS * K; ++j) acc[j] = T(0);
    const BlockScheme bsc = block_scheme(bp.max_bs);
    const int lane = threadIdx.x % kWarp;
    const int sub = lane / bp.max_bs, i = lane % bp.max_bs;
    const bool in_group = lane < bsc.gs * bp.max_bs;
    const int base = sub * bp.max_bs;  // first lane of this lane's block
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
        BlockRow<SK, MB2, T> inv;
        inv.load(bp, bsc, grp, lane, in_group);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            T rn = T(0);
            if (act) {
                if (INIT) {
                    rn = r[row * K + j];
                    p[row * K + j] = T(0);
                    const T bb = j < k ? b[row * ldb + j] : T(0);
                    acc[j] += bb * bb;
                } else if (active[j]) {
                    x[row * ldx + j] += alpha[j] * p[row * K + j];
                    rn = r[row * K + j] - alpha[j] * q[row * K + j];
                    r[row * K + j] = rn;
                }
            }
            if (!active[j]) continue;  // uniform: a frozen column keeps its z
            T zz = T(0);
#pragma unroll
            for (int c = 0; c < MB2; ++c) {
                if (c < bp.max_bs) {
                    const T rc = __shfl_sync(kFull, rn, (base + c) % kWarp);
                    if (act && c < bs) zz += inv[c] * rc;
                }
            }
            if (act) {
                z[row * K + j] = zz;
                acc[(NS - 2) * K + j] += rn * zz;
                acc[(NS - 1) * K + j] += rn * rn;
            }
        }
    }
    block_partials<T, NS * K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, NS * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            if constexpr (INIT) {
                cg_init_finish<T, K>(tot, k, ctl, sc);
            } else {
                cg_update_finish<T, K>(tot, ctl, sc);
            }
        }
    }
}

// Launches cg_block_kernel for the block size class of bp.
template <typename T, int K, bool INIT>
void launch_cg_block(int64_t n, const BlockPrec<T>& bp, const T* b, int64_t ldb, int k, T* x,
                     int64_t ldx, T* r, T* z, T* p, const T* q, SolveCtl* ctl,
                     CgScalars<T>* sc, T* partials, cudaStream_t st)
{
    const BlockScheme bsc = block_scheme(bp.max_bs);
    const int64_t ngroups = ceildiv(bp.num_blocks, bsc.gs);
    const int grid = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(ngroups, kSolverBlock / kWarp)), solver_grid()));
    const int mb2 = kMaxBs / bsc.gs;
#define B2S_CG_BLOCK(MB)                                                           \
    case MB:                                                                       \
        with_pass_kind<T, K == 1>(bp, [&](auto sk) {                               \
            auto kernel = cg_block_kernel<T, MB, K, INIT, decltype(sk)::value>;    \
            kernel<<<pgrid(kernel, grid), kSolverBlock, 0, st>>>(                  \
                n, bp, b, ldb, k, x, ldx, r, z, p, q, ctl, sc, partials);          \
        });                                                                        \
        break;
    switch (mb2) {
        B2S_CG_BLOCK(2)
        B2S_CG_BLOCK(4)
        B2S_CG_BLOCK(8)
        B2S_CG_BLOCK(16)
        B2S_CG_BLOCK(32)
    default: B2S_CG_BLOCK(1)
    }
#undef B2S_CG_BLOCK
}

struct CgLayout {
    int64_t bytes;
    int64_t off_ctl, off_sc, off_r, off_p0, off_p1, off_q, off_partials, off_z;
};

// with_z: the stored z = M^-1 r of a block preconditioner
template <typename T>
CgLayout cg_layout(int64_t n, int K, bool with_z = false)
{
    Carver c{nullptr};
    CgLayout l;
    l.off_ctl = c.take<SolveCtl>(1);
    l.off_sc = c.take<CgScalars<T>>(1);
    l.off_r = c.take<T>(n * K);
    l.off_p0 = c.take<T>(n * K);
    l.off_p1 = c.take<T>(n * K);
    l.off_q = c.take<T>(n * K);
    l.off_partials = c.take<T>(int64_t(kSolverGrid) * 3 * K);
    l.off_z = with_z ? c.take<T>(n * K) : 0;
    l.bytes = c.used;
    return l;
}

// bp: a block Jacobi preconditioner (dinv then null), or null
template <typename T>
int cg_solve(int64_t n, const int32_t* rp, const int32_t* ci, const T* v,
             int64_t max_row_nnz, const T* dinv, const BlockPrec<T>* bp, const T* b,
             int64_t ldb, T* x, int64_t ldx, int64_t k, int64_t max_iters, double reduction,
             int residual_mode, int64_t check_every, void* workspace,
             int64_t workspace_bytes,
             int64_t* iterations, double* residual_norms, uint8_t* status,
             void* stream)
{
    B2S_CHECK_ARG(n >= 0 && k >= 1 && k <= kMaxRhs, "num_rhs must be 1..16");
    B2S_CHECK_ARG(ldb >= k && ldx >= k, "leading dimension < num_rhs");
    B2S_CHECK_ARG(max_iters >= 0 && max_iters < (int64_t(1) << 30),
                  "max_iters out of range");
    B2S_CHECK_ARG(valid_residual_mode(residual_mode), "unknown residual mode %d",
                  residual_mode);
    if (bp) {
        B2S_CHECK_ARG(bp->max_bs >= 1 && bp->max_bs <= kMaxBs,
                      "max_block_size must be 1..32");
        B2S_CHECK_ARG(bp->num_blocks >= 1 && bp->ptrs && bp->blocks,
                      "block preconditioner without blocks");
    }
    const int K = rhs_bucket(k);
    const CgLayout lay = cg_layout<T>(n, K, bp != nullptr);
    if (workspace_bytes < lay.bytes) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)lay.bytes);
        return B2S_ERR_WORKSPACE;
    }
    B2S_CHECK_ARG(workspace != nullptr && b && x && rp, "null pointer");
    cudaStream_t st = as_stream(stream);
    char* w = static_cast<char*>(workspace);
    auto* ctl = reinterpret_cast<SolveCtl*>(w + lay.off_ctl);
    auto* sc = reinterpret_cast<CgScalars<T>*>(w + lay.off_sc);
    T* r = reinterpret_cast<T*>(w + lay.off_r);
    T* p[2] = {reinterpret_cast<T*>(w + lay.off_p0),
               reinterpret_cast<T*>(w + lay.off_p1)};
    T* q = reinterpret_cast<T*>(w + lay.off_q);
    T* partials = reinterpret_cast<T*>(w + lay.off_partials);
    // block preconditioner: the SpMV passes read the stored z in place of r
    T* z = bp ? reinterpret_cast<T*>(w + lay.off_z) : nullptr;
    T* zr = bp ? z : r;

    SolveCtl h{};
    h.max_iters = int(max_iters);
    h.reduction = reduction;
    h.baseline = residual_mode & ~B2S_STOP_IMPLICIT;
    h.implicit = (residual_mode & B2S_STOP_IMPLICIT) != 0;
    B2S_CUDA_TRY(cudaMemcpyAsync(ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    const int sw = solver_subwarp(max_row_nnz);
    const int64_t row_blocks = std::max<int64_t>(1, ceildiv(n * sw, kSolverBlock));
    const int grid_spmv = int(std::min<int64_t>(row_blocks, solver_grid()));
    const int grid_vec = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n, kSolverBlock)), solver_grid()));
    const int chunk = int(std::max<int64_t>(2, (check_every + 1) / 2 * 2));

    B2S_DISPATCH_RHS(K, {
        B2S_DISPATCH_SW(sw, {
            residual_kernel<T, SW, K><<<pgrid(residual_kernel<T, SW, K>, grid_spmv), kSolverBlock, 0, st>>>(
                n, rp, ci, v, x, ldx, b, ldb, int(k), r);
        });
        B2S_LAUNCH_CHECK();
        if (bp) {
            launch_cg_block<T, K, true>(n, *bp, b, ldb, int(k), x, ldx, r, z, p[0], nullptr,
                                        ctl, sc, partials, st);
        } else {
            cg_init_kernel<T, K><<<pgrid(cg_init_kernel<T, K>, grid_vec), kSolverBlock, 0, st>>>(
                n, dinv, b, ldb, int(k), r, p[0], ctl, sc, partials);
        }
        B2S_LAUNCH_CHECK();
    });
    // the split single-RHS pass (large systems)
    const int lpr = async_lanes_per_row(max_row_nnz);
    const int64_t async_need = ceildiv(ceildiv(n, kWarp / lpr), kAsyncBlock / kWarp);
    auto launch_split = [&](cudaStream_t cs, T* po, T* pn) {
        cg_pupdate_kernel<T><<<pgrid(cg_pupdate_kernel<T>, grid_vec), kSolverBlock, 0, cs>>>(n, dinv, zr, po, pn, ctl, sc);
        with_async_kernel<T, 1, false>(lpr, [&](auto kernel) {
            const int64_t grid = std::min<int64_t>(async_need, async_resident_blocks(kernel));
            kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, v, pn, 1, q, 1, nullptr, nullptr,
                                                 &ctl->all_stopped);
        });
        cg_pq_kernel<T><<<pgrid(cg_pq_kernel<T>, grid_vec), kSolverBlock, 0, cs>>>(n, pn, q, ctl, sc, partials);
        if (bp) {
            launch_cg_block<T, 1, false>(n, *bp, nullptr, 0, 1, x, ldx, r, z, pn, q, ctl, sc,
                                         partials, cs);
        } else {
            cg_update_kernel<T, 1><<<pgrid(cg_update_kernel<T, 1>, grid_vec), kSolverBlock, 0, cs>>>(n, dinv, x, ldx, r, pn,
                                                                      q, ctl, sc, partials);
        }
    };
    auto capture = [&](cudaStream_t cs) -> int {
        for (int it = 0; it < chunk; ++it) {
            T* po = p[it % 2];
            T* pn = p[(it + 1) % 2];
            if (K == 1 && n >= kCgSplitRows) {
                launch_split(cs, po, pn);
                B2S_LAUNCH_CHECK();
                continue;
            }
            B2S_DISPATCH_RHS(K, {
                if constexpr (K * sizeof(T) >= 32) {
                    // lanes own 16-byte column slices of a row
                    constexpr int VW = int(16 / sizeof(T));
                    constexpr int RPW = kWarp / (K / VW);
                    const int gs = int(std::min<int64_t>(
                        std::max<int64_t>(1, ceildiv(n, RPW * (kSolverBlock / kWarp))),
                        solver_grid()));
                    const int gu = int(std::min<int64_t>(
                        std::max<int64_t>(1, ceildiv(n * K / VW, kSolverBlock)), solver_grid()));
                    cg_spmv_lanes_kernel<T, K><<<pgrid(cg_spmv_lanes_kernel<T, K>, gs), kSolverBlock, 0, cs>>>(
                        n, rp, ci, v, dinv, zr, po, pn, q, ctl, sc, partials);
                    if (bp) {
                        launch_cg_block<T, K, false>(n, *bp, nullptr, 0, int(k), x, ldx, r, z,
                                                     pn, q, ctl, sc, partials, cs);
                    } else {
                        cg_update_lanes_kernel<T, K><<<pgrid(cg_update_lanes_kernel<T, K>, gu), kSolverBlock, 0, cs>>>(
                            n, dinv, x, ldx, r, pn, q, ctl, sc, partials);
                    }
                } else {
                    B2S_DISPATCH_SW(sw, {
                        cg_spmv_kernel<T, SW, K><<<pgrid(cg_spmv_kernel<T, SW, K>, grid_spmv), kSolverBlock, 0, cs>>>(
                            n, rp, ci, v, dinv, zr, po, pn, q, ctl, sc, partials);
                    });
                    if (bp) {
                        launch_cg_block<T, K, false>(n, *bp, nullptr, 0, int(k), x, ldx, r, z,
                                                     pn, q, ctl, sc, partials, cs);
                    } else {
                        cg_update_kernel<T, K><<<pgrid(cg_update_kernel<T, K>, grid_vec), kSolverBlock, 0, cs>>>(
                            n, dinv, x, ldx, r, pn, q, ctl, sc, partials);
                    }
                }
            });
            B2S_LAUNCH_CHECK();
        }
        return B2S_OK;
    };
    // the graph always runs an even number of iterations, so p[0] holds the
    // current direction at every replay boundary
    int rc = run_graph_loop(st, ctl, int(max_iters), chunk, capture, &h);
    if (rc != B2S_OK) return rc;
    CgScalars<T> hs;
    B2S_CUDA_TRY(cudaMemcpyAsync(&hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, st));
    B2S_CUDA_TRY(cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st));
    B2S_CUDA_TRY(cudaStreamSynchronize(st));
    if (iterations) *iterations = h.iter;
    for (int64_t j = 0; j < k; ++j) {
        if (residual_norms) residual_norms[j] = double(hs.tau[j]);
        if (status) status[j] = h.status[j];
    }
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int64_t b2s_cg_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                               int value_bytes)
{
    const int K = rhs_bucket(num_rhs);
    if (K < 0 || num_rows < 0) return -1;
    return value_bytes == 8 ? cg_layout<double>(num_rows, K).bytes
                            : cg_layout<float>(num_rows, K).bytes;
}

int64_t b2s_cg_block_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                                     int value_bytes)
{
    const int K = rhs_bucket(num_rhs);
    if (K < 0 || num_rows < 0) return -1;
    return value_bytes == 8 ? cg_layout<double>(num_rows, K, true).bytes
                            : cg_layout<float>(num_rows, K, true).bytes;
}

#define B2S_CG_ENTRY(T, S)                                                    \
    int b2s_cg_solve_##S(int64_t num_rows, const int32_t* row_ptrs,           \
                         const int32_t* col_idxs, const T* values,            \
                         int64_t max_row_nnz, const T* inv_diag, const T* b,  \
                         int64_t ldb, T* x, int64_t ldx, int64_t num_rhs,     \
                         int64_t max_iters, double reduction_factor,          \
                         int residual_mode, int64_t check_every,              \
                         void* workspace,                                     \
                         int64_t workspace_bytes, int64_t* iterations,        \
                         double* residual_norms, uint8_t* status,             \
                         void* stream)                                        \
    {                                                                         \
        return cg_solve<T>(num_rows, row_ptrs, col_idxs, values, max_row_nnz, \
                           inv_diag, nullptr, b, ldb, x, ldx, num_rhs,        \
                           max_iters, reduction_factor, residual_mode,        \
                           check_every, workspace,                            \
                           workspace_bytes, iterations, residual_norms,       \
                           status, stream);                                   \
    }                                                                         \
    int b2s_cg_block_solve_##S(                                               \
        int64_t num_rows, const int32_t* row_ptrs, const int32_t* col_idxs,  \
        const T* values, int64_t max_row_nnz, int64_t num_blocks,            \
        const int32_t* block_ptrs, int max_block_size,                        \
        const uint8_t* block_precisions, const T* blocks,       \
        const T* b, int64_t ldb, T* x, int64_t ldx, int64_t num_rhs,          \
        int64_t max_iters, double reduction_factor, int residual_mode,        \
        int64_t check_every, void* workspace, int64_t workspace_bytes,        \
        int64_t* iterations, double* residual_norms, uint8_t* status,         \
        void* stream)                                                         \
    {                                                                         \
        BlockPrec<T> bp;                                                      \
        bp.num_blocks = num_blocks;                                           \
        bp.ptrs = block_ptrs;                                                 \
        bp.max_bs = max_block_size;                                           \
        bp.blocks = blocks;                                                   \
        bp.prec = block_precisions;                                           \
        if (bp.prec && workspace && workspace_bytes >= int64_t(sizeof(int))) { \
            /* the workspace's first word as scratch, before the solve */       \
            B2S_CUDA_TRY(resolve_storage_kind(bp, static_cast<int*>(workspace), \
                                              as_stream(stream)));        \
        }                                                                 \
        return cg_solve<T>(num_rows, row_ptrs, col_idxs, values, max_row_nnz, \
                           nullptr, &bp, b, ldb, x, ldx, num_rhs, max_iters,  \
                           reduction_factor, residual_mode, check_every,      \
                           workspace, workspace_bytes, iterations,            \
                           residual_norms, status, stream);                   \
    }

B2S_CG_ENTRY(double, f64)
B2S_CG_ENTRY(float, f32)

}  // extern "C"
