// Building blocks of the fused Krylov solvers: stopping status bits, the
// device-side solver state, deterministic grid reductions (per-block
// partials summed in block order by the last block to finish) and the
// CUDA-graph driver loop that checks convergence on the host only every few
// iterations.
#pragma once

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace b2s {

constexpr int kSolverBlock = 256;
constexpr int kMaxRhs = 16;
// Grid bound of the fused kernels (8 blocks per SM, grid-stride over rows);
// it sizes their partial-sum buffers.  Launches use solver_grid(), the same
// bound on the device's own SM count.
constexpr int kSolverGrid = kMaxSMs * 8;
inline int64_t solver_grid() { return std::min(kSolverGrid, num_sms() * 8); }

// The grid of a persistent (grid-stride) solver kernel: resident_grid with
// kSolverBlock threads.
template <typename Kern>
int pgrid(Kern kernel, int64_t grid)
{
    return resident_grid(kernel, kSolverBlock, grid);
}

// stopping_status bit layout of the reference
// (include/ginkgo/core/stop/stopping_status.hpp:21-121): bit 7 converged,
// bit 6 finalized, bits 0-5 the id of the criterion that stopped it.
constexpr uint8_t kConvergedMask = 1u << 7;
constexpr uint8_t kFinalizedMask = 1u << 6;
constexpr uint8_t kIdMask = (1u << 6) - 1;
constexpr uint8_t kIterationId = 1;   // id used for the iteration limit
constexpr uint8_t kResidualId = 2;    // id used for the residual criterion

__host__ __device__ inline bool has_stopped(uint8_t s) { return s & kIdMask; }
__host__ __device__ inline bool is_finalized(uint8_t s)
{
    return s & kFinalizedMask;
}
__host__ __device__ inline void stop_status(uint8_t& s, uint8_t id, bool fin)
{
    if (!has_stopped(s)) {
        s |= (id & kIdMask);
        if (fin) s |= kFinalizedMask;
    }
}
__host__ __device__ inline void converge_status(uint8_t& s, uint8_t id,
                                                bool fin)
{
    if (!has_stopped(s)) {
        s |= kConvergedMask | (id & kIdMask);
        if (fin) s |= kFinalizedMask;
    }
}

// Control block shared by every fused solver; lives in the workspace.
struct SolveCtl {
    int iter;          // the reference's iteration counter at the last check
    int all_stopped;   // every column stopped
    unsigned ticket;   // last-block ticket of the running reduction
    int max_iters;
    double reduction;  // residual goal relative to the baseline
    int baseline;      // B2S_BASELINE_*: ||b||, ||r_0|| or 1
    int implicit;      // stop::ImplicitResidualNorm: sqrt|rho| instead of ||r||
    uint8_t status[kMaxRhs];
};

// The residual criterion's baseline (stop::ResidualNorm's starting_tau,
// core/stop/residual_norm.cpp:95-150): ||b|| (rhs_norm), the initial
// residual norm (initial_resnorm) or 1 (absolute).
template <typename T>
__device__ __forceinline__ T start_norm(const SolveCtl* ctl, T bnorm, T rnorm)
{
    return ctl->baseline == B2S_BASELINE_INITIAL_RESNORM ? rnorm
           : ctl->baseline == B2S_BASELINE_ABSOLUTE      ? T(1)
                                                         : bnorm;
}

// Whether a column meets the residual goal: ||r|| (stop::ResidualNorm) or
// sqrt|rho| of the solver's implicit squared residual norm
// (stop::ImplicitResidualNorm, reference/stop/residual_norm_kernels.cpp:80)
// against reduction * baseline.
template <typename T>
__device__ __forceinline__ bool residual_met(const SolveCtl* ctl, T tau, T rho, T start)
{
    const double m = ctl->implicit ? sqrt(fabs(double(rho))) : double(tau);
    return m <= ctl->reduction * double(start);
}

// Host check of a residual_mode argument (B2S_BASELINE_* with
// B2S_STOP_IMPLICIT or-ed in).
inline bool valid_residual_mode(int mode)
{
    const int base = mode & ~B2S_STOP_IMPLICIT;
    return base == B2S_BASELINE_RHS_NORM || base == B2S_BASELINE_INITIAL_RESNORM ||
           base == B2S_BASELINE_ABSOLUTE;
}

// Rounding-exact helpers: the same expression evaluated in two kernels must
// give the same bits, so no FMA contraction is allowed in them.
__device__ __forceinline__ double mul_rn(double a, double b)
{
    return __dmul_rn(a, b);
}
__device__ __forceinline__ float mul_rn(float a, float b)
{
    return __fmul_rn(a, b);
}
__device__ __forceinline__ double add_rn(double a, double b)
{
    return __dadd_rn(a, b);
}
__device__ __forceinline__ float add_rn(float a, float b)
{
    return __fadd_rn(a, b);
}

// Sums K values over the block and stores them as partials[blockIdx.x][K].
template <typename T, int K>
__device__ __forceinline__ void block_partials(T (&v)[K], T* __restrict__ partials,
                                               T* sm /* [warps][K] */)
{
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < K; ++j) sm[wid * K + j] = v[j];
    }
    __syncthreads();
    if (threadIdx.x < K) {
        T s = T(0);
        for (int w = 0; w < kSolverBlock / kWarp; ++w) s += sm[w * K + threadIdx.x];
        partials[blockIdx.x * K + threadIdx.x] = s;
    }
}

// True in exactly one block: the last one to finish its partials.
__device__ __forceinline__ bool last_block_done(unsigned* ticket, int* flag_sm)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        *flag_sm = (t == gridDim.x - 1);
    }
    __syncthreads();
    const bool last = *flag_sm;
    if (last) __threadfence();
    return last;
}

// In the last block: out[j] = sum over blocks of partials[b][j], summed in a
// fixed order (deterministic for a fixed grid).  M values per block; out and
// sm are shared memory ([M] and [warps][M]).
template <typename T, int M>
__device__ __forceinline__ void sum_partials(const T* partials, int nblocks,
                                             T* out, T* sm)
{
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    T acc[M];
#pragma unroll
    for (int j = 0; j < M; ++j) acc[j] = T(0);
    constexpr int kPer = (kSolverGrid + kSolverBlock - 1) / kSolverBlock;
    if (M * kPer <= 32 && nblocks <= kSolverGrid) {
        // every load of this thread in flight at once, summed in block order
        T v[kPer][M];
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int b = threadIdx.x + q * kSolverBlock;
#pragma unroll
            for (int j = 0; j < M; ++j) v[q][j] = b < nblocks ? __ldcg(partials + b * M + j) : T(0);
        }
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
#pragma unroll
            for (int j = 0; j < M; ++j) acc[j] += v[q][j];
        }
    } else {
        for (int b = threadIdx.x; b < nblocks; b += kSolverBlock) {
#pragma unroll
            for (int j = 0; j < M; ++j) acc[j] += __ldcg(partials + b * M + j);
        }
    }
#pragma unroll
    for (int j = 0; j < M; ++j) acc[j] = warp_sum(acc[j]);
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < M; ++j) sm[wid * M + j] = acc[j];
    }
    __syncthreads();
    if (threadIdx.x < M) {
        T s = T(0);
        for (int w = 0; w < kSolverBlock / kWarp; ++w) s += sm[w * M + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// r = b - A x for the first k of K columns (the rest zero); b, x strided,
// r contiguous n x K.  One subwarp of SW lanes per row, grid-stride.
template <typename T, int SW, int K>
__global__ void __launch_bounds__(kSolverBlock)
    residual_kernel(int64_t n, const int32_t* __restrict__ rp,
                    const int32_t* __restrict__ ci, const T* __restrict__ v,
                    const T* __restrict__ x, int64_t ldx,
                    const T* __restrict__ b, int64_t ldb, int k,
                    T* __restrict__ r)
{
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
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (j < k) acc[j] += a * x[c * ldx + j];
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = subwarp_sum<SW>(acc[j]);
        if (valid && lane == 0) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                r[row * K + j] = j < k ? b[row * ldb + j] - acc[j] : T(0);
            }
        }
    }
}

inline int solver_subwarp(int64_t max_row_nnz)
{
    int sw = 1;
    while (sw * 2 <= max_row_nnz && sw < 32) sw *= 2;
    return sw;
}

inline int rhs_bucket(int64_t k)
{
    for (int kk : {1, 2, 4, 8, 16}) {
        if (k <= kk) return kk;
    }
    return -1;
}

#define B2S_DISPATCH_SW(sw, ...)                               \
    switch (sw) {                                              \
    case 32: { constexpr int SW = 32; __VA_ARGS__; break; }    \
    case 16: { constexpr int SW = 16; __VA_ARGS__; break; }    \
    case 8: { constexpr int SW = 8; __VA_ARGS__; break; }      \
    case 4: { constexpr int SW = 4; __VA_ARGS__; break; }      \
    case 2: { constexpr int SW = 2; __VA_ARGS__; break; }      \
    default: { constexpr int SW = 1; __VA_ARGS__; break; }     \
    }

#define B2S_DISPATCH_RHS(kk, ...)                              \
    switch (kk) {                                              \
    case 1: { constexpr int K = 1; __VA_ARGS__; break; }       \
    case 2: { constexpr int K = 2; __VA_ARGS__; break; }       \
    case 4: { constexpr int K = 4; __VA_ARGS__; break; }       \
    case 8: { constexpr int K = 8; __VA_ARGS__; break; }       \
    default: { constexpr int K = 16; __VA_ARGS__; break; }     \
    }

// Workspace carving: 256-byte aligned bump allocation inside the caller's
// buffer (the library itself never allocates device memory).
struct Carver {
    char* base;  // unused: layouts only record byte offsets
    int64_t used = 0;
    // byte offset of a new 256-byte aligned block of count T
    template <typename T>
    int64_t take(int64_t count)
    {
        used = (used + 255) / 256 * 256;
        const int64_t off = used;
        used += count * int64_t(sizeof(T));
        return off;
    }
};

// Host loop: replays a captured CUDA graph of `chunk` iterations until the
// device reports every column stopped.  The graph is captured on a private
// stream and launched on the caller's stream; the host reads the control
// block once per replay.
template <typename Capture>
int run_graph_loop(cudaStream_t st, SolveCtl* ctl, int max_iters, int chunk,
                   Capture&& capture, SolveCtl* host_ctl)
{
    cudaStream_t cap;
    B2S_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = B2S_OK;
    do {
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            set_error("begin capture: %s", cudaGetErrorString(e));
            rc = B2S_ERR_CUDA;
            break;
        }
        rc = capture(cap);
        e = cudaStreamEndCapture(cap, &graph);
        if (rc != B2S_OK) break;
        if (e != cudaSuccess) {
            set_error("end capture: %s", cudaGetErrorString(e));
            rc = B2S_ERR_CUDA;
            break;
        }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) {
            set_error("instantiate: %s", cudaGetErrorString(e));
            rc = B2S_ERR_CUDA;
            break;
        }
        // every replay advances at least one iteration until stopped, and the
        // kernels stop every column at max_iters, so this loop is bounded
        const int64_t max_replays = int64_t(max_iters) / chunk + 2;
        for (int64_t r = 0; r < max_replays; ++r) {
            e = cudaGraphLaunch(exec, st);
            if (e == cudaSuccess) {
                e = cudaMemcpyAsync(host_ctl, ctl, sizeof(SolveCtl),
                                    cudaMemcpyDeviceToHost, st);
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                set_error("graph replay: %s", cudaGetErrorString(e));
                rc = B2S_ERR_CUDA;
                break;
            }
            if (host_ctl->all_stopped) break;
        }
    } while (false);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    return rc;
}

// One 16-byte vector of R values (R * sizeof(T) == 16, p 16-byte aligned).
template <typename T, int R>
__device__ __forceinline__ void ld_vec(const T* p, T (&o)[R])
{
    static_assert(R * sizeof(T) == 16, "one 16-byte vector");
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    memcpy(o, &u, 16);
}
template <typename T, int R>
__device__ __forceinline__ void st_vec(T* p, const T (&v)[R])
{
    uint4 u;
    memcpy(&u, v, 16);
    *reinterpret_cast<uint4*>(p) = u;
}

}  // namespace b2s
