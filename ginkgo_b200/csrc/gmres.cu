// Restarted GMRES(d) with right scalar-Jacobi preconditioning and an FP64
// restart residual, in three precisions behind one engine:
//
//   b2s_gmres_solve_f64            Arnoldi in FP64, FP64 basis
//   b2s_ir_gmres_solve_f32         mixed precision: every restart (outer
//   b2s_ir_gmres_solve_bf16basis   iteration of iterative refinement)
//                                  computes r = b - A x and ||r|| in FP64;
//                                  the Arnoldi cycle runs on an FP32 copy of
//                                  A with FP32 vectors and an FP32 or BF16
//                                  basis; x += M V y is added in FP64.
//
// Reference behaviour: core/solver/gmres.cpp:325-640 (restart, Arnoldi,
// Givens QR, solve_krylov, multi_axpy), core/solver/ir.cpp:191-257 with
// update_residual.hpp:20-60 (outer residual and check),
// reference/solver/common_gmres_kernels.cpp:29-180 (Givens formulas).
// Differences, all on the device: orthogonalisation is classical
// Gram-Schmidt with one re-orthogonalisation (CGS2, the reference's
// ortho_method::cgs2), each pass a single read of the basis; the Hessenberg
// matrix, Givens rotations and the triangular solve are FP64 in every
// variant; a cycle ends early when the Givens residual estimate reaches the
// goal, and convergence is declared only on the explicit FP64 residual.
//
// Kernels per Arnoldi step j (one CUDA graph per restart cycle):
//   spmv    v_j = round_basis(src * scale) formed on the fly (src = the
//           previous unnormalised vector, or r at j = 0) and stored;
//           w = A D^-1 v_j
//   dot     h1 = V_{0..j}^T w
//   orth    w -= V h1;  h2 = V^T w           (one basis read)
//   orth2   w -= V h2;  ||w||; last block: Hessenberg column, Givens update,
//           residual estimate, early end of the cycle, back substitution
// per cycle: update x += D^-1 V y (FP64 accumulate), residual r = b - A x.
#include <cuda_bf16.h>

#include "solver_common.cuh"

namespace b2s {
namespace {

constexpr int kMaxKrylov = 32;

struct GmresState {
    int done, cycle_done, j, final_iter;
    int total_iter, max_iters, outer_iter, converged;
    unsigned ticket;
    int krylov_dim;
    int pad[2];
    double bnorm, rnorm, reduction, inner_reduction, inner_thresh;
    double scale;  // v_j = src * scale: 1/||r|| at j = 0, 1/H(j, j-1) else
    double h1[kMaxKrylov + 1], h2[kMaxKrylov + 1];
    double H[kMaxKrylov * (kMaxKrylov + 1)];  // column j at H[j * (M + 1)]
    double g[kMaxKrylov + 1], cs[kMaxKrylov], sn[kMaxKrylov], y[kMaxKrylov];
};

template <typename TB, typename TA>
__device__ __forceinline__ TB to_basis(TA v)
{
    return TB(v);
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
__device__ __forceinline__ float from_basis<float, __nv_bfloat16>(__nv_bfloat16 v)
{
    return __bfloat162float(v);
}

// The basis value v_j[c], formed identically wherever it is needed.
template <typename TA, typename TB>
__device__ __forceinline__ TA basis_value(int j, int64_t c,
                                          const double* __restrict__ r64,
                                          const TA* __restrict__ w_src,
                                          TA scale)
{
    const TA src = j == 0 ? TA(r64[c]) : w_src[c];
    return from_basis<TA>(to_basis<TB>(mul_rn(src, scale)));
}

template <typename TA, typename TB, int SW>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_spmv_kernel(int64_t n, const int32_t* __restrict__ rp,
                      const int32_t* __restrict__ ci, const TA* __restrict__ v,
                      const TA* __restrict__ dinv,
                      const double* __restrict__ r64,
                      const TA* __restrict__ w_src, TA* __restrict__ w_dst,
                      TB* __restrict__ V, GmresState* st)
{
    if (st->done || st->cycle_done) return;
    const int j = st->j;
    const TA scale = TA(st->scale);
    TB* vj = V + int64_t(j) * n;
    const int lane = threadIdx.x % SW;
    const int64_t nsub = int64_t(gridDim.x) * kSolverBlock / SW;
    // warp-uniform trip count: all lanes of a warp run every iteration, so
    // the subwarp shuffles below always see the whole warp
    for (int64_t wbase = (blockIdx.x * int64_t(kSolverBlock) + threadIdx.x) /
                         kWarp * (kWarp / SW);
         wbase < n; wbase += nsub) {
        const int64_t row = wbase + (threadIdx.x % kWarp) / SW;
        const bool valid = row < n;
        TA acc = TA(0);
        const int end = valid ? rp[row + 1] : 0;
        for (int e = (valid ? rp[row] : end) + lane; e < end; e += SW) {
            const int64_t c = ci[e];
            const TA d = dinv ? dinv[c] : TA(1);
            acc += v[e] * mul_rn(d, basis_value<TA, TB>(j, c, r64, w_src, scale));
        }
        acc = subwarp_sum<SW>(acc);
        if (valid && lane == 0) {
            vj[row] = to_basis<TB>(basis_value<TA, TB>(j, row, r64, w_src, scale));
            w_dst[row] = acc;
        }
    }
}

// Loads V[0..j][row] (j < M) into registers.
template <typename TA, typename TB, int M>
__device__ __forceinline__ void load_basis_row(const TB* __restrict__ V,
                                               int64_t n, int j, int64_t row,
                                               TA (&vb)[M])
{
#pragma unroll
    for (int i = 0; i < M; ++i) {
        vb[i] = i <= j ? from_basis<TA>(V[int64_t(i) * n + row]) : TA(0);
    }
}

// h = V_{0..j}^T w; sums in the last block go to dst (h1 or h2).
template <typename TA, int M>
__device__ __forceinline__ void finish_dots(TA (&acc)[M], double* partials,
                                            GmresState* st, double* dst, int j)
{
    __shared__ double red[kSolverBlock / kWarp * M];
    __shared__ double tot[M];
    __shared__ int last;
    double a[M];
#pragma unroll
    for (int i = 0; i < M; ++i) a[i] = double(acc[i]);
    block_partials<double, M>(a, partials, red);
    if (last_block_done(&st->ticket, &last)) {
        sum_partials<double, M>(partials, gridDim.x, tot, red);
        if (threadIdx.x <= j && threadIdx.x < M) dst[threadIdx.x] = tot[threadIdx.x];
        if (threadIdx.x == 0) st->ticket = 0;
    }
}

template <typename TA, typename TB, int M>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_dot_kernel(int64_t n, const TB* __restrict__ V,
                     const TA* __restrict__ w, GmresState* st,
                     double* __restrict__ partials)
{
    if (st->done || st->cycle_done) return;
    const int j = st->j;
    TA acc[M];
#pragma unroll
    for (int i = 0; i < M; ++i) acc[i] = TA(0);
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        TA vb[M];
        load_basis_row<TA, TB, M>(V, n, j, row, vb);
        const TA wr = w[row];
#pragma unroll
        for (int i = 0; i < M; ++i) acc[i] += vb[i] * wr;
    }
    finish_dots<TA, M>(acc, partials, st, st->h1, j);
}

template <typename TA, typename TB, int M>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_orth_kernel(int64_t n, const TB* __restrict__ V, TA* __restrict__ w,
                      GmresState* st, double* __restrict__ partials)
{
    if (st->done || st->cycle_done) return;
    const int j = st->j;
    TA h[M];
#pragma unroll
    for (int i = 0; i < M; ++i) h[i] = i <= j ? TA(st->h1[i]) : TA(0);
    TA acc[M];
#pragma unroll
    for (int i = 0; i < M; ++i) acc[i] = TA(0);
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        TA vb[M];
        load_basis_row<TA, TB, M>(V, n, j, row, vb);
        TA wr = w[row];
#pragma unroll
        for (int i = 0; i < M; ++i) wr -= h[i] * vb[i];
        w[row] = wr;
#pragma unroll
        for (int i = 0; i < M; ++i) acc[i] += vb[i] * wr;
    }
    finish_dots<TA, M>(acc, partials, st, st->h2, j);
}

// Givens update of column j and the cycle bookkeeping (one thread).
__device__ void hessenberg_step(GmresState* st, double hnorm)
{
    constexpr int LD = kMaxKrylov + 1;
    const int j = st->j;
    double* h = st->H + j * LD;
    for (int i = 0; i <= j; ++i) h[i] = st->h1[i] + st->h2[i];
    h[j + 1] = hnorm;
    for (int i = 0; i < j; ++i) {
        const double t = st->cs[i] * h[i] + st->sn[i] * h[i + 1];
        h[i + 1] = -st->sn[i] * h[i] + st->cs[i] * h[i + 1];
        h[i] = t;
    }
    const double th = h[j], nh = h[j + 1];
    if (th == 0.0) {
        st->cs[j] = 0.0;
        st->sn[j] = 1.0;
    } else {
        const double scale = fabs(th) + fabs(nh);
        const double a = fabs(th / scale), b = fabs(nh / scale);
        const double hyp = scale * sqrt(a * a + b * b);
        st->cs[j] = th / hyp;
        st->sn[j] = nh / hyp;
    }
    h[j] = st->cs[j] * th + st->sn[j] * nh;
    h[j + 1] = 0.0;
    st->g[j + 1] = -st->sn[j] * st->g[j];
    st->g[j] = st->cs[j] * st->g[j];
    const double est = fabs(st->g[j + 1]);
    st->final_iter = j + 1;
    st->total_iter += 1;
    st->scale = hnorm > 0.0 ? 1.0 / hnorm : 0.0;
    st->j = j + 1;
    if (est <= st->inner_thresh || st->j >= st->krylov_dim ||
        st->total_iter >= st->max_iters || !(hnorm > 0.0)) {
        st->cycle_done = 1;
        // y = H \ g (back substitution over the finished columns)
        const int m = st->final_iter;
        for (int i = m - 1; i >= 0; --i) {
            double t = st->g[i];
            for (int k = i + 1; k < m; ++k) t -= st->H[k * LD + i] * st->y[k];
            st->y[i] = t / st->H[i * LD + i];
        }
    }
}

template <typename TA, typename TB, int M>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_orth2_kernel(int64_t n, const TB* __restrict__ V, TA* __restrict__ w,
                       GmresState* st, double* __restrict__ partials)
{
    __shared__ double red[kSolverBlock / kWarp];
    __shared__ double tot[1];
    __shared__ int last;
    if (st->done || st->cycle_done) return;
    const int j = st->j;
    TA h[M];
#pragma unroll
    for (int i = 0; i < M; ++i) h[i] = i <= j ? TA(st->h2[i]) : TA(0);
    double nrm = 0.0;
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        TA vb[M];
        load_basis_row<TA, TB, M>(V, n, j, row, vb);
        TA wr = w[row];
#pragma unroll
        for (int i = 0; i < M; ++i) wr -= h[i] * vb[i];
        w[row] = wr;
        nrm += double(wr) * double(wr);
    }
    double a[1] = {nrm};
    block_partials<double, 1>(a, partials, red);
    if (last_block_done(&st->ticket, &last)) {
        sum_partials<double, 1>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            st->ticket = 0;
            hessenberg_step(st, sqrt(tot[0]));
        }
    }
}

// x += D^-1 (V y) over the finished columns, accumulated into FP64 x.
template <typename TA, typename TB, int M>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_update_kernel(int64_t n, const TB* __restrict__ V,
                        const TA* __restrict__ dinv, double* __restrict__ x,
                        GmresState* st)
{
    if (st->done) return;
    const int m = st->final_iter;
    if (m == 0) return;
    TA y[M];
#pragma unroll
    for (int i = 0; i < M; ++i) y[i] = i < m ? TA(st->y[i]) : TA(0);
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        TA vb[M];
        load_basis_row<TA, TB, M>(V, n, m - 1, row, vb);
        TA u = TA(0);
#pragma unroll
        for (int i = 0; i < M; ++i) u += y[i] * vb[i];
        const TA d = dinv ? dinv[row] : TA(1);
        x[row] += double(d * u);
    }
}

// r = b - A x in FP64, ||r||, ||b||; the last block checks convergence and
// sets up the next cycle (the reference's restart kernel).
template <int SW>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_residual_kernel(int64_t n, const int32_t* __restrict__ rp,
                          const int32_t* __restrict__ ci,
                          const double* __restrict__ v,
                          const double* __restrict__ x,
                          const double* __restrict__ b,
                          double* __restrict__ r, GmresState* st,
                          double* __restrict__ partials)
{
    __shared__ double red[kSolverBlock / kWarp * 2];
    __shared__ double tot[2];
    __shared__ int last;
    if (st->done) return;
    const int lane = threadIdx.x % SW;
    const int64_t nsub = int64_t(gridDim.x) * kSolverBlock / SW;
    double acc2[2] = {0.0, 0.0};
    // warp-uniform trip count: all lanes of a warp run every iteration, so
    // the subwarp shuffles below always see the whole warp
    for (int64_t wbase = (blockIdx.x * int64_t(kSolverBlock) + threadIdx.x) /
                         kWarp * (kWarp / SW);
         wbase < n; wbase += nsub) {
        const int64_t row = wbase + (threadIdx.x % kWarp) / SW;
        const bool valid = row < n;
        double acc = 0.0;
        const int end = valid ? rp[row + 1] : 0;
        for (int e = (valid ? rp[row] : end) + lane; e < end; e += SW) acc += v[e] * x[ci[e]];
        acc = subwarp_sum<SW>(acc);
        if (valid && lane == 0) {
            const double bb = b[row];
            const double rr = bb - acc;
            r[row] = rr;
            acc2[0] += rr * rr;
            acc2[1] += bb * bb;
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
            if (rn <= st->reduction * st->bnorm) {
                st->converged = 1;
                st->done = 1;
            } else if (st->total_iter >= st->max_iters) {
                st->done = 1;
            } else {
                st->outer_iter += 1;
                st->j = 0;
                st->cycle_done = 0;
                st->g[0] = rn;
                for (int i = 1; i <= kMaxKrylov; ++i) st->g[i] = 0.0;
                st->scale = 1.0 / rn;
                st->inner_thresh = fmax(st->inner_reduction * rn,
                                        st->reduction * st->bnorm);
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

struct GmresLayout {
    int64_t bytes, off_st, off_r, off_w0, off_w1, off_v, off_partials,
        off_a32, off_d32;
};

template <typename TA, typename TB>
GmresLayout gmres_layout(int64_t n, int64_t nnz, int d, bool mixed)
{
    Carver c{nullptr};
    GmresLayout l;
    l.off_st = c.take<GmresState>(1);
    l.off_r = c.take<double>(n);
    l.off_w0 = c.take<TA>(n);
    l.off_w1 = c.take<TA>(n);
    l.off_v = c.take<TB>((int64_t(d) + 1) * n);
    l.off_partials = c.take<double>(int64_t(kSolverGrid) * (kMaxKrylov + 1));
    l.off_a32 = mixed ? c.take<float>(nnz) : 0;
    l.off_d32 = mixed ? c.take<float>(n) : 0;
    l.bytes = c.used;
    return l;
}

template <typename TA, typename TB>
int gmres_engine(int64_t n, const int32_t* rp, const int32_t* ci,
                 const double* v64, int64_t max_row_nnz, const double* dinv64,
                 const double* b, double* x, int krylov_dim,
                 int64_t max_iters, double reduction, double inner_reduction,
                 void* workspace, int64_t workspace_bytes,
                 int64_t* iterations, int64_t* restarts, double* res_norm,
                 int* converged, void* stream)
{
    constexpr bool kMixed = !std::is_same<TA, double>::value;
    B2S_CHECK_ARG(n >= 1, "GMRES needs at least one row");
    B2S_CHECK_ARG(krylov_dim >= 1 && krylov_dim <= kMaxKrylov,
                  "krylov_dim must be 1..%d", kMaxKrylov);
    B2S_CHECK_ARG(max_iters >= 0 && max_iters < (int64_t(1) << 30),
                  "max_iters out of range");
    int64_t nnz = 0;
    cudaStream_t st = as_stream(stream);
    {
        int32_t h_nnz = 0;
        B2S_CUDA_TRY(cudaMemcpyAsync(&h_nnz, rp + n, sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, st));
        B2S_CUDA_TRY(cudaStreamSynchronize(st));
        nnz = h_nnz;
    }
    const GmresLayout lay = gmres_layout<TA, TB>(n, nnz, krylov_dim, kMixed);
    if (workspace_bytes < lay.bytes) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)lay.bytes);
        return B2S_ERR_WORKSPACE;
    }
    char* w = static_cast<char*>(workspace);
    auto* gs = reinterpret_cast<GmresState*>(w + lay.off_st);
    double* r = reinterpret_cast<double*>(w + lay.off_r);
    TA* wv[2] = {reinterpret_cast<TA*>(w + lay.off_w0),
                 reinterpret_cast<TA*>(w + lay.off_w1)};
    TB* V = reinterpret_cast<TB*>(w + lay.off_v);
    double* partials = reinterpret_cast<double*>(w + lay.off_partials);
    const TA* va;
    const TA* da;
    if constexpr (kMixed) {
        float* a32 = reinterpret_cast<float*>(w + lay.off_a32);
        float* d32 = reinterpret_cast<float*>(w + lay.off_d32);
        if (nnz > 0) {
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
    h.reduction = reduction;
    h.inner_reduction = inner_reduction;
    h.cycle_done = 1;
    B2S_CUDA_TRY(cudaMemcpyAsync(gs, &h, sizeof(h), cudaMemcpyHostToDevice, st));

    const int sw = solver_subwarp(max_row_nnz);
    const int grid_spmv = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n * sw, kSolverBlock)), kSolverGrid));
    const int grid_vec = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n, kSolverBlock)), kSolverGrid));
    constexpr int M = kMaxKrylov;
    // first residual outside the graph
    B2S_DISPATCH_SW(sw, {
        gmres_residual_kernel<SW><<<grid_spmv, kSolverBlock, 0, st>>>(
            n, rp, ci, v64, x, b, r, gs, partials);
    });
    B2S_LAUNCH_CHECK();
    auto capture = [&](cudaStream_t cs) -> int {
        for (int j = 0; j < krylov_dim; ++j) {
            TA* src = wv[(j + 1) % 2];
            TA* dst = wv[j % 2];
            B2S_DISPATCH_SW(sw, {
                gmres_spmv_kernel<TA, TB, SW><<<grid_spmv, kSolverBlock, 0, cs>>>(
                    n, rp, ci, va, da, r, src, dst, V, gs);
            });
            gmres_dot_kernel<TA, TB, M><<<grid_vec, kSolverBlock, 0, cs>>>(
                n, V, dst, gs, partials);
            gmres_orth_kernel<TA, TB, M><<<grid_vec, kSolverBlock, 0, cs>>>(
                n, V, dst, gs, partials);
            gmres_orth2_kernel<TA, TB, M><<<grid_vec, kSolverBlock, 0, cs>>>(
                n, V, dst, gs, partials);
            B2S_LAUNCH_CHECK();
        }
        gmres_update_kernel<TA, TB, M><<<grid_vec, kSolverBlock, 0, cs>>>(
            n, V, da, x, gs);
        B2S_DISPATCH_SW(sw, {
            gmres_residual_kernel<SW><<<grid_spmv, kSolverBlock, 0, cs>>>(
                n, rp, ci, v64, x, b, r, gs, partials);
        });
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    };
    // the spmv of step j reads the vector written at step j - 1: the graph
    // alternates w buffers inside a cycle and every cycle restarts from r
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
        GmresState hs;
        for (int64_t cyc = 0; cyc < max_cycles; ++cyc) {
            e = cudaMemcpyAsync(&hs.done, &gs->done, sizeof(int),
                                cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) { set_error("replay: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
            if (hs.done) break;
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
    if (converged) *converged = hs.converged;
    return B2S_OK;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int64_t b2s_gmres_workspace_bytes(int64_t num_rows, int64_t nnz,
                                  int64_t krylov_dim, int variant)
{
    if (num_rows < 1 || krylov_dim < 1 || krylov_dim > kMaxKrylov) return -1;
    switch (variant) {
    case B2S_GMRES_F64:
        return gmres_layout<double, double>(num_rows, nnz, int(krylov_dim), false).bytes;
    case B2S_GMRES_MIXED_F32:
        return gmres_layout<float, float>(num_rows, nnz, int(krylov_dim), true).bytes;
    case B2S_GMRES_MIXED_BF16:
        return gmres_layout<float, __nv_bfloat16>(num_rows, nnz, int(krylov_dim), true).bytes;
    default:
        return -1;
    }
}

int b2s_gmres_solve(int variant, int64_t num_rows, const int32_t* row_ptrs,
                    const int32_t* col_idxs, const double* values,
                    int64_t max_row_nnz, const double* inv_diag,
                    const double* b, double* x, int64_t krylov_dim,
                    int64_t max_iters, double reduction_factor,
                    double inner_reduction, void* workspace,
                    int64_t workspace_bytes, int64_t* iterations,
                    int64_t* restarts, double* residual_norm, int* converged,
                    void* stream)
{
    switch (variant) {
    case B2S_GMRES_F64:
        return gmres_engine<double, double>(
            num_rows, row_ptrs, col_idxs, values, max_row_nnz, inv_diag, b, x,
            int(krylov_dim), max_iters, reduction_factor, 0.0, workspace,
            workspace_bytes, iterations, restarts, residual_norm, converged,
            stream);
    case B2S_GMRES_MIXED_F32:
        return gmres_engine<float, float>(
            num_rows, row_ptrs, col_idxs, values, max_row_nnz, inv_diag, b, x,
            int(krylov_dim), max_iters, reduction_factor, inner_reduction,
            workspace, workspace_bytes, iterations, restarts, residual_norm,
            converged, stream);
    case B2S_GMRES_MIXED_BF16:
        return gmres_engine<float, __nv_bfloat16>(
            num_rows, row_ptrs, col_idxs, values, max_row_nnz, inv_diag, b, x,
            int(krylov_dim), max_iters, reduction_factor, inner_reduction,
            workspace, workspace_bytes, iterations, restarts, residual_norm,
            converged, stream);
    default:
        set_error("unknown GMRES variant %d", variant);
        return B2S_ERR_INVALID_ARG;
    }
}

}  // extern "C"
