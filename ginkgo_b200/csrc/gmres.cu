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
// Kernels per Arnoldi step j (one CUDA graph per restart cycle):
//   prepare v_j = round_basis(src * scale) stored in the basis (src = the
//           previous unnormalised vector, or r at j = 0); y = D^-1 v_j
//   spmv    w = A y with the pipelined Csr kernel (values and column
//           indices of the next row group copied with cp.async while the
//           current group is summed)
//   dots    h1 = V_{0..j}^T w and G(:, j) = V_{0..j}^T v_j, eight basis
//           vectors per pass over the rows; last block: h = (2I - G) h1
//   update  w'' = w - V h and ||w''||; last block: Hessenberg column,
//           Givens update, residual estimate, early end of the cycle, back
//           substitution
// per cycle: x += D^-1 V y (FP64 accumulate) with r = b, then r -= A x with
// the pipelined kernel in FP64, then ||r||, ||b|| and the restart check.
// The serial parts (Givens chain, back substitution, (2I - G) h1) run in
// the last block on shared-memory copies of the small arrays.
#include <cuda_bf16.h>

#include "csr_async.cuh"
#include "solver_common.cuh"

namespace b2s {
namespace {

constexpr int kMaxKrylov = 32;
constexpr int kLd = kMaxKrylov + 1;

struct GmresState {
    int done, cycle_done, j, final_iter;
    int total_iter, max_iters, outer_iter, converged;
    int krylov_dim;
    int idle;  // done || cycle_done: the Arnoldi kernels have nothing to do
    unsigned ticket;
    int pad;
    double bnorm, rnorm, reduction, inner_reduction, inner_thresh;
    double scale;  // v_j = src * scale: 1/||r|| at j = 0, 1/H(j, j-1) else
    double minus_one, one;       // alpha, beta of r = b - A x
    double h[kLd];               // combined projection coefficients of step j
    double H[kMaxKrylov * kLd];  // column j at H[j * kLd]
    double G[kLd * kLd];         // Gram matrix of the stored basis
    double g[kLd], cs[kMaxKrylov], sn[kMaxKrylov], y[kMaxKrylov];
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

// Step j, part 1: v_j = round_basis(src * scale) stored in the basis and
// y = D^-1 v_j, the SpMV input (src = the previous unnormalised vector, or
// r at j = 0).  One pass over n entries.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_prepare_kernel(int64_t n, const TA* __restrict__ dinv,
                         const double* __restrict__ r64,
                         const TA* __restrict__ w_src, TB* __restrict__ V,
                         TA* __restrict__ y, GmresState* st)
{
    if (st->idle) return;
    const int j = st->j;
    const TA scale = TA(st->scale);
    TB* vj = V + int64_t(j) * n;
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        const TA src = j == 0 ? TA(r64[row]) : w_src[row];
        const TB vb = to_basis<TB>(mul_rn(src, scale));
        vj[row] = vb;
        const TA va = from_basis<TA>(vb);
        y[row] = dinv ? dinv[row] * va : va;
    }
}

// Sums each of the 16 values v[0..15] over the warp with 16 shuffles (a
// butterfly that halves the values a lane carries at every level, instead
// of 16 separate reductions of 5 shuffles each).  Returns, in lane l, the
// warp total of value l / 2.
__device__ __forceinline__ double butterfly16(double (&v)[16], int lane)
{
    constexpr unsigned kFull = 0xffffffffu;
#pragma unroll
    for (int half = 8; half >= 1; half /= 2) {
        const bool up = lane & (2 * half);
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const double send = up ? v[i] : v[i + half];
            const double keep = up ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(kFull, send, 2 * half);
        }
    }
    return v[0] + __shfl_xor_sync(kFull, v[0], 1);
}

// Step j, part 3: h1 = V_{0..j}^T w and G(:, j) = V_{0..j}^T v_j, eight
// basis vectors per pass over the rows (w and v_j stay in L1/L2 between
// passes), two rows per thread and iteration.  Launched with a few blocks
// per SM, so the per-pass block reduction is amortised over many rows.
// Partials: per block 2 * kLd entries.  The last block completes G's row
// and column j and forms h = (2I - G) h1.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_dots_kernel(int64_t n, const TB* __restrict__ V,
                      const TA* __restrict__ w, GmresState* st,
                      double* __restrict__ partials)
{
    constexpr int C = 8;
    __shared__ double red[kSolverBlock / kWarp][2 * C];
    __shared__ double tot[2 * kLd];
    __shared__ double Gs[kLd * kLd];
    __shared__ int last;
    if (st->idle) return;
    const int j = st->j;
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
    const TB* vj = V + int64_t(j) * n;
    double* part = partials + int64_t(blockIdx.x) * 2 * kLd;
    const int64_t stride = int64_t(gridDim.x) * kSolverBlock;
    for (int i0 = 0; i0 <= j; i0 += C) {
        const int nv = j + 1 - i0 < C ? j + 1 - i0 : C;  // vectors this pass
        TA a[C], g[C];
#pragma unroll
        for (int u = 0; u < C; ++u) a[u] = g[u] = TA(0);
        int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x;
        for (; row + stride < n; row += 2 * stride) {
            const int64_t r1 = row + stride;
            const TA w0 = w[row], w1 = w[r1];
            const TA v0 = from_basis<TA>(vj[row]), v1 = from_basis<TA>(vj[r1]);
            TA x0[C], x1[C];
#pragma unroll
            for (int u = 0; u < C; ++u) {
                if (u < nv) {
                    x0[u] = from_basis<TA>(V[int64_t(i0 + u) * n + row]);
                    x1[u] = from_basis<TA>(V[int64_t(i0 + u) * n + r1]);
                }
            }
#pragma unroll
            for (int u = 0; u < C; ++u) {
                if (u < nv) {
                    a[u] += x0[u] * w0;
                    g[u] += x0[u] * v0;
                    a[u] += x1[u] * w1;
                    g[u] += x1[u] * v1;
                }
            }
        }
        if (row < n) {
            const TA w0 = w[row];
            const TA v0 = from_basis<TA>(vj[row]);
#pragma unroll
            for (int u = 0; u < C; ++u) {
                if (u < nv) {
                    const TA x0 = from_basis<TA>(V[int64_t(i0 + u) * n + row]);
                    a[u] += x0 * w0;
                    g[u] += x0 * v0;
                }
            }
        }
        double vals[2 * C];
#pragma unroll
        for (int u = 0; u < C; ++u) {
            vals[u] = double(a[u]);
            vals[C + u] = double(g[u]);
        }
        const double t = butterfly16(vals, lane);
        if ((lane & 1) == 0) red[wid][lane / 2] = t;
        __syncthreads();
        if (threadIdx.x < 2 * C) {
            const int u = threadIdx.x % C;
            if (u < nv) {
                double sum = 0.0;
                for (int k = 0; k < kSolverBlock / kWarp; ++k) sum += red[k][threadIdx.x];
                part[(threadIdx.x < C ? 0 : kLd) + i0 + u] = sum;
            }
        }
        __syncthreads();
    }
    if (last_block_done(&st->ticket, &last)) {
        // block-ordered sums of the 2 (j + 1) used entries
        for (int e = wid; e < 2 * kLd; e += kSolverBlock / kWarp) {
            if ((e % kLd) > j) continue;
            double s = 0.0;
            for (int b = lane; b < int(gridDim.x); b += kWarp) {
                s += __ldcg(partials + int64_t(b) * 2 * kLd + e);
            }
            s = warp_sum(s);
            if (lane == 0) tot[e] = s;
        }
        // G(0..j-1, 0..j-1) from the earlier steps of this cycle
        for (int e = threadIdx.x; e < j * kLd; e += kSolverBlock) Gs[e] = st->G[e];
        __syncthreads();
        if (threadIdx.x <= j) {
            const int i = threadIdx.x;
            const double gij = tot[kLd + i];
            Gs[i * kLd + j] = gij;
            Gs[j * kLd + i] = gij;
            st->G[i * kLd + j] = gij;
            st->G[j * kLd + i] = gij;
        }
        __syncthreads();
        // h = (2I - G) h1: CGS2's second projection from G
        if (threadIdx.x <= j) {
            const int i = threadIdx.x;
            double gh = 0.0;
            for (int k = 0; k <= j; ++k) gh += Gs[i * kLd + k] * tot[k];
            st->h[i] = 2.0 * tot[i] - gh;
        }
        if (threadIdx.x == 0) st->ticket = 0;
    }
}

// The end of Arnoldi step j, run by the whole last block of the update
// kernel: Givens update of column j, residual estimate, cycle bookkeeping
// and, when the cycle ends, the back substitution y = H \ g.  The small
// arrays are staged in shared memory, so the serial chain runs at
// shared-memory latency.
__device__ void close_step(GmresState* st, double hnorm)
{
    __shared__ double hc[kLd], gS[kLd], csS[kMaxKrylov], snS[kMaxKrylov];
    __shared__ double Hs[kMaxKrylov * kLd], ts[kMaxKrylov];
    __shared__ int fin;
    const int j = st->j;
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
        st->scale = hnorm > 0.0 ? 1.0 / hnorm : 0.0;
        st->j = j + 1;
        fin = est <= st->inner_thresh || j + 1 >= st->krylov_dim ||
              total >= st->max_iters || !(hnorm > 0.0);
        if (fin) {
            st->cycle_done = 1;
            st->idle = 1;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= j + 1; i += kSolverBlock) st->H[j * kLd + i] = hc[i];
    if (!fin) return;
    // y = H \ g over the m = j + 1 finished columns: one warp, column by
    // column from the last (t -= H(:, k) y_k after each y_k)
    const int m = j + 1;
    for (int e = threadIdx.x; e < j * kLd; e += kSolverBlock) Hs[e] = st->H[e];
    for (int i = threadIdx.x; i <= j; i += kSolverBlock) {
        Hs[j * kLd + i] = hc[i];
        ts[i] = gS[i];
    }
    __syncthreads();
    if (threadIdx.x < kWarp) {
        const int lane = threadIdx.x;
        for (int k = m - 1; k >= 0; --k) {
            const double yk = ts[k] / Hs[k * kLd + k];
            if (lane == 0) st->y[k] = yk;
            for (int i = lane; i < k; i += kWarp) ts[i] -= Hs[k * kLd + i] * yk;
            __syncwarp();
        }
    }
}

// w'' = w - V h, ||w''||; the last block closes the Arnoldi step.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_update_kernel(int64_t n, const TB* __restrict__ V, TA* __restrict__ w,
                        GmresState* st, double* __restrict__ partials)
{
    __shared__ double red[kSolverBlock / kWarp];
    __shared__ double tot[1];
    __shared__ TA hs[kLd];
    __shared__ int last;
    if (st->idle) return;
    const int j = st->j;
    for (int i = threadIdx.x; i <= j; i += kSolverBlock) hs[i] = TA(st->h[i]);
    __syncthreads();
    double nrm = 0.0;
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        TA wr = w[row];
        // eight basis loads in flight, subtracted in order i = 0..j
        for (int i0 = 0; i0 <= j; i0 += 8) {
            TA x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (i0 + u <= j) x[u] = from_basis<TA>(V[int64_t(i0 + u) * n + row]);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (i0 + u <= j) wr -= hs[i0 + u] * x[u];
            }
        }
        w[row] = wr;
        nrm += double(wr) * double(wr);
    }
    double a[1] = {nrm};
    block_partials<double, 1>(a, partials, red);
    if (last_block_done(&st->ticket, &last)) {
        sum_partials<double, 1>(partials, gridDim.x, tot, red);
        close_step(st, sqrt(tot[0]));
    }
}

// x += D^-1 (V y) over the finished columns, accumulated into FP64 x, and
// r = b (the start of r = b - A x).
template <typename TA, typename TB>
__global__ void __launch_bounds__(kSolverBlock)
    gmres_xupdate_kernel(int64_t n, const TB* __restrict__ V,
                         const TA* __restrict__ dinv, double* __restrict__ x,
                         const double* __restrict__ b, double* __restrict__ r,
                         GmresState* st)
{
    __shared__ TA ys[kMaxKrylov];
    if (st->done) return;
    const int m = st->final_iter;
    for (int i = threadIdx.x; i < m; i += kSolverBlock) ys[i] = TA(st->y[i]);
    __syncthreads();
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        if (m > 0) {
            TA u = TA(0);
            for (int i0 = 0; i0 < m; i0 += 8) {
                TA xv[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (i0 + q < m) xv[q] = from_basis<TA>(V[int64_t(i0 + q) * n + row]);
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (i0 + q < m) u += ys[i0 + q] * xv[q];
                }
            }
            const TA d = dinv ? dinv[row] : TA(1);
            x[row] += double(d * u);
        }
        r[row] = b[row];
    }
}

// ||r||, ||b|| of r = b - A x; the last block checks convergence and sets up
// the next cycle (the reference's restart step).
__global__ void __launch_bounds__(kSolverBlock)
    gmres_restart_kernel(int64_t n, const double* __restrict__ r,
                         const double* __restrict__ b, GmresState* st,
                         double* __restrict__ partials)
{
    __shared__ double red[kSolverBlock / kWarp * 2];
    __shared__ double tot[2];
    __shared__ int last;
    if (st->done) return;
    double acc2[2] = {0.0, 0.0};
    for (int64_t row = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; row < n;
         row += int64_t(gridDim.x) * kSolverBlock) {
        const double rr = r[row], bb = b[row];
        acc2[0] += rr * rr;
        acc2[1] += bb * bb;
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
    int64_t bytes, off_st, off_r, off_w0, off_w1, off_y, off_v, off_partials,
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
    l.off_y = c.take<TA>(n);
    l.off_v = c.take<TB>((int64_t(d) + 1) * n);
    l.off_partials = c.take<double>(int64_t(kSolverGrid) * 2 * kLd);
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
    TA* y = reinterpret_cast<TA*>(w + lay.off_y);
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
    h.idle = 1;
    h.minus_one = -1.0;
    h.one = 1.0;
    B2S_CUDA_TRY(cudaMemcpyAsync(gs, &h, sizeof(h), cudaMemcpyHostToDevice, st));

    const int grid_vec = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n, kSolverBlock)), kSolverGrid));
    const int grid_dots = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n, 2 * kSolverBlock)), int64_t(kNumSMs) * 2));
    // pipelined SpMV: persistent grid, as many blocks as fit at once
    const int lpr = async_lanes_per_row(max_row_nnz);
    const int64_t async_need = ceildiv(ceildiv(n, kWarp / lpr), kAsyncBlock / kWarp);
    // x += D^-1 V y and r = b; r -= A x (FP64); ||r||, ||b|| and the check
    auto restart = [&](cudaStream_t cs) {
        gmres_xupdate_kernel<TA, TB><<<grid_vec, kSolverBlock, 0, cs>>>(n, V, da, x, b,
                                                                        r, gs);
        with_async_kernel<double, 1, false>(lpr, [&](auto kernel) {
            const int64_t grid = std::min<int64_t>(async_need, async_resident_blocks(kernel));
            kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, v64, x, 1, r, 1,
                                                 &gs->minus_one, &gs->one, &gs->done);
        });
        gmres_restart_kernel<<<grid_vec, kSolverBlock, 0, cs>>>(n, r, b, gs, partials);
    };
    // first residual outside the graph (final_iter = 0: x is not touched)
    restart(st);
    B2S_LAUNCH_CHECK();
    auto capture = [&](cudaStream_t cs) -> int {
        for (int j = 0; j < krylov_dim; ++j) {
            TA* src = wv[(j + 1) % 2];
            TA* dst = wv[j % 2];
            gmres_prepare_kernel<TA, TB><<<grid_vec, kSolverBlock, 0, cs>>>(
                n, da, r, src, V, y, gs);
            with_async_kernel<TA, 1, false>(lpr, [&](auto kernel) {
                const int64_t grid = std::min<int64_t>(async_need,
                                                       async_resident_blocks(kernel));
                kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, va, y, 1, dst, 1,
                                                     nullptr, nullptr, &gs->idle);
            });
            gmres_dots_kernel<TA, TB><<<grid_dots, kSolverBlock, 0, cs>>>(
                n, V, dst, gs, partials);
            gmres_update_kernel<TA, TB><<<grid_vec, kSolverBlock, 0, cs>>>(
                n, V, dst, gs, partials);
            B2S_LAUNCH_CHECK();
        }
        restart(cs);
        B2S_LAUNCH_CHECK();
        return B2S_OK;
    };
    // the spmv of step j reads the vector prepared at step j; the update of
    // step j - 1 wrote the other w buffer, which prepare reads
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
