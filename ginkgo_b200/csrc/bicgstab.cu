// Fused preconditioned BiCGStab (scalar Jacobi, block Jacobi or identity),
// the loop of core/solver/bicgstab.cpp:95-250 with the kernels of
// common/unified/solver/bicgstab_kernels.cpp:23-195 regrouped into three
// passes per iteration, no host synchronisation inside the loop:
//
//   spmv1   p' = r + tmp (p - omega v), tmp = rho/prev_rho * alpha/omega
//           (p' = r when prev_rho * omega == 0) formed on the fly at every
//           column index; v' = A D^-1 p'; dot(rr, v') in-kernel; the last
//           block sets alpha = rho / dot(rr, v')   (step_1 + precond + SpMV
//           + dot + the alpha of step_2)
//   spmv2   s = r - alpha v' formed on the fly; t = A D^-1 s; dot(s, t),
//           dot(t, t), ||s||^2; the last block checks ||s|| (a column that
//           converges here is finalised by the next pass) and sets
//           omega = dot(s, t) / dot(t, t)     (step_2 + check + precond +
//           SpMV + the dots of step_3)
//   update  x += alpha D^-1 p' + omega D^-1 s, r = s - omega t (or only
//           x += alpha D^-1 p' for a column finalised at s); dot(rr, r),
//           ||r||^2; the last block advances the iteration and checks
//           (step_3 / finalize + next dot + check)
//
// p and v are double-buffered so every row reads the previous iterate.
//
// One right-hand side on a large system runs the two SpMV passes split, so
// the matrix streams through the pipelined Csr kernel with one gather per
// stored entry (forming p' and s at every gathered column triples the
// gathers once the vectors no longer sit in L2); four or more right-hand
// sides always run split, with the column-slice SpMV (bicg_vec_k_kernel,
// rhs_lanes_kernel, bicg_dot1k/2k_kernel), as does block Jacobi:
//   bicg_pupdate  p' and y = D^-1 p'      csr_async  v = A y
//   bicg_dot1     dot(rr, v) -> alpha      bicg_supdate  s, z = D^-1 s
//   csr_async     t = A z                  bicg_dot2  dot(s, t), dot(t, t),
//                                          ||s|| -> the check on s, omega
// then the update pass as above.  Every vector entry is rounded as in the
// fused passes.
#include "csr_async.cuh"
#include "jacobi_scheme.cuh"
#include "rhs_lanes.cuh"
#include "solver_common.cuh"

namespace b2s {
namespace {

template <typename T>
struct BicgScalars {
    T rho[kMaxRhs], prev_rho[kMaxRhs], alpha[kMaxRhs], omega[kMaxRhs],
        start[kMaxRhs], tau[kMaxRhs];
};

template <typename T>
__device__ __forceinline__ T bicg_p(T r, T p, T v, T tmp, T omega, bool from_r)
{
    return from_r ? r : add_rn(r, mul_rn(tmp, add_rn(p, -mul_rn(omega, v))));
}

template <typename T>
__device__ __forceinline__ T bicg_s(T r, T v, T alpha)
{
    return add_rn(r, -mul_rn(alpha, v));
}

// The last block's part of the update pass (thread 0): tot holds dot(rr, r)
// and ||r||^2 per column; finalises the columns that stopped at s, advances
// the iteration, swaps rho and applies the checks.
template <typename T, int K>
__device__ void bicg_update_finish(const T* tot, SolveCtl* ctl, BicgScalars<T>* sc)
{
    ctl->ticket = 0;
    int all_after_s = 1;
    for (int j = 0; j < K; ++j) all_after_s &= has_stopped(ctl->status[j]);
    const int iter = all_after_s ? ctl->iter : ctl->iter + 1;
    ctl->iter = iter;
    int all = 1;
    for (int j = 0; j < K; ++j) {
        uint8_t st = ctl->status[j];
        if (has_stopped(st)) {
            st |= kFinalizedMask;
        } else {
            sc->prev_rho[j] = sc->rho[j];
            sc->rho[j] = tot[j];
            sc->tau[j] = sqrt(tot[K + j]);
            if (residual_met(ctl, sc->tau[j], sc->rho[j], sc->start[j])) {
                converge_status(st, kResidualId, true);
            }
            if (iter >= ctl->max_iters) stop_status(st, kIterationId, true);
        }
        ctl->status[j] = st;
        all &= has_stopped(st);
    }
    ctl->all_stopped = all;
}

// The last block's part of the pass after the first SpMV (thread j < K):
// alpha = rho / dot(rr, v).
template <typename T, int K>
__device__ void bicg_alpha_finish(const T* tot, SolveCtl* ctl, BicgScalars<T>* sc)
{
    const int j = threadIdx.x;
    if (j < K && !has_stopped(ctl->status[j])) {
        const T bv = tot[j];
        sc->alpha[j] = bv != T(0) ? sc->rho[j] / bv : T(0);
    }
    if (threadIdx.x == 0) ctl->ticket = 0;
}

// The last block's part of the pass after the second SpMV (thread 0): tot
// holds dot(s, t), dot(t, t) and ||s||^2 per column; the check on s
// (without finalising: the update pass adds alpha y) and omega.
template <typename T, int K>
__device__ void bicg_omega_finish(const T* tot, SolveCtl* ctl, BicgScalars<T>* sc)
{
    ctl->ticket = 0;
    for (int j = 0; j < K; ++j) {
        uint8_t st = ctl->status[j];
        if (has_stopped(st)) continue;
        const T tau_s = sqrt(tot[2 * K + j]);
        if (residual_met(ctl, tau_s, sc->rho[j], sc->start[j])) {
            converge_status(st, kResidualId, false);
            sc->tau[j] = tau_s;
        }
        ctl->status[j] = st;
        const T tt = tot[K + j];
        sc->omega[j] = tt != T(0) ? tot[j] / tt : T(0);
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_init_kernel(int64_t n, const T* __restrict__ b, int64_t ldb, int k,
                     const T* __restrict__ r, T* __restrict__ rr,
                     T* __restrict__ p, T* __restrict__ v, SolveCtl* ctl,
                     BicgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * 3 * K];
    __shared__ T tot[3 * K];
    __shared__ int last;
    T acc[3 * K];
#pragma unroll
    for (int j = 0; j < 3 * K; ++j) acc[j] = T(0);
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const T ri = r[i * K + j];
            const T bb = j < k ? b[i * ldb + j] : T(0);
            rr[i * K + j] = ri;
            p[i * K + j] = T(0);
            v[i * K + j] = T(0);
            acc[j] += bb * bb;
            acc[K + j] += ri * ri;  // dot(rr, r) with rr = r
            acc[2 * K + j] += ri * ri;
        }
    }
    block_partials<T, 3 * K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 3 * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            ctl->ticket = 0;
            ctl->iter = 0;
            int all = 1;
            for (int j = 0; j < K; ++j) {
                uint8_t s = 0;
                if (j >= k) stop_status(s, kIterationId, true);
                sc->start[j] = start_norm(ctl, T(sqrt(tot[j])), T(sqrt(tot[2 * K + j])));
                sc->rho[j] = tot[K + j];
                sc->prev_rho[j] = T(1);
                sc->alpha[j] = T(1);
                sc->omega[j] = T(1);
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
    }
}

template <typename T, int SW, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_spmv1_kernel(int64_t n, const int32_t* __restrict__ rp,
                      const int32_t* __restrict__ ci, const T* __restrict__ a,
                      const T* __restrict__ dinv, const T* __restrict__ r,
                      const T* __restrict__ rr, const T* __restrict__ p_old,
                      const T* __restrict__ v_old, T* __restrict__ p_new,
                      T* __restrict__ v_new, SolveCtl* ctl, BicgScalars<T>* sc,
                      T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * K];
    __shared__ T tot[K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    bool active[K], from_r[K];
    T tmp[K], om[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = !has_stopped(ctl->status[j]);
        om[j] = sc->omega[j];
        from_r[j] = sc->prev_rho[j] * om[j] == T(0);
        tmp[j] = from_r[j] ? T(0) : sc->rho[j] / sc->prev_rho[j] * sc->alpha[j] / om[j];
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
            const T av = a[e];
            const int64_t c = ci[e];
            const T d = dinv ? dinv[c] : T(1);
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (active[j]) {
                    const T pc = bicg_p(r[c * K + j], p_old[c * K + j],
                                        v_old[c * K + j], tmp[j], om[j], from_r[j]);
                    acc[j] += av * mul_rn(d, pc);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = subwarp_sum<SW>(acc[j]);
        if (valid && lane == 0) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (active[j]) {
                    p_new[row * K + j] = bicg_p(r[row * K + j], p_old[row * K + j],
                                                v_old[row * K + j], tmp[j], om[j],
                                                from_r[j]);
                    v_new[row * K + j] = acc[j];
                    dot[j] += rr[row * K + j] * acc[j];
                }
            }
        }
    }
    block_partials<T, K>(dot, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, K>(partials, gridDim.x, tot, red);
        if (threadIdx.x < K) {
            const T bv = tot[threadIdx.x];
            sc->alpha[threadIdx.x] = bv != T(0) ? sc->rho[threadIdx.x] / bv : T(0);
        }
        if (threadIdx.x == 0) ctl->ticket = 0;
    }
}

template <typename T, int SW, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_spmv2_kernel(int64_t n, const int32_t* __restrict__ rp,
                      const int32_t* __restrict__ ci, const T* __restrict__ a,
                      const T* __restrict__ dinv, const T* __restrict__ r,
                      const T* __restrict__ vv, T* __restrict__ s,
                      T* __restrict__ t, SolveCtl* ctl, BicgScalars<T>* sc,
                      T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * 3 * K];
    __shared__ T tot[3 * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    bool active[K];
    T alpha[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = !has_stopped(ctl->status[j]);
        alpha[j] = sc->alpha[j];
    }
    T acc3[3 * K];
#pragma unroll
    for (int j = 0; j < 3 * K; ++j) acc3[j] = T(0);
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
            const T av = a[e];
            const int64_t c = ci[e];
            const T d = dinv ? dinv[c] : T(1);
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (active[j]) {
                    acc[j] += av * mul_rn(d, bicg_s(r[c * K + j], vv[c * K + j], alpha[j]));
                }
            }
        }
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] = subwarp_sum<SW>(acc[j]);
        if (valid && lane == 0) {
#pragma unroll
            for (int j = 0; j < K; ++j) {
                if (active[j]) {
                    const T sr = bicg_s(r[row * K + j], vv[row * K + j], alpha[j]);
                    s[row * K + j] = sr;
                    t[row * K + j] = acc[j];
                    acc3[j] += sr * acc[j];
                    acc3[K + j] += acc[j] * acc[j];
                    acc3[2 * K + j] += sr * sr;
                }
            }
        }
    }
    block_partials<T, 3 * K>(acc3, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 3 * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            ctl->ticket = 0;
            for (int j = 0; j < K; ++j) {
                uint8_t st = ctl->status[j];
                if (has_stopped(st)) continue;
                const T tau_s = sqrt(tot[2 * K + j]);
                // check on s without finalising (core/solver/bicgstab.cpp
                // second check): the update pass adds alpha y and finalises
                if (residual_met(ctl, tau_s, sc->rho[j], sc->start[j])) {
                    converge_status(st, kResidualId, false);
                    sc->tau[j] = tau_s;
                }
                ctl->status[j] = st;
                const T tt = tot[K + j];
                sc->omega[j] = tt != T(0) ? tot[j] / tt : T(0);
            }
        }
    }
}

// zs: block Jacobi, x += alpha p + omega zs with p = M p' and zs = M s
// already formed (dinv then null); null: x += alpha D^-1 p + omega D^-1 s.
template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_update_kernel(int64_t n, const T* __restrict__ dinv,
                       T* __restrict__ x, int64_t ldx, T* __restrict__ r,
                       const T* __restrict__ rr, const T* __restrict__ p,
                       const T* __restrict__ s, const T* __restrict__ t,
                       SolveCtl* ctl, BicgScalars<T>* sc,
                       T* __restrict__ partials, const T* __restrict__ zs = nullptr)
{
    __shared__ T red[kSolverBlock / kWarp * 2 * K];
    __shared__ T tot[2 * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    int mode[K];  // 0 frozen, 1 finalise at s, 2 full update
    T alpha[K], omega[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const uint8_t st = ctl->status[j];
        mode[j] = !has_stopped(st) ? 2 : (is_finalized(st) ? 0 : 1);
        alpha[j] = sc->alpha[j];
        omega[j] = sc->omega[j];
    }
    T acc[2 * K];
#pragma unroll
    for (int j = 0; j < 2 * K; ++j) acc[j] = T(0);
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T d = dinv ? dinv[i] : T(1);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (mode[j] == 1) {
                x[i * ldx + j] += alpha[j] * mul_rn(d, p[i * K + j]);
            } else if (mode[j] == 2) {
                const T si = s[i * K + j];
                const T zi = zs ? zs[i * K + j] : mul_rn(d, si);
                x[i * ldx + j] += alpha[j] * mul_rn(d, p[i * K + j]) + omega[j] * zi;
                const T ri = si - omega[j] * t[i * K + j];
                r[i * K + j] = ri;
                acc[j] += rr[i * K + j] * ri;
                acc[K + j] += ri * ri;
            }
        }
    }
    block_partials<T, 2 * K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 2 * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) bicg_update_finish<T, K>(tot, ctl, sc);
    }
}

constexpr int64_t kBicgSplitRows = int64_t(1) << 19;

template <typename T>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_pupdate_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r,
                        const T* __restrict__ p_old, const T* __restrict__ v_old,
                        T* __restrict__ p_new, T* __restrict__ y, SolveCtl* ctl,
                        BicgScalars<T>* sc)
{
    if (ctl->all_stopped) return;
    const T om = sc->omega[0];
    const bool from_r = sc->prev_rho[0] * om == T(0);
    const T tmp = from_r ? T(0) : sc->rho[0] / sc->prev_rho[0] * sc->alpha[0] / om;
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T pc = bicg_p(r[i], p_old[i], v_old[i], tmp, om, from_r);
        p_new[i] = pc;
        y[i] = dinv ? mul_rn(dinv[i], pc) : pc;
    }
}

template <typename T>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_dot1_kernel(int64_t n, const T* __restrict__ rr, const T* __restrict__ v,
                     SolveCtl* ctl, BicgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp];
    __shared__ T tot[1];
    __shared__ int last;
    if (ctl->all_stopped) return;
    T acc[1] = {T(0)};
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        acc[0] += rr[i] * v[i];
    }
    block_partials<T, 1>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 1>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            const T bv = tot[0];
            sc->alpha[0] = bv != T(0) ? sc->rho[0] / bv : T(0);
            ctl->ticket = 0;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_supdate_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r,
                        const T* __restrict__ v, T* __restrict__ s, T* __restrict__ z,
                        SolveCtl* ctl, BicgScalars<T>* sc)
{
    if (ctl->all_stopped) return;
    const T alpha = sc->alpha[0];
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T sr = bicg_s(r[i], v[i], alpha);
        s[i] = sr;
        z[i] = dinv ? mul_rn(dinv[i], sr) : sr;
    }
}

template <typename T>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_dot2_kernel(int64_t n, const T* __restrict__ s, const T* __restrict__ t,
                     SolveCtl* ctl, BicgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * 3];
    __shared__ T tot[3];
    __shared__ int last;
    if (ctl->all_stopped) return;
    T acc[3] = {T(0), T(0), T(0)};
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T si = s[i], ti = t[i];
        acc[0] += si * ti;
        acc[1] += ti * ti;
        acc[2] += si * si;
    }
    block_partials<T, 3>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 3>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) {
            ctl->ticket = 0;
            uint8_t st = ctl->status[0];
            if (!has_stopped(st)) {
                const T tau_s = sqrt(tot[2]);
                // the check on s without finalising, as in bicg_spmv2_kernel
                if (residual_met(ctl, tau_s, sc->rho[0], sc->start[0])) {
                    converge_status(st, kResidualId, false);
                    sc->tau[0] = tau_s;
                }
                ctl->status[0] = st;
                sc->omega[0] = tot[1] != T(0) ? tot[0] / tot[1] : T(0);
            }
        }
    }
}

// The split passes' vector updates for K columns (several right-hand
// sides): STEP 1 p' = r + tmp (p - omega v) and y = D^-1 p'; STEP 2
// s = r - alpha v and z = D^-1 s.  Stopped columns are left as they are.
template <typename T, int K, int STEP>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_vec_k_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r,
                      const T* __restrict__ a_old, const T* __restrict__ v_old,
                      T* __restrict__ out, T* __restrict__ prec, SolveCtl* ctl,
                      BicgScalars<T>* sc)
{
    if (ctl->all_stopped) return;
    bool active[K], from_r[K];
    T c1[K], c2[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = !has_stopped(ctl->status[j]);
        if (STEP == 1) {
            c2[j] = sc->omega[j];
            from_r[j] = sc->prev_rho[j] * c2[j] == T(0);
            c1[j] = from_r[j] ? T(0) : sc->rho[j] / sc->prev_rho[j] * sc->alpha[j] / c2[j];
        } else {
            from_r[j] = false;
            c1[j] = sc->alpha[j];
            c2[j] = T(0);
        }
    }
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
        const T d = dinv ? dinv[i] : T(1);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (!active[j]) continue;
            const int64_t e = i * K + j;
            const T val = STEP == 1 ? bicg_p(r[e], a_old[e], v_old[e], c1[j], c2[j], from_r[j])
                                    : bicg_s(r[e], a_old[e], c1[j]);
            out[e] = val;
            prec[e] = dinv ? mul_rn(d, val) : val;
        }
    }
}

// ---------------------------------------------------------------------------
// The split passes for K >= 4 right-hand sides with 16-byte column slices
// (K a multiple of VW = 16 / sizeof(T)): the n x K blocks are walked as one
// flat array of 16-byte vectors, thread t owning the VW columns
// (t mod KL) * VW.. of row t / KL (KL = K / VW); the grid stride is a
// multiple of KL, so a thread keeps its columns and the per-column sums
// reduce over the lanes that share them (shuffles over lane offsets KL,
// 2 KL, ...), then over the block's warps and the blocks (partials
// [sum][block][K], deterministic).  Same arithmetic as the row-wise
// kernels above; stopped columns keep their values.
// ---------------------------------------------------------------------------
template <typename T, int K, int STEP>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_vec_lanes_kernel(int64_t n, const T* __restrict__ dinv, const T* __restrict__ r,
                          const T* __restrict__ a_old, const T* __restrict__ v_old,
                          T* __restrict__ out, T* __restrict__ prec, SolveCtl* ctl,
                          BicgScalars<T>* sc)
{
    constexpr int VW = int(16 / sizeof(T));
    constexpr int KL = K / VW;
    if (ctl->all_stopped) return;
    const int64_t t0 = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x;
    const int col0 = int(t0 % KL) * VW;
    bool active[VW], from_r[VW];
    T c1[VW], c2[VW];
#pragma unroll
    for (int u = 0; u < VW; ++u) {
        const int j = col0 + u;
        active[u] = !has_stopped(ctl->status[j]);
        if (STEP == 1) {
            c2[u] = sc->omega[j];
            from_r[u] = sc->prev_rho[j] * c2[u] == T(0);
            c1[u] = from_r[u] ? T(0) : sc->rho[j] / sc->prev_rho[j] * sc->alpha[j] / c2[u];
        } else {
            from_r[u] = false;
            c1[u] = sc->alpha[j];
            c2[u] = T(0);
        }
    }
    const int64_t nvec = n * KL;
    for (int64_t t = t0; t < nvec; t += int64_t(gridDim.x) * kSolverBlock) {
        const int64_t i = t / KL, e = t * VW;
        const T d = dinv ? dinv[i] : T(1);
        T rv[VW], av[VW], vv[VW], val[VW], pv[VW];
        ld_vec<T, VW>(r + e, rv);
        ld_vec<T, VW>(a_old + e, av);
        if (STEP == 1) ld_vec<T, VW>(v_old + e, vv);
#pragma unroll
        for (int u = 0; u < VW; ++u) {
            if (active[u]) {
                val[u] = STEP == 1 ? bicg_p(rv[u], av[u], vv[u], c1[u], c2[u], from_r[u])
                                   : bicg_s(rv[u], av[u], c1[u]);
            } else {
                val[u] = STEP == 1 ? av[u] : rv[u];
            }
            pv[u] = dinv ? mul_rn(d, val[u]) : val[u];
        }
        st_vec<T, VW>(out + e, val);
        st_vec<T, VW>(prec + e, pv);
    }
}

// Sums NS products per column over the lanes that share the column slice,
// the block's warps (red[W][NS * K]) and the blocks: partials[m][block][K].
template <typename T, int K, int NS>
__device__ __forceinline__ void lanes_partials(T (&acc)[NS][int(16 / sizeof(T))], int col0,
                                               T* __restrict__ partials, T* red)
{
    constexpr int VW = int(16 / sizeof(T));
    constexpr int KL = K / VW;
    constexpr int W = kSolverBlock / kWarp;
    const int lane = threadIdx.x % kWarp, wid = threadIdx.x / kWarp;
#pragma unroll
    for (int off = KL; off < kWarp; off *= 2) {
#pragma unroll
        for (int m = 0; m < NS; ++m) {
#pragma unroll
            for (int u = 0; u < VW; ++u) {
                acc[m][u] += __shfl_xor_sync(0xffffffffu, acc[m][u], off);
            }
        }
    }
    if (lane < KL) {
#pragma unroll
        for (int m = 0; m < NS; ++m) {
#pragma unroll
            for (int u = 0; u < VW; ++u) red[wid * NS * K + m * K + col0 + u] = acc[m][u];
        }
    }
    __syncthreads();
    if (threadIdx.x < NS * K) {
        T s = T(0);
        for (int w = 0; w < W; ++w) s += red[w * NS * K + threadIdx.x];
        const int m = threadIdx.x / K, j = threadIdx.x % K;
        partials[int64_t(m) * gridDim.x * K + int64_t(blockIdx.x) * K + j] = s;
    }
}

// The last block: tot[m * K + j] = sum over blocks of partials[m][.][j].
template <typename T, int K, int NS>
__device__ __forceinline__ void lanes_totals(const T* __restrict__ partials, T* tot, T* red)
{
#pragma unroll
    for (int m = 0; m < NS; ++m) {
        sum_partials<T, K>(partials + int64_t(m) * gridDim.x * K, gridDim.x, tot + m * K, red);
    }
}

// NS = 1: dot(rr, v) -> alpha; NS = 3: dot(s, t), dot(t, t), ||s||^2 ->
// the check on s and omega
template <typename T, int K, int NS>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_dots_lanes_kernel(int64_t n, const T* __restrict__ a, const T* __restrict__ b,
                           SolveCtl* ctl, BicgScalars<T>* sc, T* __restrict__ partials)
{
    constexpr int VW = int(16 / sizeof(T));
    constexpr int KL = K / VW;
    __shared__ T red[kSolverBlock / kWarp * NS * K];
    __shared__ T tot[NS * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    const int64_t t0 = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x;
    const int col0 = int(t0 % KL) * VW;
    T acc[NS][VW];
#pragma unroll
    for (int m = 0; m < NS; ++m) {
#pragma unroll
        for (int u = 0; u < VW; ++u) acc[m][u] = T(0);
    }
    const int64_t nvec = n * KL;
    for (int64_t t = t0; t < nvec; t += int64_t(gridDim.x) * kSolverBlock) {
        T av[VW], bv[VW];
        ld_vec<T, VW>(a + t * VW, av);
        ld_vec<T, VW>(b + t * VW, bv);
#pragma unroll
        for (int u = 0; u < VW; ++u) {
            acc[0][u] += av[u] * bv[u];
            if constexpr (NS == 3) {
                acc[1][u] += bv[u] * bv[u];
                acc[2][u] += av[u] * av[u];
            }
        }
    }
    lanes_partials<T, K, NS>(acc, col0, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        lanes_totals<T, K, NS>(partials, tot, red);
        if constexpr (NS == 1) {
            bicg_alpha_finish<T, K>(tot, ctl, sc);
        } else {
            if (threadIdx.x == 0) bicg_omega_finish<T, K>(tot, ctl, sc);
        }
    }
}

// x += alpha y + omega z (alpha y alone for a column finalised at s),
// r = s - omega t, then dot(rr, r) and ||r||^2 per column
template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_update_lanes_kernel(int64_t n, T* __restrict__ x, int64_t ldx, T* __restrict__ r,
                             const T* __restrict__ rr, const T* __restrict__ y,
                             const T* __restrict__ s, const T* __restrict__ t,
                             const T* __restrict__ z, SolveCtl* ctl, BicgScalars<T>* sc,
                             T* __restrict__ partials)
{
    constexpr int VW = int(16 / sizeof(T));
    constexpr int KL = K / VW;
    __shared__ T red[kSolverBlock / kWarp * 2 * K];
    __shared__ T tot[2 * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    const int64_t t0 = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x;
    const int col0 = int(t0 % KL) * VW;
    int mode[VW];  // 0 frozen, 1 finalise at s, 2 full update
    T alpha[VW], omega[VW];
#pragma unroll
    for (int u = 0; u < VW; ++u) {
        const uint8_t st = ctl->status[col0 + u];
        mode[u] = !has_stopped(st) ? 2 : (is_finalized(st) ? 0 : 1);
        alpha[u] = sc->alpha[col0 + u];
        omega[u] = sc->omega[col0 + u];
    }
    T acc[2][VW];
#pragma unroll
    for (int u = 0; u < VW; ++u) acc[0][u] = acc[1][u] = T(0);
    const int64_t nvec = n * KL;
    for (int64_t q = t0; q < nvec; q += int64_t(gridDim.x) * kSolverBlock) {
        const int64_t i = q / KL, e = q * VW;
        T yv[VW], sv[VW], tv[VW], zv[VW], rv[VW], hv[VW];
        ld_vec<T, VW>(y + e, yv);
        ld_vec<T, VW>(s + e, sv);
        ld_vec<T, VW>(t + e, tv);
        ld_vec<T, VW>(z + e, zv);
        ld_vec<T, VW>(r + e, rv);
        ld_vec<T, VW>(rr + e, hv);
        T* xr = x + i * ldx + col0;
#pragma unroll
        for (int u = 0; u < VW; ++u) {
            if (mode[u] == 1) {
                xr[u] += alpha[u] * yv[u];
            } else if (mode[u] == 2) {
                xr[u] += alpha[u] * yv[u] + omega[u] * zv[u];
                const T ri = sv[u] - omega[u] * tv[u];
                rv[u] = ri;
                acc[0][u] += hv[u] * ri;
                acc[1][u] += ri * ri;
            }
        }
        st_vec<T, VW>(r + e, rv);
    }
    lanes_partials<T, K, 2>(acc, col0, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        lanes_totals<T, K, 2>(partials, tot, red);
        if (threadIdx.x == 0) bicg_update_finish<T, K>(tot, ctl, sc);
    }
}

// ---------------------------------------------------------------------------
// Block Jacobi (right preconditioning by the block-diagonal inverse M): the
// preconditioned vectors M p' and M s are no longer row-wise scales, so the
// iteration runs split for any number of right-hand sides:
//   bicg_block_vec  p' = r + tmp (p - omega v) and y = M p'   (STEP 1)
//   csr_async       v = A y
//   bicg_dot1k      dot(rr, v) -> alpha
//   bicg_block_vec  s = r - alpha v and z = M s             (STEP 2)
//   csr_async       t = A z
//   bicg_dot2k      dot(s, t), dot(t, t), ||s|| -> check on s, omega
//   bicg_update     x += alpha y + omega z, r = s - omega t (zs = z)
// bicg_block_vec runs one warp per group of the block-interleaved storage,
// lane (sub, i) owning row i of block sub: the block's lanes form their
// rows' entries, then M times them by shuffles (apply_block's column order,
// reference/preconditioner/jacobi_kernels.cpp:419-445).  The sequence is
// core/solver/bicgstab.cpp:190-250 with the preconditioner applies at
// :194 and :229.
// ---------------------------------------------------------------------------
template <typename T, int MB2, int K, int STEP, int SK>
__global__ void __launch_bounds__(kSolverBlock, (MB2 > 8 ? 0 : SK == kF16 ? 6 : SK >= 0 ? 5 : 0))
    bicg_block_vec_kernel(int64_t n, BlockPrec<T> bp, const T* __restrict__ r,
                          const T* __restrict__ a_old, const T* __restrict__ v_old,
                          T* __restrict__ out, T* __restrict__ prec, SolveCtl* ctl,
                          BicgScalars<T>* sc)
{
    constexpr unsigned kFull = 0xffffffffu;
    if (ctl->all_stopped) return;
    bool active[K], from_r[K];
    T c1[K], c2[K];  // STEP 1: tmp, omega; STEP 2: alpha
#pragma unroll
    for (int j = 0; j < K; ++j) {
        active[j] = !has_stopped(ctl->status[j]);
        if (STEP == 1) {
            c2[j] = sc->omega[j];
            from_r[j] = sc->prev_rho[j] * c2[j] == T(0);
            c1[j] = from_r[j] ? T(0) : sc->rho[j] / sc->prev_rho[j] * sc->alpha[j] / c2[j];
        } else {
            from_r[j] = false;
            c1[j] = sc->alpha[j];
            c2[j] = T(0);
        }
    }
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
        int s0 = 0, bs = 0;
        const bool in_block = in_group && blk < bp.num_blocks &&
                              block_extent(bp.ptrs, blk, n, bp.max_bs, s0, bs);
        const bool act = in_block && i < bs;
        const int64_t row = s0 + i;
        BlockRow<SK, MB2, T> inv;
        inv.load(bp, bsc, grp, lane, in_group);
#pragma unroll
        for (int j = 0; j < K; ++j) {
            if (!active[j]) continue;  // uniform
            T val = T(0);
            if (act) {
                const int64_t e = row * K + j;
                val = STEP == 1 ? bicg_p(r[e], a_old[e], v_old[e], c1[j], c2[j], from_r[j])
                                : bicg_s(r[e], a_old[e], c1[j]);
                out[e] = val;
            }
            T mz = T(0);
#pragma unroll
            for (int c = 0; c < MB2; ++c) {
                if (c < bp.max_bs) {
                    const T vc = __shfl_sync(kFull, val, (base + c) % kWarp);
                    if (act && c < bs) mz += inv[c] * vc;
                }
            }
            if (act) prec[row * K + j] = mz;
        }
    }
}

// dot(rr, v) per column; the last block sets alpha (as bicg_spmv1_kernel)
template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_dot1k_kernel(int64_t n, const T* __restrict__ rr, const T* __restrict__ v,
                      SolveCtl* ctl, BicgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * K];
    __shared__ T tot[K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    T acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = T(0);
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] += rr[i * K + j] * v[i * K + j];
    }
    block_partials<T, K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, K>(partials, gridDim.x, tot, red);
        bicg_alpha_finish<T, K>(tot, ctl, sc);
    }
}

// dot(s, t), dot(t, t), ||s||^2 per column; the last block checks s and
// sets omega (as bicg_spmv2_kernel)
template <typename T, int K>
__global__ void __launch_bounds__(kSolverBlock)
    bicg_dot2k_kernel(int64_t n, const T* __restrict__ s, const T* __restrict__ t,
                      SolveCtl* ctl, BicgScalars<T>* sc, T* __restrict__ partials)
{
    __shared__ T red[kSolverBlock / kWarp * 3 * K];
    __shared__ T tot[3 * K];
    __shared__ int last;
    if (ctl->all_stopped) return;
    T acc[3 * K];
#pragma unroll
    for (int j = 0; j < 3 * K; ++j) acc[j] = T(0);
    for (int64_t i = blockIdx.x * int64_t(kSolverBlock) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kSolverBlock) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const T si = s[i * K + j], ti = t[i * K + j];
            acc[j] += si * ti;
            acc[K + j] += ti * ti;
            acc[2 * K + j] += si * si;
        }
    }
    block_partials<T, 3 * K>(acc, partials, red);
    if (last_block_done(&ctl->ticket, &last)) {
        sum_partials<T, 3 * K>(partials, gridDim.x, tot, red);
        if (threadIdx.x == 0) bicg_omega_finish<T, K>(tot, ctl, sc);
    }
}

// grid of the warp-per-group block kernels
template <typename T>
int bicg_block_grid(const BlockPrec<T>& bp)
{
    const BlockScheme bsc = block_scheme(bp.max_bs);
    const int64_t ngroups = ceildiv(bp.num_blocks, bsc.gs);
    return int(std::min<int64_t>(std::max<int64_t>(1, ceildiv(ngroups, kSolverBlock / kWarp)),
                                 solver_grid()));
}

template <typename T, int K, int STEP>
void launch_bicg_block_vec(int64_t n, const BlockPrec<T>& bp, const T* r, const T* a_old,
                           const T* v_old, T* out, T* prec, SolveCtl* ctl,
                           BicgScalars<T>* sc, cudaStream_t st)
{
    const int grid = bicg_block_grid(bp);
#define B2S_BICG_BLOCK(MB)                                                        \
    case MB:                                                                      \
        with_pass_kind<T, K == 1>(bp, [&](auto sk) {                              \
            auto kernel = bicg_block_vec_kernel<T, MB, K, STEP, decltype(sk)::value>; \
            kernel<<<pgrid(kernel, grid), kSolverBlock, 0, st>>>(                 \
                n, bp, r, a_old, v_old, out, prec, ctl, sc);                      \
        });                                                                       \
        break;
    switch (kMaxBs / block_scheme(bp.max_bs).gs) {
        B2S_BICG_BLOCK(2)
        B2S_BICG_BLOCK(4)
        B2S_BICG_BLOCK(8)
        B2S_BICG_BLOCK(16)
        B2S_BICG_BLOCK(32)
    default: B2S_BICG_BLOCK(1)
    }
#undef B2S_BICG_BLOCK
}

struct BicgLayout {
    int64_t bytes, off_ctl, off_sc, off_r, off_rr, off_p0, off_p1, off_v0,
        off_v1, off_s, off_t, off_partials, off_y, off_z;
};

template <typename T>
BicgLayout bicg_layout(int64_t n, int K, bool with_yz = false)
{
    Carver c{nullptr};
    BicgLayout l;
    l.off_ctl = c.take<SolveCtl>(1);
    l.off_sc = c.take<BicgScalars<T>>(1);
    l.off_r = c.take<T>(n * K);
    l.off_rr = c.take<T>(n * K);
    l.off_p0 = c.take<T>(n * K);
    l.off_p1 = c.take<T>(n * K);
    l.off_v0 = c.take<T>(n * K);
    l.off_v1 = c.take<T>(n * K);
    l.off_s = c.take<T>(n * K);
    l.off_t = c.take<T>(n * K);
    l.off_partials = c.take<T>(int64_t(kSolverGrid) * 3 * K);
    // the SpMV inputs of the split passes (single column, or block Jacobi)
    l.off_y = K == 1 || K >= 4 || with_yz ? c.take<T>(n * K) : 0;
    l.off_z = K == 1 || K >= 4 || with_yz ? c.take<T>(n * K) : 0;
    l.bytes = c.used;
    return l;
}

// bp: a block Jacobi preconditioner (dinv then null), or null
template <typename T>
int bicgstab_solve(int64_t n, const int32_t* rp, const int32_t* ci, const T* v,
                   int64_t max_row_nnz, const T* dinv, const BlockPrec<T>* bp,
                   const T* b, int64_t ldb,
                   T* x, int64_t ldx, int64_t k, int64_t max_iters,
                   double reduction, int residual_mode, int64_t check_every,
                   void* workspace,
                   int64_t workspace_bytes, int64_t* iterations,
                   double* residual_norms, uint8_t* status, void* stream)
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
    const BicgLayout lay = bicg_layout<T>(n, K, bp != nullptr);
    if (workspace_bytes < lay.bytes) {
        set_error("workspace of %lld bytes < %lld", (long long)workspace_bytes,
                  (long long)lay.bytes);
        return B2S_ERR_WORKSPACE;
    }
    B2S_CHECK_ARG(workspace != nullptr && b && x && rp, "null pointer");
    cudaStream_t st = as_stream(stream);
    char* w = static_cast<char*>(workspace);
    auto* ctl = reinterpret_cast<SolveCtl*>(w + lay.off_ctl);
    auto* sc = reinterpret_cast<BicgScalars<T>*>(w + lay.off_sc);
    T* r = reinterpret_cast<T*>(w + lay.off_r);
    T* rr = reinterpret_cast<T*>(w + lay.off_rr);
    T* p[2] = {reinterpret_cast<T*>(w + lay.off_p0), reinterpret_cast<T*>(w + lay.off_p1)};
    T* vv[2] = {reinterpret_cast<T*>(w + lay.off_v0), reinterpret_cast<T*>(w + lay.off_v1)};
    T* s = reinterpret_cast<T*>(w + lay.off_s);
    T* t = reinterpret_cast<T*>(w + lay.off_t);
    T* partials = reinterpret_cast<T*>(w + lay.off_partials);
    T* yv = K == 1 || K >= 4 || bp ? reinterpret_cast<T*>(w + lay.off_y) : nullptr;
    T* zv = K == 1 || K >= 4 || bp ? reinterpret_cast<T*>(w + lay.off_z) : nullptr;

    SolveCtl h{};
    h.max_iters = int(max_iters);
    h.reduction = reduction;
    h.baseline = residual_mode & ~B2S_STOP_IMPLICIT;
    h.implicit = (residual_mode & B2S_STOP_IMPLICIT) != 0;
    B2S_CUDA_TRY(cudaMemcpyAsync(ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    const int sw = solver_subwarp(max_row_nnz);
    const int grid_spmv = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n * sw, kSolverBlock)), solver_grid()));
    const int grid_vec = int(std::min<int64_t>(
        std::max<int64_t>(1, ceildiv(n, kSolverBlock)), solver_grid()));
    const int chunk = int(std::max<int64_t>(2, (check_every + 1) / 2 * 2));
    B2S_DISPATCH_RHS(K, {
        B2S_DISPATCH_SW(sw, {
            residual_kernel<T, SW, K><<<pgrid(residual_kernel<T, SW, K>, grid_spmv), kSolverBlock, 0, st>>>(
                n, rp, ci, v, x, ldx, b, ldb, int(k), r);
        });
        B2S_LAUNCH_CHECK();
        bicg_init_kernel<T, K><<<pgrid(bicg_init_kernel<T, K>, grid_vec), kSolverBlock, 0, st>>>(
            n, b, ldb, int(k), r, rr, p[0], vv[0], ctl, sc, partials);
        B2S_LAUNCH_CHECK();
    });
    // the split single-RHS passes (large systems)
    const int lpr = async_lanes_per_row(max_row_nnz);
    const int64_t async_need = ceildiv(ceildiv(n, kWarp / lpr), kAsyncBlock / kWarp);
    auto async_spmv = [&](cudaStream_t cs, const T* in, T* out) {
        with_async_kernel<T, 1, false>(lpr, [&](auto kernel) {
            const int64_t grid = std::min<int64_t>(async_need, async_resident_blocks(kernel));
            kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, v, in, 1, out, 1, nullptr,
                                                 nullptr, &ctl->all_stopped);
        });
    };
    const bool split = K == 1 && n >= kBicgSplitRows;
    // the split passes with K columns: block Jacobi (any K), and four or
    // more right-hand sides (forming p' and s at every gathered column
    // would read 3 K values per stored entry); the SpMVs with lanes owning
    // 16-byte column slices where K allows, else the pipelined kernel
    auto split_k_iteration = [&](cudaStream_t cs, int o, int nw) {
        B2S_DISPATCH_RHS(K, {
            auto spmv_k = [&](const T* in, T* out) {
                if constexpr (K >= 4 && K % Vec16<T>::width == 0) {
                    launch_csr_lanes<T, K>(n, rp, ci, v, in, K, out, K, nullptr, nullptr, cs,
                                           &ctl->all_stopped);
                } else {
                    with_async_kernel<T, K, (K >= 2)>(lpr, [&](auto kernel) {
                        const int64_t grid = std::min<int64_t>(async_need,
                                                               async_resident_blocks(kernel));
                        kernel<<<grid, kAsyncBlock, 0, cs>>>(n, rp, ci, v, in, K, out, K,
                                                             nullptr, nullptr,
                                                             &ctl->all_stopped);
                    });
                }
            };
            constexpr bool kLanes = K >= 4 && K % Vec16<T>::width == 0;
            // the flat vector passes: one wave of 16-byte vectors per thread
            const int grid_lanes = int(std::min<int64_t>(
                std::max<int64_t>(1, ceildiv(n * K / Vec16<T>::width, kSolverBlock)),
                solver_grid()));
            if (bp) {
                launch_bicg_block_vec<T, K, 1>(n, *bp, r, p[o], vv[o], p[nw], yv, ctl, sc, cs);
            } else if constexpr (kLanes) {
                bicg_vec_lanes_kernel<T, K, 1><<<pgrid(bicg_vec_lanes_kernel<T, K, 1>, grid_lanes), kSolverBlock, 0, cs>>>(
                    n, dinv, r, p[o], vv[o], p[nw], yv, ctl, sc);
            } else {
                bicg_vec_k_kernel<T, K, 1><<<pgrid(bicg_vec_k_kernel<T, K, 1>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, dinv, r, p[o], vv[o], p[nw], yv, ctl, sc);
            }
            spmv_k(yv, vv[nw]);
            if constexpr (kLanes) {
                bicg_dots_lanes_kernel<T, K, 1><<<pgrid(bicg_dots_lanes_kernel<T, K, 1>, grid_lanes), kSolverBlock, 0, cs>>>(
                    n, rr, vv[nw], ctl, sc, partials);
            } else {
                bicg_dot1k_kernel<T, K><<<pgrid(bicg_dot1k_kernel<T, K>, grid_vec), kSolverBlock, 0, cs>>>(n, rr, vv[nw], ctl,
                                                                          sc, partials);
            }
            if (bp) {
                launch_bicg_block_vec<T, K, 2>(n, *bp, r, vv[nw], nullptr, s, zv, ctl, sc, cs);
            } else if constexpr (kLanes) {
                bicg_vec_lanes_kernel<T, K, 2><<<pgrid(bicg_vec_lanes_kernel<T, K, 2>, grid_lanes), kSolverBlock, 0, cs>>>(
                    n, dinv, r, vv[nw], nullptr, s, zv, ctl, sc);
            } else {
                bicg_vec_k_kernel<T, K, 2><<<pgrid(bicg_vec_k_kernel<T, K, 2>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, dinv, r, vv[nw], nullptr, s, zv, ctl, sc);
            }
            spmv_k(zv, t);
            if constexpr (kLanes) {
                bicg_dots_lanes_kernel<T, K, 3><<<pgrid(bicg_dots_lanes_kernel<T, K, 3>, grid_lanes), kSolverBlock, 0, cs>>>(
                    n, s, t, ctl, sc, partials);
                bicg_update_lanes_kernel<T, K><<<pgrid(bicg_update_lanes_kernel<T, K>, grid_lanes), kSolverBlock, 0, cs>>>(
                    n, x, ldx, r, rr, yv, s, t, zv, ctl, sc, partials);
            } else {
                bicg_dot2k_kernel<T, K><<<pgrid(bicg_dot2k_kernel<T, K>, grid_vec), kSolverBlock, 0, cs>>>(n, s, t, ctl, sc,
                                                                          partials);
                bicg_update_kernel<T, K><<<pgrid(bicg_update_kernel<T, K>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, nullptr, x, ldx, r, rr, yv, s, t, ctl, sc, partials, zv);
            }
        });
    };
    const bool split_k = bp != nullptr || K >= 4;
    auto capture = [&](cudaStream_t cs) -> int {
        for (int it = 0; it < chunk; ++it) {
            const int o = it % 2, nw = (it + 1) % 2;
            if (split_k) {
                split_k_iteration(cs, o, nw);
                B2S_LAUNCH_CHECK();
                continue;
            }
            if (split) {
                bicg_pupdate_kernel<T><<<pgrid(bicg_pupdate_kernel<T>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, dinv, r, p[o], vv[o], p[nw], yv, ctl, sc);
                async_spmv(cs, yv, vv[nw]);
                bicg_dot1_kernel<T><<<pgrid(bicg_dot1_kernel<T>, grid_vec), kSolverBlock, 0, cs>>>(n, rr, vv[nw], ctl, sc,
                                                                      partials);
                bicg_supdate_kernel<T><<<pgrid(bicg_supdate_kernel<T>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, dinv, r, vv[nw], s, zv, ctl, sc);
                async_spmv(cs, zv, t);
                bicg_dot2_kernel<T><<<pgrid(bicg_dot2_kernel<T>, grid_vec), kSolverBlock, 0, cs>>>(n, s, t, ctl, sc,
                                                                      partials);
                bicg_update_kernel<T, 1><<<pgrid(bicg_update_kernel<T, 1>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, dinv, x, ldx, r, rr, p[nw], s, t, ctl, sc, partials);
                B2S_LAUNCH_CHECK();
                continue;
            }
            B2S_DISPATCH_RHS(K, {
                B2S_DISPATCH_SW(sw, {
                    bicg_spmv1_kernel<T, SW, K><<<pgrid(bicg_spmv1_kernel<T, SW, K>, grid_spmv), kSolverBlock, 0, cs>>>(
                        n, rp, ci, v, dinv, r, rr, p[o], vv[o], p[nw], vv[nw],
                        ctl, sc, partials);
                    bicg_spmv2_kernel<T, SW, K><<<pgrid(bicg_spmv2_kernel<T, SW, K>, grid_spmv), kSolverBlock, 0, cs>>>(
                        n, rp, ci, v, dinv, r, vv[nw], s, t, ctl, sc, partials);
                });
                bicg_update_kernel<T, K><<<pgrid(bicg_update_kernel<T, K>, grid_vec), kSolverBlock, 0, cs>>>(
                    n, dinv, x, ldx, r, rr, p[nw], s, t, ctl, sc, partials);
            });
            B2S_LAUNCH_CHECK();
        }
        return B2S_OK;
    };
    int rc = run_graph_loop(st, ctl, int(max_iters), chunk, capture, &h);
    if (rc != B2S_OK) return rc;
    BicgScalars<T> hs;
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

int64_t b2s_bicgstab_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                                     int value_bytes)
{
    const int K = rhs_bucket(num_rhs);
    if (K < 0 || num_rows < 0) return -1;
    return value_bytes == 8 ? bicg_layout<double>(num_rows, K).bytes
                            : bicg_layout<float>(num_rows, K).bytes;
}

int64_t b2s_bicgstab_block_workspace_bytes(int64_t num_rows, int64_t num_rhs,
                                           int value_bytes)
{
    const int K = rhs_bucket(num_rhs);
    if (K < 0 || num_rows < 0) return -1;
    return value_bytes == 8 ? bicg_layout<double>(num_rows, K, true).bytes
                            : bicg_layout<float>(num_rows, K, true).bytes;
}

#define B2S_BICG_ENTRY(T, S)                                                  \
    int b2s_bicgstab_solve_##S(                                               \
        int64_t num_rows, const int32_t* row_ptrs, const int32_t* col_idxs,   \
        const T* values, int64_t max_row_nnz, const T* inv_diag, const T* b,  \
        int64_t ldb, T* x, int64_t ldx, int64_t num_rhs, int64_t max_iters,   \
        double reduction_factor, int residual_mode, int64_t check_every,     \
        void* workspace,                                                      \
        int64_t workspace_bytes, int64_t* iterations, double* residual_norms, \
        uint8_t* status, void* stream)                                        \
    {                                                                         \
        return bicgstab_solve<T>(num_rows, row_ptrs, col_idxs, values,        \
                                 max_row_nnz, inv_diag, nullptr, b, ldb, x,   \
                                 ldx, num_rhs, max_iters, reduction_factor,   \
                                 residual_mode, check_every, workspace,       \
                                 workspace_bytes,                             \
                                 iterations, residual_norms, status, stream); \
    }                                                                         \
    int b2s_bicgstab_block_solve_##S(                                         \
        int64_t num_rows, const int32_t* row_ptrs, const int32_t* col_idxs,   \
        const T* values, int64_t max_row_nnz, int64_t num_blocks,             \
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
        return bicgstab_solve<T>(num_rows, row_ptrs, col_idxs, values,        \
                                 max_row_nnz, nullptr, &bp, b, ldb, x, ldx,   \
                                 num_rhs, max_iters, reduction_factor,        \
                                 residual_mode, check_every, workspace,       \
                                 workspace_bytes, iterations, residual_norms, \
                                 status, stream);                             \
    }

B2S_BICG_ENTRY(double, f64)
B2S_BICG_ENTRY(float, f32)

}  // extern "C"
