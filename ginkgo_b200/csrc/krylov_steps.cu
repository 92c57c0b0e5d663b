// Kernel-level drop-ins for the reference's Krylov step kernels, for a
// caller that keeps the reference's own solver loop and only swaps the
// backend.  Dense operands are row-major views {values, stride}; scalars are
// device arrays of num_rhs entries; stop_status is the reference's uint8
// stopping_status array (bit 7 converged, bit 6 finalized, bits 0-5 id).
// Semantics follow the reference executor:
//   cg          reference/solver/cg_kernels.cpp:25-98
//   bicgstab    reference/solver/bicgstab_kernels.cpp:26-160
//   gmres       reference/solver/gmres_kernels.cpp:27-100
//   common_gmres reference/solver/common_gmres_kernels.cpp:29-180
//   dot / norm2 reference/matrix/dense_kernels.cpp (compute_conj_dot,
//               compute_norm2), deterministic two-level reduction here
//   residual_norm common/cuda_hip/stop/residual_norm_kernels.cpp:42-50
// The fused solvers (b2s_cg_solve_* ...) are the fast path; these exist so
// the stock loop can run on the B200 kernels unchanged.
#include "solver_common.cuh"

namespace b2s {
namespace {

constexpr int kB = 256;

__device__ __forceinline__ bool stopped(const uint8_t* st, int64_t j)
{
    return has_stopped(st[j]);
}

#define B2S_ELEMWISE_LOOP(n, k)                                             \
    for (int64_t idx_ = blockIdx.x * int64_t(kB) + threadIdx.x;             \
         idx_ < (n) * (k); idx_ += int64_t(gridDim.x) * kB)                 \
        for (int64_t i = idx_ / (k), j = idx_ % (k), once_ = 1; once_;      \
             once_ = 0)

template <typename T>
__global__ void cg_initialize_k(int64_t n, int64_t k, const T* b, int64_t ldb,
                                T* r, int64_t ldr, T* z, int64_t ldz, T* p,
                                int64_t ldp, T* q, int64_t ldq, T* prev_rho,
                                T* rho, uint8_t* st)
{
    const int64_t g = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (g < k) {
        rho[g] = T(0);
        prev_rho[g] = T(1);
        st[g] = 0;
    }
    B2S_ELEMWISE_LOOP(n, k)
    {
        r[i * ldr + j] = b[i * ldb + j];
        z[i * ldz + j] = p[i * ldp + j] = q[i * ldq + j] = T(0);
    }
}

template <typename T>
__global__ void cg_step_1_k(int64_t n, int64_t k, T* p, int64_t ldp,
                            const T* z, int64_t ldz, const T* rho,
                            const T* prev_rho, const uint8_t* st)
{
    B2S_ELEMWISE_LOOP(n, k)
    {
        if (stopped(st, j)) continue;
        if (prev_rho[j] == T(0)) {
            p[i * ldp + j] = z[i * ldz + j];
        } else {
            const T tmp = rho[j] / prev_rho[j];
            p[i * ldp + j] = z[i * ldz + j] + tmp * p[i * ldp + j];
        }
    }
}

template <typename T>
__global__ void cg_step_2_k(int64_t n, int64_t k, T* x, int64_t ldx, T* r,
                            int64_t ldr, const T* p, int64_t ldp, const T* q,
                            int64_t ldq, const T* beta, const T* rho,
                            const uint8_t* st)
{
    B2S_ELEMWISE_LOOP(n, k)
    {
        if (stopped(st, j) || beta[j] == T(0)) continue;
        const T tmp = rho[j] / beta[j];
        x[i * ldx + j] += tmp * p[i * ldp + j];
        r[i * ldr + j] -= tmp * q[i * ldq + j];
    }
}

template <typename T>
__global__ void bicg_step_1_k(int64_t n, int64_t k, const T* r, int64_t ldr,
                              T* p, int64_t ldp, const T* v, int64_t ldv,
                              const T* rho, const T* prev_rho, const T* alpha,
                              const T* omega, const uint8_t* st)
{
    B2S_ELEMWISE_LOOP(n, k)
    {
        if (stopped(st, j)) continue;
        if (prev_rho[j] * omega[j] != T(0)) {
            const T tmp = rho[j] / prev_rho[j] * alpha[j] / omega[j];
            p[i * ldp + j] = r[i * ldr + j] +
                             tmp * (p[i * ldp + j] - omega[j] * v[i * ldv + j]);
        } else {
            p[i * ldp + j] = r[i * ldr + j];
        }
    }
}

// alpha is written by one thread per column before the vector update reads
// it, so the column value is computed redundantly from rho and beta instead
template <typename T>
__global__ void bicg_step_2_k(int64_t n, int64_t k, const T* r, int64_t ldr,
                              T* s, int64_t lds, const T* v, int64_t ldv,
                              const T* rho, T* alpha, const T* beta,
                              const uint8_t* st)
{
    const int64_t g = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (g < k && !stopped(st, g)) {
        alpha[g] = beta[g] != T(0) ? rho[g] / beta[g] : T(0);
    }
    B2S_ELEMWISE_LOOP(n, k)
    {
        if (stopped(st, j)) continue;
        const T a = beta[j] != T(0) ? rho[j] / beta[j] : T(0);
        s[i * lds + j] = r[i * ldr + j] - a * v[i * ldv + j];
    }
}

template <typename T>
__global__ void bicg_step_3_k(int64_t n, int64_t k, T* x, int64_t ldx, T* r,
                              int64_t ldr, const T* s, int64_t lds, const T* t,
                              int64_t ldt, const T* y, int64_t ldy, const T* z,
                              int64_t ldz, const T* alpha, const T* beta,
                              const T* gamma, T* omega, const uint8_t* st)
{
    const int64_t g = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (g < k && !stopped(st, g)) {
        omega[g] = beta[g] != T(0) ? gamma[g] / beta[g] : T(0);
    }
    B2S_ELEMWISE_LOOP(n, k)
    {
        if (stopped(st, j)) continue;
        const T om = beta[j] != T(0) ? gamma[j] / beta[j] : T(0);
        x[i * ldx + j] += alpha[j] * y[i * ldy + j] + om * z[i * ldz + j];
        r[i * ldr + j] = s[i * lds + j] - om * t[i * ldt + j];
    }
}

template <typename T>
__global__ void bicg_finalize_k(int64_t n, int64_t k, T* x, int64_t ldx,
                                const T* y, int64_t ldy, const T* alpha,
                                uint8_t* st)
{
    B2S_ELEMWISE_LOOP(n, k)
    {
        const uint8_t s = st[j];
        if (has_stopped(s) && !is_finalized(s)) {
            x[i * ldx + j] += alpha[j] * y[i * ldy + j];
        }
    }
}

__global__ void finalize_status_k(int64_t k, uint8_t* st)
{
    const int64_t g = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (g < k && has_stopped(st[g])) st[g] |= kFinalizedMask;
}

// Givens update of Hessenberg column `iter` per unstopped column (one
// thread per right-hand side), the reference's hessenberg_qr.
template <typename T>
__global__ void hessenberg_qr_k(int64_t k, int64_t iter, T* gs, int64_t ldgs,
                                T* gc, int64_t ldgc, T* resnorm, T* rnc,
                                int64_t ldrnc, T* h, int64_t ldh,
                                int64_t* final_iter_nums, const uint8_t* st)
{
    const int64_t c = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (c >= k) return;
    if (!stopped(st, c)) final_iter_nums[c]++;
    if (stopped(st, c)) return;
#define H_(i) h[(i) * ldh + c]
#define S_(i) gs[(i) * ldgs + c]
#define C_(i) gc[(i) * ldgc + c]
    for (int64_t j = 0; j < iter; ++j) {
        const T t = C_(j) * H_(j) + S_(j) * H_(j + 1);
        H_(j + 1) = -S_(j) * H_(j) + C_(j) * H_(j + 1);
        H_(j) = t;
    }
    if (H_(iter) == T(0)) {
        C_(iter) = T(0);
        S_(iter) = T(1);
    } else {
        const T th = H_(iter), nh = H_(iter + 1);
        const T scale = abs(th) + abs(nh);
        const T a = abs(th / scale), b = abs(nh / scale);
        const T hyp = scale * sqrt(a * a + b * b);
        C_(iter) = th / hyp;
        S_(iter) = nh / hyp;
    }
    H_(iter) = C_(iter) * H_(iter) + S_(iter) * H_(iter + 1);
    H_(iter + 1) = T(0);
    rnc[(iter + 1) * ldrnc + c] = -S_(iter) * rnc[iter * ldrnc + c];
    rnc[iter * ldrnc + c] = C_(iter) * rnc[iter * ldrnc + c];
    resnorm[c] = abs(rnc[(iter + 1) * ldrnc + c]);
#undef H_
#undef S_
#undef C_
}

template <typename T>
__global__ void solve_krylov_k(int64_t k, const T* rnc, int64_t ldrnc,
                               const T* h, int64_t ldh, T* y, int64_t ldy,
                               const int64_t* final_iter_nums,
                               const uint8_t* st)
{
    const int64_t c = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (c >= k || is_finalized(st[c])) return;
    for (int64_t i = final_iter_nums[c] - 1; i >= 0; --i) {
        T t = rnc[i * ldrnc + c];
        for (int64_t j = i + 1; j < final_iter_nums[c]; ++j) {
            t -= h[j * ldh + i * k + c] * y[j * ldy + c];
        }
        y[i * ldy + c] = t / h[i * ldh + i * k + c];
    }
}

// Deterministic dot / squared norm per column: per-block partials, then a
// single block sums them in order.
template <typename T, bool NORM>
__global__ void col_partials_k(int64_t n, int64_t k, const T* a, int64_t lda,
                               const T* b, int64_t ldb, T* partials)
{
    // block-strided over rows; column j reduced by the whole block
    __shared__ T red[kB / kWarp];
    for (int64_t j = 0; j < k; ++j) {
        T acc = T(0);
        for (int64_t i = blockIdx.x * int64_t(kB) + threadIdx.x; i < n;
             i += int64_t(gridDim.x) * kB) {
            const T x = a[i * lda + j];
            acc += NORM ? x * x : x * b[i * ldb + j];
        }
        acc = warp_sum(acc);
        if (threadIdx.x % kWarp == 0) red[threadIdx.x / kWarp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            T s = T(0);
            for (int w = 0; w < kB / kWarp; ++w) s += red[w];
            partials[j * gridDim.x + blockIdx.x] = s;
        }
        __syncthreads();
    }
}

template <typename T, bool NORM>
__global__ void col_finish_k(int64_t k, int nblocks, const T* partials, T* out)
{
    __shared__ T red[kB / kWarp];
    for (int64_t j = 0; j < k; ++j) {
        T acc = T(0);
        for (int b = threadIdx.x; b < nblocks; b += kB) acc += partials[j * nblocks + b];
        acc = warp_sum(acc);
        if (threadIdx.x % kWarp == 0) red[threadIdx.x / kWarp] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            T s = T(0);
            for (int w = 0; w < kB / kWarp; ++w) s += red[w];
            out[j] = NORM ? sqrt(s) : s;
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void residual_norm_k(int64_t k, const T* tau, const T* orig_tau,
                                double goal, uint8_t stopping_id,
                                int set_finalized, uint8_t* st, int* flags)
{
    // flags[0]: all converged/stopped, flags[1]: one changed (preset by the
    // host entry to 1 / 0, as the reference's init_kernel does)
    const int64_t c = blockIdx.x * int64_t(kB) + threadIdx.x;
    if (c >= k) return;
    if (double(tau[c]) <= goal * double(orig_tau[c])) {
        uint8_t s = st[c];
        converge_status(s, stopping_id, set_finalized != 0);
        st[c] = s;
        flags[1] = 1;
    } else if (!has_stopped(st[c])) {
        flags[0] = 0;
    }
}

inline int grid_for(int64_t work)
{
    return int(std::max<int64_t>(1, std::min<int64_t>(ceildiv(work, kB), 16 * num_sms())));
}

constexpr int kDotBlocks = 4 * kMaxSMs;  // grid-stride partials, any SM count

}  // namespace
}  // namespace b2s

using namespace b2s;

#define B2S_STEP_ENTRIES(T, S)                                                 \
    extern "C" int b2s_cg_initialize_##S(                                      \
        int64_t n, int64_t k, const T* b, int64_t ldb, T* r, int64_t ldr,      \
        T* z, int64_t ldz, T* p, int64_t ldp, T* q, int64_t ldq, T* prev_rho,  \
        T* rho, uint8_t* stop_status, void* stream)                            \
    {                                                                          \
        cg_initialize_k<T><<<grid_for(std::max(n * k, k)), kB, 0,              \
                             as_stream(stream)>>>(n, k, b, ldb, r, ldr, z,     \
                                                  ldz, p, ldp, q, ldq,         \
                                                  prev_rho, rho, stop_status); \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_cg_step_1_##S(int64_t n, int64_t k, T* p, int64_t ldp,  \
                                     const T* z, int64_t ldz, const T* rho,    \
                                     const T* prev_rho,                        \
                                     const uint8_t* stop_status, void* stream) \
    {                                                                          \
        if (n * k == 0) return B2S_OK;                                         \
        cg_step_1_k<T><<<grid_for(n * k), kB, 0, as_stream(stream)>>>(        \
            n, k, p, ldp, z, ldz, rho, prev_rho, stop_status);                 \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_cg_step_2_##S(                                          \
        int64_t n, int64_t k, T* x, int64_t ldx, T* r, int64_t ldr,            \
        const T* p, int64_t ldp, const T* q, int64_t ldq, const T* beta,       \
        const T* rho, const uint8_t* stop_status, void* stream)                \
    {                                                                          \
        if (n * k == 0) return B2S_OK;                                         \
        cg_step_2_k<T><<<grid_for(n * k), kB, 0, as_stream(stream)>>>(        \
            n, k, x, ldx, r, ldr, p, ldp, q, ldq, beta, rho, stop_status);     \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_bicgstab_step_1_##S(                                    \
        int64_t n, int64_t k, const T* r, int64_t ldr, T* p, int64_t ldp,      \
        const T* v, int64_t ldv, const T* rho, const T* prev_rho,              \
        const T* alpha, const T* omega, const uint8_t* stop_status,            \
        void* stream)                                                          \
    {                                                                          \
        if (n * k == 0) return B2S_OK;                                         \
        bicg_step_1_k<T><<<grid_for(n * k), kB, 0, as_stream(stream)>>>(      \
            n, k, r, ldr, p, ldp, v, ldv, rho, prev_rho, alpha, omega,         \
            stop_status);                                                      \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_bicgstab_step_2_##S(                                    \
        int64_t n, int64_t k, const T* r, int64_t ldr, T* s, int64_t lds,      \
        const T* v, int64_t ldv, const T* rho, T* alpha, const T* beta,        \
        const uint8_t* stop_status, void* stream)                              \
    {                                                                          \
        bicg_step_2_k<T><<<grid_for(std::max(n * k, k)), kB, 0,                \
                           as_stream(stream)>>>(n, k, r, ldr, s, lds, v, ldv,  \
                                                rho, alpha, beta,              \
                                                stop_status);                  \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_bicgstab_step_3_##S(                                    \
        int64_t n, int64_t k, T* x, int64_t ldx, T* r, int64_t ldr,            \
        const T* s, int64_t lds, const T* t, int64_t ldt, const T* y,          \
        int64_t ldy, const T* z, int64_t ldz, const T* alpha, const T* beta,   \
        const T* gamma, T* omega, const uint8_t* stop_status, void* stream)    \
    {                                                                          \
        bicg_step_3_k<T><<<grid_for(std::max(n * k, k)), kB, 0,                \
                           as_stream(stream)>>>(                               \
            n, k, x, ldx, r, ldr, s, lds, t, ldt, y, ldy, z, ldz, alpha, beta, \
            gamma, omega, stop_status);                                        \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_bicgstab_finalize_##S(                                  \
        int64_t n, int64_t k, T* x, int64_t ldx, const T* y, int64_t ldy,      \
        const T* alpha, uint8_t* stop_status, void* stream)                    \
    {                                                                          \
        cudaStream_t st = as_stream(stream);                                   \
        if (n * k > 0) {                                                       \
            bicg_finalize_k<T><<<grid_for(n * k), kB, 0, st>>>(                \
                n, k, x, ldx, y, ldy, alpha, stop_status);                     \
            B2S_LAUNCH_CHECK();                                                \
        }                                                                      \
        finalize_status_k<<<grid_for(k), kB, 0, st>>>(k, stop_status);         \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_gmres_hessenberg_qr_##S(                                \
        int64_t k, int64_t iter, T* givens_sin, int64_t ld_sin,                \
        T* givens_cos, int64_t ld_cos, T* residual_norm,                       \
        T* residual_norm_collection, int64_t ld_rnc, T* hessenberg_iter,       \
        int64_t ld_h, int64_t* final_iter_nums, const uint8_t* stop_status,    \
        void* stream)                                                          \
    {                                                                          \
        hessenberg_qr_k<T><<<grid_for(k), kB, 0, as_stream(stream)>>>(         \
            k, iter, givens_sin, ld_sin, givens_cos, ld_cos, residual_norm,    \
            residual_norm_collection, ld_rnc, hessenberg_iter, ld_h,           \
            final_iter_nums, stop_status);                                     \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_gmres_solve_krylov_##S(                                 \
        int64_t k, const T* residual_norm_collection, int64_t ld_rnc,          \
        const T* hessenberg, int64_t ld_h, T* y, int64_t ld_y,                 \
        const int64_t* final_iter_nums, const uint8_t* stop_status,            \
        void* stream)                                                          \
    {                                                                          \
        solve_krylov_k<T><<<grid_for(k), kB, 0, as_stream(stream)>>>(          \
            k, residual_norm_collection, ld_rnc, hessenberg, ld_h, y, ld_y,    \
            final_iter_nums, stop_status);                                     \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_dense_compute_dot_##S(                                  \
        int64_t n, int64_t k, const T* a, int64_t lda, const T* b,             \
        int64_t ldb, T* result, void* workspace, int64_t workspace_bytes,      \
        void* stream)                                                          \
    {                                                                          \
        const int64_t need = int64_t(kDotBlocks) * k * int64_t(sizeof(T));    \
        if (workspace_bytes < need) {                                          \
            set_error("workspace of %lld bytes < %lld",                        \
                      (long long)workspace_bytes, (long long)need);            \
            return B2S_ERR_WORKSPACE;                                          \
        }                                                                      \
        if (k == 0) return B2S_OK;                                             \
        cudaStream_t st = as_stream(stream);                                   \
        T* part = static_cast<T*>(workspace);                                  \
        col_partials_k<T, false><<<kDotBlocks, kB, 0, st>>>(n, k, a, lda, b,   \
                                                            ldb, part);        \
        col_finish_k<T, false><<<1, kB, 0, st>>>(k, kDotBlocks, part, result); \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_dense_compute_norm2_##S(                                \
        int64_t n, int64_t k, const T* a, int64_t lda, T* result,              \
        void* workspace, int64_t workspace_bytes, void* stream)                \
    {                                                                          \
        const int64_t need = int64_t(kDotBlocks) * k * int64_t(sizeof(T));    \
        if (workspace_bytes < need) {                                          \
            set_error("workspace of %lld bytes < %lld",                        \
                      (long long)workspace_bytes, (long long)need);            \
            return B2S_ERR_WORKSPACE;                                          \
        }                                                                      \
        if (k == 0) return B2S_OK;                                             \
        cudaStream_t st = as_stream(stream);                                   \
        T* part = static_cast<T*>(workspace);                                  \
        col_partials_k<T, true><<<kDotBlocks, kB, 0, st>>>(n, k, a, lda, a,    \
                                                           lda, part);         \
        col_finish_k<T, true><<<1, kB, 0, st>>>(k, kDotBlocks, part, result);  \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }                                                                          \
    extern "C" int b2s_residual_norm_check_##S(                                \
        int64_t k, const T* tau, const T* orig_tau, double goal,               \
        int stopping_id, int set_finalized, uint8_t* stop_status,              \
        int* device_flags, void* stream)                                       \
    {                                                                          \
        cudaStream_t st = as_stream(stream);                                   \
        const int init[2] = {1, 0};                                            \
        B2S_CUDA_TRY(cudaMemcpyAsync(device_flags, init, sizeof(init),         \
                                     cudaMemcpyHostToDevice, st));             \
        residual_norm_k<T><<<grid_for(k), kB, 0, st>>>(                        \
            k, tau, orig_tau, goal, uint8_t(stopping_id), set_finalized,       \
            stop_status, device_flags);                                        \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }

B2S_STEP_ENTRIES(double, f64)
B2S_STEP_ENTRIES(float, f32)

extern "C" int64_t b2s_dense_reduction_workspace_bytes(int64_t num_rhs,
                                                       int value_bytes)
{
    return int64_t(b2s::kDotBlocks) * num_rhs * value_bytes;
}
