// Batched BiCGStab over thousands of independent systems of uneven size,
// stored as a ragged batch Ell.  Each system is solved by one group of G
// threads (G = 32..256, several groups per block); the rows of a system are
// spread over the group, RPT rows per thread, and the solver vectors of a
// thread's rows live in registers.  Only the two SpMV inputs (p_hat, s_hat)
// go to shared memory (or a global scratch, the autotuner decides), so one
// SM holds many systems at once.  Systems are sorted into size buckets;
// every bucket is a persistent kernel whose groups walk the bucket's system
// list, and all buckets run from one CUDA graph on parallel branches.
//
// Algorithm per system: reference/solver/batch_bicgstab_kernels.hpp:175-348
// (the same order of updates, stop test ||r|| <= tol ||b|| (relative) or
// ||r|| <= tol (absolute) checked at the loop top and on s, iteration count
// logged as the batch logger does), scalar Jacobi as
// reference/preconditioner/batch_scalar_jacobi.hpp:40-58 (first stored
// diagonal entry, zero -> 1).  Four group reductions per iteration.
//
// Batch Ell layout: system b has n_b = row_offsets[b+1] - row_offsets[b]
// rows and its entries at values[width * row_offsets[b] + j * n_b + r],
// column-major inside the system with local column indices (-1 = padding);
// for equal sizes this is the reference's batch::matrix::Ell value layout
// (include/ginkgo/core/matrix/batch_ell.hpp:149-221) with the column indices
// stored per system.  The uniform entry points take the reference's own
// batch::matrix::Ell: every system n rows, one col_idxs array of n * width
// entries shared by all systems (core/matrix/batch_struct.hpp:268-280).
#include <algorithm>
#include <map>
#include <vector>

#include "solver_common.cuh"

namespace b2s {
namespace {

constexpr int kBatchBlock = 256;

template <int G>
__device__ __forceinline__ void group_sync(int group)
{
    if constexpr (G == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(G) : "memory");
    }
}

// Sum over the G threads of a group, M <= kMaxSums values at once; every
// thread gets the totals.  red: [2][G/32][kMaxSums] per group; consecutive
// calls alternate between the two halves.  The halves have a fixed size
// whatever M is, so a call never writes entries that the previous call (on
// the other half) may still be reading: a warp reaches call c + 2's writes
// only after call c + 1's barrier, which every warp passes after its reads
// of call c.
constexpr int kMaxSums = 2;

template <typename T, int G, int M>
__device__ __forceinline__ void group_sum(T (&v)[M], T* red, int& parity,
                                          int group)
{
    static_assert(M <= kMaxSums, "group_sum: too many values");
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = warp_sum(v[m]);
    if constexpr (G > 32) {
        constexpr int W = G / 32;
        T* slot = red + parity * W * kMaxSums;
        const int lane = threadIdx.x % 32, wig = (threadIdx.x % G) / 32;
        if (lane == 0) {
#pragma unroll
            for (int m = 0; m < M; ++m) slot[wig * M + m] = v[m];
        }
        group_sync<G>(group);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            T s = T(0);
#pragma unroll
            for (int w = 0; w < W; ++w) s += slot[w * M + m];
            v[m] = s;
        }
        parity ^= 1;
    } else {
        __syncwarp();  // order the group's shared-memory traffic
    }
}

struct BatchArgs {
    const int32_t* row_offsets;  // ragged batch; unused when uniform_n > 0
    int uniform_n;               // > 0: every system has this many rows and
                                 // the column indices are shared
    const int32_t* sys_list;  // systems of this bucket
    int num_sys;
    int width;
    int max_iters;
    int tol_absolute;
    int use_jacobi;
    double tol;
    int32_t* iters_out;
    double* res_out;
};

template <typename T, int G, int RPT, bool SMEM>
__global__ void __launch_bounds__(kBatchBlock, 1)
    batch_bicgstab_kernel(BatchArgs a, const int32_t* __restrict__ ci,
                          const T* __restrict__ val, const T* __restrict__ b,
                          T* __restrict__ x, T* __restrict__ gscratch)
{
    constexpr int GPB = kBatchBlock / G;  // groups per block
    constexpr int NMAX = G * RPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int group = threadIdx.x / G;
    const int t = threadIdx.x % G;
    T* red = reinterpret_cast<T*>(smem_raw) + group * 2 * (G / 32) * kMaxSums;
    T* vecs;
    if constexpr (SMEM) {
        vecs = reinterpret_cast<T*>(smem_raw) + GPB * 2 * (G / 32) * kMaxSums +
               group * 2 * NMAX;
    } else {
        vecs = gscratch + (int64_t(blockIdx.x) * GPB + group) * 2 * NMAX;
    }
    T* phat = vecs;
    T* shat = vecs + NMAX;
    int parity = 0;
    const int total_groups = gridDim.x * GPB;
    for (int q = blockIdx.x * GPB + group; q < a.num_sys; q += total_groups) {
        const int sys = a.sys_list[q];
        const int off = a.uniform_n ? sys * a.uniform_n : a.row_offsets[sys];
        const int n = a.uniform_n ? a.uniform_n : a.row_offsets[sys + 1] - off;
        const int64_t vbase = int64_t(a.width) * off;
        const int32_t* cs = a.uniform_n ? ci : ci + vbase;
        const T* vs = val + vbase;
        T r[RPT], rh[RPT], p[RPT], v[RPT], s[RPT], tt[RPT], xx[RPT], pr[RPT];
        T bb2 = T(0);
        // preconditioner, x, r = b - A x with x staged as the SpMV input
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int row = t + k * G;
            pr[k] = T(1);
            xx[k] = T(0);
            if (row < n) {
                if (a.use_jacobi) {
                    for (int j = 0; j < a.width; ++j) {
                        if (cs[row + j * n] == row) {
                            const T d = vs[row + j * n];
                            if (d != T(0)) pr[k] = T(1) / d;
                            break;
                        }
                    }
                }
                xx[k] = x[off + row];
                phat[row] = xx[k];
                const T bv = b[off + row];
                r[k] = bv;
                bb2 += bv * bv;
            }
        }
        group_sync<G>(group);
        T rr2 = T(0);
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int row = t + k * G;
            if (row < n) {
                T acc = T(0);
                for (int j = 0; j < a.width; ++j) {
                    const int c = cs[row + j * n];
                    if (unsigned(c) < unsigned(n)) acc += vs[row + j * n] * phat[c];
                }
                r[k] -= acc;
                rr2 += r[k] * r[k];
            } else {
                r[k] = T(0);
            }
            rh[k] = r[k];
            p[k] = T(0);
            v[k] = T(0);
        }
        T red2[2] = {bb2, rr2};
        group_sum<T, G, 2>(red2, red, parity, group);
        const T rhs_norm = sqrt(red2[0]);
        T res_norm = sqrt(red2[1]);
        const T goal = a.tol_absolute ? T(a.tol) : T(a.tol) * rhs_norm;
        T rho_old = T(1), omega = T(1), alpha = T(1);
        // rho_new for the first iteration: r_hat . r = ||r||^2
        T rho_new = red2[1];
        int iter = 0;
        for (iter = 0; iter < a.max_iters; ++iter) {
            if (res_norm <= goal) break;
            const T beta = (rho_new / rho_old) * (alpha / omega);
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int row = t + k * G;
                p[k] = r[k] + beta * (p[k] - omega * v[k]);
                if (row < n) phat[row] = pr[k] * p[k];
            }
            group_sync<G>(group);
            T d1[1] = {T(0)};
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int row = t + k * G;
                if (row < n) {
                    T acc = T(0);
                    for (int j = 0; j < a.width; ++j) {
                        const int c = cs[row + j * n];
                        if (unsigned(c) < unsigned(n)) acc += vs[row + j * n] * phat[c];
                    }
                    v[k] = acc;
                    d1[0] += rh[k] * acc;
                }
            }
            group_sum<T, G, 1>(d1, red, parity, group);
            alpha = rho_new / d1[0];
            T d2[1] = {T(0)};
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int row = t + k * G;
                s[k] = r[k] - alpha * v[k];
                if (row < n) {
                    shat[row] = pr[k] * s[k];
                    d2[0] += s[k] * s[k];
                }
            }
            group_sum<T, G, 1>(d2, red, parity, group);
            res_norm = sqrt(d2[0]);
            if (res_norm <= goal) {
#pragma unroll
                for (int k = 0; k < RPT; ++k) xx[k] += alpha * (pr[k] * p[k]);
                break;
            }
            T d3[2] = {T(0), T(0)};
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int row = t + k * G;
                if (row < n) {
                    T acc = T(0);
                    for (int j = 0; j < a.width; ++j) {
                        const int c = cs[row + j * n];
                        if (unsigned(c) < unsigned(n)) acc += vs[row + j * n] * shat[c];
                    }
                    tt[k] = acc;
                    d3[0] += acc * s[k];
                    d3[1] += acc * acc;
                } else {
                    tt[k] = T(0);
                }
            }
            group_sum<T, G, 2>(d3, red, parity, group);
            omega = d3[0] / d3[1];
            T d4[2] = {T(0), T(0)};
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int row = t + k * G;
                xx[k] += alpha * (pr[k] * p[k]) + omega * (pr[k] * s[k]);
                r[k] = s[k] - omega * tt[k];
                if (row < n) {
                    d4[0] += r[k] * r[k];
                    d4[1] += rh[k] * r[k];
                }
            }
            group_sum<T, G, 2>(d4, red, parity, group);
            res_norm = sqrt(d4[0]);
            rho_old = rho_new;
            rho_new = d4[1];
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int row = t + k * G;
            if (row < n) x[off + row] = xx[k];
        }
        if (t == 0) {
            a.iters_out[sys] = iter;
            a.res_out[sys] = double(res_norm);
        }
        // the next system reuses phat/shat
        group_sync<G>(group);
    }
}

template <typename T, int G, int RPT>
size_t batch_smem_bytes(bool smem_vecs)
{
    constexpr int GPB = kBatchBlock / G;
    size_t bytes = size_t(GPB) * 2 * (G / 32) * kMaxSums * sizeof(T);
    if (smem_vecs) bytes += size_t(GPB) * 2 * G * RPT * sizeof(T);
    return bytes;
}

// Launch configurations: (G, RPT) with G * RPT >= the bucket's largest
// system; RPT <= 16 keeps the eight register vectors within budget.
struct BatchConfig {
    int G, RPT;
    bool smem;
};

template <typename T>
int launch_bucket(const BatchConfig& cfg, const BatchArgs& a,
                  const int32_t* ci, const T* val, const T* b, T* x,
                  T* gscratch, int64_t gscratch_entries, cudaStream_t st)
{
    if (a.num_sys == 0) return B2S_OK;
#define B2S_BATCH_CASE(GG, RR)                                                 \
    if (cfg.G == GG && cfg.RPT == RR) {                                        \
        constexpr int GPB = kBatchBlock / GG;                                  \
        const int need = int(ceildiv(a.num_sys, GPB));                         \
        int grid;                                                              \
        if (cfg.smem) {                                                        \
            auto k = batch_bicgstab_kernel<T, GG, RR, true>;                   \
            const size_t sm = batch_smem_bytes<T, GG, RR>(true);               \
            B2S_CUDA_TRY(cudaFuncSetAttribute(                                 \
                k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));     \
            int per_sm = 0;                                                    \
            B2S_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(        \
                &per_sm, k, kBatchBlock, sm));                                 \
            grid = std::max(1, std::min(need, std::max(per_sm, 1) * num_sms())); \
            k<<<grid, kBatchBlock, sm, st>>>(a, ci, val, b, x, gscratch);      \
        } else {                                                               \
            auto k = batch_bicgstab_kernel<T, GG, RR, false>;                  \
            const size_t sm = batch_smem_bytes<T, GG, RR>(false);              \
            int per_sm = 0;                                                    \
            B2S_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(        \
                &per_sm, k, kBatchBlock, sm));                                 \
            grid = std::max(1, std::min(need, std::max(per_sm, 1) * num_sms())); \
            const int64_t need_scratch = int64_t(grid) * GPB * 2 * GG * RR;    \
            if (need_scratch > gscratch_entries) {                             \
                grid = int(gscratch_entries / (int64_t(GPB) * 2 * GG * RR));   \
                if (grid < 1) {                                                \
                    set_error("batch scratch too small");                      \
                    return B2S_ERR_WORKSPACE;                                  \
                }                                                              \
            }                                                                  \
            k<<<grid, kBatchBlock, sm, st>>>(a, ci, val, b, x, gscratch);      \
        }                                                                      \
        B2S_LAUNCH_CHECK();                                                    \
        return B2S_OK;                                                         \
    }
    B2S_BATCH_CASE(32, 1)
    B2S_BATCH_CASE(32, 2)
    B2S_BATCH_CASE(32, 4)
    B2S_BATCH_CASE(32, 8)
    B2S_BATCH_CASE(32, 16)
    B2S_BATCH_CASE(64, 1)
    B2S_BATCH_CASE(64, 2)
    B2S_BATCH_CASE(64, 4)
    B2S_BATCH_CASE(64, 8)
    B2S_BATCH_CASE(64, 16)
    B2S_BATCH_CASE(128, 1)
    B2S_BATCH_CASE(128, 2)
    B2S_BATCH_CASE(128, 4)
    B2S_BATCH_CASE(128, 8)
    B2S_BATCH_CASE(256, 1)
    B2S_BATCH_CASE(256, 2)
    B2S_BATCH_CASE(256, 4)
#undef B2S_BATCH_CASE
    set_error("unsupported batch configuration G=%d RPT=%d", cfg.G, cfg.RPT);
    return B2S_ERR_UNSUPPORTED;
}

// Size buckets by powers of two of the largest row count they hold.
constexpr int kBuckets = 12;  // up to 2^11 = 2048 rows
inline int bucket_of(int n)
{
    int bkt = 0;
    while ((1 << (bkt + 1)) < n && bkt + 1 < kBuckets) ++bkt;
    return (1 << bkt) >= n ? bkt : bkt + 1;
}

inline std::vector<BatchConfig> candidates(int nmax)
{
    std::vector<BatchConfig> out;
    for (int G : {32, 64, 128, 256}) {
        int rpt = 1;
        while (G * rpt < nmax) rpt *= 2;
        const int max_rpt = 8;  // eight register vectors of RPT rows
        if (rpt > max_rpt) continue;
        out.push_back({G, rpt, true});
        out.push_back({G, rpt, false});
    }
    return out;
}

// Default when no tuned table is given: the smallest group that keeps four
// rows per thread or fewer, vectors in shared memory.
inline BatchConfig default_config(int nmax)
{
    for (int G : {32, 64, 128, 256}) {
        int rpt = 1;
        while (G * rpt < nmax) rpt *= 2;
        if (rpt <= 4) return {G, rpt, true};
    }
    int rpt = 1;
    while (256 * rpt < nmax) rpt *= 2;
    return {256, rpt, true};
}

struct BucketPlan {
    int bucket, nmax, first, count;  // slice of the sorted system list
};

template <typename T>
int batch_solve(int64_t num_sys, const int32_t* row_offsets,
                const int32_t* host_row_offsets, int64_t width,
                const int32_t* ci, const T* val, const T* b, T* x,
                int64_t max_iters, double tol, int tol_absolute,
                int use_jacobi, const int32_t* tune_table, void* workspace,
                int64_t workspace_bytes, int32_t* iters_out, double* res_out,
                void* stream, int32_t* tune_out, int uniform_n = 0)
{
    B2S_CHECK_ARG(num_sys >= 0 && width >= 1 && width <= 64, "bad batch shape");
    B2S_CHECK_ARG(host_row_offsets != nullptr, "host row offsets required");
    B2S_CHECK_ARG(max_iters >= 0 && max_iters < (1 << 30), "max_iters out of range");
    if (num_sys == 0) return B2S_OK;
    cudaStream_t st = as_stream(stream);
    // sort systems by bucket (stable) on the host
    std::vector<std::vector<int32_t>> lists(kBuckets);
    int max_n = 0;
    for (int64_t s = 0; s < num_sys; ++s) {
        const int n = host_row_offsets[s + 1] - host_row_offsets[s];
        B2S_CHECK_ARG(n >= 0 && n <= (1 << (kBuckets - 1)),
                      "system %lld has %d rows (1..%d supported)", (long long)s,
                      n, 1 << (kBuckets - 1));
        lists[bucket_of(std::max(n, 1))].push_back(int32_t(s));
        max_n = std::max(max_n, n);
    }
    std::vector<int32_t> order;
    std::vector<BucketPlan> plans;
    for (int bk = 0; bk < kBuckets; ++bk) {
        if (lists[bk].empty()) continue;
        plans.push_back({bk, 1 << bk, int(order.size()), int(lists[bk].size())});
        order.insert(order.end(), lists[bk].begin(), lists[bk].end());
    }
    // workspace: system list, then the global scratch for SpMV inputs
    const int64_t list_bytes = (num_sys * 4 + 255) / 256 * 256;
    B2S_CHECK_ARG(workspace_bytes >= list_bytes, "workspace too small");
    int32_t* dev_list = static_cast<int32_t*>(workspace);
    T* gscratch = reinterpret_cast<T*>(static_cast<char*>(workspace) + list_bytes);
    const int64_t gscratch_entries = (workspace_bytes - list_bytes) / int64_t(sizeof(T));
    B2S_CUDA_TRY(cudaMemcpyAsync(dev_list, order.data(), num_sys * 4,
                                 cudaMemcpyHostToDevice, st));
    B2S_CUDA_TRY(cudaStreamSynchronize(st));  // order lives on the host stack

    auto args_for = [&](const BucketPlan& pl) {
        BatchArgs a;
        a.row_offsets = row_offsets;
        a.uniform_n = uniform_n;
        a.sys_list = dev_list + pl.first;
        a.num_sys = pl.count;
        a.width = int(width);
        a.max_iters = int(max_iters);
        a.tol_absolute = tol_absolute;
        a.use_jacobi = use_jacobi;
        a.tol = tol;
        a.iters_out = iters_out;
        a.res_out = res_out;
        return a;
    };

    std::vector<BatchConfig> chosen(plans.size());
    for (size_t i = 0; i < plans.size(); ++i) {
        const int bk = plans[i].bucket;
        if (tune_table && tune_table[2 * bk] > 0) {
            chosen[i] = {tune_table[2 * bk], 0, tune_table[2 * bk + 1] != 0};
            int rpt = 1;
            while (chosen[i].G * rpt < plans[i].nmax) rpt *= 2;
            chosen[i].RPT = rpt;
        } else {
            chosen[i] = default_config(plans[i].nmax);
        }
    }

    if (tune_out) {
        // autotune: time every candidate on the bucket, x restored between
        // trials from a copy kept in the scratch tail
        int64_t total_rows = host_row_offsets[num_sys] - host_row_offsets[0];
        B2S_CHECK_ARG(gscratch_entries > total_rows, "workspace too small for tuning");
        T* x_save = gscratch + gscratch_entries - total_rows;
        const int64_t scratch_avail = gscratch_entries - total_rows;
        B2S_CUDA_TRY(cudaMemcpyAsync(x_save, x + host_row_offsets[0],
                                     total_rows * sizeof(T),
                                     cudaMemcpyDeviceToDevice, st));
        cudaEvent_t e0, e1;
        B2S_CUDA_TRY(cudaEventCreate(&e0));
        B2S_CUDA_TRY(cudaEventCreate(&e1));
        for (int k = 0; k < 2 * kBuckets; ++k) tune_out[k] = 0;
        for (size_t i = 0; i < plans.size(); ++i) {
            float best = 1e30f;
            BatchConfig best_cfg = chosen[i];
            for (const BatchConfig& cfg : candidates(plans[i].nmax)) {
                float ms_min = 1e30f;
                for (int rep = 0; rep < 2; ++rep) {
                    B2S_CUDA_TRY(cudaMemcpyAsync(
                        x + host_row_offsets[0], x_save, total_rows * sizeof(T),
                        cudaMemcpyDeviceToDevice, st));
                    B2S_CUDA_TRY(cudaEventRecord(e0, st));
                    int rc = launch_bucket<T>(cfg, args_for(plans[i]), ci, val, b,
                                              x, gscratch, scratch_avail, st);
                    if (rc != B2S_OK) return rc;
                    B2S_CUDA_TRY(cudaEventRecord(e1, st));
                    B2S_CUDA_TRY(cudaEventSynchronize(e1));
                    float ms = 0;
                    B2S_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
                    ms_min = std::min(ms_min, ms);
                }
                if (ms_min < best) {
                    best = ms_min;
                    best_cfg = cfg;
                }
            }
            chosen[i] = best_cfg;
            tune_out[2 * plans[i].bucket] = best_cfg.G;
            tune_out[2 * plans[i].bucket + 1] = best_cfg.smem ? 1 : 0;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        B2S_CUDA_TRY(cudaMemcpyAsync(x + host_row_offsets[0], x_save,
                                     total_rows * sizeof(T),
                                     cudaMemcpyDeviceToDevice, st));
    }

    // one graph, every bucket on its own branch
    cudaStream_t cap;
    B2S_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    std::vector<cudaStream_t> branches(plans.size());
    for (auto& s : branches) B2S_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t fork, join;
    B2S_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    B2S_CUDA_TRY(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = B2S_OK;
    // the scratch is split evenly between the buckets that use it
    const int64_t per_bucket = gscratch_entries / int64_t(std::max<size_t>(plans.size(), 1));
    do {
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { set_error("capture: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
        cudaEventRecord(fork, cap);
        for (size_t i = 0; i < plans.size() && rc == B2S_OK; ++i) {
            cudaStreamWaitEvent(branches[i], fork, 0);
            rc = launch_bucket<T>(chosen[i], args_for(plans[i]), ci, val, b, x,
                                  gscratch + int64_t(i) * per_bucket, per_bucket,
                                  branches[i]);
            cudaEventRecord(join, branches[i]);
            cudaStreamWaitEvent(cap, join, 0);
        }
        e = cudaStreamEndCapture(cap, &graph);
        if (rc != B2S_OK) break;
        if (e != cudaSuccess) { set_error("capture: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; break; }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { set_error("batch graph: %s", cudaGetErrorString(e)); rc = B2S_ERR_CUDA; }
    } while (false);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    for (auto& s : branches) cudaStreamDestroy(s);
    cudaStreamDestroy(cap);
    return rc;
}

}  // namespace
}  // namespace b2s

using namespace b2s;

extern "C" {

int64_t b2s_batch_bicgstab_workspace_bytes(int64_t num_systems,
                                           int64_t total_rows, int value_bytes)
{
    if (num_systems < 0 || total_rows < 0) return -1;
    // system list + scratch for the SpMV inputs of every concurrently
    // resident group (bounded by the SM count) + a copy of x for tuning
    const int64_t list = (num_systems * 4 + 255) / 256 * 256;
    const int64_t pool = int64_t(64) << 20;  // SpMV-input scratch of the groups
    return list + pool + total_rows * value_bytes;
}

#define B2S_BATCH_ENTRY(T, S)                                                  \
    int b2s_batch_ell_bicgstab_solve_##S(                                      \
        int64_t num_systems, const int32_t* row_offsets,                       \
        const int32_t* host_row_offsets, int64_t width,                        \
        const int32_t* col_idxs, const T* values, const T* b, T* x,            \
        int64_t max_iters, double tolerance, int tolerance_absolute,           \
        int use_jacobi, const int32_t* tune_table, void* workspace,            \
        int64_t workspace_bytes, int32_t* iterations, double* residual_norms, \
        void* stream)                                                          \
    {                                                                          \
        return batch_solve<T>(num_systems, row_offsets, host_row_offsets,      \
                              width, col_idxs, values, b, x, max_iters,        \
                              tolerance, tolerance_absolute, use_jacobi,       \
                              tune_table, workspace, workspace_bytes,          \
                              iterations, residual_norms, stream, nullptr);    \
    }                                                                          \
    int b2s_batch_ell_bicgstab_tune_##S(                                       \
        int64_t num_systems, const int32_t* row_offsets,                       \
        const int32_t* host_row_offsets, int64_t width,                        \
        const int32_t* col_idxs, const T* values, const T* b, T* x,            \
        int64_t max_iters, double tolerance, int tolerance_absolute,           \
        int use_jacobi, void* workspace, int64_t workspace_bytes,              \
        int32_t* iterations, double* residual_norms, int32_t* tune_table_out,  \
        void* stream)                                                          \
    {                                                                          \
        return batch_solve<T>(num_systems, row_offsets, host_row_offsets,      \
                              width, col_idxs, values, b, x, max_iters,        \
                              tolerance, tolerance_absolute, use_jacobi,       \
                              nullptr, workspace, workspace_bytes, iterations, \
                              residual_norms, stream, tune_table_out);         \
    }

B2S_BATCH_ENTRY(double, f64)
B2S_BATCH_ENTRY(float, f32)

// The reference's uniform batch::matrix::Ell: num_systems systems of
// num_rows rows each, column indices shared (num_rows * width entries).
#define B2S_BATCH_UNIFORM_ENTRY(T, S)                                          \
    int b2s_batch_ell_uniform_bicgstab_solve_##S(                              \
        int64_t num_systems, int64_t num_rows, int64_t width,                  \
        const int32_t* col_idxs, const T* values, const T* b, T* x,            \
        int64_t max_iters, double tolerance, int tolerance_absolute,           \
        int use_jacobi, const int32_t* tune_table, void* workspace,            \
        int64_t workspace_bytes, int32_t* iterations, double* residual_norms, \
        void* stream, int32_t* tune_table_out)                                 \
    {                                                                          \
        B2S_CHECK_ARG(num_systems >= 0 && num_rows >= 1 &&                     \
                          num_rows <= (1 << (kBuckets - 1)),                   \
                      "uniform batch: num_rows must be 1..%d",                 \
                      1 << (kBuckets - 1));                                    \
        B2S_CHECK_ARG(num_systems * num_rows < (int64_t(1) << 31),             \
                      "uniform batch too large for int32 row offsets");        \
        std::vector<int32_t> offs(size_t(num_systems) + 1);                    \
        for (int64_t s = 0; s <= num_systems; ++s)                             \
            offs[size_t(s)] = int32_t(s * num_rows);                           \
        return batch_solve<T>(num_systems, nullptr, offs.data(), width,        \
                              col_idxs, values, b, x, max_iters, tolerance,    \
                              tolerance_absolute, use_jacobi,                  \
                              tune_table_out ? nullptr : tune_table,           \
                              workspace, workspace_bytes, iterations,          \
                              residual_norms, stream, tune_table_out,          \
                              int(num_rows));                                  \
    }

B2S_BATCH_UNIFORM_ENTRY(double, f64)
B2S_BATCH_UNIFORM_ENTRY(float, f32)

}  // extern "C"
